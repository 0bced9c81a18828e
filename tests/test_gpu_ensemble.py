"""The batched ensemble: CUDA-graph replay over several streams gives the
same fields, bit for bit, as stepping the members one by one."""
import numpy as np
import pytest

torch = pytest.importorskip('torch')

from atmdyn import ic
from atmdyn.ensemble import Ensemble

pytestmark = pytest.mark.gpu


def members():
    out = []
    for i, (n, L) in enumerate(((32, 8), (48, 12), (40, 10), (64, 6), (24, 8))):
        if i % 2:
            st = ic.jet_case(n, n, L, 25e3 * 1024 / n / 4, 25e3 * 1024 / n / 4, width=300e3, seed=10 + i)
            st.dt = 30.0
        else:
            st = ic.bubble_case(n, n, L, 50e3 * 128 / n, 50e3 * 128 / n, seed=10 + i)
        st.remap_every = 5
        out.append(st)
    return out


@pytest.mark.parametrize('precision', ['mixed', 'fp64'])
def test_graph_replay_matches_eager(precision):
    a = Ensemble(members(), precision, nstreams=3)
    b = Ensemble(members(), precision, nstreams=3)
    a.step_eager(15)
    b.step_eager(5)
    b.capture(5)
    b.replay(2)
    torch.cuda.synchronize()
    for da, db in zip(a.dyn, b.dyn):
        for f in ('dp', 'pt', 'ud', 'vd'):
            np.testing.assert_array_equal(da.get(f, halo=True), db.get(f, halo=True))
    assert a.stable() and b.stable()
    a.close()
    b.close()


def test_whole_run_as_one_graph_matches_eager():
    """Four remap cycles (20 steps) captured as one graph and replayed as
    one launch."""
    a = Ensemble(members(), 'mixed', nstreams=3)
    b = Ensemble(members(), 'mixed', nstreams=3)
    a.step_eager(25)
    b.step_eager(5)
    b.capture(5, cycles=4)
    assert b.cycle == 20
    b.replay(1)
    torch.cuda.synchronize()
    for da, db in zip(a.dyn, b.dyn):
        for f in ('dp', 'pt', 'ud', 'vd'):
            np.testing.assert_array_equal(da.get(f, halo=True), db.get(f, halo=True))
    a.close()
    b.close()
