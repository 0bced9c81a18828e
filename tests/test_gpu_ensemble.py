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


def _fields(ens):
    return [{f: d.get(f, halo=True) for f in ('dp', 'pt', 'ud', 'vd')} for d in ens.dyn]


def _assert_same(a, b):
    for fa, fb in zip(a, b):
        for f in fa:
            np.testing.assert_array_equal(fa[f], fb[f], err_msg=f)


@pytest.mark.parametrize('strips', [None, {32: 16, 48: 32, 40: 16, 64: 64, 24: 32}])
@pytest.mark.parametrize('dataflow', [True, False])
def test_persistent_kernel_matches_eager(strips, dataflow):
    """One launch of the persistent kernel advances every member (uneven
    sizes and layer counts) by 10 steps with two remaps, bit for bit as
    stepping the members one by one, whatever the strip heights, with the
    dataflow schedule and with the stage barriers."""
    a = Ensemble(members(), 'mixed', nstreams=3)
    b = Ensemble(members(), 'mixed', nstreams=3)
    a.step_eager(10)
    if strips:
        b.set_strips(strips)
    b.set_schedule(dataflow)
    b.run_persistent(10, 5)
    torch.cuda.synchronize()
    assert not b.barrier_timed_out()
    _assert_same(_fields(a), _fields(b))
    assert a.stable() and b.stable()
    a.close()
    b.close()


def test_persistent_launch_as_graph_replays():
    """Two remap cycles as one persistent launch (dataflow schedule)
    captured in a CUDA graph, replayed twice: 20 steps, bit-identical to
    eager stepping."""
    a = Ensemble(members(), 'mixed', nstreams=3)
    b = Ensemble(members(), 'mixed', nstreams=3)
    a.step_eager(20)
    b.set_schedule(True)
    b.capture_persistent(5, cycles=2)
    b.replay(2)
    torch.cuda.synchronize()
    assert b.steps_done == 20
    assert not b.barrier_timed_out()
    _assert_same(_fields(a), _fields(b))
    a.close()
    b.close()


def test_autotune_keeps_the_state():
    """The strip-height autotuner times trial launches and restores every
    member's state afterwards."""
    b = Ensemble(members(), 'mixed', nstreams=3)
    before = _fields(b)
    table = b.autotune(steps=2, reps=1)
    assert set(table) == {st.nx for st in b.members} and set(table.values()) <= {16, 32, 64}
    _assert_same(before, _fields(b))
    b.close()


def test_persistent_barrier_wait_runs_out():
    """The grid barrier's wait is bounded: a launch whose barrier waits for
    one block more than the grid holds ends with the timeout status instead
    of hanging, and the device keeps working."""
    import ctypes
    from atmdyn import load
    lib = load()
    out = ctypes.c_int(0)
    assert lib.atm_ensemble_barrier_check(5_000_000, ctypes.byref(out)) == 0
    assert out.value == 1
    a = Ensemble(members()[:2], 'mixed', nstreams=1)
    a.run_persistent(5, 5)
    assert not a.barrier_timed_out() and a.stable()
    a.close()


def test_persistent_stage_profile():
    """Per-stage timing of a persistent launch: every stage that ran has a
    positive time, the remap stages run only on remap steps, and the stages
    add up to about the launch's own duration."""
    b = Ensemble(members(), 'mixed', nstreams=1)
    b.run_persistent(2, 0)
    b.profile_persistent(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    b.run_persistent(4, 0)  # no remap
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    st = b.persistent_stage_ms()
    assert all(st[s] > 0 for s in st if not s.startswith('remap'))
    assert all(st[s] == 0 for s in ('remap_ring', 'remap_winds', 'remap_energy'))
    assert 0.5 * ms < sum(st.values()) <= 1.05 * ms + 0.05
    b.close()


def test_dataflow_odd_step_counts():
    """The dataflow schedule's phase arithmetic: a launch whose remap cycle
    does not divide its step count (7 steps, remap every 3: remaps after
    steps 3 and 6, none after step 7) and a launch without remap, bit-
    identical to eager stepping."""
    a = Ensemble(members(), 'mixed', nstreams=3)
    b = Ensemble(members(), 'mixed', nstreams=3)
    for n in range(1, 9):
        for st, d in zip(a.members, a.dyn):
            d.step(st.dt, remap=(n <= 7 and n % 3 == 0), check_stable=False)
    b.set_schedule(True)
    b.run_persistent(7, 3)  # 7 steps and 2 remaps: 9 swaps of the time levels
    b.run_persistent(1, 0)  # one step more: 10 swaps
    torch.cuda.synchronize()
    assert not b.barrier_timed_out()
    _assert_same(_fields(a), _fields(b))
    a.close()
    b.close()
