"""The mass sweeps run one block per strip of sub-tiles in y and keep the
stencil rows neighbouring sub-tiles share instead of recomputing them.  A
kept row is the row a fresh tile computes from the same inputs, so the
fields cannot depend on the strip length: every strip length, ragged last
strips included, gives the same fields bit for bit, in both forms (the
mixed form has no oracle of its own; this is its check of the strips).
"""
import numpy as np
import pytest

from atmdyn import ic, Dycore, subtiles

pytestmark = pytest.mark.gpu


def _run(precision, strip, nsteps=6):
    # 70 x 45: tiles of 32 columns leave a ragged last column of tiles, and
    # no strip length below divides the rows evenly
    st = ic.jet_case(70, 45, 8, 25e3 * 1024 / 70 / 4, 25e3 * 1024 / 70 / 4, width=500e3 * 70 / 256, seed=5)
    st.dt = 30.0
    g = Dycore(st, precision)
    with subtiles(strip):
        for n in range(1, nsteps + 1):
            assert g.step(st.dt, remap=n % 3 == 0, check_stable=True)
    out = {f: g.get(f, halo=True) for f in ('dp', 'pt', 'ud', 'vd')}
    g.close()
    return out


@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
def test_fields_do_not_depend_on_strip_length(precision):
    ref = _run(precision, 1)
    for strip in (2, 3, 5, 16):
        got = _run(precision, strip)
        for f in ref:
            np.testing.assert_array_equal(got[f], ref[f], err_msg='%s, %d sub-tiles per strip' % (f, strip))
