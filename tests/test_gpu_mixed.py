"""The mixed form (FP32 sweeps on an FP64 state) against the FP64 form.

* Total mass: the sweeps' tendencies are applied in flux form to the FP64
  state, so sum(dp) telescopes and changes only by FP64 round-off.
* Error: after 50 steps of a 256 x 256 x 32 jet (dt 30 s, remap every 8)
  the relative L2 errors of dp, pt and ud against the FP64 form stay far
  below 1e-5, and vd (whose norm is the small perturbation of a zonal jet)
  below 1e-4.
* The mixed form is stable and deterministic: the same run twice is bit
  for bit the same.
"""
import numpy as np
import pytest

from atmdyn import ic, Dycore

pytestmark = pytest.mark.gpu


def jet():
    st = ic.jet_case(256, 256, 32, 25e3, 25e3, seed=1)
    st.dt = 30.0
    return st


def run(precision, nsteps=50, remap_every=8):
    st = jet()
    g = Dycore(st, precision)
    m0 = g.mass()
    for n in range(1, nsteps + 1):
        assert g.step(st.dt, remap=n % remap_every == 0, check_stable=True)
    out = {f: g.get(f) for f in ('dp', 'pt', 'ud', 'vd')}
    out['mass_change'] = (g.mass() - m0) / m0
    g.close()
    return out


def test_mixed_form_mass_and_error_against_fp64():
    a = run('fp64')
    b = run('mixed')
    assert abs(b['mass_change']) < 1e-13
    assert abs(a['mass_change']) < 1e-13
    rel = {f: np.linalg.norm(b[f] - a[f]) / np.linalg.norm(a[f]) for f in ('dp', 'pt', 'ud', 'vd')}
    assert rel['dp'] < 1e-7 and rel['pt'] < 1e-7 and rel['ud'] < 1e-5, rel
    assert rel['vd'] < 1e-4, rel
    assert rel['ud'] > 0  # the sweeps did run in FP32


def test_mixed_form_is_deterministic():
    a = run('mixed', nsteps=12)
    b = run('mixed', nsteps=12)
    for f in ('dp', 'pt', 'ud', 'vd'):
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)

