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


def _remap_state(kind, nlay):
    if kind == 'ridged':  # some face coordinates not monotone: the sequential all-pairs path
        st = ic.bubble_case(24, 20, nlay, 266e3, 266e3, radius=200e3)
        pat = (np.where(np.isin(np.arange(st.ny) % 4, (1, 2)), 400.0, 9000.0)[:, None] * 0.5 +
               np.where(np.isin(np.arange(st.nx) % 4, (1, 2)), 400.0, 9000.0)[None, :] * 0.5)
        st.dp = st.dp.copy()
        st.dp[3] = pat
        return st
    st = ic.jet_case(48, 40, nlay, 100e3, 100e3, width=600e3, seed=3)
    rng = np.random.default_rng(nlay)
    st.dp = st.dp * (1 + rng.uniform(-0.3, 0.3, st.dp.shape))  # source and target interfaces apart
    st.pt = st.pt * (1 + rng.normal(0, 1e-3, st.pt.shape))
    st.v = st.v + rng.normal(0, 1.0, st.v.shape)
    return st


@pytest.mark.parametrize('kind,nlay', [('jet', 20), ('jet', 64), ('jet', 100), ('ridged', 8)])
def test_warp_remap_matches_sequential_remap(kind, nlay):
    """The mixed form remaps with the warp-cooperative kernels (one warp per
    column, scans with shuffles); the FP64 form with the sequential ones.
    On the same FP64 state one remap of each agrees to rounding: the sums
    are associated differently."""
    st = _remap_state(kind, nlay)
    out = {}
    for form in ('fp64', 'mixed'):
        g = Dycore(st, form)
        g.remap()
        assert g.check_stability()
        out[form] = {f: g.get(f, halo=True) for f in ('dp', 'pt', 'ud', 'vd')}
        g.close()
    for f in ('dp', 'pt', 'ud', 'vd'):
        a, b = out['fp64'][f], out['mixed'][f]
        rel = np.abs(a - b).max() / np.abs(a).max()
        assert rel <= 1e-11, (f, rel)
