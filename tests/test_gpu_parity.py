"""Parity of the CUDA library's FP64 form with the CPU oracle.

The FP64 form evaluates the same IEEE operations in the same order as the
oracle (no fused multiply-add on either side, the same portable pow/log),
so every comparison here is bit-exact: max |difference| == 0.
"""
import numpy as np
import pytest

from atmdyn import ic, model, Dycore, device_pow_log
import pyoracle

pytestmark = pytest.mark.gpu

HALO = 7
KAPPA = ic.KAPPA


def _bubble(n=24, m=None, L=8, **kw):
    m = m or n
    return ic.bubble_case(n, m, L, 50e3 * 128 / n, 50e3 * 128 / n, radius=500e3 * n / 128 * 2, **kw)


def _jet(n=32, m=None, L=10, seed=0):
    m = m or n
    return ic.jet_case(n, m, L, 25e3 * 1024 / n / 4, 25e3 * 1024 / n / 4, width=500e3 * n / 256, seed=seed)


def _assert_same(a, b, what):
    d = np.abs(a - b)
    bad = ~(d == 0) & ~(np.isnan(a) & np.isnan(b))
    if bad.any():
        idx = np.argwhere(bad)[0]
        raise AssertionError('%s differs at %s: %r vs %r (max %g, %d points)' % (
            what, tuple(idx), a[tuple(idx)], b[tuple(idx)], np.nanmax(d), bad.sum()))


def test_device_pow_log_bit_identical_to_host():
    rng = np.random.default_rng(0)
    x = np.concatenate([np.exp(rng.uniform(np.log(1e2), np.log(2e5), 50000)),
                        rng.uniform(0.5, 1.5, 50000), [1.0, 2.0, 1e-300, 1e300]])
    p_dev, l_dev = device_pow_log(x, KAPPA)
    _assert_same(p_dev, pyoracle.pow_array(x, KAPPA), 'pow')
    _assert_same(l_dev, pyoracle.log_array(x), 'log')


@pytest.mark.parametrize('case', ['bubble', 'jet', 'ragged'])
def test_cgrid_step_bit_exact(case):
    st = {'bubble': _bubble(), 'jet': _jet(), 'ragged': _bubble(37, 23, 7)}[case]
    dt = st.dt
    g = Dycore(st)
    o = pyoracle.OracleModel(st)
    for a in (g, o):
        a.cgrid_step(dt / 2)
    nx, ny = st.nx, st.ny
    sl2 = (slice(None), slice(HALO - 2, HALO + ny + 2), slice(HALO - 2, HALO + nx + 2))
    sl0 = (slice(None), slice(HALO, HALO + ny), slice(HALO, HALO + nx))
    _assert_same(g.get('dpc', halo=True)[sl2], o.get(pyoracle.DPC, halo=True)[sl2], 'dpc')
    _assert_same(g.get('ptc', halo=True)[sl2], o.get(pyoracle.PTC, halo=True)[sl2], 'ptc')
    _assert_same(g.get('uc', halo=True)[sl0], o.get(pyoracle.UC, halo=True)[sl0], 'uc')
    _assert_same(g.get('vc', halo=True)[sl0], o.get(pyoracle.VC, halo=True)[sl0], 'vc')
    for a in (g, o):
        a.cgrid_halo()
    for name, f in (('dpc', pyoracle.DPC), ('ptc', pyoracle.PTC), ('uc', pyoracle.UC), ('vc', pyoracle.VC)):
        _assert_same(g.get(name, halo=True), o.get(f, halo=True), name + ' after halo')


@pytest.mark.parametrize('case', ['bubble', 'jet', 'ragged'])
def test_dgrid_step_and_remap_bit_exact(case):
    st = {'bubble': _bubble(), 'jet': _jet(), 'ragged': _bubble(37, 23, 7)}[case]
    dt = st.dt
    g = Dycore(st)
    o = pyoracle.OracleModel(st)
    for a in (g, o):
        a.cgrid_step(dt / 2)
        a.cgrid_halo()
        a.dgrid_step(dt)
    # the whole arrays, halo included, as the reference leaves them
    for name, f in (('dp', pyoracle.DP), ('pt', pyoracle.PT), ('ud', pyoracle.UD), ('vd', pyoracle.VD)):
        _assert_same(g.get(name, halo=True), o.get(f, halo=True), name + ' after D step')
    trace_o = o.enable_trace()
    trace_g, fallback = g.remap_trace()
    for a in (g, o):
        a.remap()
    for name, f in (('dp', pyoracle.DP), ('pt', pyoracle.PT), ('ud', pyoracle.UD), ('vd', pyoracle.VD)):
        _assert_same(g.get(name, halo=True), o.get(f, halo=True), name + ' after remap')
    np.testing.assert_array_equal(trace_g, trace_o)
    for a in (g, o):
        a.dgrid_halo()
    for name, f in (('dp', pyoracle.DP), ('pt', pyoracle.PT), ('ud', pyoracle.UD), ('vd', pyoracle.VD)):
        _assert_same(g.get(name, halo=True), o.get(f, halo=True), name + ' after halo')
    assert g.check_stability() and o.check_stability()


def test_bubble_100_steps_bit_exact_and_mass():
    """The bubble case with the reference's time loop, remap every 5 steps."""
    st = _bubble(32, 32, 10)
    tc = model.schedule_for(st.dt, 100, 5)
    g = Dycore(st)
    o = pyoracle.OracleModel(st, threads=4)
    m0 = g.mass()
    rg = model.run_model(g, tc)
    ro = model.run_model(o, tc)
    assert rg.stable and ro.stable and rg.steps == ro.steps == 100 and rg.remap_steps == ro.remap_steps
    for name, f in (('dp', pyoracle.DP), ('pt', pyoracle.PT), ('ud', pyoracle.UD), ('vd', pyoracle.VD)):
        _assert_same(g.get(name, halo=True), o.get(f, halo=True), name)
    assert abs(g.mass() - m0) / m0 <= 1e-13


def test_division_by_constants_is_ieee_division():
    import ctypes
    from atmdyn import load
    lib = load()
    bad = ctypes.c_longlong(-1)
    assert lib.atm_device_div_check(400_000_000, 12345, ctypes.byref(bad)) == 0
    assert bad.value == 0


def _ridged(nx=24, ny=20, L=8, layer=3):
    """A state whose face-interpolated interface pressures are not monotone:
    in one layer the thickness alternates thin, thin, thick, thick along y
    (and along x), so that at some faces the outer pair of the (7/12, -1/12)
    interpolation (src/mod_remap.f90:84-100) outweighs the inner pair."""
    st = _bubble(nx, ny, L)
    thin, thick = 400.0, 9000.0
    jy = (np.arange(ny) % 4)[:, None]
    ix = (np.arange(nx) % 4)[None, :]
    pat = np.where((jy == 1) | (jy == 2), thin, thick) * 0.5 + np.where((ix == 1) | (ix == 2), thin, thick) * 0.5
    st.dp = st.dp.copy()
    st.dp[layer] = pat
    st.u = st.u + 0.5 * np.sin(np.arange(nx) * 0.7)[None, None, :]
    st.v = st.v + 0.3 * np.cos(np.arange(ny) * 0.9)[None, :, None]
    return st


def test_remap_all_pairs_branch_bit_exact():
    """Columns with non-monotone coordinates take the reference's all-pairs
    loop (src/mod_remap.f90:176-283); the forward result and the (k, m,
    case) sets match the oracle there too."""
    st = _ridged()
    g = Dycore(st)
    o = pyoracle.OracleModel(st)
    trace_o = o.enable_trace()
    trace_g, fallback = g.remap_trace()
    for a in (g, o):
        a.remap()
    assert fallback.value > 0, 'no column took the all-pairs branch'
    for name, f in (('dp', pyoracle.DP), ('pt', pyoracle.PT), ('ud', pyoracle.UD), ('vd', pyoracle.VD)):
        _assert_same(g.get(name, halo=True), o.get(f, halo=True), name + ' after remap')
    np.testing.assert_array_equal(trace_g, trace_o)
    g.close()
