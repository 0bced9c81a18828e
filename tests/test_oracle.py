"""Known-answer tests of the CPU oracle (the FP64 restatement of the
reference's dycore).  The reference has no tests or golden data, so these
analytic properties pin the restatement."""
import math

import numpy as np
import pytest

from atmdyn import ic, model
import pyoracle

HALO = 7
KAPPA = ic.KAPPA


def _rest_state(n=16, L=6):
    st = ic.bubble_case(n, n, L, 100e3, 100e3, amplitude=0.0, u0=0.0)
    # horizontally uniform layers at the target grid, so the remap target
    # equals the source grid
    return st


def _run_step(o, dt, remap=True):
    o.cgrid_step(dt / 2.)
    o.cgrid_halo()
    o.dgrid_step(dt)
    if remap:
        o.remap()
    o.dgrid_halo()


def test_resting_uniform_atmosphere_is_steady_bit_for_bit():
    st = _rest_state()
    o = pyoracle.OracleModel(st)
    before = o.state()
    for _ in range(3):
        _run_step(o, st.dt, remap=False)
    after = o.state()
    for k in before:
        np.testing.assert_array_equal(before[k], after[k], err_msg=k)


def test_remap_onto_own_grid_is_identity():
    """dp equals the target grid, so every pair is case 5 with an
    integral factor of exactly one (src/mod_remap.f90:255-260)."""
    st = ic.bubble_case(12, 10, 7, 100e3, 100e3, amplitude=1.0, radius=300e3)
    st.u = st.u + np.random.default_rng(1).normal(0, 1, st.u.shape)
    o = pyoracle.OracleModel(st)
    before = o.state()
    trace = o.enable_trace()
    o.remap()
    after = o.state()
    np.testing.assert_array_equal(before['dp'], after['dp'])
    np.testing.assert_array_equal(before['ud'], after['ud'])
    np.testing.assert_array_equal(before['vd'], after['vd'])
    rel = np.abs(after['pt'] - before['pt']) / np.abs(before['pt'])
    assert rel.max() < 1e-13
    # every destination layer gets exactly its own source layer, case 5
    t = trace[0, 1:-1, 1:-1]
    L = st.nlay
    np.testing.assert_array_equal(t[..., 0], np.broadcast_to(np.arange(1, L + 1), t.shape[:-1]))
    np.testing.assert_array_equal(t[..., 1], t[..., 0])
    assert (t[..., 2] == 5).all() and (t[..., 4] == 1).all()


def test_halo_fill_is_periodic_wrap():
    st = ic.jet_case(20, 14, 4, 50e3, 50e3, width=200e3, seed=3)
    o = pyoracle.OracleModel(st)
    for f in (pyoracle.DP, pyoracle.PT, pyoracle.UD, pyoracle.VD):
        a = o.get(f, halo=True)
        inner = a[:, HALO:-HALO, HALO:-HALO]
        wrapped = np.pad(inner, ((0, 0), (HALO, HALO), (HALO, HALO)), mode='wrap')
        np.testing.assert_array_equal(a, wrapped)


def test_mass_conserved_and_serial_equals_threads_and_checked_build():
    st = ic.bubble_case(24, 20, 6, 200e3, 200e3, radius=800e3)
    tc = model.schedule_for(st.dt, 12, 5)
    runs = {}
    for name, kw in (('serial', {}), ('threads', {'threads': 4}),
                     ('checked', {'variant': 'checked', 'poison': True})):
        o = pyoracle.OracleModel(st, **kw)
        m0 = math.fsum(o.get(pyoracle.DP).ravel())
        r = model.run_model(o, tc)
        assert r.stable and r.steps == 12 and r.remap_steps == [5, 10]
        m1 = math.fsum(o.get(pyoracle.DP).ravel())
        assert abs(m1 - m0) / m0 < 1e-13
        runs[name] = o.state()
    for k in runs['serial']:
        np.testing.assert_array_equal(runs['serial'][k], runs['threads'][k], err_msg=k)
        np.testing.assert_array_equal(runs['serial'][k], runs['checked'][k], err_msg=k)


def test_portable_pow_log_accuracy():
    from decimal import Decimal, getcontext
    getcontext().prec = 40
    rng = np.random.default_rng(0)
    x = np.exp(rng.uniform(np.log(1e2), np.log(2e5), 2000))
    p = pyoracle.pow_array(x, KAPPA)
    kd = Decimal(KAPPA)
    worst = 0.0
    for xi, pi in zip(x, p):
        t = (kd * Decimal(xi).ln()).exp()
        worst = max(worst, float(abs((Decimal(pi) - t) / Decimal(float(np.spacing(pi))))))
    assert worst < 0.52
    y = rng.uniform(0.5, 1.5, 2000)
    lg = pyoracle.log_array(y)
    worst = 0.0
    for yi, li in zip(y, lg):
        t = Decimal(yi).ln()
        worst = max(worst, float(abs((Decimal(li) - t) / Decimal(float(np.spacing(abs(li)))))))
    assert worst < 0.51
    # within one ulp of the C library everywhere
    glibc = pyoracle.pow_array(x, KAPPA, variant='libm')
    assert (np.abs(p - glibc) <= np.spacing(glibc)).all()


def test_literals_and_constants():
    assert ic.R_DRY == float(np.float32(287.052874))
    assert ic.KAPPA == ic.R_DRY / 1005.0


# ------------------------------------------------------------- physics ----
def physics_state(n=12, L=8, seed=3, unstable=True):
    """Horizontally uniform layers (so the D-grid interpolation of a wind
    tendency is the tendency itself) with sheared winds, and, when
    unstable, potential temperature falling with height across layers 3-5."""
    st = ic.bubble_case(n, n, L, 100e3, 100e3, amplitude=0.0, u0=0.0)
    shear = np.linspace(-4.0, 6.0, L)[:, None, None]
    st.u = np.broadcast_to(shear, st.u.shape).copy()
    st.v = np.broadcast_to(-0.5 * shear, st.v.shape).copy()
    if unstable:
        st.pt = st.pt.copy()
        st.pt[3] = st.pt[2] * (1 - 2e-3)
        st.pt[4] = st.pt[2] * (1 - 4e-3)
    st.ts = np.full((n, n), 288.0)
    return st


def test_physics_stable_column_leaves_winds_and_theta():
    """Stable stratification with weak shear: no interface mixes, the wind
    tendencies are exactly zero and theta only moves by the round-off of
    its recovery from the energy (mod_physics.f90:146-166)."""
    st = physics_state(unstable=False)
    st.u = np.zeros_like(st.u)
    st.v = np.zeros_like(st.v)
    o = pyoracle.OracleModel(st)
    before = o.state()
    o.physics_tendencies()
    o.apply_physics(600.0)
    after = o.state()
    np.testing.assert_array_equal(after['ud'], before['ud'])
    np.testing.assert_array_equal(after['vd'], before['vd'])
    np.testing.assert_array_equal(after['dp'], before['dp'])
    assert np.max(np.abs(after['pt'] / before['pt'] - 1)) < 1e-12
    np.testing.assert_array_equal(o.get(pyoracle.TS), 288.0)


def test_physics_mixing_conserves_column_momentum():
    """The exchange of mod_physics.f90:111-133 moves momentum between
    layers k and k+1 in proportion to 1/dp, so sum(dp * du) over a column
    vanishes."""
    st = physics_state()
    o = pyoracle.OracleModel(st)
    before = o.state()
    o.physics_tendencies()
    o.apply_physics(600.0)  # one mixing timescale
    after = o.state()
    dp = before['dp']
    du = after['ud'] - before['ud']
    dv = after['vd'] - before['vd']
    assert np.max(np.abs(du)) > 1e-3  # the unstable band mixed
    scale = np.sum(dp * np.abs(du), axis=0)
    assert np.max(np.abs(np.sum(dp * du, axis=0)) / scale) < 1e-12
    assert np.max(np.abs(np.sum(dp * dv, axis=0)) / np.sum(dp * np.abs(dv), axis=0)) < 1e-12
    assert np.max(np.abs(du[3:5])) > 1e-3  # the layers around the unstable interfaces


def test_physics_surface_heating_and_ts_halo():
    """ts_tend = net_flux(level 1) / 208400 (mod_physics.f90:178-185) on the
    interior; physics_halo_exchange makes the halo the periodic image."""
    st = physics_state(unstable=False)
    o = pyoracle.OracleModel(st)
    rng = np.random.default_rng(1)
    nf = np.zeros((st.nlay + 1, st.ny + 2 * HALO, st.nx + 2 * HALO))
    nf[0] = rng.normal(0, 100.0, nf[0].shape)
    o.set_net_flux(nf)
    o.physics_tendencies()
    o.apply_physics(120.0)
    ts = o.get(pyoracle.TS)[0]
    np.testing.assert_array_equal(ts, 288.0 + 120.0 * (nf[0, HALO:-HALO, HALO:-HALO] / 208400.0))
    o.physics_halo()
    th = o.get(pyoracle.TS, halo=True)[0]
    np.testing.assert_array_equal(th[:HALO, HALO:-HALO], th[st.ny:st.ny + HALO, HALO:-HALO])
    np.testing.assert_array_equal(th[HALO:-HALO, :HALO], th[HALO:-HALO, st.nx:st.nx + HALO])
    np.testing.assert_array_equal(th[:HALO, :HALO], th[st.ny:st.ny + HALO, st.nx:st.nx + HALO])
