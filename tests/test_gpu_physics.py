"""The column physics (src/mod_physics.f90) on the GPU against the FP64
restatement, bit for bit: tendencies and their application, the surface
heating from a net flux, the ts halo, whole steps with the physics in the
time loop, and the ts output mean."""
import numpy as np
import pytest

from atmdyn import ic, Dycore, model
import pyoracle

pytestmark = pytest.mark.gpu

H = 7
ORC = {'dp': pyoracle.DP, 'pt': pyoracle.PT, 'ud': pyoracle.UD, 'vd': pyoracle.VD, 'ts': pyoracle.TS}


def unstable_state(nx=40, ny=24, nlay=10, seed=11):
    """A bubble with noisy winds, thickness and potential temperature, so
    that some interfaces mix (Richardson number below 1/4) and others
    do not, and a noisy surface temperature."""
    st = ic.bubble_case(nx, ny, nlay, 100e3, 100e3, seed=seed)
    rng = np.random.default_rng(seed)
    st.u = st.u + rng.normal(0, 3.0, st.u.shape)
    st.v = st.v + rng.normal(0, 3.0, st.v.shape)
    st.pt = st.pt * (1 + rng.normal(0, 3e-3, st.pt.shape))
    st.dp = st.dp + rng.normal(0, 20.0, st.dp.shape)
    st.ts = 288.0 + rng.normal(0, 2.0, (ny, nx))
    return st


def assert_same(g, o, names=('dp', 'pt', 'ud', 'vd', 'ts')):
    for n in names:
        a = g.get(n, halo=True)
        b = o.get(ORC[n], halo=True)
        np.testing.assert_array_equal(a, b, err_msg=n)


def test_tendencies_and_application_bit_exact():
    st = unstable_state()
    g, o = Dycore(st), pyoracle.OracleModel(st)
    assert_same(g, o)
    before = g.get('ud')
    for dyn in (g, o):
        dyn.physics_tendencies()
        dyn.apply_physics(st.dt)
    assert np.max(np.abs(g.get('ud') - before)) > 1e-4  # some columns mixed
    assert_same(g, o)


def test_surface_heating_and_ts_halo_bit_exact():
    st = unstable_state(seed=12)
    g, o = Dycore(st), pyoracle.OracleModel(st)
    rng = np.random.default_rng(3)
    nf = np.zeros((st.nlay + 1, st.ny + 2 * H, st.nx + 2 * H))
    nf[0] = rng.normal(0, 150.0, nf[0].shape)
    g.set_net_flux(nf)
    o.set_net_flux(nf)
    for dyn in (g, o):
        dyn.physics_tendencies()
        dyn.apply_physics(90.0)
        dyn.physics_halo()
    assert_same(g, o)


def test_apply_before_tendencies_is_an_error():
    st = unstable_state(16, 16, 4)
    g = Dycore(st)
    with pytest.raises(Exception):
        g.apply_physics(st.dt)


@pytest.mark.parametrize('dt_physics_steps', [1, 3])
def test_steps_with_physics_bit_exact(dt_physics_steps):
    """run_model with the physics due every dt_physics_steps steps and the
    remap every 4: C half step, halo, D step, physics applied, remap, halo,
    ts halo, as src/mod_model.f90:138-166."""
    st = unstable_state(seed=13)
    st.dt = 60.0
    tc = model.TimeControl(dt_max=st.dt, run_duration=8 * st.dt, dt_physics=dt_physics_steps * st.dt,
                           dt_remap=4 * st.dt)
    g, o = Dycore(st), pyoracle.OracleModel(st)
    rg = model.run_model(g, tc, physics=True)
    ro = model.run_model(o, tc, physics=True)
    assert rg.steps == ro.steps == 8 and rg.remap_steps == ro.remap_steps == [4, 8]
    assert_same(g, o)


def test_mixed_form_physics_is_fp64():
    """The prognostic state is FP64 in both forms and the physics runs in
    FP64: on the same state the mixed form's tendencies are the FP64 ones."""
    st = unstable_state(seed=14)
    g64, gmx = Dycore(st), Dycore(st, 'mixed')
    for dyn in (g64, gmx):
        dyn.physics_tendencies()
        dyn.apply_physics(st.dt)
    for n in ('dp', 'pt', 'ud', 'vd', 'ts'):
        np.testing.assert_array_equal(g64.get(n, halo=True), gmx.get(n, halo=True), err_msg=n)


def test_ts_output_mean():
    """accumulate_output adds dt * ts (src/mod_output.f90:101); the mean is
    the plain FP64 sum divided by the accumulated time."""
    st = unstable_state(seed=15)
    g = Dycore(st)
    rng = np.random.default_rng(4)
    nf = np.zeros((st.nlay + 1, st.ny + 2 * H, st.nx + 2 * H))
    nf[0] = rng.normal(0, 150.0, nf[0].shape)
    g.set_net_flux(nf)
    g.output_enable()
    acc, t = 0., 0.
    g.physics_tendencies()
    for dt in (60.0, 45.0, 60.0):
        g.apply_physics(dt)
        g.physics_halo()
        g.accumulate_output(dt)
        acc = acc + dt * g.get('ts')[0]
        t = t + dt
    np.testing.assert_array_equal(g.output_read('ts')[0], acc / t)
