"""The radiation (src/mod_radiation.f90) on the GPU against the FP64
restatement, bit for bit: net fluxes of one call at three layer counts
(the kernel's 32-, 64- and 128-level instances) on the reference's tables
and on synthetic ones, with noisy surface temperatures and cell axes off
the origin; both forms; the net-flux halo; the table-range stop and the
context after it; whole runs with radiation and physics in the time
loop; and sampled columns of the benchmark's 1024 x 1024 x 64 domain."""
import numpy as np
import pytest

from atmdyn import ic, Dycore, model, gas_optics
from atmdyn._lib import AtmError
import pyoracle

pytestmark = pytest.mark.gpu

H = 7


def tables():
    out = [('synthetic', gas_optics.synthetic(3))]
    go = gas_optics.load_default()
    if go is not None:
        out.append(('reference', go))
    return out


def radiative_state(nx, ny, nlay, seed=0):
    st = ic.bubble_case(nx, ny, nlay, 100e3, 100e3, seed=seed)
    rng = np.random.default_rng(seed)
    st.pt = st.pt * (1 + rng.normal(0, 2e-3, st.pt.shape))
    st.dp = st.dp * (1 + rng.normal(0, 2e-3, st.dp.shape))
    st.ts = 288.0 + rng.normal(0, 3.0, (ny, nx))
    return st


def oracle_flux(st, go, dy, xc, yc):
    return pyoracle.radiative_heating(go, dy.get('dp'), dy.get('pt'), dy.get('ts')[0], xc, yc, st.ak[0],
                                      st.gravity, threads=8)


@pytest.mark.parametrize('nlay', [20, 48, 100])
@pytest.mark.parametrize('which', ['synthetic', 'reference'])
def test_net_flux_bit_exact(nlay, which):
    found = dict(tables())
    if which not in found:
        pytest.skip('no extracted gas-optics tables')
    go = found[which]
    st = radiative_state(24, 20, nlay, seed=nlay)
    xc, yc = ic.cell_axes(st)
    xc = xc + 3.0e5  # off-centre, so the irradiance varies over the domain
    dy = Dycore(st)
    dy.set_radiation(go, xc, yc)
    dy.radiative_heating(0.0)
    got = dy.get('net_flux')
    want = oracle_flux(st, go, dy, xc, yc)
    np.testing.assert_array_equal(got, want)
    assert np.all(np.isfinite(got))
    dy.close()


def test_mixed_form_and_parameters():
    """The radiation is FP64 in the mixed form too (its state is FP64);
    non-default zenith angle, albedo and emissivity."""
    go = tables()[-1][1]
    st = radiative_state(20, 16, 30, seed=5)
    xc, yc = ic.cell_axes(st)
    dy = Dycore(st, 'mixed')
    dy.set_radiation(go, xc, yc)
    dy.radiative_heating(3600.0, solar_zenith_angle=0.6, surface_albedo=0.12, surface_emissivity=0.95)
    want = pyoracle.radiative_heating(go, dy.get('dp'), dy.get('pt'), dy.get('ts')[0], xc, yc, st.ak[0],
                                      st.gravity, solar_zenith_angle=0.6, surface_albedo=0.12,
                                      surface_emissivity=0.95)
    np.testing.assert_array_equal(dy.get('net_flux'), want)
    dy.close()


def test_halo_and_range_stop():
    """radiation_halo_exchange makes the halo the periodic image; a surface
    temperature above the Planck table gives ATM_ERR_RANGE (where the
    reference stops) and leaves the context usable."""
    go = tables()[-1][1]
    st = radiative_state(16, 12, 20, seed=7)
    dy = Dycore(st)
    dy.set_radiation(go)
    dy.radiative_heating()
    dy.radiation_halo()
    nf = dy.get('net_flux', halo=True)
    np.testing.assert_array_equal(nf, pyoracle.periodic_halo(nf[:, H:-H, H:-H]))
    hot = np.pad(np.full((1, st.ny, st.nx), 1000.0), ((0, 0), (H, H), (H, H)))
    dy.upload('ts', hot)
    with pytest.raises(AtmError, match='outside the gas-optics tables'):
        dy.radiative_heating()
    dy.upload('ts', np.pad(st.ts[None], ((0, 0), (H, H), (H, H))))
    dy.radiative_heating()
    assert dy.check_stability()
    dy.close()


@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
def test_run_with_radiation_and_physics(precision):
    """run_model with radiation every 4 steps, physics every 2, remap every
    5: the FP64 form bit-identical to the oracle after 12 steps; the mixed
    form within its sweep tolerance (its radiation is FP64 and its heating
    term follows the same net flux)."""
    go = tables()[-1][1]
    st = radiative_state(32, 24, 20, seed=9)
    dt = 60.0
    tc = model.TimeControl(dt_max=dt, run_duration=12 * dt, dt_radiation=4 * dt, dt_physics=2 * dt,
                           dt_remap=5 * dt)
    g = Dycore(st, precision)
    o = pyoracle.OracleModel(st, threads=8)
    xc, yc = ic.cell_axes(st)
    g.set_radiation(go, xc, yc)
    o.set_radiation(go, xc, yc)
    calls = []
    orig = g.radiative_heating

    def counted(time=0.0, **kw):
        calls.append(time)
        return orig(time, **kw)
    g.radiative_heating = counted
    rg = model.run_model(g, tc, physics=True, radiation=True)
    ro = model.run_model(o, tc, physics=True, radiation=True)
    assert rg.steps == ro.steps == 12 and rg.stable and ro.stable
    assert calls == [0.0, 4 * dt, 8 * dt]
    names = (('dp', pyoracle.DP), ('pt', pyoracle.PT), ('ud', pyoracle.UD), ('vd', pyoracle.VD),
             ('ts', pyoracle.TS), ('net_flux', pyoracle.NET_FLUX))
    for n, f in names:
        a, b = g.get(n), o.get(f)
        if precision == 'fp64':
            np.testing.assert_array_equal(a, b, err_msg=n)
        else:
            assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b), n
    g.close()


def test_full_size_sampled_columns():
    """At the benchmark's size (jet 1024 x 1024 x 64, the reference's tables
    when present): the net flux of 8 x 8 sampled columns (a sub-grid of the
    domain, so that their cell axes are a subset of the domain's) is
    bit-identical to the oracle's on the same columns."""
    go = tables()[-1][1]
    st = ic.jet_case(1024, 1024, 64, 25e3, 25e3, seed=0)
    rng = np.random.default_rng(5)
    st.ts = 288.0 + rng.normal(0, 2.0, (st.ny, st.nx))
    xc, yc = ic.cell_axes(st)
    dy = Dycore(st)
    dy.set_radiation(go, xc, yc)
    dy.radiative_heating()
    nf = dy.get('net_flux')
    ii = np.sort(rng.choice(st.nx, 8, replace=False))
    jj = np.sort(rng.choice(st.ny, 8, replace=False))
    dp, pt, ts = dy.get('dp'), dy.get('pt'), dy.get('ts')[0]
    sub = np.ix_(jj, ii)
    want = pyoracle.radiative_heating(go, dp[:, sub[0], sub[1]], pt[:, sub[0], sub[1]], ts[sub], xc[ii], yc[jj],
                                      st.ak[0], st.gravity)
    np.testing.assert_array_equal(nf[:, sub[0], sub[1]], want)
    dy.close()
