"""The radiation oracle (src/mod_radiation.f90) pinned on the CPU: the
table reader against a Fortran snippet, the reference's own tables (when
the package build extracted them), closed forms of the two-stream and
adding equations for a purely absorbing shortwave and an isothermal
longwave atmosphere (written here from the mathematics, not from the
oracle's code), the table-range stop, and the distance between the
portable exp/log/pow and the C library's."""
import os

import numpy as np
import pytest

from atmdyn import gas_optics, ic
import pyoracle

KAPPA = ic.KAPPA
F32 = lambda x: float(np.float32(x))  # noqa: E731


def test_fortran_reader():
    """Default-real literals are rounded to single precision, d exponents
    and kind suffixes stay double; reshape order (t, p, g) -> [g][p][t];
    continuation lines and comments are skipped."""
    body = ['   real(rk), parameter :: pressures(n_pressures) = [ &',
            '      1.0e+00, 1.0e+05] ! Pa',
            '   real(rk), parameter :: &',
            '      temperatures(n_temperatures, n_pressures) = reshape( &',
            '      [1.0e2, 2.0e2, 1.5e2, 2.5e2], (/n_temperatures, n_pressures/))']
    for name in ('shortwave_absorption_lut', 'longwave_absorption_lut'):
        body += ['      real(rk), parameter :: &',
                 '         %s(n_temperatures, n_pressures, n_g_points) &' % name,
                 '         = reshape([0.1, 0.2, 0.3, 0.4, &',
                 '                    0.5d0, 0.6_rk, 0.7, 0.8], (/n_temperatures, n_pressures, n_g_points/))']
    body += ['      real(rk), parameter :: &',
             '         rayleigh_scattering_lut(n_g_points) = [ &',
             '         1.0e-5, 2.0e-5]',
             '      real(rk), parameter :: &',
             '         planckian_temperatures(n_planckian_temperatures) = [ &',
             '         1.0e2, 2.0e2, 3.0e2]',
             '      real(rk), parameter :: &',
             '         planckian_lut(n_planckian_temperatures, n_g_points) = reshape( &',
             '         [1., 2., 3., 4., 5., 6.], (/n_planckian_temperatures, n_g_points/))']
    solar = ('   real(rk), parameter :: irradiance_fraction(n_g_points) = &\n'
             '                          [0.3, 0.7]\n')
    go = gas_optics.from_fortran_text('\n'.join(body) + '\n', solar)
    assert go.sw_absorption.shape == (2, 2, 2) and go.planck.shape == (2, 3)
    assert go.sw_absorption[0, 0, 1] == F32(0.2) and go.sw_absorption[0, 1, 0] == F32(0.3)
    assert go.sw_absorption[1, 0, 0] == 0.5 and go.sw_absorption[1, 0, 1] == 0.6  # double literals
    assert go.temperatures[1, 1] == 250.0 and go.planck[1, 0] == 4.0
    assert go.irradiance_fraction[0] == F32(0.3)


def test_reference_tables_shapes():
    """The reference's tables as the package build extracted them: 16
    g-points, 53 pressures x 6 temperatures, 231 Planck temperatures,
    ascending axes, irradiance fractions summing to one."""
    go = gas_optics.load_default()
    if go is None:
        pytest.skip('no extracted gas-optics tables (the package build writes them from a reference checkout)')
    assert go.sw_absorption.shape == (16, 53, 6) and go.lw_absorption.shape == (16, 53, 6)
    assert go.planck.shape == (16, 231) and go.planck_temperatures.shape == (231,)
    assert abs(go.irradiance_fraction.sum() - 1.0) < 1e-6
    assert np.all(go.sw_absorption > 0) and np.all(go.lw_absorption > 0) and np.all(go.planck > 0)
    # every value is a widened single-precision literal
    for a in (go.pressures, go.temperatures, go.sw_absorption, go.lw_absorption, go.planck):
        np.testing.assert_array_equal(a, a.astype(np.float32).astype(np.float64))


# ---- closed forms --------------------------------------------------------------------------

def column_state(nx=3, ny=2, nlay=9, ptop=1.0e4, psurf=1.0e5, seed=0):
    """dp, pt with some noise, a potential temperature giving about 220-290 K."""
    rng = np.random.default_rng(seed)
    dp = np.full((nlay, ny, nx), (psurf - ptop) / nlay) * (1 + rng.uniform(-.2, .2, (nlay, ny, nx)))
    plev = ptop + np.cumsum(dp[::-1], axis=0)[::-1]
    t = 220.0 + 70.0 * (plev / psurf) ** 2 + rng.uniform(-3, 3, dp.shape)
    pt = t / plev ** KAPPA
    ts = 288.0 + rng.uniform(-2, 2, (ny, nx))
    xc = np.linspace(-1.5e6, 1.5e6, nx)
    yc = np.linspace(-4e5, 4e5, ny)
    return dp, pt, ts, xc, yc, ptop


def layer_properties(dp, ptop):
    """play, T_layer, T_level (1-based on the first axis) of
    calculate_radiative_heating (mod_radiation.f90:54-103), from the
    definitions: pkap = p**kappa, play = dp / ln(p_k / p_k+1), T = pt *
    layer-mean p**kappa, levels interpolated linearly in ln p."""
    nlay = dp.shape[0]
    plev = np.empty((nlay + 2,) + dp.shape[1:])
    plev[nlay + 1] = ptop
    for k in range(nlay, 0, -1):
        plev[k] = plev[k + 1] + dp[k - 1]
    pk = plev ** KAPPA
    lnr = np.log(plev[1:nlay + 1] / plev[2:nlay + 2])
    play = np.concatenate([np.zeros((1,) + dp.shape[1:]), dp / lnr])
    playkap = np.concatenate([np.zeros((1,) + dp.shape[1:]), (pk[2:nlay + 2] - pk[1:nlay + 1]) / (-lnr * KAPPA)])
    return plev, play, playkap


def temperatures(pt, plev, play, playkap):
    nlay = pt.shape[0]
    tl = np.concatenate([np.zeros((1,) + pt.shape[1:]), pt * playkap[1:]])
    lp = np.log(np.maximum(play, 1e-300))
    tv = np.empty((nlay + 2,) + pt.shape[1:])
    for k in range(1, nlay):
        lq = np.log(plev[k + 1])
        tv[k + 1] = (tl[k] * (lp[k + 1] - lq) + tl[k + 1] * (lq - lp[k])) / (lp[k + 1] - lp[k])
    lq = np.log(plev[nlay + 1])
    tv[nlay + 1] = (tl[nlay - 1] * (lp[nlay] - lq) + tl[nlay] * (lq - lp[nlay - 1])) / (lp[nlay] - lp[nlay - 1])
    lq = np.log(plev[1])
    tv[1] = (tl[1] * (lp[2] - lq) + tl[2] * (lq - lp[1])) / (lp[2] - lp[1])
    return tl, tv


def linear_tables(a_sw, a_lw, planck_slope, frac):
    """One g-point; absorption a + b p + c T, linear in both lookup axes, so
    any bilinear interpolation returns it; Planck function linear in T."""
    p = np.linspace(1.0, 1.2e5, 7)
    temps = np.tile(np.linspace(100.0, 400.0, 4), (7, 1)) + np.linspace(0, 10, 7)[:, None]

    def lin(a):
        return (a[0] + a[1] * p[:, None] + a[2] * temps)[None]
    pt_ = np.linspace(100.0, 400.0, 31)
    return gas_optics.GasOptics(p, temps, lin(a_sw), np.zeros(1), lin(a_lw), pt_,
                                (planck_slope * (pt_ - 50.0))[None], np.array([frac])).validate()


def kabs(a, play, tl):
    return a[0] + a[1] * play + a[2] * tl


def test_shortwave_pure_absorption_closed_form():
    """No scattering, no thermal emission: the direct beam decays as
    exp(-tau / mu0); the diffuse field has reflectance 0 and transmittance
    exp(-lambda tau) with the lambda of the direct-beam coefficients
    (gamma1 = 7/4, gamma2 = -1/4 at g = 0, mu0 = 1: sqrt(3)), which the
    reference reuses for the diffuse layer (mod_radiation.f90:254-260);
    the top diffuse input is the beam itself (:264), the beam is added to
    the downward flux (:266), and the surface reflects A of the diffuse
    flux that reaches it."""
    dp, pt, ts, xc, yc, ptop = column_state()
    g = 9.80665
    a = (2e-6, 1e-10, 3e-9)
    go = linear_tables(a, (1e-5, 0, 0), 0.0, 1.0)
    nf = pyoracle.radiative_heating(go, dp, pt, ts, xc, yc, ptop, g)
    plev, play, playkap = layer_properties(dp, ptop)
    tl, _ = temperatures(pt, plev, play, playkap)
    nlay = dp.shape[0]
    tau = np.concatenate([np.zeros((1,) + dp.shape[1:]), kabs(a, play[1:], tl[1:]) * dp / g])
    r = np.sqrt(xc[None, :] ** 2 + yc[:, None] ** 2)
    irr = 600 * (1 + F32(.2) / (1 + (r / 1e8) ** 2))
    lam = np.sqrt(1.75 ** 2 - .25 ** 2)
    A = F32(.3)
    beam = np.empty((nlay + 2,) + dp.shape[1:])
    fdn = np.empty_like(beam)
    beam[nlay + 1] = irr
    fdn[nlay + 1] = irr
    for k in range(nlay, 0, -1):
        beam[k] = np.exp(-tau[k]) * beam[k + 1]
        fdn[k] = np.exp(-lam * tau[k]) * fdn[k + 1]
    alb = np.empty_like(beam)
    alb[1] = A
    for k in range(1, nlay + 1):
        alb[k + 1] = np.exp(-lam * tau[k]) ** 2 * alb[k]
    want = (fdn + beam - alb * fdn)[1:]
    np.testing.assert_allclose(nf, want, rtol=1e-12, atol=1e-9)


def test_longwave_nonscattering_closed_form():
    """No sunlight: reflectance 0, transmittance exp(-2 tau) (gamma1 = 2,
    gamma2 = 0), sources pi (B_k+1 - T B_k + d) and pi (B_k - T B_k+1 - d)
    with d = (1 - T)(B_k - B_k+1) / (2 tau) for a Planck function linear in
    optical depth; surface emission eps pi B(ts), reflection 1 - eps."""
    dp, pt, ts, xc, yc, ptop = column_state(seed=4)
    g = 9.80665
    a = (3e-5, 2e-10, -4e-8)
    slope = 0.01
    go = linear_tables((1e-6, 0, 0), a, slope, 0.0)
    nf = pyoracle.radiative_heating(go, dp, pt, ts, xc, yc, ptop, g)
    plev, play, playkap = layer_properties(dp, ptop)
    tl, tv = temperatures(pt, plev, play, playkap)
    nlay = dp.shape[0]
    B = slope * (tv - 50.0)
    Bs = slope * (ts - 50.0)
    eps = F32(.99)
    pi = F32(np.pi)
    up = np.zeros((nlay + 2,) + dp.shape[1:])
    dn = np.zeros_like(up)
    em = np.zeros_like(up)
    alb = np.zeros_like(up)
    T = np.zeros_like(up)
    sd = np.zeros_like(up)
    alb[1] = 1 - eps
    em[1] = eps * pi * Bs
    for k in range(1, nlay + 1):
        tau = kabs(a, play[k], tl[k]) * dp[k - 1] / g
        T[k] = np.exp(-2 * tau)
        d = (1 - T[k]) * (B[k] - B[k + 1]) / (2 * tau)
        su = pi * (B[k + 1] - T[k] * B[k] + d)
        sd[k] = pi * (B[k] - T[k] * B[k + 1] - d)
        alb[k + 1] = T[k] ** 2 * alb[k]
        em[k + 1] = su + T[k] * (em[k] + sd[k] * alb[k])
    up[nlay + 1] = em[nlay + 1]
    for k in range(nlay, 0, -1):
        dn[k] = sd[k] + T[k] * dn[k + 1]
        up[k] = alb[k] * dn[k] + em[k]
    want = (dn - up)[1:]
    np.testing.assert_allclose(nf, want, rtol=1e-11, atol=1e-9)


def test_range_stop():
    """A surface temperature above the Planck table stops the reference
    (mod_gas_optics.f90:4562-4566); so does a layer pressure below it."""
    dp, pt, ts, xc, yc, ptop = column_state()
    go = linear_tables((1e-6, 0, 0), (1e-5, 0, 0), 0.01, 0.5)
    with pytest.raises(pyoracle.RadiationRangeError):
        pyoracle.radiative_heating(go, dp, pt, ts + 200.0, xc, yc, ptop, 9.8)
    go.pressures[0] = 2.0e4
    with pytest.raises(pyoracle.RadiationRangeError):
        pyoracle.radiative_heating(go, dp, pt, ts, xc, yc, ptop, 9.8)


def test_portable_math_against_libm():
    """The oracle's portable exp/log/pow against the C library's (the
    reference's gfortran calls libm): net fluxes within 1e-12 relative on
    the reference's tables or, without them, on synthetic ones."""
    go = gas_optics.load_default() or gas_optics.synthetic(1)
    st = ic.bubble_case(16, 12, 20, 100e3, 100e3, seed=2)
    ts = np.full((st.ny, st.nx), 288.0)
    xc, yc = ic.cell_axes(st)
    a = pyoracle.radiative_heating(go, st.dp, st.pt, ts, xc, yc, st.ak[0], st.gravity)
    b = pyoracle.radiative_heating(go, st.dp, st.pt, ts, xc, yc, st.ak[0], st.gravity, variant='libm')
    scale = np.abs(a).max()
    assert np.abs(a - b).max() <= 1e-12 * scale
    assert np.all(np.isfinite(a))


def test_gas_optics_struct_matches_header():
    """The ctypes atm_gas_optics has the fields of include/atmdyn.h's struct,
    in its order and with its types."""
    import os
    import re
    import ctypes
    from atmdyn import _lib
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with open(os.path.join(here, 'include', 'atmdyn.h')) as f:
        h = f.read()
    body = re.search(r'typedef struct \{(.*?)\} atm_gas_optics;', h, re.S).group(1)
    decl = [(t.strip(), [n.strip(' *') for n in names.split(',')])
            for t, names in re.findall(r'^\s*(int|const double\*)\s+([^;]+);', body, re.M)]
    fields = [(n, t) for t, ns in decl for n in ns]
    got = _lib.GasOpticsC._fields_
    assert [n for n, _ in fields] == [n for n, _ in got]
    for (n, t), (_, ct) in zip(fields, got):
        assert (ct is ctypes.c_int) == (t == 'int'), n
    go = gas_optics.synthetic(0)
    st = _lib.gas_optics_struct(go)
    assert (st.n_g, st.n_p, st.n_t, st.n_planck) == (16, 53, 6, 231)
    assert ctypes.addressof(st.planck.contents) == go.planck.ctypes.data


def test_gas_optics_validation():
    """Tables with a descending axis or mismatched shapes are rejected."""
    go = gas_optics.synthetic(0)
    bad = gas_optics.GasOptics(**{f: getattr(go, f).copy() for f in go.__dataclass_fields__})
    bad.pressures = bad.pressures[::-1].copy()
    with pytest.raises(ValueError, match='ascending'):
        bad.validate()
    bad = gas_optics.GasOptics(**{f: getattr(go, f).copy() for f in go.__dataclass_fields__})
    bad.planck = bad.planck[:, :-1]
    with pytest.raises(ValueError, match='shape'):
        bad.validate()
