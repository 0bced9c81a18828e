"""Seeded initial conditions for the dynamical core, in the style of the
reference's scripts/ic_generator.py (hydrostatic layers, layer-mean
potential temperature consistent with the interface geopotential,
``pt = |d(gz)/d(p**kappa)| / cp``, scripts/ic_generator.py:140-143).

Conventions of the model (src/mod_fields.f90, src/mod_input.f90:151-245):
* fields are Fortran arrays (i, j, k) with i fastest; here they are numpy
  arrays of shape (nlay, ny, nx) in C order, which is the same memory;
* k = 1 is the lowest layer; interface k is the bottom of layer k and
  interface nlay+1 is the model top, ``plev(nlay+1) = ak(1)``;
* the model's potential temperature is T / p**kappa (no reference pressure),
  so ``pt = theta / p0**kappa`` with p0 = 1000 hPa;
* the D-grid u sits on the x-directed cell edges (x_c, y_f), v on the
  y-directed edges (x_f, y_c) (src/mod_sw_dyn.f90:45-64).

Two cases:
* ``bubble``: resting, uniform wind u0, theta(p) = 300 K (1000 hPa/p)^0.1
  plus a Gaussian warm bubble;
* ``jet``: a zonal jet u(y, p) = U(y) ln(ps/p)/ln(ps/ptop) with
  U(y) = 30 m/s sech^2((y - Ly/2)/500 km) minus its domain mean, in
  thermal-wind balance with a meridional temperature anomaly
  dT/dy = -f U(y) / (R ln(ps/ptop)), plus seeded white-noise theta
  perturbations smoothed by a 3-cell Gaussian and rescaled to 0.5 K rms.
"""
from __future__ import annotations

from dataclasses import dataclass, field
import numpy as np

# src/mod_constants.f90:11-14 (R_dry is a default-real literal)
R_DRY = float(np.float32(287.052874))
CP_DRY = 1005.0
KAPPA = R_DRY / CP_DRY
P0 = 1.0e5


@dataclass
class InitialState:
    """A complete dycore set-up: grid, coordinate, constants and fields."""
    nx: int
    ny: int
    nlay: int
    dx: float
    dy: float
    ak: np.ndarray            # (nlay+1,)
    bk: np.ndarray            # (nlay+1,)
    dp: np.ndarray            # (nlay, ny, nx)
    pt: np.ndarray
    u: np.ndarray
    v: np.ndarray
    gzs: np.ndarray           # (ny, nx) surface geopotential
    gravity: float = 9.807
    coriolis: float = 1e-4
    divdamp: float = 0.15
    vortdamp: float = 0.005
    dt: float = 60.0
    remap_every: int = 5
    nsteps: int = 100
    name: str = ''
    extra: dict = field(default_factory=dict)
    ts: np.ndarray | None = None  # (ny, nx) surface temperature (the physics' only 2-D prognostic)
    xc: np.ndarray | None = None  # (nx,) cell-centre x axis of the initial file (default: see cell_axes)
    yc: np.ndarray | None = None  # (ny,)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nlay


def cell_axes(st):
    """The cell-centre axes (xc, yc): the state's own (read from its initial
    file), else the reference generator's, centred on the domain
    (scripts/ic_generator.py:20-22: linspace((dx-Lx)/2, (Lx-dx)/2, nx))."""
    xc, yc = getattr(st, 'xc', None), getattr(st, 'yc', None)
    if xc is None:
        lx = st.nx * st.dx
        xc = np.linspace((st.dx - lx) / 2, (lx - st.dx) / 2, st.nx)
    if yc is None:
        ly = st.ny * st.dy
        yc = np.linspace((st.dy - ly) / 2, (ly - st.dy) / 2, st.ny)
    return np.asarray(xc, dtype=np.float64), np.asarray(yc, dtype=np.float64)


def sigma_coordinate(nlay: int, ptop: float = 1.0e4):
    """Pure-sigma coefficients: Ak = ptop, Bk = (nlay+1-k)/nlay (k = 1 is the
    surface).  Ak(1) = ptop as src/mod_remap.f90:362 assumes."""
    k = np.arange(1, nlay + 2, dtype=np.float64)
    ak = np.full(nlay + 1, ptop)
    bk = (nlay + 1 - k) / nlay
    return ak, bk


def _layer_pt(p_bot, p_top, t_of_p_integral):
    """Layer-mean model theta from hydrostatic geopotential thickness."""
    dgz = R_DRY * t_of_p_integral(p_bot, p_top)
    return dgz / (CP_DRY * (p_bot ** KAPPA - p_top ** KAPPA))


def _base_integral(p_bot, p_top):
    # integral of T dp/p for theta(p) = 300 K (p0/p)^0.1, T = theta (p/p0)^kappa
    a = KAPPA - 0.1
    return 300.0 / a * ((p_bot / P0) ** a - (p_top / P0) ** a)


def _interfaces(ak, bk, ps):
    """plev(k), k = 1..nlay+1, for surface pressure ps (broadcast)."""
    return ak[:, None, None] + bk[:, None, None] * (ps[None] - ak[0])


def bubble_case(nx=128, ny=128, nlay=20, dx=50e3, dy=50e3, ptop=1.0e4,
                ps=1.0e5, u0=10.0, amplitude=2.0, radius=500e3,
                p_centre=7.0e4, p_halfwidth=2.0e4, seed=0, **kw) -> InitialState:
    ak, bk = sigma_coordinate(nlay, ptop)
    psurf = np.full((ny, nx), ps)
    plev = _interfaces(ak, bk, psurf)                 # (nlay+1, ny, nx)
    p_bot, p_top = plev[:-1], plev[1:]
    dp = p_bot - p_top
    pt = _layer_pt(p_bot, p_top, _base_integral)
    xc = (np.arange(nx) + 0.5) * dx
    yc = (np.arange(ny) + 0.5) * dy
    X, Y = np.meshgrid(xc, yc)
    r2 = ((X - nx * dx / 2) ** 2 + (Y - ny * dy / 2) ** 2) / radius ** 2
    pmid = 0.5 * (p_bot + p_top)
    dtheta = amplitude * np.exp(-r2)[None] * np.exp(-((pmid - p_centre) / p_halfwidth) ** 2)
    pt = pt + dtheta / P0 ** KAPPA
    u = np.full((nlay, ny, nx), u0)
    v = np.zeros((nlay, ny, nx))
    gzs = np.zeros((ny, nx))
    st = InitialState(nx, ny, nlay, dx, dy, ak, bk, np.ascontiguousarray(dp),
                      np.ascontiguousarray(pt), u, v, gzs, name='bubble')
    for key, val in kw.items():
        setattr(st, key, val)
    return st


def _gaussian_smooth_periodic(a: np.ndarray, sigma_cells: float) -> np.ndarray:
    ny, nx = a.shape[-2:]
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.rfftfreq(nx)[None, :]
    g = np.exp(-2.0 * (np.pi * sigma_cells) ** 2 * (kx ** 2 + ky ** 2))
    return np.fft.irfft2(np.fft.rfft2(a) * g, s=(ny, nx))


def jet_case(nx=1024, ny=1024, nlay=64, dx=25e3, dy=25e3, ptop=1.0e4,
             ps=1.0e5, u_jet=30.0, width=500e3, coriolis=1e-4,
             noise_k=0.5, smooth_cells=3.0, seed=0, **kw) -> InitialState:
    rng = np.random.default_rng(seed)
    ak, bk = sigma_coordinate(nlay, ptop)
    psurf = np.full((ny, nx), ps)
    plev = _interfaces(ak, bk, psurf)
    p_bot, p_top = plev[:-1], plev[1:]
    dp = p_bot - p_top
    Ly = ny * dy
    a = width

    def U(y):
        return u_jet / np.cosh((y - Ly / 2) / a) ** 2

    ubar = u_jet * 2 * a * np.tanh(Ly / (2 * a)) / Ly

    def intU(y):   # integral of (U - ubar) from 0 to y
        return u_jet * a * (np.tanh((y - Ly / 2) / a) - np.tanh(-Ly / (2 * a))) - ubar * y

    lnr = np.log(ps / ptop)
    yc = (np.arange(ny) + 0.5) * dy
    yf = np.arange(ny) * dy
    dT = -coriolis / (R_DRY * lnr) * intU(yc)          # (ny,)
    dT = np.broadcast_to(dT[None, :, None], p_bot.shape)

    def integral(pb, pt_):
        return _base_integral(pb, pt_) + dT * np.log(pb / pt_)

    pt = _layer_pt(p_bot, p_top, integral)
    noise = rng.normal(0.0, noise_k, size=(nlay, ny, nx))
    noise = _gaussian_smooth_periodic(noise, smooth_cells)
    noise *= noise_k / max(noise.std(), 1e-30)
    pt = pt + noise / P0 ** KAPPA
    pmid = 0.5 * (p_bot + p_top)
    w = np.log(ps / pmid) / lnr                           # (nlay, ny, nx)
    u = (U(yf) - ubar)[None, :, None] * w
    v = np.zeros((nlay, ny, nx))
    gzs = np.zeros((ny, nx))
    st = InitialState(nx, ny, nlay, dx, dy, ak, bk, np.ascontiguousarray(dp),
                      np.ascontiguousarray(pt), np.ascontiguousarray(u), v, gzs,
                      coriolis=coriolis, name='jet')
    for key, val in kw.items():
        setattr(st, key, val)
    return st


# The five benchmark configurations (sizes, steps and remap intervals).
def config(n: int, **over) -> InitialState:
    if n == 1:
        st = bubble_case(128, 128, 20, 50e3, 50e3, seed=0)
        st.dt, st.remap_every, st.nsteps = 60.0, 5, 100
    elif n == 2:
        st = jet_case(1024, 1024, 64, 25e3, 25e3, seed=0)
        st.dt, st.remap_every, st.nsteps = 30.0, 8, 200
    elif n == 3:
        st = jet_case(2048, 2048, 64, 25e3, 25e3, seed=1)
        st.dt, st.remap_every, st.nsteps = 30.0, 8, 200
    elif n == 4:
        st = jet_case(512, 512, 32, 25e3, 25e3, seed=2)
        st.dt, st.remap_every, st.nsteps = 30.0, 5, 20
    else:
        raise ValueError('configs 1-4 are single grids; see ensemble_members() for 5')
    for key, val in over.items():
        setattr(st, key, val)
    st.name = 'config%d' % n
    return st


def ensemble_members(n_members=64, seed=3):
    """Config 5: members of uneven sizes, grids from {64,128,256,512}^2,
    layers from {20,32,48,64}, each a bubble or jet case."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n_members):
        n = int(rng.choice([64, 128, 256, 512]))
        L = int(rng.choice([20, 32, 48, 64]))
        kind = 'bubble' if rng.integers(2) == 0 else 'jet'
        dx = 50e3 * 128 / n
        if kind == 'bubble':
            st = bubble_case(n, n, L, dx, dx, seed=int(seed * 1000 + m))
            st.dt = 60.0 * 128 / n
        else:
            st = jet_case(n, n, L, dx, dx, seed=int(seed * 1000 + m))
            st.dt = 30.0 * 1024 / n / 2
        st.remap_every, st.nsteps = 5, 100
        st.name = 'member%d_%s' % (m, kind)
        out.append(st)
    return out
