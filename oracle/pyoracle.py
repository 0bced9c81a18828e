"""ctypes wrapper of the CPU oracle (test infrastructure only).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module.  PARITY UNPINNED: see atm_oracle.h.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HALO = 7
DP, PT, UD, VD, GZ, PLEV, PKAP, NET_FLUX, DPC, PTC, UC, VC, TS = range(13)

_libs: dict = {}
_P = ctypes.POINTER(ctypes.c_double)


def build():
    subprocess.run(['make', '-s', '-C', HERE], check=True)


def load(variant: str = 'portable'):
    """variant: 'portable' (the pow/log the CUDA library reproduces bit for
    bit), 'libm' (the C library's pow/log) or 'checked' (bounds checks)."""
    if variant in _libs:
        return _libs[variant]
    name = {'portable': 'liboracle.so', 'libm': 'liboracle_libm.so',
            'checked': 'liboracle_chk.so'}[variant]
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        build()
    lib = ctypes.CDLL(path)
    lib.orc_create.restype = ctypes.c_void_p
    lib.orc_create.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 2 + [_P, _P] + [ctypes.c_double] * 4
    vp = [ctypes.c_void_p]
    lib.orc_destroy.argtypes = vp
    lib.orc_set_field.argtypes = vp + [ctypes.c_int, _P, ctypes.c_int]
    lib.orc_get_field.argtypes = vp + [ctypes.c_int, _P, ctypes.c_int]
    lib.orc_field_levels.argtypes = vp + [ctypes.c_int]
    for f in ('orc_init', 'orc_cgrid_halo', 'orc_remap', 'orc_dgrid_halo'):
        getattr(lib, f).argtypes = vp
    lib.orc_cgrid_step.argtypes = vp + [ctypes.c_double]
    lib.orc_dgrid_step.argtypes = vp + [ctypes.c_double]
    lib.orc_physics_tendencies.argtypes = vp
    lib.orc_apply_physics.argtypes = vp + [ctypes.c_double]
    lib.orc_physics_halo.argtypes = vp
    lib.orc_check_stability.argtypes = vp
    lib.orc_mass.argtypes = vp
    lib.orc_mass.restype = ctypes.c_double
    lib.orc_set_threads.argtypes = vp + [ctypes.c_int]
    lib.orc_set_poison.argtypes = vp + [ctypes.c_int]
    lib.orc_set_remap_trace.argtypes = vp + [ctypes.POINTER(ctypes.c_int32)]
    lib.orc_pow_array.argtypes = [_P, ctypes.c_double, _P, ctypes.c_int]
    lib.orc_log_array.argtypes = [_P, _P, ctypes.c_int]
    lib.orc_radiative_heating.argtypes = [ctypes.c_int] * 3 + [_P] * 5 + [ctypes.c_double] * 2 + \
        [ctypes.c_void_p] + [ctypes.c_double] * 3 + [_P, ctypes.c_int]
    _libs[variant] = lib
    return lib


def _ptr(a):
    return a.ctypes.data_as(_P)


class OracleModel:
    """The oracle with the stepper interface of atmdyn.model.run_model."""

    def __init__(self, st, threads: int = 1, variant: str = 'portable', poison: bool = False):
        self.lib = load(variant)
        self.st = st
        self.nx, self.ny, self.nlay = st.nx, st.ny, st.nlay
        ak = np.ascontiguousarray(st.ak, dtype=np.float64)
        bk = np.ascontiguousarray(st.bk, dtype=np.float64)
        self.s = self.lib.orc_create(st.nx, st.ny, st.nlay, st.dx, st.dy, _ptr(ak), _ptr(bk),
                                     st.gravity, st.coriolis, st.divdamp, st.vortdamp)
        if not self.s:
            raise ValueError('orc_create rejected the configuration')
        self.lib.orc_set_threads(self.s, threads)
        self.threads, self.variant = threads, variant
        self.lib.orc_set_poison(self.s, int(poison))
        for f, a in ((DP, st.dp), (PT, st.pt), (UD, st.u), (VD, st.v)):
            self.set(f, a)
        gz = np.zeros((st.nlay + 1, st.ny, st.nx))
        gz[0] = st.gzs
        self.set(GZ, gz)
        if getattr(st, 'ts', None) is not None:
            self.set(TS, np.asarray(st.ts)[None])
        self.lib.orc_init(self.s)
        if getattr(st, 'ts', None) is not None:
            self.physics_halo()  # initial_halo_exchange of ts (mod_input.f90:251)
        self._trace = None

    def __del__(self):
        if getattr(self, 's', None):
            self.lib.orc_destroy(self.s)
            self.s = None

    def levels(self, field):
        return self.lib.orc_field_levels(self.s, field)

    def set(self, field, a, halo=False):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if self.lib.orc_set_field(self.s, field, _ptr(a), int(halo)) != 0:
            raise ValueError('bad field')

    def get(self, field, halo=False):
        K = self.levels(field)
        shape = (K, self.ny + 2 * HALO, self.nx + 2 * HALO) if halo else (K, self.ny, self.nx)
        out = np.empty(shape)
        self.lib.orc_get_field(self.s, field, _ptr(out), int(halo))
        return out

    # stepper interface
    def cgrid_step(self, dt_half):
        self.lib.orc_cgrid_step(self.s, dt_half)

    def cgrid_halo(self):
        self.lib.orc_cgrid_halo(self.s)

    def dgrid_step(self, dt):
        self.lib.orc_dgrid_step(self.s, dt)

    def remap(self):
        self.lib.orc_remap(self.s)

    def dgrid_halo(self):
        self.lib.orc_dgrid_halo(self.s)

    def physics_tendencies(self):
        self.lib.orc_physics_tendencies(self.s)

    def apply_physics(self, dt):
        self.lib.orc_apply_physics(self.s, dt)

    def physics_halo(self):
        self.lib.orc_physics_halo(self.s)

    def set_net_flux(self, nf_halo):
        self.set(NET_FLUX, nf_halo, halo=True)

    # radiation (the stepper interface of run_model)
    def set_radiation(self, go, xc, yc, threads=None, **params):
        self._rad = (go, xc, yc, threads or self.threads, params)

    def radiative_heating(self, time=0.0):
        go, xc, yc, threads, params = self._rad
        ts = self.get(TS)[0]
        self._nf = radiative_heating(go, self.get(DP), self.get(PT), ts, xc, yc, float(self.st.ak[0]),
                                     self.st.gravity, threads=threads, variant=self.variant, **params)

    def radiation_halo(self):
        self.set_net_flux(periodic_halo(self._nf))

    def check_stability(self):
        return bool(self.lib.orc_check_stability(self.s))

    def mass(self):
        return self.lib.orc_mass(self.s)

    def enable_trace(self):
        self._trace = np.full((3, self.ny + 2, self.nx + 2, self.nlay, 5), -1, dtype=np.int32)
        self.lib.orc_set_remap_trace(self.s, self._trace.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        return self._trace

    def disable_trace(self):
        self.lib.orc_set_remap_trace(self.s, None)
        self._trace = None

    def state(self):
        return {name: self.get(f) for name, f in (('dp', DP), ('pt', PT), ('ud', UD), ('vd', VD))}


def periodic_halo(a):
    """(K, ny, nx) interior -> (K, ny+14, nx+14) with the periodic halo
    (the single-image halo_exchange, src/mod_sync.f90:67-217)."""
    K, ny, nx = a.shape
    iy = (np.arange(-HALO, ny + HALO)) % ny
    ix = (np.arange(-HALO, nx + HALO)) % nx
    return np.ascontiguousarray(a[:, iy][:, :, ix])


class RadiationRangeError(ValueError):
    """A layer pressure or temperature outside the gas-optics tables (the
    reference stops there)."""


def radiative_heating(go, dp, pt, ts, xc, yc, ptop, gravity, solar_zenith_angle=0.0,
                      surface_albedo=float(np.float32(.3)), surface_emissivity=float(np.float32(.99)),
                      threads=1, variant='portable'):
    """calculate_radiative_heating of the oracle: net_flux (nlay+1, ny, nx)
    from interior dp, pt (nlay, ny, nx), ts (ny, nx) and the cell axes."""
    lib = load(variant)
    nlay, ny, nx = dp.shape
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (dp, pt, ts, xc, yc)]
    tabs = [np.ascontiguousarray(getattr(go, n), dtype=np.float64) for n in
            ('pressures', 'temperatures', 'sw_absorption', 'sw_scattering', 'lw_absorption',
             'planck_temperatures', 'planck', 'irradiance_fraction')]

    class _GO(ctypes.Structure):
        _fields_ = [('n_g', ctypes.c_int), ('n_p', ctypes.c_int), ('n_t', ctypes.c_int),
                    ('n_planck', ctypes.c_int)] + [('p%d' % q, _P) for q in range(8)]
    st = _GO(tabs[3].shape[0], tabs[0].shape[0], tabs[1].shape[1], tabs[5].shape[0], *[_ptr(t) for t in tabs])
    out = np.zeros((nlay + 1, ny, nx))
    rc = lib.orc_radiative_heating(nx, ny, nlay, *[_ptr(a) for a in arrs], float(ptop), float(gravity),
                                   ctypes.cast(ctypes.byref(st), ctypes.c_void_p), float(solar_zenith_angle),
                                   float(surface_albedo), float(surface_emissivity), _ptr(out), int(threads))
    if rc == 1:
        raise RadiationRangeError('a layer pressure or temperature is outside the gas-optics tables')
    if rc:
        raise ValueError('orc_radiative_heating rejected the sizes')
    return out


def pow_array(x, y, variant='portable'):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    load(variant).orc_pow_array(_ptr(x), float(y), _ptr(out), x.size)
    return out


def log_array(x, variant='portable'):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    load(variant).orc_log_array(_ptr(x), _ptr(out), x.size)
    return out


class TLMModel:
    """Tangent-linear model of the oracle (dual numbers, branches frozen at
    the FP64 trajectory); the stepper interface of atmdyn.model.run_model."""

    def __init__(self, st, tangents=None, threads: int = 1):
        self.lib = load('portable')
        lib = self.lib
        if not hasattr(lib, '_tlm_ready'):
            vp = [ctypes.c_void_p]
            lib.tlm_create.restype = ctypes.c_void_p
            lib.tlm_create.argtypes = lib.orc_create.argtypes
            lib.tlm_destroy.argtypes = vp
            lib.tlm_set_field.argtypes = vp + [ctypes.c_int, _P, _P, ctypes.c_int]
            lib.tlm_get_field.argtypes = vp + [ctypes.c_int, _P, _P, ctypes.c_int]
            for f in ('tlm_init', 'tlm_cgrid_halo', 'tlm_remap', 'tlm_dgrid_halo'):
                getattr(lib, f).argtypes = vp
            lib.tlm_cgrid_step.argtypes = vp + [ctypes.c_double]
            lib.tlm_dgrid_step.argtypes = vp + [ctypes.c_double]
            lib.tlm_set_threads.argtypes = vp + [ctypes.c_int]
            lib._tlm_ready = True
        self.st = st
        self.nx, self.ny, self.nlay = st.nx, st.ny, st.nlay
        ak = np.ascontiguousarray(st.ak, dtype=np.float64)
        bk = np.ascontiguousarray(st.bk, dtype=np.float64)
        self.s = lib.tlm_create(st.nx, st.ny, st.nlay, st.dx, st.dy, _ptr(ak), _ptr(bk),
                                st.gravity, st.coriolis, st.divdamp, st.vortdamp)
        lib.tlm_set_threads(self.s, threads)
        tangents = tangents or {}
        for name, f, a in (('dp', DP, st.dp), ('pt', PT, st.pt), ('ud', UD, st.u), ('vd', VD, st.v)):
            self.set(f, a, tangents.get(name))
        gz = np.zeros((st.nlay + 1, st.ny, st.nx))
        gz[0] = st.gzs
        self.set(GZ, gz, None)
        lib.tlm_init(self.s)

    def __del__(self):
        if getattr(self, 's', None):
            self.lib.tlm_destroy(self.s)
            self.s = None

    def levels(self, field):
        return self.nlay + 1 if field in (GZ, PLEV, PKAP, NET_FLUX) else self.nlay

    def set(self, field, val, tan=None, halo=False):
        val = np.ascontiguousarray(val, dtype=np.float64)
        t = None if tan is None else np.ascontiguousarray(tan, dtype=np.float64)
        assert self.lib.tlm_set_field(self.s, field, _ptr(val), None if t is None else _ptr(t), int(halo)) == 0

    def get(self, field, halo=False):
        K = self.levels(field)
        shape = (K, self.ny + 2 * HALO, self.nx + 2 * HALO) if halo else (K, self.ny, self.nx)
        v = np.empty(shape)
        t = np.empty(shape)
        assert self.lib.tlm_get_field(self.s, field, _ptr(v), _ptr(t), int(halo)) == 0
        return v, t

    def cgrid_step(self, dt_half):
        self.lib.tlm_cgrid_step(self.s, dt_half)

    def cgrid_halo(self):
        self.lib.tlm_cgrid_halo(self.s)

    def dgrid_step(self, dt):
        self.lib.tlm_dgrid_step(self.s, dt)

    def remap(self):
        self.lib.tlm_remap(self.s)

    def dgrid_halo(self):
        self.lib.tlm_dgrid_halo(self.s)

    def check_stability(self):
        return True
