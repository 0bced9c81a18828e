"""Host-side mirror of the reference's dycore interface over libatmdyn.

:class:`Dycore` exposes the routines of src/mod_sw_dyn.f90:17-19 and
src/mod_remap.f90:13 (``cgrid_step``/``cgrid_halo``/``dgrid_step``/
``remap``/``dgrid_halo``) plus ``check_stability`` of src/mod_fields.f90:69,
so :func:`atmdyn.model.run_model` drives it exactly like the reference's
time loop drives the Fortran modules.  Fields are numpy arrays of shape
(K, ny, nx) (interior) or (K, ny+14, nx+14) (with the 7-wide halo), the
memory layout of the reference's Fortran arrays.
"""
from __future__ import annotations

import ctypes
import numpy as np

from . import _lib
from ._lib import check, ATM_DP, ATM_PT, ATM_UD, ATM_VD, ATM_GZ, ATM_PLEV, ATM_PKAP, ATM_NET_FLUX, ATM_TS

HALO = 7
FIELDS = {'dp': ATM_DP, 'pt': ATM_PT, 'ud': ATM_UD, 'vd': ATM_VD, 'gz': ATM_GZ,
          'plev': ATM_PLEV, 'pkap': ATM_PKAP, 'net_flux': ATM_NET_FLUX,
          'dpc': 8, 'ptc': 9, 'uc': 10, 'vc': 11, 'ts': ATM_TS}
_P = ctypes.POINTER(ctypes.c_double)


def _ptr(a):
    return a.ctypes.data_as(_P)


def with_halo(interior: np.ndarray) -> np.ndarray:
    """(K, ny, nx) interior -> (K, ny+14, nx+14) array with a zero halo."""
    K, ny, nx = interior.shape
    out = np.zeros((K, ny + 2 * HALO, nx + 2 * HALO))
    out[:, HALO:HALO + ny, HALO:HALO + nx] = interior
    return out


class Dycore:
    """One single-image dycore domain on the current CUDA device."""

    def __init__(self, st, precision: str = 'fp64'):
        self.lib = _lib.load()
        self.st = st
        self.nx, self.ny, self.nlay = st.nx, st.ny, st.nlay
        self.precision = precision
        ak = np.ascontiguousarray(st.ak, dtype=np.float64)
        bk = np.ascontiguousarray(st.bk, dtype=np.float64)
        ctx = ctypes.c_void_p()
        prec = {'fp64': _lib.ATM_FP64, 'mixed': _lib.ATM_MIXED}[precision]
        rc = self.lib.atm_create(ctypes.byref(ctx), st.nx, st.ny, st.nlay, st.dx, st.dy, _ptr(ak), _ptr(bk),
                                 st.gravity, st.coriolis, st.divdamp, st.vortdamp, prec, 0)
        check(rc, None, 'atm_create')
        self.ctx = ctx
        for f, a in ((ATM_DP, st.dp), (ATM_PT, st.pt), (ATM_UD, st.u), (ATM_VD, st.v)):
            self.upload(f, with_halo(np.asarray(a, dtype=np.float64)))
        gz = np.zeros((st.nlay + 1, st.ny, st.nx))
        gz[0] = st.gzs
        self.upload(ATM_GZ, with_halo(gz))
        if getattr(st, 'ts', None) is not None:
            self.upload(ATM_TS, with_halo(np.asarray(st.ts, dtype=np.float64)[None]))
        check(self.lib.atm_init(self.ctx), self.ctx, 'atm_init')

    def close(self):
        if getattr(self, 'ctx', None):
            self.lib.atm_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def levels(self, field):
        if field == ATM_TS:
            return 1
        return self.nlay + 1 if field in (ATM_GZ, ATM_PLEV, ATM_PKAP, ATM_NET_FLUX) else self.nlay

    def upload(self, field, a):
        if isinstance(field, str):
            field = FIELDS[field]
        a = np.ascontiguousarray(a, dtype=np.float64)
        check(self.lib.atm_upload(self.ctx, field, _ptr(a)), self.ctx, 'atm_upload')

    def get(self, field, halo=False):
        if isinstance(field, str):
            field = FIELDS[field]
        K = self.levels(field)
        out = np.empty((K, self.ny + 2 * HALO, self.nx + 2 * HALO))
        check(self.lib.atm_download(self.ctx, field, _ptr(out)), self.ctx, 'atm_download')
        return out if halo else out[:, HALO:HALO + self.ny, HALO:HALO + self.nx].copy()

    def get_into(self, field, out):
        """Download a field with its halo straight into ``out`` (a contiguous
        float64 array of shape (K, ny+14, nx+14), e.g. pinned host memory)."""
        if isinstance(field, str):
            field = FIELDS[field]
        assert out.dtype == np.float64 and out.flags.c_contiguous
        assert out.shape == (self.levels(field), self.ny + 2 * HALO, self.nx + 2 * HALO)
        check(self.lib.atm_download(self.ctx, field, _ptr(out)), self.ctx, 'atm_download')
        return out

    def set_net_flux(self, nf_halo):
        if nf_halo is None:
            check(self.lib.atm_set_net_flux(self.ctx, None), self.ctx, 'atm_set_net_flux')
            return
        a = np.ascontiguousarray(nf_halo, dtype=np.float64)
        check(self.lib.atm_set_net_flux(self.ctx, _ptr(a)), self.ctx, 'atm_set_net_flux')

    # the reference's dycore entry points
    def cgrid_step(self, dt_half):
        check(self.lib.atm_cgrid_step(self.ctx, dt_half), self.ctx, 'atm_cgrid_step')

    def cgrid_halo(self):
        check(self.lib.atm_cgrid_halo(self.ctx), self.ctx, 'atm_cgrid_halo')

    def dgrid_step(self, dt):
        check(self.lib.atm_dgrid_step(self.ctx, dt), self.ctx, 'atm_dgrid_step')

    def remap(self):
        check(self.lib.atm_remap(self.ctx), self.ctx, 'atm_remap')

    def dgrid_halo(self):
        check(self.lib.atm_dgrid_halo(self.ctx), self.ctx, 'atm_dgrid_halo')

    def check_stability(self):
        s = ctypes.c_int(0)
        check(self.lib.atm_check_stability(self.ctx, ctypes.byref(s)), self.ctx, 'atm_check_stability')
        return bool(s.value)

    def step(self, dt, remap=False, check_stable=True):
        s = ctypes.c_int(1)
        check(self.lib.atm_step(self.ctx, dt, int(remap), ctypes.byref(s) if check_stable else None),
              self.ctx, 'atm_step')
        return bool(s.value)

    # column physics (src/mod_physics.f90)
    def physics_tendencies(self):
        check(self.lib.atm_physics_tendencies(self.ctx), self.ctx, 'atm_physics_tendencies')

    def apply_physics(self, dt):
        check(self.lib.atm_apply_physics(self.ctx, dt), self.ctx, 'atm_apply_physics')

    def physics_halo(self):
        check(self.lib.atm_physics_halo(self.ctx), self.ctx, 'atm_physics_halo')

    # radiation (src/mod_radiation.f90)
    def set_radiation(self, go, xc=None, yc=None):
        """Upload the gas-optics tables (:class:`atmdyn.gas_optics.GasOptics`)
        and the cell-centre axes the solar irradiance depends on (default:
        the state's, see :func:`atmdyn.ic.cell_axes`)."""
        from .ic import cell_axes
        self._go = go.validate()
        check(self.lib.atm_set_gas_optics(self.ctx, ctypes.byref(_lib.gas_optics_struct(self._go))), self.ctx,
              'atm_set_gas_optics')
        if xc is None or yc is None:
            xc, yc = cell_axes(self.st)
        xc = np.ascontiguousarray(xc, dtype=np.float64)
        yc = np.ascontiguousarray(yc, dtype=np.float64)
        assert xc.shape == (self.nx,) and yc.shape == (self.ny,)
        check(self.lib.atm_set_cell_coordinates(self.ctx, _ptr(xc), _ptr(yc)), self.ctx, 'atm_set_cell_coordinates')

    def radiative_heating(self, time=0.0, solar_zenith_angle=None, surface_albedo=None, surface_emissivity=None):
        """calculate_radiative_heating (src/mod_radiation.f90:41-156): the
        net flux of the current state; the parameters default to the
        reference's fixed values.  Raises AtmError (ATM_ERR_RANGE) where the
        reference stops on a lookup outside its tables."""
        from . import gas_optics as g
        sza = g.SOLAR_ZENITH_ANGLE if solar_zenith_angle is None else solar_zenith_angle
        alb = g.SURFACE_ALBEDO if surface_albedo is None else surface_albedo
        emi = g.SURFACE_EMISSIVITY if surface_emissivity is None else surface_emissivity
        check(self.lib.atm_radiative_heating(self.ctx, time, sza, alb, emi), self.ctx, 'atm_radiative_heating')

    def radiation_halo(self):
        check(self.lib.atm_radiation_halo(self.ctx), self.ctx, 'atm_radiation_halo')

    def mass(self):
        m = ctypes.c_double(0.)
        check(self.lib.atm_mass(self.ctx, ctypes.byref(m)), self.ctx, 'atm_mass')
        return m.value

    def sync(self):
        check(self.lib.atm_sync(self.ctx), self.ctx, 'atm_sync')

    def remap_trace(self):
        """Arm the pair trace for the next remap; returns (buffer, fallback)."""
        buf = np.full((3, self.ny + 2, self.nx + 2, self.nlay, 5), -1, dtype=np.int32)
        fb = ctypes.c_int(0)
        self._trace_keep = (buf, fb)
        check(self.lib.atm_remap_trace(self.ctx, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                       ctypes.byref(fb)), self.ctx, 'atm_remap_trace')
        return buf, fb

    def set_stream(self, stream_ptr):
        """Run on an external CUDA stream (an int cudaStream_t, or 0 for own)."""
        check(self.lib.atm_set_stream(self.ctx, ctypes.c_void_p(stream_ptr or None)), self.ctx, 'atm_set_stream')

    def profile(self, enable=True):
        check(self.lib.atm_profile(self.ctx, int(enable)), self.ctx, 'atm_profile')

    def profile_read(self):
        """{stage: (total ms, launches)} since profile(True)."""
        n = 0
        names = []
        while True:
            nm = self.lib.atm_profile_stage(n)
            if nm is None:
                break
            names.append(nm.decode())
            n += 1
        ms = np.zeros(n)
        cnt = np.zeros(n, dtype=np.int32)
        check(self.lib.atm_profile_read(self.ctx, _ptr(ms), cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n),
              self.ctx, 'atm_profile_read')
        return {names[i]: (float(ms[i]), int(cnt[i])) for i in range(n)}

    def launch_count(self):
        v = ctypes.c_longlong(0)
        check(self.lib.atm_launch_count(self.ctx, ctypes.byref(v)), self.ctx, 'atm_launch_count')
        return v.value

    def state(self):
        return {name: self.get(f) for name, f in (('dp', ATM_DP), ('pt', ATM_PT), ('ud', ATM_UD), ('vd', ATM_VD))}

    # device-resident access (torch tensors or raw device pointers)
    def upload_device(self, field, t, dtype_bytes=None):
        """Interior (nlay, ny, nx) from a contiguous device buffer; the halo
        becomes the periodic image of the interior."""
        if isinstance(field, str):
            field = FIELDS[field]
        ptr = t if isinstance(t, int) else t.data_ptr()
        nb = dtype_bytes or (8 if isinstance(t, int) else t.element_size())
        check(self.lib.atm_upload_device(self.ctx, field, ctypes.c_void_p(ptr), nb), self.ctx, 'atm_upload_device')

    def download_device(self, field, t, dtype_bytes=None):
        if isinstance(field, str):
            field = FIELDS[field]
        ptr = t if isinstance(t, int) else t.data_ptr()
        nb = dtype_bytes or (8 if isinstance(t, int) else t.element_size())
        check(self.lib.atm_download_device(self.ctx, field, ctypes.c_void_p(ptr), nb), self.ctx, 'atm_download_device')

    # output accumulation on the device (accumulate_output / write_output)
    def output_enable(self):
        check(self.lib.atm_output_enable(self.ctx), self.ctx, 'atm_output_enable')

    def output_reset(self):
        check(self.lib.atm_output_reset(self.ctx), self.ctx, 'atm_output_reset')

    def accumulate_output(self, dt):
        check(self.lib.atm_accumulate_output(self.ctx, dt), self.ctx, 'atm_accumulate_output')

    def output_read(self, name):
        """Mean over the interval of 'dp', 'pt', 'u', 'v', 'nflx' or 'ts', (K, ny, nx)."""
        which = {'dp': 0, 'pt': 1, 'u': 2, 'v': 3, 'nflx': 4, 'ts': 5}[name]
        K = self.nlay + 1 if name == 'nflx' else 1 if name == 'ts' else self.nlay
        out = np.empty((K, self.ny, self.nx))
        check(self.lib.atm_output_read(self.ctx, which, _ptr(out)), self.ctx, 'atm_output_read')
        return out

    # ---- adjoint (FP64 form): hand-written reverse mode of the step
    def adj_enable(self):
        check(self.lib.atm_adj_enable(self.ctx), self.ctx, 'atm_adj_enable')

    def adj_zero(self):
        check(self.lib.atm_adj_zero(self.ctx), self.ctx, 'atm_adj_zero')

    def adj_set(self, slot, field, a_halo):
        """Adjoint field of slot 'in'/'out' (dp, pt, ud, vd) or a C-grid
        adjoint (dpc, ptc, uc, vc) from a (K, ny+14, nx+14) array."""
        if isinstance(field, str):
            field = FIELDS[field]
        a = np.ascontiguousarray(a_halo, dtype=np.float64)
        check(self.lib.atm_adj_set(self.ctx, _SLOTS[slot], field, _ptr(a)), self.ctx, 'atm_adj_set')

    def adj_get(self, slot, field, halo=True):
        if isinstance(field, str):
            field = FIELDS[field]
        out = np.empty((self.nlay, self.ny + 2 * HALO, self.nx + 2 * HALO))
        check(self.lib.atm_adj_get(self.ctx, _SLOTS[slot], field, _ptr(out)), self.ctx, 'atm_adj_get')
        return out if halo else out[:, HALO:HALO + self.ny, HALO:HALO + self.nx].copy()

    def adj_set_device(self, slot, field, ptr):
        """Interior adjoint from a contiguous float64 (nlay, ny, nx) device buffer."""
        if isinstance(field, str):
            field = FIELDS[field]
        check(self.lib.atm_adj_set_device(self.ctx, _SLOTS[slot], field, ctypes.c_void_p(ptr)), self.ctx,
              'atm_adj_set_device')

    def adj_get_device(self, slot, field, ptr):
        if isinstance(field, str):
            field = FIELDS[field]
        check(self.lib.atm_adj_get_device(self.ctx, _SLOTS[slot], field, ctypes.c_void_p(ptr)), self.ctx,
              'atm_adj_get_device')

    def adj_step(self, dt, remap=False):
        check(self.lib.atm_adj_step(self.ctx, dt, int(remap)), self.ctx, 'atm_adj_step')

    def adj_halo(self, slot='out'):
        check(self.lib.atm_adj_halo(self.ctx, _SLOTS[slot]), self.ctx, 'atm_adj_halo')

    def adj_cgrid_halo(self):
        check(self.lib.atm_adj_cgrid_halo(self.ctx), self.ctx, 'atm_adj_cgrid_halo')

    def adj_cgrid_step(self, dt_half):
        check(self.lib.atm_adj_cgrid_step(self.ctx, dt_half), self.ctx, 'atm_adj_cgrid_step')

    def adj_dgrid_step(self, dt):
        check(self.lib.atm_adj_dgrid_step(self.ctx, dt), self.ctx, 'atm_adj_dgrid_step')

    def adj_remap(self):
        check(self.lib.atm_adj_remap(self.ctx), self.ctx, 'atm_adj_remap')

    def tape_bytes(self):
        n = ctypes.c_longlong(0)
        check(self.lib.atm_tape_bytes(self.ctx, ctypes.byref(n)), self.ctx, 'atm_tape_bytes')
        return n.value

    def step_tape(self, dt, remap, ptr):
        """A step that records its forward products at the device address ptr."""
        check(self.lib.atm_step_tape(self.ctx, dt, int(remap), ctypes.c_void_p(ptr)), self.ctx, 'atm_step_tape')

    def adj_step_tape(self, dt, remap, ptr):
        check(self.lib.atm_adj_step_tape(self.ctx, dt, int(remap), ctypes.c_void_p(ptr)), self.ctx,
              'atm_adj_step_tape')

    def state_bytes(self):
        n = ctypes.c_longlong(0)
        check(self.lib.atm_state_bytes(self.ctx, ctypes.byref(n)), self.ctx, 'atm_state_bytes')
        return n.value

    def state_save(self, ptr):
        check(self.lib.atm_state_save(self.ctx, ctypes.c_void_p(ptr)), self.ctx, 'atm_state_save')

    def state_load(self, ptr):
        check(self.lib.atm_state_load(self.ctx, ctypes.c_void_p(ptr)), self.ctx, 'atm_state_load')


def device_pow_log(x, y):
    lib = _lib.load()
    x = np.ascontiguousarray(x, dtype=np.float64)
    p = np.empty_like(x)
    lg = np.empty_like(x)
    check(lib.atm_device_pow_log(_ptr(x), float(y), _ptr(p), _ptr(lg), x.size), None, 'atm_device_pow_log')
    return p, lg


_SLOTS = {'in': _lib.ATM_ADJ_IN, 'out': _lib.ATM_ADJ_OUT, _lib.ATM_ADJ_IN: _lib.ATM_ADJ_IN,
          _lib.ATM_ADJ_OUT: _lib.ATM_ADJ_OUT}
