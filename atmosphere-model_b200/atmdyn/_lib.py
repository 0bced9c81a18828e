"""ctypes binding of libatmdyn.so (the C ABI declared in include/atmdyn.h).

The library is built in-tree by ``make -C atmosphere-model_b200/csrc`` (or
``__graft_entry__.build()``).  There is no fallback: if the shared library is
missing or a CUDA call fails, the calls raise.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
# ATMDYN_LIBRARY selects another build of the library (e.g. an installed copy)
LIB_PATH = os.environ.get('ATMDYN_LIBRARY') or os.path.join(HERE, 'libatmdyn.so')
CSRC = os.path.join(os.path.dirname(HERE), 'csrc')

ATM_DP, ATM_PT, ATM_UD, ATM_VD, ATM_GZ, ATM_PLEV, ATM_PKAP, ATM_NET_FLUX = range(8)
ATM_DPC, ATM_PTC, ATM_UC, ATM_VC = range(8, 12)
ATM_TS = 12
ATM_FP64, ATM_MIXED = 0, 1
STATUS = {0: 'ATM_OK', 1: 'ATM_ERR_ARG', 2: 'ATM_ERR_CUDA', 3: 'ATM_ERR_STATE',
          4: 'ATM_ERR_NOMEM', 5: 'ATM_ERR_UNSUPPORTED', 6: 'ATM_ERR_TOO_LARGE', 7: 'ATM_ERR_RANGE'}

# every entry point of include/atmdyn.h
EXPORTS = ('atm_create', 'atm_upload', 'atm_download', 'atm_init', 'atm_cgrid_step', 'atm_cgrid_halo',
           'atm_dgrid_step', 'atm_remap', 'atm_dgrid_halo', 'atm_check_stability', 'atm_mass',
           'atm_set_net_flux', 'atm_step', 'atm_sync', 'atm_destroy', 'atm_last_error',
           'atm_upload_device', 'atm_download_device', 'atm_set_stream', 'atm_remap_trace',
           'atm_device_pow_log', 'atm_version', 'atm_profile', 'atm_profile_read', 'atm_profile_stage',
           'atm_launch_count', 'atm_remap_noalloc', 'atm_device_div_check',
           'atm_adj_enable', 'atm_adj_zero', 'atm_adj_set', 'atm_adj_get', 'atm_adj_set_device',
           'atm_adj_get_device', 'atm_adj_step', 'atm_adj_halo', 'atm_adj_cgrid_halo', 'atm_adj_cgrid_step',
           'atm_adj_dgrid_step', 'atm_adj_remap', 'atm_state_bytes', 'atm_state_save', 'atm_state_load',
           'atm_tape_bytes', 'atm_step_tape', 'atm_adj_step_tape', 'atm_output_enable', 'atm_output_reset',
           'atm_accumulate_output', 'atm_output_read', 'atm_output_time', 'atm_physics_tendencies',
           'atm_apply_physics', 'atm_physics_halo', 'atm_device_wait_check',
           'atm_ensemble_create', 'atm_ensemble_set_strips', 'atm_ensemble_set_stream', 'atm_ensemble_prepare',
           'atm_ensemble_run', 'atm_ensemble_status', 'atm_ensemble_blocks', 'atm_ensemble_destroy',
           'atm_ensemble_barrier_check', 'atm_ensemble_profile', 'atm_ensemble_stage_ms',
           'atm_ensemble_set_schedule', 'atm_set_gas_optics', 'atm_set_cell_coordinates',
           'atm_radiative_heating', 'atm_radiation_halo', 'atm_device_kappa_pow')
ATM_ADJ_IN, ATM_ADJ_OUT = 0, 1

# the entry points every build must export
CORE = ('atm_create', 'atm_upload', 'atm_download', 'atm_init', 'atm_cgrid_step', 'atm_cgrid_halo',
        'atm_dgrid_step', 'atm_remap', 'atm_dgrid_halo', 'atm_check_stability', 'atm_mass', 'atm_step',
        'atm_sync', 'atm_destroy', 'atm_last_error', 'atm_set_stream')

_lib = None


class GasOpticsC(ctypes.Structure):
    """atm_gas_optics of include/atmdyn.h."""
    _fields_ = [('n_g', ctypes.c_int), ('n_p', ctypes.c_int), ('n_t', ctypes.c_int), ('n_planck', ctypes.c_int)] + \
        [(n, ctypes.POINTER(ctypes.c_double)) for n in
         ('pressures', 'temperatures', 'sw_absorption', 'sw_scattering', 'lw_absorption', 'planck_temperatures',
          'planck', 'irradiance_fraction')]


def gas_optics_struct(go):
    """An atm_gas_optics over the arrays of a :class:`atmdyn.gas_optics.GasOptics`
    (which must outlive the struct)."""
    P = ctypes.POINTER(ctypes.c_double)
    n_p, n_t = go.temperatures.shape
    return GasOpticsC(go.n_g, n_p, n_t, go.planck_temperatures.shape[0],
                      *[getattr(go, n).ctypes.data_as(P) for n in
                        ('pressures', 'temperatures', 'sw_absorption', 'sw_scattering', 'lw_absorption',
                         'planck_temperatures', 'planck', 'irradiance_fraction')])


class AtmError(RuntimeError):
    pass


def build():
    subprocess.run(['make', '-s', '-C', CSRC], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise AtmError('libatmdyn.so is not built (run make -C %s)' % CSRC)
    lib = ctypes.CDLL(LIB_PATH)
    missing = [f for f in CORE if not hasattr(lib, f)]
    if missing:
        raise AtmError('libatmdyn.so lacks %s' % ', '.join(missing))
    P = ctypes.POINTER(ctypes.c_double)
    vp = ctypes.c_void_p
    i = ctypes.c_int
    d = ctypes.c_double
    lib.atm_create.argtypes = [ctypes.POINTER(vp), i, i, i, d, d, P, P, d, d, d, d, i, i]
    lib.atm_upload.argtypes = [vp, i, P]
    lib.atm_download.argtypes = [vp, i, P]
    for f in ('atm_init', 'atm_cgrid_halo', 'atm_remap', 'atm_dgrid_halo', 'atm_sync', 'atm_destroy'):
        getattr(lib, f).argtypes = [vp]
    lib.atm_cgrid_step.argtypes = [vp, d]
    lib.atm_dgrid_step.argtypes = [vp, d]
    lib.atm_check_stability.argtypes = [vp, ctypes.POINTER(i)]
    lib.atm_mass.argtypes = [vp, P]
    lib.atm_set_net_flux.argtypes = [vp, P]
    lib.atm_step.argtypes = [vp, d, i, ctypes.POINTER(i)]
    lib.atm_last_error.argtypes = [vp]
    lib.atm_last_error.restype = ctypes.c_char_p
    lib.atm_upload_device.argtypes = [vp, i, vp, i]
    lib.atm_download_device.argtypes = [vp, i, vp, i]
    lib.atm_set_stream.argtypes = [vp, vp]
    lib.atm_remap_trace.argtypes = [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(i)]
    lib.atm_device_pow_log.argtypes = [P, d, P, P, i]
    lib.atm_version.restype = ctypes.c_char_p
    # measurement and test entry points (an older build may lack some)
    optional = {
        'atm_profile': ([vp, i], None),
        'atm_profile_read': ([vp, P, ctypes.POINTER(i), i], None),
        'atm_profile_stage': ([i], ctypes.c_char_p),
        'atm_launch_count': ([vp, ctypes.POINTER(ctypes.c_longlong)], None),
        'atm_device_div_check': ([ctypes.c_longlong, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)], None),
        'atm_adj_enable': ([vp], None),
        'atm_adj_zero': ([vp], None),
        'atm_adj_set': ([vp, i, i, P], None),
        'atm_adj_get': ([vp, i, i, P], None),
        'atm_adj_set_device': ([vp, i, i, vp], None),
        'atm_adj_get_device': ([vp, i, i, vp], None),
        'atm_adj_step': ([vp, d, i], None),
        'atm_adj_halo': ([vp, i], None),
        'atm_adj_cgrid_halo': ([vp], None),
        'atm_adj_cgrid_step': ([vp, d], None),
        'atm_adj_dgrid_step': ([vp, d], None),
        'atm_adj_remap': ([vp], None),
        'atm_state_bytes': ([vp, ctypes.POINTER(ctypes.c_longlong)], None),
        'atm_state_save': ([vp, vp], None),
        'atm_state_load': ([vp, vp], None),
        'atm_tape_bytes': ([vp, ctypes.POINTER(ctypes.c_longlong)], None),
        'atm_step_tape': ([vp, d, i, vp], None),
        'atm_adj_step_tape': ([vp, d, i, vp], None),
        'atm_output_enable': ([vp], None),
        'atm_output_reset': ([vp], None),
        'atm_accumulate_output': ([vp, d], None),
        'atm_output_read': ([vp, i, P], None),
        'atm_output_time': ([vp, P], None),
        'atm_physics_tendencies': ([vp], None),
        'atm_apply_physics': ([vp, d], None),
        'atm_physics_halo': ([vp], None),
        'atm_device_wait_check': ([i, ctypes.POINTER(i)], None),
        'atm_ensemble_create': ([ctypes.POINTER(vp), ctypes.POINTER(vp), P, i], None),
        'atm_ensemble_set_strips': ([vp, i, i], None),
        'atm_ensemble_set_stream': ([vp, vp], None),
        'atm_ensemble_prepare': ([vp], None),
        'atm_ensemble_run': ([vp, i, i], None),
        'atm_ensemble_status': ([vp, ctypes.POINTER(i)], None),
        'atm_ensemble_blocks': ([vp, ctypes.POINTER(i)], None),
        'atm_ensemble_profile': ([vp, i], None),
        'atm_ensemble_set_schedule': ([vp, i], None),
        'atm_ensemble_stage_ms': ([vp, ctypes.POINTER(ctypes.c_double), i], None),
        'atm_ensemble_destroy': ([vp], None),
        'atm_ensemble_barrier_check': ([ctypes.c_longlong, ctypes.POINTER(i)], None),
        'atm_set_gas_optics': ([vp, ctypes.POINTER(GasOpticsC)], None),
        'atm_set_cell_coordinates': ([vp, P, P], None),
        'atm_radiative_heating': ([vp, d, d, d, d], None),
        'atm_radiation_halo': ([vp], None),
        'atm_device_kappa_pow': ([P, P, i], None),
    }
    for f, (args, res) in optional.items():
        if hasattr(lib, f):
            getattr(lib, f).argtypes = args
            if res is not None:
                getattr(lib, f).restype = res
    _lib = lib
    return lib


def check(rc: int, ctx=None, what: str = ''):
    if rc != 0:
        msg = ''
        if ctx is not None and _lib is not None:
            try:
                msg = _lib.atm_last_error(ctx).decode()
            except Exception:
                msg = ''
        raise AtmError('%s failed with %s %s' % (what, STATUS.get(rc, rc), msg))
