"""atm_remap_noalloc: the vertical remap for callers that cannot let the
library allocate device memory (a time loop whose device-memory budget is
fixed at start-up, or one that must avoid the device-wide synchronisation
of cudaMalloc/cudaFree mid-step).  Its scratch is a fixed file-scope device
array, so the test calls it several times in a row through the C ABI and
checks each result against the context-based atm_remap of the FP64 form,
bit for bit (the tolerance of the FP64 parity tests), together with the
status the entry point reports (finite results, columns that took the
all-pairs search) and that the calls after the first one leave the free
device memory unchanged.  The file sorts last so that a run stopping at
the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from atmdyn import ic, Dycore, load

pytestmark = pytest.mark.gpu

HALO = 7
_P = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
NAMES = ('dp', 'pt', 'ud', 'vd')


def _fn():
    fn = load().atm_remap_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int] * 3 + [_P, _P] + [ctypes.c_void_p] * 10 + [_I, _I]
    return fn


def _prepared(nx=40, ny=28, nlay=9):
    """A context just before its remap: C step, C halo and D step done."""
    st = ic.bubble_case(nx, ny, nlay, 160e3, 160e3, radius=1200e3, u0=15.0)
    st.v = st.v + 3.0
    g = Dycore(st, 'fp64')
    g.cgrid_step(st.dt / 2.)
    g.cgrid_halo()
    g.dgrid_step(st.dt)
    return st, g


def _ridged():
    """A state at rest whose face-interpolated interface pressures are not
    monotone in one layer (thin and thick thicknesses alternating in pairs),
    so that some wind columns take the all-pairs search."""
    nx, ny, nlay = 24, 20, 8
    st = ic.bubble_case(nx, ny, nlay, 266e3, 266e3, radius=200e3)
    pat = (np.where(np.isin(np.arange(ny) % 4, (1, 2)), 400.0, 9000.0)[:, None] * 0.5 +
           np.where(np.isin(np.arange(nx) % 4, (1, 2)), 400.0, 9000.0)[None, :] * 0.5)
    st.dp = st.dp.copy()
    st.dp[3] = pat
    return st, Dycore(st, 'fp64')


def _call(fn, st, before, gzs, plant_nan=False):
    import torch
    dev_in = {n: torch.from_numpy(before[n]).cuda().contiguous() for n in NAMES}
    if plant_nan:  # a non-finite input value, planted on the host side
        k, j, i = st.nlay // 2, HALO + st.ny // 2, HALO + st.nx // 2
        dev_in['pt'][k, j, i] = float('nan')
    dev_out = {n: dev_in[n].clone() for n in NAMES}
    dev_gzs = torch.from_numpy(gzs).cuda().contiguous()
    ak = np.ascontiguousarray(st.ak, dtype=np.float64)
    bk = np.ascontiguousarray(st.bk, dtype=np.float64)
    stable, fallback = ctypes.c_int(-1), ctypes.c_int(-1)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rc = fn(st.nx, st.ny, st.nlay, ak.ctypes.data_as(_P), bk.ctypes.data_as(_P),
            dev_in['dp'].data_ptr(), dev_in['pt'].data_ptr(), dev_in['ud'].data_ptr(), dev_in['vd'].data_ptr(),
            dev_gzs.data_ptr(), dev_out['dp'].data_ptr(), dev_out['pt'].data_ptr(), dev_out['ud'].data_ptr(),
            dev_out['vd'].data_ptr(), None, ctypes.byref(stable), ctypes.byref(fallback))
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert rc == 0, 'atm_remap_noalloc returned %d' % rc
    return {n: dev_out[n].cpu().numpy() for n in NAMES}, stable.value, fallback.value, free0 - free1


def test_remap_noalloc_matches_atm_remap_in_a_row():
    import torch
    torch.cuda.set_device(0)
    fn = _fn()
    # a different state for each call, so that nothing of one call can make
    # the next one pass; 9-10 layers use the 32-level column kernels, 40 the
    # 64-level ones
    cases = [('bubble', (40, 28, 9)), ('bubble', (44, 30, 10)), ('bubble', (24, 24, 40)), ('ridged', None)]
    for call, (kind, size) in enumerate(cases):
        if kind == 'ridged':
            st, g = _ridged()
        else:
            st, g = _prepared(*size)
        before = {n: g.get(n, halo=True) for n in NAMES}
        gzs = g.get('gz', halo=True)[0].copy()
        _, fb_ctx = g.remap_trace()
        g.remap()
        expect = {n: g.get(n, halo=True) for n in NAMES}
        got, stable, fallback, mem_used = _call(fn, st, before, gzs)
        for n in NAMES:
            assert got[n].shape == expect[n].shape
            # whole arrays: the interior is remapped, the halo is untouched in both
            np.testing.assert_array_equal(got[n], expect[n], err_msg='%s, call %d' % (n, call + 1))
        assert stable == 1
        assert fallback == fb_ctx.value, (fallback, fb_ctx.value)
        if kind == 'ridged':
            assert fallback > 0
        if call > 0:  # the first call may load the library's module (and its array)
            assert mem_used == 0, 'free device memory changed by %d bytes' % mem_used
        g.close()


def test_remap_noalloc_reports_non_finite_results():
    import torch
    torch.cuda.set_device(0)
    fn = _fn()
    st, g = _prepared()
    before = {n: g.get(n, halo=True) for n in NAMES}
    gzs = g.get('gz', halo=True)[0].copy()
    _, stable, _, _ = _call(fn, st, before, gzs, plant_nan=True)
    assert stable == 0
    _, stable, _, _ = _call(fn, st, before, gzs)  # the next call starts clean
    assert stable == 1
    g.close()


def test_remap_noalloc_rejects_sizes_beyond_its_scratch():
    fn = _fn()
    ak = np.full(65, 1e4)
    bk = np.linspace(1, 0, 65)
    # distinct, never dereferenced: the size check comes before any use
    ptrs = [ctypes.c_void_p(4096 * (i + 1)) for i in range(9)]
    rc = fn(1024, 1024, 64, ak.ctypes.data_as(_P), bk.ctypes.data_as(_P), *ptrs, None, None, None)
    assert rc == 6  # ATM_ERR_TOO_LARGE
