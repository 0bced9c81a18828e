"""atm_remap_noalloc: the vertical remap for callers that cannot let the
library allocate device memory (a time loop whose device-memory budget is
fixed at start-up, or one that must avoid the device-wide synchronisation
of cudaMalloc/cudaFree mid-step).  Its scratch is a fixed file-scope device
array, so the test calls it twice in a row through the C ABI and checks
each result against the context-based atm_remap of the FP64 form, bit for
bit (the tolerance of the FP64 parity tests).  The file sorts last so that
a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from atmdyn import ic, Dycore, load

pytestmark = pytest.mark.gpu

HALO = 7
_P = ctypes.POINTER(ctypes.c_double)


def _prepared(nx=40, ny=28, nlay=9):
    """A context just before its remap: C step, C halo and D step done."""
    st = ic.bubble_case(nx, ny, nlay, 160e3, 160e3, radius=1200e3, u0=15.0)
    st.v = st.v + 3.0
    g = Dycore(st, 'fp64')
    g.cgrid_step(st.dt / 2.)
    g.cgrid_halo()
    g.dgrid_step(st.dt)
    return st, g


def test_remap_noalloc_matches_atm_remap_twice():
    import torch
    torch.cuda.set_device(0)
    lib = load()
    fn = lib.atm_remap_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int] * 3 + [_P, _P] + [ctypes.c_void_p] * 9 + [ctypes.c_void_p]

    for call in range(2):
        # a different state for each call, so that nothing of the first call
        # can make the second one pass
        st, g = _prepared(40 + 4 * call, 28 + 2 * call, 9 + call)
        names = ('dp', 'pt', 'ud', 'vd')
        before = {n: g.get(n, halo=True) for n in names}
        gzs = g.get('gz', halo=True)[0].copy()
        g.remap()
        expect = {n: g.get(n, halo=True) for n in names}

        dev_in = {n: torch.from_numpy(before[n]).cuda().contiguous() for n in names}
        dev_out = {n: dev_in[n].clone() for n in names}
        dev_gzs = torch.from_numpy(gzs).cuda().contiguous()
        ak = np.ascontiguousarray(st.ak, dtype=np.float64)
        bk = np.ascontiguousarray(st.bk, dtype=np.float64)
        torch.cuda.synchronize()
        rc = fn(st.nx, st.ny, st.nlay, ak.ctypes.data_as(_P), bk.ctypes.data_as(_P),
                dev_in['dp'].data_ptr(), dev_in['pt'].data_ptr(), dev_in['ud'].data_ptr(), dev_in['vd'].data_ptr(),
                dev_gzs.data_ptr(), dev_out['dp'].data_ptr(), dev_out['pt'].data_ptr(), dev_out['ud'].data_ptr(),
                dev_out['vd'].data_ptr(), None)
        assert rc == 0, 'atm_remap_noalloc returned %d' % rc
        torch.cuda.synchronize()
        for n in names:
            got = dev_out[n].cpu().numpy()
            assert got.shape == expect[n].shape
            # whole arrays: the interior is remapped, the halo is untouched in both
            np.testing.assert_array_equal(got, expect[n], err_msg='%s, call %d' % (n, call + 1))
        g.close()


def test_remap_noalloc_rejects_sizes_beyond_its_scratch():
    lib = load()
    fn = lib.atm_remap_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int] * 3 + [_P, _P] + [ctypes.c_void_p] * 9 + [ctypes.c_void_p]
    ak = np.full(65, 1e4)
    bk = np.linspace(1, 0, 65)
    # distinct, never dereferenced: the size check comes before any use
    ptrs = [ctypes.c_void_p(4096 * (i + 1)) for i in range(9)]
    rc = fn(1024, 1024, 64, ak.ctypes.data_as(_P), bk.ctypes.data_as(_P), *ptrs, None)
    assert rc == 6  # ATM_ERR_TOO_LARGE
