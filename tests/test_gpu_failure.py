"""Failure detection without a GPU fault.

* The tile kernels' bounded mbarrier wait, made to run out on a barrier
  that nothing completes, gives up after its poll limit and reports it; the
  context stays usable.
* A non-finite value planted in the state (the host makes the failure) is
  reported by the stability check and by the step's own flags; a context
  with a clean state steps normally afterwards.
"""
import ctypes

import numpy as np
import pytest

from atmdyn import ic, Dycore, _lib

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_the_device_stays_usable():
    lib = _lib.load()
    t = ctypes.c_int(-1)
    assert lib.atm_device_wait_check(64, ctypes.byref(t)) == 0
    assert t.value == 1
    st = ic.bubble_case(32, 24, 6, 100e3, 100e3, seed=1)
    g = Dycore(st)
    assert g.step(st.dt, remap=True, check_stable=True)
    assert np.isfinite(g.get('dp')).all()


@pytest.mark.parametrize('field', ['dp', 'pt', 'ud', 'vd'])
def test_nonfinite_state_is_reported(field):
    st = ic.bubble_case(32, 24, 6, 100e3, 100e3, seed=2)
    a = {'dp': st.dp, 'pt': st.pt, 'ud': st.u, 'vd': st.v}[field].copy()
    a[3, 10, 12] = np.nan
    setattr(st, {'dp': 'dp', 'pt': 'pt', 'ud': 'u', 'vd': 'v'}[field], a)
    g = Dycore(st)
    assert not g.check_stability()
    assert not g.step(st.dt, remap=False, check_stable=True)
    g.close()
    clean = ic.bubble_case(32, 24, 6, 100e3, 100e3, seed=2)
    h = Dycore(clean)
    assert h.step(clean.dt, remap=True, check_stable=True)
