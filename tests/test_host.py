"""Host-side logic and the C ABI surface, without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from atmdyn import ic, model
from atmdyn import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()  # loads libatmdyn.so (no CUDA call is made)
    hdr = open(os.path.join(ROOT, 'include', 'atmdyn.h')).read()
    declared = set(re.findall(r'^(?:int|const char\*)\s+(atm_\w+)\(', hdr, flags=re.M))
    assert len(declared) >= 20
    for name in declared:
        getattr(lib, name)
    assert set(_lib.EXPORTS) == declared
    assert lib.atm_version().decode().startswith('libatmdyn')


def test_create_rejects_bad_arguments_without_touching_the_gpu():
    lib = _lib.load()
    ctx = ctypes.c_void_p()
    ak = np.full(5, 1e4)
    bk = np.linspace(1, 0, 5)
    P = ctypes.POINTER(ctypes.c_double)
    # nx below the halo width, nlay too small, bad precision: all ATM_ERR_ARG
    for nx, ny, nl, prec in ((6, 16, 4, 0), (16, 16, 2, 0), (16, 16, 4, 7), (16, 16, 200, 0)):
        rc = lib.atm_create(ctypes.byref(ctx), nx, ny, nl, 1e3, 1e3, ak.ctypes.data_as(P), bk.ctypes.data_as(P),
                            9.8, 1e-4, 0.1, 0.0, prec, 0)
        assert rc == 1
    # the wait check's poll limit is bounded before any launch
    t = ctypes.c_int(-1)
    for polls in (0, -5, 100001):
        assert lib.atm_device_wait_check(polls, ctypes.byref(t)) == 1 and t.value == -1


def test_schedule_matches_calculate_dt():
    """calculate_dt (src/mod_model.f90:201-237): remap every 5 steps of 60 s,
    a last step shortened to reach t_final exactly."""
    tc = model.schedule_for(60.0, 12, 5)
    sch = model.Schedule(tc)
    t, remaps, steps = 0.0, [], 0
    while t < sch.t_final:
        steps += 1
        dt = sch.calculate_dt(t)
        if sch.remap_this_step:
            remaps.append(steps)
            sch.remap_this_step = False
        t += dt
    assert steps == 12 and remaps == [5, 10] and t == 720.0
    tc = model.TimeControl(dt_max=120.0, run_duration=1000.0, dt_remap=300.0)
    sch = model.Schedule(tc)
    t, dts = 0.0, []
    while t < sch.t_final:
        dts.append(sch.calculate_dt(t))
        t += dts[-1]
    # output/remap events shorten steps so that events land exactly
    assert dts == [120.0, 120.0, 60.0, 120.0, 120.0, 60.0, 120.0, 120.0, 60.0, 100.0]


class _CountingStepper:
    def __init__(self, unstable_at=None):
        self.calls = []
        self.unstable_at = unstable_at

    def cgrid_step(self, dt):
        self.calls.append(('c', dt))

    def cgrid_halo(self):
        self.calls.append(('ch',))

    def dgrid_step(self, dt):
        self.calls.append(('d', dt))

    def remap(self):
        self.calls.append(('r',))

    def dgrid_halo(self):
        self.calls.append(('dh',))

    def check_stability(self):
        n = sum(1 for c in self.calls if c[0] == 'd')
        return self.unstable_at is None or n < self.unstable_at


def test_run_model_call_order_and_instability_exit():
    s = _CountingStepper()
    r = model.run_model(s, model.schedule_for(30.0, 8, 4))
    assert r.steps == 8 and r.remap_steps == [4, 8] and r.stable
    assert s.calls[:5] == [('c', 15.0), ('ch',), ('d', 30.0), ('dh',), ('c', 15.0)]
    i = s.calls.index(('r',))
    assert s.calls[i - 1] == ('d', 30.0) and s.calls[i + 1] == ('dh',)
    s = _CountingStepper(unstable_at=3)
    r = model.run_model(s, model.schedule_for(30.0, 8, 4))
    assert not r.stable and r.steps == 3


class _PhysicsRadiationStepper(_CountingStepper):
    def physics_tendencies(self):
        self.calls.append(('pt',))

    def apply_physics(self, dt):
        self.calls.append(('pa', dt))

    def physics_halo(self):
        self.calls.append(('ph',))

    def radiative_heating(self, time):
        self.calls.append(('rad', time))

    def radiation_halo(self):
        self.calls.append(('radh',))


def test_run_model_radiation_schedule():
    """run_model (mod_model.f90:112-199) with radiation: radiative heating
    and its halo at the first step and whenever dt_radiation has passed,
    before the physics tendencies and the C-grid step of that step, at the
    step's start time; none without radiation=True."""
    tc = model.TimeControl(dt_max=60.0, run_duration=600.0, dt_radiation=240.0, dt_physics=120.0, dt_remap=300.0)
    s = _PhysicsRadiationStepper()
    r = model.run_model(s, tc, physics=True, radiation=True)
    assert r.steps == 10 and r.stable
    rad = [c[1] for c in s.calls if c[0] == 'rad']
    assert rad == [0.0, 240.0, 480.0]
    for t in rad:
        i = s.calls.index(('rad', t))
        assert s.calls[i + 1] == ('radh',)
        assert s.calls[i + 2][0] in ('pt', 'c')  # then the physics tendencies when due, or the C-grid step
    assert s.calls[:4] == [('rad', 0.0), ('radh',), ('pt',), ('c', 30.0)]
    s = _PhysicsRadiationStepper()
    model.run_model(s, tc, physics=True, radiation=False)
    assert not any(c[0] in ('rad', 'radh') for c in s.calls)


def test_initial_conditions_are_hydrostatic_and_seeded():
    a = ic.jet_case(32, 32, 8, 50e3, 50e3, width=200e3, seed=5)
    b = ic.jet_case(32, 32, 8, 50e3, 50e3, width=200e3, seed=5)
    c = ic.jet_case(32, 32, 8, 50e3, 50e3, width=200e3, seed=6)
    np.testing.assert_array_equal(a.pt, b.pt)
    assert not np.array_equal(a.pt, c.pt)
    assert np.allclose(a.dp.sum(axis=0), 9e4)
    assert (a.pt > 0).all() and np.isfinite(a.u).all()
    st = ic.config(1)
    assert (st.nx, st.ny, st.nlay, st.dt, st.remap_every, st.nsteps) == (128, 128, 20, 60.0, 5, 100)
    assert st.ak[0] == 1e4 and st.bk[0] == 1.0 and st.bk[-1] == 0.0


def test_ensemble_balance():
    """Longest-processing-time assignment of the ensemble members to streams."""
    from atmdyn.ensemble import balance
    sizes = [64 ** 2 * 20, 512 ** 2 * 64, 128 ** 2 * 32, 256 ** 2 * 48, 64 ** 2 * 64, 512 ** 2 * 20, 256 ** 2 * 20]
    b = balance(sizes, 3)
    assert len(b) == len(sizes) and set(b) <= {0, 1, 2}
    loads = [sum(s for s, k in zip(sizes, b) if k == j) for j in range(3)]
    assert max(loads) <= sum(sizes) / 3 + max(sizes)
    assert b[1] != b[5]  # the two largest members run on different streams


class _TapeRecorder:
    """Stands in for a Dycore in the tape recording of atmdyn.adjoint."""

    def __init__(self):
        self.calls = []

    def tape_bytes(self):
        return 64

    def step_tape(self, dt, remap, ptr):
        self.calls.append(bool(remap))


def test_recompute_stops_before_the_last_remap_only():
    """A backward's recompute (final_state=False) skips the remap of the
    segment's last step only, whose tape already holds the pre-remap state;
    the forward's recording keeps every remap (its final state is the
    segment's output)."""
    torch = pytest.importorskip('torch')
    from atmdyn.adjoint import _record
    like = torch.zeros(1, dtype=torch.float64)
    remaps = [False, True, False, True]
    for final_state, want in ((True, remaps), (False, [False, True, False, False])):
        dyn = _TapeRecorder()
        tapes = _record(dyn, 30.0, remaps, like, final_state=final_state)
        assert dyn.calls == want
        assert len(tapes) == len(remaps) and all(t.numel() == 8 for t in tapes)
    dyn = _TapeRecorder()
    _record(dyn, 30.0, [False, False], like, final_state=False)
    assert dyn.calls == [False, False]


def test_math_tables_reproducible():
    """atm_math_tables.h and atm_kappa_tables.h are what their generator writes."""
    import subprocess
    import sys
    import os
    here = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'atmosphere-model_b200', 'csrc')
    for args, name in (([], 'atm_math_tables.h'), (['--kappa'], 'atm_kappa_tables.h')):
        got = subprocess.run([sys.executable, 'gen_math_tables.py'] + args, cwd=here, check=True,
                             capture_output=True, text=True).stdout
        with open(os.path.join(here, name)) as f:
            assert got == f.read(), name
