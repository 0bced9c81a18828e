"""Host-side time loop of the dynamical core, mirroring the reference's
``run_model`` (src/mod_model.f90:91-199) and ``calculate_dt``
(src/mod_model.f90:201-237).

A *stepper* is anything with the reference's dycore entry points:
``cgrid_step(dt_half)``, ``cgrid_halo()``, ``dgrid_step(dt)``, ``remap()``,
``dgrid_halo()`` and ``check_stability() -> bool``, and, for a run with
physics, ``physics_tendencies()``, ``apply_physics(dt)`` and
``physics_halo()``, and for a run with radiation ``radiative_heating(time)``
and ``radiation_halo()``.  The CUDA library (:class:`atmdyn.Dycore`) is one; the
CPU oracle used by the tests is another.
"""
from __future__ import annotations

from dataclasses import dataclass
import numpy as np

# mod_model.f90:205, a default-real literal
TIME_EPS = float(np.float32(1e-2))
NEVER = 1.0e30


@dataclass
class TimeControl:
    """The ``time_control`` namelist, in seconds (src/mod_config.f90:42-45)."""
    dt_max: float
    run_duration: float
    dt_output: float = NEVER
    dt_radiation: float = NEVER
    dt_physics: float = NEVER
    dt_remap: float = NEVER
    t_initial: float = 0.0


class Schedule:
    """``calculate_dt`` and the event flags it sets (mod_model.f90:201-237)."""

    def __init__(self, tc: TimeControl):
        self.tc = tc
        self.t_final = tc.t_initial + tc.run_duration   # mod_input.f90:243
        t0 = tc.t_initial
        self.previous_write_time = t0
        self.previous_radiation_time = t0
        self.previous_physics_time = t0
        self.previous_remap_time = t0
        self.write_this_step = False
        self.calculate_radiation_this_step = True       # mod_model.f90:73
        self.calculate_physics_this_step = True         # mod_model.f90:76
        self.remap_this_step = False

    def calculate_dt(self, time: float) -> float:
        tc = self.tc
        cand = [tc.dt_max,
                self.t_final - time,
                self.previous_write_time + tc.dt_output - time,
                self.previous_radiation_time + tc.dt_radiation - time,
                self.previous_physics_time + tc.dt_physics - time,
                self.previous_remap_time + tc.dt_remap - time]
        positive = [c for c in cand if c > 0]
        dt = min(positive)
        if abs(dt - cand[2]) < TIME_EPS:
            self.write_this_step = True
            self.previous_write_time = time + dt
        if abs(dt - cand[3]) < TIME_EPS:
            self.calculate_radiation_this_step = True
            self.previous_radiation_time = time + dt
        if abs(dt - cand[4]) < TIME_EPS:
            self.calculate_physics_this_step = True
            self.previous_physics_time = time + dt
        if abs(dt - cand[5]) < TIME_EPS:
            self.remap_this_step = True
            self.previous_remap_time = time + dt
        return dt


def schedule_for(dt: float, nsteps: int, remap_every: int) -> TimeControl:
    """Time control that takes ``nsteps`` steps of ``dt`` and remaps every
    ``remap_every`` steps."""
    return TimeControl(dt_max=dt, run_duration=dt * nsteps,
                       dt_remap=dt * remap_every if remap_every > 0 else NEVER)


@dataclass
class RunResult:
    steps: int
    time: float
    stable: bool
    remap_steps: list


def run_model(stepper, tc: TimeControl, max_steps: int | None = None,
              on_step=None, accumulate=None, write=None, physics: bool = False,
              before_remap=None, radiation: bool = False) -> RunResult:
    """``run_model`` (mod_model.f90:112-193): each step is [radiative
    heating and its halo when due], [physics tendencies when due], C-grid
    half step, halo, D-grid step,
    [apply the physics tendencies], remap if due, halo, [physics halo],
    stability check, then ``accumulate(dt)`` (accumulate_output) and, when
    the schedule says so, ``write(time_stamp)`` (write_output, stamped
    .5 (previous_write_time + time) as the reference does).  The bracketed
    physics calls run when ``physics`` is true, the radiation when
    ``radiation`` is true (at the first step and every dt_radiation);
    without it the net flux is whatever the caller set (zero by default).  ``before_remap(n)``, when
    given, runs just before the remap of step n (the tests arm the remap's
    pair trace there)."""
    sch = Schedule(tc)
    time = tc.t_initial
    n = 0
    stable = True
    remaps = []
    while time < sch.t_final:
        if sch.calculate_radiation_this_step:        # mod_model.f90:117-127
            if radiation:
                stepper.radiative_heating(time)
                stepper.radiation_halo()
            sch.calculate_radiation_this_step = False
        n += 1
        dt = sch.calculate_dt(time)
        if sch.calculate_physics_this_step:
            if physics:
                stepper.physics_tendencies()
            sch.calculate_physics_this_step = False
        stepper.cgrid_step(dt / 2.0)
        stepper.cgrid_halo()
        stepper.dgrid_step(dt)
        if physics:
            stepper.apply_physics(dt)
        if sch.remap_this_step:
            if before_remap is not None:
                before_remap(n)
            stepper.remap()
            sch.remap_this_step = False
            remaps.append(n)
        stepper.dgrid_halo()
        if physics:
            stepper.physics_halo()
        stable = bool(stepper.check_stability())
        if not stable:
            break
        time = time + dt
        if accumulate is not None:
            accumulate(dt)
        if sch.write_this_step:
            if write is not None:
                write(.5 * (sch.previous_write_time + time))
            sch.write_this_step = False
        if on_step is not None:
            on_step(n, time)
        if max_steps is not None and n >= max_steps:
            break
    return RunResult(n, time, stable, remaps)
