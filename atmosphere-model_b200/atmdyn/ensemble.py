"""Batched ensemble of independent dycore domains on one GPU.

The ensemble workload is many small, uneven domains (64 members of 64^2 to
512^2 columns and 20 to 64 layers).  One member's step is a dozen short
kernels, so launching members one after another leaves the GPU mostly
idle.  :class:`Ensemble` therefore

* spreads the members over several CUDA streams, balanced by cell count
  (longest-processing-time first), so kernels of different members run
  concurrently on the 148 SMs;
* captures remap cycles of every member (``remap_every`` steps, the remap
  on the last; one cycle up to a whole run) into a single CUDA graph: the
  forks and joins across the streams become graph edges, and advancing the
  whole ensemble by the captured steps is one graph launch.

Every member is a full :class:`Dycore` (FP64 or mixed form) whose kernels
are those of a single domain; the graph changes only how they are launched,
so the results are bit-identical to stepping the members one by one.

For the mixed form, :meth:`Ensemble.run_persistent` and
:meth:`Ensemble.capture_persistent` advance every member with ONE launch of
the library's persistent kernel (``atm_ensemble_*``): the stages of every
step are queues of warp-sized work items that all members take together,
stage after stage, between bounded grid-wide barriers, or, with
:meth:`Ensemble.set_schedule` (True), that each member takes on its own (a
per-member ticket, so the stages of different members overlap).  Each
member's sweeps use the strip height of an autotuned table keyed on its
grid size (:meth:`Ensemble.autotune`).  The results are again bit-identical
to stepping the members one by one.
"""
from __future__ import annotations

import ctypes
import heapq

import numpy as np
import torch

from . import _lib
from .dycore import Dycore


def balance(sizes, nbins):
    """Assign items (by size) to nbins bins, largest first into the lightest
    bin; returns the bin of each item."""
    heap = [(0, b) for b in range(nbins)]
    heapq.heapify(heap)
    out = [0] * len(sizes)
    for i in sorted(range(len(sizes)), key=lambda i: -sizes[i]):
        load, b = heapq.heappop(heap)
        out[i] = b
        heapq.heappush(heap, (load + sizes[i], b))
    return out


class Ensemble:
    def __init__(self, members, precision: str = 'mixed', nstreams: int = 8):
        self.members = list(members)
        self.dyn = [Dycore(st, precision) for st in self.members]
        self.nstreams = max(1, min(nstreams, len(self.members)))
        self.streams = [torch.cuda.Stream() for _ in range(self.nstreams)]
        self.bin = balance([st.cells for st in self.members], self.nstreams)
        for d, b in zip(self.dyn, self.bin):
            d.set_stream(self.streams[b].cuda_stream)
        self.cells = sum(st.cells for st in self.members)
        self.graph = None
        self.steps_done = 0

    def close(self):
        self.graph = None
        if getattr(self, 'ens', None) is not None:
            _lib.load().atm_ensemble_destroy(self.ens)
            self.ens = None
        for d in self.dyn:
            d.close()

    # ---- the persistent kernel (mixed form)
    def _ens(self):
        if getattr(self, 'ens', None) is None:
            lib = _lib.load()
            n = len(self.dyn)
            ctxs = (ctypes.c_void_p * n)(*[d.ctx.value for d in self.dyn])
            dts = np.ascontiguousarray([st.dt for st in self.members], dtype=np.float64)
            h = ctypes.c_void_p()
            _lib.check(lib.atm_ensemble_create(ctypes.byref(h), ctxs, dts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               n), None, 'atm_ensemble_create')
            self.ens = h
            self.strips = {}
        return self.ens

    def set_strips(self, table):
        """Strip height of the marching sweeps per member grid size, {nx: rows}."""
        lib = _lib.load()
        e = self._ens()
        for i, st in enumerate(self.members):
            rows = table.get(st.nx, 32)
            _lib.check(lib.atm_ensemble_set_strips(e, i, rows), None, 'atm_ensemble_set_strips')
        self.strips = dict(table)

    def _prepare(self, stream):
        lib = _lib.load()
        e = self._ens()
        _lib.check(lib.atm_ensemble_set_stream(e, ctypes.c_void_p(stream)), None, 'atm_ensemble_set_stream')
        torch.cuda.synchronize()
        _lib.check(lib.atm_ensemble_prepare(e), None, 'atm_ensemble_prepare')

    def run_persistent(self, nsteps: int, remap_every: int):
        """One launch of the persistent kernel: nsteps steps of every member
        from the current one (which must follow a remap when remap_every > 0,
        as the remap is due after every remap_every-th step of the launch)."""
        assert remap_every == 0 or self.steps_done % remap_every == 0
        lib = _lib.load()
        stream = torch.cuda.current_stream()
        self._prepare(stream.cuda_stream)
        _lib.check(lib.atm_ensemble_run(self.ens, nsteps, remap_every), None, 'atm_ensemble_run')
        self.steps_done += nsteps

    def set_schedule(self, dataflow: bool = False):
        """Schedule of the persistent kernel: a grid barrier after every
        stage (the default), or dataflow (members advance on their own,
        stages of different members overlap).  Measured on the 64-member
        workload, the dataflow schedule is the slower one."""
        _lib.check(_lib.load().atm_ensemble_set_schedule(self._ens(), int(bool(dataflow))), None,
                   'atm_ensemble_set_schedule')

    STAGES = ('c_mass', 'c_column', 'c_mom', 'c_halo', 'd_ring', 'd_mass', 'd_column', 'd_corners', 'd_mom',
              'remap_ring', 'remap_winds', 'remap_energy', 'd_halo')

    def profile_persistent(self, enable=True):
        """Per-stage timing of the following persistent launches (block 0's
        clock between barrier exits)."""
        _lib.check(_lib.load().atm_ensemble_profile(self._ens(), int(enable)), None, 'atm_ensemble_profile')

    def persistent_stage_ms(self):
        """{stage: milliseconds summed over the launches since profiling began}."""
        out = (ctypes.c_double * len(self.STAGES))()
        _lib.check(_lib.load().atm_ensemble_stage_ms(self._ens(), out, len(self.STAGES)), None,
                   'atm_ensemble_stage_ms')
        return {n: out[i] for i, n in enumerate(self.STAGES)}

    def barrier_timed_out(self):
        v = ctypes.c_int(0)
        _lib.check(_lib.load().atm_ensemble_status(self._ens(), ctypes.byref(v)), None, 'atm_ensemble_status')
        return bool(v.value)

    def capture_persistent(self, remap_every: int, cycles: int):
        """The persistent launch of cycles remap cycles as a CUDA graph (one
        kernel node): each replay advances every member by remap_every *
        cycles steps.  The launch must swap the time levels an even number of
        times: (remap_every + 1) * cycles even."""
        assert self.steps_done % remap_every == 0 and ((remap_every + 1) * cycles) % 2 == 0
        lib = _lib.load()
        cap = torch.cuda.Stream()
        self._prepare(cap.cuda_stream)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=cap):
            _lib.check(lib.atm_ensemble_run(self.ens, remap_every * cycles, remap_every), None, 'atm_ensemble_run')
        self.graph = g
        self.cycle = remap_every * cycles
        return g

    def autotune(self, rows=(16, 32, 64), steps: int = 2, reps: int = 2):
        """The strip height of each grid size's members: for each size (in
        turn, the others at their best so far) the fastest of ``rows`` over
        ``steps`` steps of the persistent kernel without remap, timed on the
        device; the members' states are restored afterwards.  Returns the
        table {nx: rows}."""
        assert steps % 2 == 0  # the time levels come back where they were
        saved = []
        for d in self.dyn:
            buf = torch.empty(d.state_bytes() // 8, dtype=torch.float64, device='cuda')
            d.state_save(buf.data_ptr())
            saved.append(buf)
        torch.cuda.synchronize()
        lib = _lib.load()
        table = {st.nx: 32 for st in self.members}
        done = self.steps_done
        timings = {}
        for nx in sorted(table):
            best = None
            for r in rows:
                trial = dict(table)
                trial[nx] = r
                self.set_strips(trial)
                ms = []
                for _ in range(reps):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    self._prepare(torch.cuda.current_stream().cuda_stream)
                    e0.record()
                    _lib.check(lib.atm_ensemble_run(self.ens, steps, 0), None, 'atm_ensemble_run')
                    e1.record()
                    torch.cuda.synchronize()
                    ms.append(e0.elapsed_time(e1))
                t = min(ms)
                timings[(nx, r)] = t
                if best is None or t < best[0]:
                    best = (t, r)
            table[nx] = best[1]
        for d, buf in zip(self.dyn, saved):
            d.state_load(buf.data_ptr())
        torch.cuda.synchronize()
        self.steps_done = done
        self.set_strips(table)
        self.autotune_ms = timings
        return table

    def _cycle(self, remap_every):
        for _ in range(remap_every):
            self.steps_done += 1
            for st, d in zip(self.members, self.dyn):
                d.step(st.dt, remap=self.steps_done % st.remap_every == 0, check_stable=False)

    def step_eager(self, nsteps):
        """Advance every member by nsteps, launching kernel by kernel."""
        for _ in range(nsteps):
            self.steps_done += 1
            for st, d in zip(self.members, self.dyn):
                d.step(st.dt, remap=self.steps_done % st.remap_every == 0, check_stable=False)

    def capture(self, remap_every: int, cycles: int | None = None):
        """Capture remap cycles of every member into one CUDA graph (the
        members must share remap_every, and capture starts right after a
        remap).  A step and a remap each swap a member's two time levels;
        the graph holds an even number of swaps (cycles defaults to one
        cycle when remap_every is odd, two otherwise, and must be even when
        remap_every is even) so that each replay starts from the buffers
        the capture started from."""
        assert all(st.remap_every == remap_every for st in self.members)
        assert self.steps_done % remap_every == 0
        unit = 1 if (remap_every + 1) % 2 == 0 else 2
        cycles = unit if cycles is None else cycles
        assert cycles >= 1 and cycles % unit == 0
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream()
        start = self.steps_done
        with torch.cuda.graph(g, stream=cap):
            for s in self.streams:
                s.wait_stream(cap)
            for _ in range(cycles):
                self._cycle(remap_every)
            for s in self.streams:
                cap.wait_stream(s)
        # capture records the launches without running them
        self.steps_done = start
        self.graph = g
        self.cycle = remap_every * cycles
        return g

    def replay(self, cycles: int):
        for _ in range(cycles):
            self.graph.replay()
            self.steps_done += self.cycle

    def synchronize(self):
        torch.cuda.synchronize()

    def stable(self):
        return all(d.check_stability() for d in self.dyn)
