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
"""
from __future__ import annotations

import heapq

import torch

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
        for d in self.dyn:
            d.close()

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
