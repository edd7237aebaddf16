"""Independent designs advanced together on one GPU.

A single design on these grids is a chain of thousands of short, latency-bound
kernels that leaves most of the B200 idle.  `DesignSweep` runs several
designs (different grids, volume fractions and load sets allowed) side by
side: every design owns its libtof context, its CUDA stream and a host thread
that issues its iteration, so the kernels of different designs overlap on
the device.  libtof releases the Python GIL inside every call, and a design's
iteration only synchronises its own stream.  Results are identical to running
the designs one after another (every reduction in libtof has a fixed order).

After each design iteration the design's modes are ranked by effective mass
in the thrust direction (sims/modal_participation.py:37-57, 89-94).
"""
from __future__ import annotations

import threading
import time

import torch

from .modal import EXCITABLE_FRAC


class DesignSweep:
    """designs: list of (name, geom, fem, opt) with opt a
    tof_b200.topopt.SIMPOptimizer built on fem (see workloads.sweep_designs)."""

    def __init__(self, designs):
        self.designs = list(designs)
        torch.cuda.synchronize()                   # set-up work on the creating stream is done
        self.streams = [torch.cuda.Stream() for _ in self.designs]
        self.ranking = {name: [] for name, *_ in self.designs}
        self.errors = []

    def _one(self, i):
        name, geom, fem, opt = self.designs[i]
        try:
            with torch.cuda.stream(self.streams[i]):
                opt.step()
                if opt.modal_active and opt.X4 is not None:
                    n = opt.n_modes_track
                    eff = opt.ctx.effective_mass(opt.X4[:n].contiguous(), 2)
                    order = sorted(range(n), key=lambda k: -eff[k])
                    first = next((k for k in range(n) if eff[k] >= EXCITABLE_FRAC), None)
                    self.ranking[name].append(dict(order=order, eff=list(map(float, eff)), first_excitable=first))
        except Exception as e:            # reported to the caller after all threads joined
            self.errors.append((name, e))

    def step(self, concurrent: bool = True) -> float:
        """One design iteration of every design; returns the wall time (s)
        from the first launch to the last design's completion."""
        self.errors = []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if concurrent:
            threads = [threading.Thread(target=self._one, args=(i,)) for i in range(len(self.designs))]
            for t in threads:
                t.start()
            for t in threads:
                t.join()
        else:
            for i in range(len(self.designs)):
                self._one(i)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if self.errors:
            name, e = self.errors[0]
            raise RuntimeError(f"design {name}: {e}") from e
        return dt

    def histories(self):
        return {name: opt.history for name, _, _, opt in self.designs}
