"""Refinement that moves with an oscillating body.

The reference's dynamic remeshing (Grid_Manager_dynamic.cpp) is not
compiled into its step, so a moving body there keeps a static mesh.  Here a
direct-forcing sphere oscillating along y is run in windows of a few coarse
steps: each window's lattice is classified on the device with its
refinement boxes and forcing band around the displacements the sphere takes
during that window only (`df_sphere_case(window=...)`), and the state of the
previous window is carried onto it (`mt_case_remap`).  The finest level
then covers the sphere instead of its whole swept path.  The markers follow
the path of the whole run; the forcing step counter carries over, so the
markers' path continues across windows.
"""
from __future__ import annotations

import time

import numpy as np

from .case import df_sphere_case
from .serving import AMPLITUDE, PERIOD


def path_window(t0: int, t1: int, amp: float, period: int) -> tuple:
    """Smallest and largest centre displacement y = amp sin(2 pi t / period)
    over the finest steps t0 .. t1 (inclusive)."""
    t = np.arange(t0, t1 + 1)
    y = amp * np.sin(2.0 * np.pi * (t % period) / period)
    return float(y.min()), float(y.max())


class MovingSphere:
    """An oscillating direct-forcing sphere whose refinement follows it."""

    def __init__(self, ctx, radius=8, max_level=3, re=150.0, u=0.1, storage="f16", window=16,
                 amplitude=AMPLITUDE, period=PERIOD, scaling="standard", storage_shift=None):
        self.ctx = ctx
        self.kw = dict(radius=radius, max_level=max_level, re=re, u=u, oscillating=True, period=period,
                       amplitude=amplitude, mesh="device")
        self.r, self.L = int(radius), max_level
        self.amp = amplitude * int(radius)
        self.period = period
        self.storage = storage
        self.window = window
        self.scaling = scaling
        self.storage_shift = storage_shift
        self.mgr = None
        self.coarse = 0          # coarse steps done
        self.force = np.zeros(4)  # accumulated over the finished windows
        self.remesh_s = 0.0
        self.remesh_times = []   # per re-mesh: (build, remap, release) seconds
        self.windows = 0

    def _case(self):
        s = 1 << self.L
        t0 = self.coarse * s
        t1 = (self.coarse + self.window) * s
        return df_sphere_case(window=path_window(t0, t1, self.amp, self.period), **self.kw)

    def step(self, n: int):
        """n coarse steps, re-meshing at every window boundary."""
        from .lbm import LBM_Manager
        while n > 0:
            if self.mgr is None or self.coarse % self.window == 0:
                # the previous window's steps finish first (not re-meshing time)
                self.ctx.synchronize()
                t = time.perf_counter()
                new = LBM_Manager(self.ctx, self._case(), self.storage, schedule="fused", scaling=self.scaling,
                                  storage_shift=self.storage_shift)
                self.ctx.synchronize()
                t1 = time.perf_counter()
                if self.mgr is not None:
                    new.remap_from(self.mgr, counts=False)
                    self.ctx.synchronize()
                    t2 = time.perf_counter()
                    self.force += self.mgr.force()
                    self.mgr.close()
                else:
                    t2 = t1
                self.mgr = new
                self.ctx.synchronize()
                t3 = time.perf_counter()
                self.remesh_s += t3 - t
                self.remesh_times.append((t1 - t, t2 - t1, t3 - t2))
                self.windows += 1
            k = min(n, self.window - self.coarse % self.window)
            self.mgr.fluidSimulate(k)
            self.coarse += k
            n -= k

    def total_force(self) -> np.ndarray:
        """(fx, fy, fz, forcing steps) accumulated over the whole run."""
        return self.force + (self.mgr.force() if self.mgr is not None else 0.0)

    def close(self):
        if self.mgr is not None:
            self.mgr.close()
            self.mgr = None
