"""pardiso2_b200 — B200-native Stokes multigrid behind the Pardiso2 entry points.

The product is the CUDA library libp2cuda.so (sm_100a) with a plain C ABI
(include/p2cuda.h).  This package holds its sources (csrc/), the in-tree
build (build.py), a ctypes binding (capi.py), the reference-layout model
generator used by tests and benchmarks (model.py), and StokesProblem, a thin
host mirror of the reference's two entry points for one model:
  ronurecalc()  -> marker -> node fields   (pardiso/mark3mg.c:630)
  vpiterate()   -> Stokes solve            (pardiso/move3mgNew.c:1791)
"""
from __future__ import annotations

from typing import Dict, Optional

import numpy as np

from . import capi, model
from .capi import Context, P2Error, Params, SolveInfo, default_params

__all__ = ["capi", "model", "Context", "P2Error", "Params", "SolveInfo", "default_params", "StokesProblem",
           "params_for"]


def params_for(m: "model.Model", precision: int = 0, tol: float = 1e-8, npre=None, npost=None, omega: float = 0.7,
               restart: int = 16, max_iter: int = 200, use_graphs: bool = True, smoother: int = 1,
               sweep_growth: int = 1, sweep_max: int = 64) -> Params:
    """C-ABI parameters for a model (its mode.t3c-equivalent knobs plus solver controls)."""
    p = default_params()
    sp = m.params
    p.p0koef, p.p1koef, p.p2koef, p.v0koef, p.v1koef = sp.p0koef, sp.p1koef, sp.p2koef, sp.v0koef, sp.v1koef
    p.nubeg, p.nuend, p.nukoef = sp.nubeg, sp.nuend, sp.nukoef
    p.gxkoef, p.gykoef, p.gzkoef, p.pinit = sp.gx, sp.gy, sp.gz, sp.pinit
    p.pxinit, p.pyinit, p.pzinit = sp.pin
    p.viscmod = sp.viscmod
    p.multinum = m.multinum
    nl = m.multinum + 1
    for l in range(nl):
        p.npre[l] = (npre[l] if npre is not None else min(sweep_max, 4 * sweep_growth ** l))
        p.npost[l] = (npost[l] if npost is not None else min(sweep_max, 4 * sweep_growth ** l))
    p.tol, p.max_iter, p.precision, p.restart, p.omega = tol, max_iter, precision, restart, omega
    p.use_graphs = 1 if use_graphs else 0
    p.smoother = smoother
    return p


class StokesProblem:
    """One model resident on one GPU: grid + boundary tables + markers."""

    def __init__(self, m: "model.Model", device: int = 0, **kw):
        self.m = m
        self.ctx = Context(device)
        self.params = params_for(m, **kw)
        self.ctx.set_grid(m.gx, m.gy, m.gz, self.params)
        self.ctx.set_bc(m.bc.bondm, m.bc.bondv1, m.bc.bondn1)

    def close(self):
        self.ctx.close()

    def ronurecalc(self, init: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        n = self.m.nodenum
        keys = ("nu", "ro", "nxx", "nxy", "nxz", "nyz")
        f = {k: (np.array(init[k], np.float32) if init is not None else np.zeros(n, np.float32)) for k in keys}
        r = self.m.rocks
        return self.ctx.ronurecalc(self.m.markx, self.m.marky, self.m.markz, self.m.markt, r.n0, r.n1, r.ro, f)

    def set_nodes(self, f: Dict[str, np.ndarray]):
        self.ctx.set_nodes(f)

    def vpiterate(self, vx=None, vy=None, vz=None, pr=None):
        """Solve; returns (solution dict of float/double host arrays, SolveInfo)."""
        n = self.m.nodenum
        vx = np.zeros(n, np.float32) if vx is None else vx
        vy = np.zeros(n, np.float32) if vy is None else vy
        vz = np.zeros(n, np.float32) if vz is None else vz
        pr = np.zeros(n, np.float64) if pr is None else pr
        info = self.ctx.stokes_solve(vx, vy, vz, pr)
        return {"vx": vx, "vy": vy, "vz": vz, "pr": pr}, info

    def autotune(self, trial_iters: int = 16):
        """Choose smoother and sweep schedule for this model (p2_autotune)."""
        return self.ctx.autotune(trial_iters)

    def solve_fp64(self):
        """Solve on the resident node fields; FP64 solution arrays + info."""
        info = self.ctx.solve_resident()
        return self.ctx.solution(self.m.nodenum), info
