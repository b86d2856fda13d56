"""Converged solutions of the larger benchmark workloads, as test fixtures.

The oracle port (oracle/libp2oracle.so: the C restatement of the reference's
discretisation, pinned to the reference's own exact discrete solutions by
tests/test_oracle_golden.py) solves the seeded spheres129 (config 3) and
layered257 (config 5) models to a true relative residual of 1e-10 (at
contrast 1e6 the FP64 iteration levels off near 1.2e-11).  A full
solution is 70 MB (129^3) or 540 MB (257^3), so each fixture keeps:
  sub_{pr,vx,vy,vz}   the solution on the sub-lattice of every `stride`-th
                      node along each axis (stride 4 at 129^3, 8 at 257^3:
                      33^3 nodes), float64
  norm_{pr,vx,vy,vz}  the 2-norm of the full field (entries that are not
                      unknowns are zero)
  sum_{pr,vx,vy,vz}   the sum of the full field
  hist                the oracle's relative residual per outer iteration
  oracle_smoother, oracle_sweeps   the oracle's smoother and sweeps per level
  stride, shape
GPU tests and bench.py compare the GPU solution on the same sub-lattice
(relative L2 per field) and its full-field norms against these.

Usage: OMP_NUM_THREADS=<cores> python tests/golden/make_solution_fixtures.py [3] [5]
"""
import ctypes as C
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from oracle import oracle as O  # noqa: E402
from pardiso2_b200 import model as M  # noqa: E402

KEYS = ("pr", "vx", "vy", "vz")
# workload -> (fixture file, sub-lattice stride, oracle smoother, sweeps per level)
CASES = {
    3: ("spheres129_solution.npz", 4, 1, lambda nl: [4 * 2 ** l for l in range(nl)]),
    5: ("layered257_solution.npz", 8, 2, lambda nl: [4 * 2 ** l for l in range(nl)]),
}
TOL = 1e-10


def sub_lattice(field, shape, stride):
    """field in the node layout (y fastest, then x, then z) -> the nodes
    with every coordinate a multiple of stride, as a flat float64 array."""
    nx, ny, nz = shape
    a = np.asarray(field, np.float64).reshape(nz, nx, ny)
    return np.ascontiguousarray(a[::stride, ::stride, ::stride]).reshape(-1)


def make(cfg):
    name, stride, smoother, sweeps = CASES[cfg]
    t0 = time.time()
    m = M.config_model(cfg)
    f = O.ronurecalc(m)
    nl = m.multinum + 1
    C.c_int.in_dll(O.lib(), "p2o_smoother").value = smoother
    s = O.OracleSolver(m, npre=sweeps(nl), npost=sweeps(nl))
    s.set_fields(f)
    hist = s.solve(tol=TOL, max_cycles=400, restart=16)
    sol = s.solution()  # entries that are not unknowns are zero
    s.close()
    if hist[-1] > TOL:
        raise RuntimeError("oracle did not reach %g: %s" % (TOL, hist[-5:]))
    out = {"stride": np.int64(stride), "shape": np.array(m.shape, np.int64), "hist": hist,
           "oracle_smoother": np.int64(smoother), "oracle_sweeps": np.array(sweeps(nl), np.int64)}
    for k in KEYS:
        out["sub_" + k] = sub_lattice(sol[k], m.shape, stride)
        out["norm_" + k] = np.float64(np.linalg.norm(sol[k]))
        out["sum_" + k] = np.float64(sol[k].sum())
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("%s: %d iterations, residual %.2e, %.0f s" % (name, len(hist) - 1, hist[-1], time.time() - t0), flush=True)


if __name__ == "__main__":
    for a in sys.argv[1:] or ["3", "5"]:
        make(int(a))
