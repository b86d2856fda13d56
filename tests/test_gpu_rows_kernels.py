"""The operator rows (x-, y-, z-Stokes and continuity rows of a level,
move3mgNew.c:796-1576) from the two row kernels: k_rows (one thread per
node, reads from global memory) and k_rows_zm (z-marching columns with rings
of node and stress planes in shared memory; the default for FP32 rows on
large levels).  Both evaluate the same expressions, so A x agrees to
rounding (a stress read back from shared memory is not contracted into a
fused multiply-add with the difference that uses it), on grids whose blocks
are partial along every axis; and whole solves with either kernel take the
same iterations (within one) to the same solution (within 1e-6)."""
import numpy as np
import pytest

import pardiso2_b200 as P
from pardiso2_b200 import capi
from pardiso2_b200 import model as M

pytestmark = pytest.mark.gpu


def unknown_mask(shape):
    nx, ny, nz = shape
    k, i, j = np.meshgrid(np.arange(nz), np.arange(nx), np.arange(ny), indexing="ij")
    valid = [(i > 0) & (j > 0) & (k > 0), (j < ny - 1) & (k < nz - 1), (i < nx - 1) & (k < nz - 1),
             (i < nx - 1) & (j < ny - 1)]
    return np.stack([v.reshape(-1) for v in valid], axis=1).reshape(-1)


@pytest.fixture(scope="module")
def spheres_odd():
    """Level 0 of 113 x 97 x 65 nodes (partial blocks of every kernel along
    every axis), level 1 of 59 x 51 x 35."""
    m = M.random_spheres_model(113, 4, 10, (1e-2, 1e3), markers=(2, 2, 2), seed=9, name="spheres113",
                               shape=(113, 97, 65))
    prob = P.StokesProblem(m)
    f = prob.ronurecalc()
    prob.close()
    return m, f


@pytest.mark.parametrize("level", [0, 1])
def test_row_kernels_agree(spheres_odd, level):
    m, f = spheres_odd
    lv = m.levels
    shape = (lv.mgx[level], lv.mgy[level], lv.mgz[level])
    n = shape[0] * shape[1] * shape[2]
    rng = np.random.Generator(np.random.PCG64(300 + level))
    x = np.where(unknown_mask(shape), rng.standard_normal(4 * n), 0.0)
    prob = P.StokesProblem(m)
    prob.set_nodes(f)
    H = capi.DebugHooks(prob.ctx)
    out = {}
    for variant in (1, 2):
        H.rows_kernel(variant)
        out[variant] = H.apply(level, x)
    H.rows_kernel(0)
    prob.close()
    ref = out[1]
    scale = np.abs(ref).max()
    assert scale > 0
    d = np.abs(out[2] - ref).max() / scale
    assert d < 1e-13, d


def test_solves_with_row_kernels_agree(spheres_odd):
    m, f = spheres_odd
    sols, its = [], []
    for variant in (1, 2):
        prob = P.StokesProblem(m, tol=1e-8, sweep_growth=2)
        prob.set_nodes(f)
        capi.DebugHooks(prob.ctx).rows_kernel(variant)
        sol, info = prob.solve_fp64()
        prob.close()
        assert info.status == 0, info.as_dict()
        sols.append(sol)
        its.append(info.iterations)
    # the FP32 cycle's rounding differs between the kernels, and the mixed
    # solve's iteration count can move by one with it
    assert abs(its[0] - its[1]) <= 1, its
    for k in ("vx", "vy", "vz", "pr"):
        d = np.linalg.norm(sols[0][k] - sols[1][k]) / np.linalg.norm(sols[1][k])
        assert d < 1e-6, (k, d)
