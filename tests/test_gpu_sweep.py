"""The fused smoother sweep (smoother 5, k_vanka_sweep: both colours of a
sweep in one launch, z-marching tiles with the red-updated planes held in
shared memory) against the two colour passes of the default smoother
(smoother 1: k_vanka_stored per colour, each followed by the boundary rows).
Both apply the same update to every cell in the same order of colours, so the states after a few sweeps
agree to rounding (the fused kernel's arithmetic is the same expression
sequence; only the compiler's contraction may differ), and whole solves take
the same iterations and reach the same solution."""
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


def level_shape(m, l):
    lv = m.levels
    return (lv.mgx[l], lv.mgy[l], lv.mgz[l])


def smooth_with(m, fields, smoother, precision, level, sweeps, b, x):
    prob = P.StokesProblem(m, smoother=smoother, precision=precision)
    prob.set_nodes(fields)
    out = capi.DebugHooks(prob.ctx).smooth(level, sweeps, b, x)
    prob.close()
    return out


@pytest.fixture(scope="module")
def spheres113():
    m = M.random_spheres_model(113, 4, 10, (1e-2, 1e3), markers=(2, 2, 2), seed=9, name="spheres113",
                               shape=(113, 97, 65))
    prob = P.StokesProblem(m)
    f = prob.ronurecalc()
    prob.close()
    return m, f


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("sweeps", [2, 3])
def test_fused_sweep_matches_colour_passes(spheres113, precision, sweeps):
    m, f = spheres113
    for level in (0, 1):
        shape = level_shape(m, level)
        n = shape[0] * shape[1] * shape[2]
        rng = np.random.Generator(np.random.PCG64(100 + level))
        mask = unknown_mask(shape)
        b = np.where(mask, rng.standard_normal(4 * n), 0.0)
        x = np.where(mask, rng.standard_normal(4 * n) * 1e-2, 0.0)
        fused = smooth_with(m, f, 5, precision, level, sweeps, b, x)
        split = smooth_with(m, f, 1, precision, level, sweeps, b, x)
        assert np.all(np.isfinite(fused))
        tol = 1e-5 if precision == 0 else 1e-12
        for c in range(4):
            d = np.linalg.norm(fused[c::4] - split[c::4]) / np.linalg.norm(split[c::4] - x[c::4])
            assert d < tol, (level, c, d)


def test_fused_and_split_solves_agree(spheres113):
    m, f = spheres113
    sols, its = [], []
    for smoother in (5, 1):
        prob = P.StokesProblem(m, smoother=smoother, tol=1e-8, sweep_growth=2)
        prob.set_nodes(f)
        sol, info = prob.solve_fp64()
        prob.close()
        assert info.status == 0, info.as_dict()
        sols.append(sol)
        its.append(info.iterations)
    assert abs(its[0] - its[1]) <= 1, its
    for k in ("vx", "vy", "vz", "pr"):
        d = np.linalg.norm(sols[0][k] - sols[1][k]) / np.linalg.norm(sols[1][k])
        assert d < 1e-6, (k, d)
