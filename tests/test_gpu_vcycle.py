"""One preconditioning V-cycle (p2_debug_vcycle: the solver's precision,
exact coarsest solve, from a zero guess) on the 65^3 workload contracts the
residual of a consistent right-hand side b = A x (A the level-0 operator of
the reference's discretisation, move3mgNew.c:796-1576): ||b - A V(b)|| is
well below ||b|| for both the FP32 and the FP64 cycle and both smoothers the
autotuner chooses from, and the FP32 and FP64 cycles agree to the FP32
cycle's rounding."""
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
def spheres65():
    m = M.config_model(2)
    prob = P.StokesProblem(m)
    f = prob.ronurecalc()
    prob.close()
    return m, f


@pytest.mark.parametrize("smoother", [1, 0])
def test_vcycle_contracts(spheres65, smoother):
    m, f = spheres65
    n = m.nodenum
    mask = unknown_mask(m.shape)
    rng = np.random.Generator(np.random.PCG64(77))
    x = np.where(mask, rng.standard_normal(4 * n), 0.0)
    prob = P.StokesProblem(m)
    prob.set_nodes(f)
    H = capi.DebugHooks(prob.ctx)
    b = H.apply(0, x)
    prob.close()
    out = {}
    for precision in (0, 1):
        prob = P.StokesProblem(m, precision=precision, smoother=smoother)
        prob.set_nodes(f)
        H = capi.DebugHooks(prob.ctx)
        v = H.vcycle(b)
        r = b - H.apply(0, v)
        prob.close()
        assert np.all(np.isfinite(v))
        red = np.linalg.norm(r[mask]) / np.linalg.norm(b[mask])
        assert red < 0.5, (precision, red)
        out[precision] = (v, red)
    # the FP32 and FP64 cycles reduce the residual alike
    assert abs(out[0][1] - out[1][1]) < 0.05 * out[1][1] + 1e-3, (out[0][1], out[1][1])
