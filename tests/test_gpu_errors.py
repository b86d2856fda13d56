"""Error behaviour of the C ABI on the GPU (every call returns a status;
nothing faults, traps or hangs the device)."""
import ctypes

import numpy as np
import pytest

import pardiso2_b200 as P
from pardiso2_b200 import capi
from pardiso2_b200 import model as M

pytestmark = pytest.mark.gpu


def small():
    return M.sphere_model(13, 1, (2, 2, 2), seed=4)


def test_periodic_is_rejected():
    m = small()
    ctx = capi.Context(0)
    with pytest.raises(capi.P2Error) as e:
        ctx.set_grid(m.gx, m.gy, m.gz, P.params_for(m), periodic=(1, 0, 0))
    assert e.value.code == 8
    ctx.close()


def test_open_boundary_rows_are_rejected():
    m = small()
    ctx = capi.Context(0)
    ctx.set_grid(m.gx, m.gy, m.gz, P.params_for(m))
    bondm = m.bc.bondm.copy()
    # drop the wall rows of Vx on the x=0 plane of level 0
    n = m.shape[0]
    for k in range(n - 1):
        for j in range(n - 1):
            bondm[(k * n * n + j) * 4 + 1] = 0
    with pytest.raises(capi.P2Error) as e:
        ctx.set_bc(bondm, m.bc.bondv1, m.bc.bondn1)
    assert e.value.code == 8
    ctx.close()


def test_solve_before_setup_is_a_state_error():
    ctx = capi.Context(0)
    info = capi.SolveInfo()
    st = ctx.L.p2_stokes_solve_resident(ctx.h, ctypes.byref(info))
    assert st == 7
    ctx.close()


def test_nan_viscosity_reports_nan():
    m = small()
    prob = P.StokesProblem(m, tol=1e-8, max_iter=20)
    f = prob.ronurecalc()
    f["nxx"][f["nxx"].size // 2] = np.nan
    prob.set_nodes(f)
    info = prob.ctx.solve_resident(check=False)
    assert info.status == 5  # P2_ERR_NAN
    prob.close()


def test_iteration_cap_reports_not_converged():
    m = small()
    prob = P.StokesProblem(m, tol=1e-14, max_iter=2)
    prob.ronurecalc()
    info = prob.ctx.solve_resident(check=False)
    assert info.status == 4 and info.iterations == 2
    prob.close()


def test_power_law_rock_is_rejected():
    m = small()
    prob = P.StokesProblem(m)
    r = m.rocks
    with pytest.raises(capi.P2Error) as e:
        prob.ctx.upload_markers(m.markx, m.marky, m.markz, m.markt, r.n0, r.n1 * 2, r.ro)
    assert e.value.code == 8
    prob.close()


def test_context_survives_errors():
    m = small()
    prob = P.StokesProblem(m, tol=1e-8)
    with pytest.raises(capi.P2Error):
        prob.ctx.set_grid(m.gx[::-1].copy(), m.gy, m.gz, prob.params)  # decreasing lines
    # the context is still usable after a rejected call
    prob2 = P.StokesProblem(m, tol=1e-8)
    prob2.ronurecalc()
    _, info = prob2.solve_fp64()
    assert info.status == 0
    prob.close()
    prob2.close()


def test_singular_coarsest_system_reports_singular():
    """A coarsest-level cell whose six faces are all fixed-value boundary rows
    leaves its pressure with neither an equation nor a coupling in the
    coarsest system: the direct solve meets an exactly zero pivot and the
    solve returns P2_ERR_SINGULAR (a status, not a device fault)."""
    m = small()
    lv = m.levels
    c = lv.multinum
    nx, ny, off = lv.mgx[c], lv.mgy[c], lv.mgp[c]
    i, j, k = nx // 2, ny // 2, lv.mgz[c] // 2
    faces = [(i - 1, j - 1, k - 1, 1), (i, j - 1, k - 1, 1), (i - 1, j - 1, k - 1, 2), (i - 1, j, k - 1, 2),
             (i - 1, j - 1, k - 1, 3), (i - 1, j - 1, k, 3)]
    bondm = m.bc.bondm.copy()
    bondv1 = [m.bc.bondv1]
    bondn1 = [m.bc.bondn1]
    row = m.bc.bondnum
    for (a, b, d, comp) in faces:
        u = off + d * lv.mgxy[c] + a * ny + b
        assert bondm[4 * u + comp] == 0
        row += 1
        bondm[4 * u + comp] = row
        bondv1.append(np.array([[0.0, 0.0]], np.float32))
        bondn1.append(np.array([0], np.int32))
    prob = P.StokesProblem(m, tol=1e-8)
    prob.ctx.set_bc(bondm, np.concatenate(bondv1), np.concatenate(bondn1))
    prob.ronurecalc()
    with pytest.raises(capi.P2Error) as e:
        prob.ctx.solve_resident()
    assert e.value.code == 6  # P2_ERR_SINGULAR
    # the context stays usable: the original tables solve
    prob.ctx.set_bc(m.bc.bondm, m.bc.bondv1, m.bc.bondn1)
    prob.ronurecalc()
    _, info = prob.solve_fp64()
    assert info.status == 0
    prob.close()
