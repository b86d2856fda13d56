"""CUDA path (through the C ABI) vs the reference's golden vectors and the
oracle restatement.

Tolerances:
  * marker -> node fields: bit-exact (the same float accumulation order as
    the single-threaded reference);
  * level-0 operator rows: 1e-13 relative (FP64, same inputs);
  * coarse rows / restriction: 2e-7 (coarse viscosities are float);
  * solutions: 1e-6 relative L2 per field at a relative residual of 1e-8,
    for the FP32-V-cycle (mixed) and the FP64-V-cycle solves.
"""
import os

import numpy as np
import pytest

import pardiso2_b200 as P
from pardiso2_b200 import capi
from pardiso2_b200 import model as M
from tests.golden.make_golden import CASES, probe_vector
from tests.test_oracle_golden import load_case, pin_mask, rel

pytestmark = pytest.mark.gpu
FIELDS = ("nu", "ro", "nxx", "nxy", "nxz", "nyz")


@pytest.fixture(scope="module", params=sorted(CASES))
def gcase(request):
    m, g = load_case(request.param)
    prob = P.StokesProblem(m, tol=1e-10)
    yield m, g, prob
    prob.close()


def test_ronurecalc_bit_exact_vs_reference(gcase):
    m, g, prob = gcase
    f = prob.ronurecalc()
    for k in FIELDS:
        assert np.array_equal(f[k], g["node_" + k]), k


def test_operator_rows_vs_reference(gcase):
    m, g, prob = gcase
    prob.set_nodes({k: g["node_" + k] for k in FIELDS})
    H = capi.DebugHooks(prob.ctx)
    for lev in range(m.multinum):
        x = probe_vector(m.levels.mgn[lev], lev)
        y = H.apply(lev, x)
        has = g["op_rows_lev%d" % lev]
        ref = g["op_lev%d" % lev]
        err = np.abs(y - ref)[has].max() / np.abs(ref[has]).max()
        assert err < (1e-13 if lev == 0 else 2e-7), (lev, err)


def test_transfers_vs_reference(gcase):
    m, g, prob = gcase
    prob.set_nodes({k: g["node_" + k] for k in FIELDS})
    H = capi.DebugHooks(prob.ctx)
    for lc in range(1, m.multinum + 1):
        nc, nf = m.levels.mgn[lc], m.levels.mgn[lc - 1]
        got = H.restrict(lc, g["restrict_in_lev%d" % lc], nc, compat=False)
        ref = g["restrict_lev%d" % lc]
        mask = pin_mask(m, lc)
        assert np.abs(got - ref)[mask].max() <= 2e-7 * np.abs(ref[mask]).max()
        got = H.prolong(lc, probe_vector(nc, 20 + lc), probe_vector(nf, 30 + lc))
        assert np.abs(got - g["prolong_lev%d" % lc]).max() <= 1e-13 * np.abs(g["prolong_lev%d" % lc]).max()


def test_coarse_viscosity_restriction_vs_reference(gcase):
    m, g, prob = gcase
    prob.set_nodes({k: g["node_" + k] for k in FIELDS})
    H = capi.DebugHooks(prob.ctx)
    nu, ro = H.level_fields(m.levels.total_nodes)
    lv = m.levels
    for l in range(1, m.multinum + 1):
        a, b = lv.mgp[l], lv.mgp[l] + lv.mgn[l]
        assert np.abs(nu[a:b] - g["level_nu"][a:b]).max() <= 2e-7 * np.abs(g["level_nu"][a:b]).max()
        assert np.abs(ro[a:b] - g["level_ro"][a:b]).max() <= 2e-7 * max(np.abs(g["level_ro"][a:b]).max(), 1.0)


@pytest.mark.parametrize("precision", [0, 1])
def test_solve_vs_reference_solution(gcase, precision):
    m, g, _ = gcase
    prob = P.StokesProblem(m, precision=precision, tol=1e-8)
    prob.set_nodes({k: g["node_" + k] for k in FIELDS})
    sol, info = prob.solve_fp64()
    prob.close()
    assert info.status == 0 and info.rel_residual <= 1e-8
    for k in ("vx", "vy", "vz", "pr"):
        assert rel(sol[k], g["sol_" + k]) < 1e-6, (k, rel(sol[k], g["sol_" + k]))


@pytest.mark.parametrize("smoother", [0, 1, 2, 3])
def test_every_smoother_reaches_the_reference_solution(gcase, smoother):
    """Diagonal and full cell-block smoothers are preconditioners only: all
    converge to the same discrete solution."""
    m, g, _ = gcase
    prob = P.StokesProblem(m, tol=1e-8, smoother=smoother, sweep_growth=2)
    prob.set_nodes({k: g["node_" + k] for k in FIELDS})
    sol, info = prob.solve_fp64()
    prob.close()
    assert info.status == 0 and info.rel_residual <= 1e-8
    for k in ("vx", "vy", "vz", "pr"):
        assert rel(sol[k], g["sol_" + k]) < 1e-6, (k, rel(sol[k], g["sol_" + k]))


def test_full_cell_block_variants_agree(gcase):
    """The full cell-block smoother with stored cell factors (1), factored on
    every sweep from shared stresses (3) or row by row (2): the same
    iteration up to rounding, so the outer iterations agree."""
    m, g, _ = gcase
    its, sols = [], []
    for sm in (1, 3, 2):
        prob = P.StokesProblem(m, tol=1e-8, smoother=sm)
        prob.set_nodes({k: g["node_" + k] for k in FIELDS})
        sol, info = prob.solve_fp64()
        prob.close()
        assert info.status == 0
        its.append(info.iterations)
        sols.append(sol)
    assert max(its) - min(its) <= 1, its
    for s in sols[1:]:
        for k in ("vx", "vy", "vz", "pr"):
            assert rel(sols[0][k], s[k]) < 1e-6, k


def test_autotune_choice_reaches_the_reference_solution(gcase):
    m, g, _ = gcase
    prob = P.StokesProblem(m, tol=1e-8)
    prob.set_nodes({k: g["node_" + k] for k in FIELDS})
    tune = prob.autotune(6)
    assert tune.candidates == 12 and tune.smoother in (0, 1) and tune.sweep_growth in (1, 2)
    assert tune.sweeps0 in (prob.params.npre[0], prob.params.npre[0] // 2)
    assert tune.sweep_max in (16, 64)
    assert tune.restart in (12, 16)
    assert np.isfinite(tune.est_ms) and 0 < tune.rate < 1
    sol, info = prob.solve_fp64()
    prob.close()
    assert info.status == 0 and info.rel_residual <= 1e-8
    for k in ("vx", "vy", "vz", "pr"):
        assert rel(sol[k], g["sol_" + k]) < 1e-6, k


def test_vpiterate_host_arrays(gcase):
    """The reference-shaped call: float vx/vy/vz and double pr in/out."""
    m, g, _ = gcase
    prob = P.StokesProblem(m, tol=1e-8)
    prob.set_nodes({k: g["node_" + k] for k in FIELDS})
    sol, info = prob.vpiterate()
    prob.close()
    assert sol["vx"].dtype == np.float32 and sol["pr"].dtype == np.float64
    for k in ("vx", "vy", "vz", "pr"):
        assert rel(sol[k].astype(np.float64), g["sol_" + k]) < 1e-6, k


def test_sphere33_full_path_vs_oracle(oracle_mod):
    """The 33^3 CPU-runnable case (4x4x4 markers per cell): GPU marker ->
    node fields bit-exact with the oracle, GPU solves within 1e-6 of the
    oracle's FP64 multigrid solution."""
    m = M.config_model(1)
    prob = P.StokesProblem(m, tol=1e-8)
    f = prob.ronurecalc()
    fo = oracle_mod.ronurecalc(m)
    for k in FIELDS:
        assert np.array_equal(f[k], fo[k]), k
    s = oracle_mod.OracleSolver(m, npre=[4] * 3, npost=[4] * 3)
    s.set_fields(fo)
    s.solve(tol=1e-11, max_cycles=300)
    ref = s.solution()
    for precision in (0, 1):
        p2 = P.StokesProblem(m, precision=precision, tol=1e-8)
        p2.set_nodes(f)
        sol, info = p2.solve_fp64()
        p2.close()
        assert info.status == 0
        for k in ("vx", "vy", "vz", "pr"):
            assert rel(sol[k], ref[k]) < 1e-6, (precision, k, rel(sol[k], ref[k]))
    prob.close()


def test_determinism():
    m = M.random_spheres_model(33, 2, 6, (1e-2, 1e2), markers=(2, 2, 2), seed=21, name="det33")
    prob = P.StokesProblem(m, tol=1e-9)
    f1 = prob.ronurecalc()
    f2 = prob.ronurecalc()
    for k in FIELDS:
        assert np.array_equal(f1[k], f2[k])
    prob.set_nodes(f1)
    s1, i1 = prob.solve_fp64()
    s2, i2 = prob.solve_fp64()
    prob.close()
    assert i1.iterations == i2.iterations
    for k in s1:
        assert np.array_equal(s1[k], s2[k]), k


def test_spheres65_properties(oracle_mod):
    """65^3, 8 spheres, viscosity contrast 1e6: the FP64 residual of the GPU
    solution, evaluated independently by the oracle's matrix-free rows, meets
    1e-8; mixed and FP64 V-cycles agree within 1e-6."""
    m = M.config_model(2)
    sols = {}
    for precision in (0, 1):
        prob = P.StokesProblem(m, precision=precision, tol=1e-8)
        f = prob.ronurecalc()
        sol, info = prob.solve_fp64()
        prob.close()
        assert info.status == 0, info.as_dict()
        sols[precision] = sol
    s = oracle_mod.OracleSolver(m)
    s.set_fields(f)
    s.set_solution(sols[0])
    assert s.rel_residual() <= 1.05e-8
    for k in ("vx", "vy", "vz", "pr"):
        assert rel(sols[0][k], sols[1][k]) < 1e-6, k
