"""The oracle restatement pinned against golden vectors produced by the
reference's own C code (tests/golden/make_golden.py), and — when the
reference build oracle/_ref is present — against the live reference (CPU)."""
import os

import numpy as np
import pytest

from pardiso2_b200 import model as M
from tests.golden.make_golden import CASES, probe_vector

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load_case(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    m = CASES[name]()
    # the exact marker inputs the reference saw
    m.markx, m.marky, m.markz, m.markt = g["markx"], g["marky"], g["markz"], g["markt"]
    return m, g


def pin_mask(m, lev):
    lv = m.levels
    off = lv.mgp[lev]
    mask = np.ones(lv.mgn[lev] * 4, bool)
    for u in range(lv.mgn[lev]):
        b = m.bc.bondm[(off + u) * 4]
        if b and m.bc.bondn1[b] == 0:
            mask[u * 4] = False
    return mask


def vmax_valid(m, v, c):
    """max |v| over the valid positions of velocity component c (1..3)."""
    nx, ny, nz = m.shape
    k, i, j = np.meshgrid(np.arange(nz), np.arange(nx), np.arange(ny), indexing="ij")
    ok = [(j < ny - 1) & (k < nz - 1), (i < nx - 1) & (k < nz - 1), (i < nx - 1) & (j < ny - 1)][c - 1].ravel()
    return float(np.abs(v[ok]).max())


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request, oracle_mod):
    m, g = load_case(request.param)
    O = oracle_mod
    f = O.ronurecalc(m)
    s = O.OracleSolver(m, npre=[4] * (m.multinum + 1), npost=[4] * (m.multinum + 1))
    s.set_fields({k: g["node_" + k] for k in ("nu", "ro", "nxx", "nxy", "nxz", "nyz")})
    yield request.param, m, g, f, s
    s.close()


def test_ronurecalc_bit_exact(case):
    """mark3mg.c:630-1133 restated: identical float node fields to the
    single-threaded reference."""
    _, m, g, f, _ = case
    for k in ("nu", "ro", "nxx", "nxy", "nxz", "nyz"):
        assert np.array_equal(f[k], g["node_" + k]), k


def test_operator_matches_reference_rows(case):
    """Matrix-free rows vs the reference's assembled 57-coefficient row store."""
    _, m, g, _, s = case
    for lev in range(m.multinum):
        x = probe_vector(m.levels.mgn[lev], lev)
        y = s.apply(lev, x)
        has = g["op_rows_lev%d" % lev]
        ref = g["op_lev%d" % lev]
        err = np.abs(y - ref)[has].max() / np.abs(ref[has]).max()
        # level 0 uses the same float node fields (FP64 arithmetic order only);
        # coarse levels see the reference's float-accumulated nu (ronurestrict)
        assert err < (1e-13 if lev == 0 else 2e-7), (lev, err)


def test_rhs_matches_reference(case):
    _, m, g, _, s = case
    b = s.rhs()
    has = g["op_rows_lev0"]
    assert np.array_equal(b[has], g["rhs"][has])  # same float sums, same FP64 ops


def test_transfers_match_reference(case, oracle_mod):
    _, m, g, _, s = case
    for lc in range(1, m.multinum + 1):
        nc = m.levels.mgn[lc]
        got = oracle_mod.restrict(s, lc, g["restrict_in_lev%d" % lc], nc, compat=False)
        ref = g["restrict_lev%d" % lc]
        mask = pin_mask(m, lc)
        assert np.abs(got - ref)[mask].max() <= 2e-7 * np.abs(ref[mask]).max()
        nf = m.levels.mgn[lc - 1]
        got = oracle_mod.prolong(s, lc, probe_vector(nc, 20 + lc), probe_vector(nf, 30 + lc))
        assert np.abs(got - g["prolong_lev%d" % lc]).max() <= 1e-13 * np.abs(g["prolong_lev%d" % lc]).max()


def test_solution_matches_reference_discrete_solution(case):
    """The oracle's multigrid converges to the exact solution of the
    reference's level-0 system (direct sparse LU of its rows)."""
    _, m, g, _, s = case
    hist = s.solve(tol=1e-12, max_cycles=200)
    assert hist[-1] <= 1e-12
    sol = s.solution()
    for k in ("vx", "vy", "vz", "pr"):
        assert rel(sol[k], g["sol_" + k]) < 1e-8, k


def test_golden_system_solution_is_tight():
    for name in CASES:
        g = np.load(os.path.join(GOLDEN, name + ".npz"))
        assert float(g["sol_rel_residual"]) < 1e-11


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(__file__)),
                                                    "oracle", "_ref", "libp2ref.so")),
                    reason="reference build oracle/_ref not present")
def test_live_reference_ronurecalc_and_rows(oracle_mod):
    """Live run of the reference's own ronurecalc/assembly (one model per process)."""
    from oracle import refdrv
    m = M.random_spheres_model(15, 1, 3, (1e-1, 1e1), markers=(2, 2, 2), seed=11, name="live15")
    r = refdrv.RefModel(m)
    r.ronurecalc()
    nodes = r.nodes()
    f = oracle_mod.ronurecalc(m)
    for k in nodes:
        assert np.array_equal(nodes[k], f[k]), k
    r.fill_stress(-7.0)
    r.set_step(0.01, 1e30)
    r.first_iteration()
    # vpiterate's post-solve stresses, strain rates and time-step limit
    w = r.written()
    vel = (w["vx"], w["vy"], w["vz"])
    st = r.written_stress()
    ost = oracle_mod.stress_strain(m, vel, nodes, init=-7.0)
    for k in st:
        assert np.array_equal(st[k].view(np.uint32), ost[k].view(np.uint32)), k
    assert r.timestep() == min(0.01 / vmax_valid(m, v, c) for c, v in enumerate(vel, 1))
    s = oracle_mod.OracleSolver(m)
    s.set_fields(nodes)
    row, col, val, rhs = r.rows(0)
    x = probe_vector(m.nodenum, 5)
    ref = np.zeros(m.nodenum * 4)
    np.add.at(ref, row, val * x[col])
    has = np.zeros(ref.size, bool)
    has[row] = True
    y = s.apply(0, x)
    assert np.abs(y - ref)[has].max() < 1e-13 * np.abs(ref[has]).max()


@pytest.mark.parametrize("variant", ["rk4_og0", "rk4_og1", "rk4_og2", "simple_og0"])
def test_oracle_movemark_vs_reference_golden(oracle_mod, variant):
    """Marker advection (movemark, mark3mg.c:174): positions and the markk
    reset bit-exact with the reference's own run (move17.npz)."""
    from tests.golden.make_golden import MOVE_VARIANTS
    g = np.load(os.path.join(GOLDEN, "move17.npz"))
    m = M.sphere_model(17, 2, (1, 1, 1), seed=3, eta_sphere=1e3)
    markmod, outgrid = MOVE_VARIANTS[variant]
    ins = (g["in_x"], g["in_y"], g["in_z"], g["in_t"])
    out = oracle_mod.movemark(m, (g["vx"], g["vy"], g["vz"]), float(g["dt"]), markmod, outgrid, markers=ins,
                              markk=np.full(ins[0].size, 300.0, np.float32))
    for a, c in zip(out, "xyzk"):
        assert np.array_equal(a.view(np.uint32), g["out_%s_%s" % (variant, c)].view(np.uint32)), c
    moved = (out[0] != ins[0]) | (out[1] != ins[1]) | (out[2] != ins[2])
    assert moved.sum() > ins[0].size // 2


def test_oracle_stress_strain_vs_reference_golden(oracle_mod):
    """The post-solve stress / strain-rate pass (move3mgNew.c:2908-3038)
    bit-exact with the reference's value-mode stencils (move17.npz)."""
    g = np.load(os.path.join(GOLDEN, "move17.npz"))
    src = np.load(os.path.join(GOLDEN, "sphere17.npz"))
    m = M.sphere_model(17, 2, (1, 1, 1), seed=3, eta_sphere=1e3)
    nodes = {k: src["node_" + k] for k in ("nxx", "nxy", "nxz", "nyz")}
    out = oracle_mod.stress_strain(m, (g["vx"], g["vy"], g["vz"]), nodes, init=-7.0)
    for k, a in out.items():
        assert np.array_equal(a.view(np.uint32), g["st_" + k].view(np.uint32)), k
        assert (a != -7.0).sum() > 0.7 * a.size * (0.75 if k[1] != k[2] else 1.0), k


@pytest.mark.parametrize("variant", ["rk4_og0", "simple_og0"])
def test_oracle_movemark_strain_outputs_vs_reference_golden(oracle_mod, variant):
    """movemark's strain-rate outputs (epscalc1 at the markers, val1; the
    Runge-Kutta brittle strain marke): bit-exact with the reference's run."""
    from tests.golden.make_golden import MOVE_VARIANTS
    g = np.load(os.path.join(GOLDEN, "move17.npz"))
    m = M.sphere_model(17, 2, (1, 1, 1), seed=3, eta_sphere=1e3)
    markmod, outgrid = MOVE_VARIANTS[variant]
    strain = [g["st_" + k] for k in ("exx", "eyy", "ezz", "exy", "exz", "eyz")]
    me_in = g["marke_in"] if markmod == 2 else np.zeros_like(g["marke_in"])
    out = oracle_mod.movemark(m, (g["vx"], g["vy"], g["vz"]), float(g["dt"]), markmod, outgrid,
                              markers=(g["in_x"], g["in_y"], g["in_z"], g["in_t"]), strain=strain,
                              val1=np.full(me_in.size, -1.0), marke=me_in)
    for a, k in zip(out, ("x", "y", "z", "val1", "marke")):
        ref = g["strain_%s_%s" % (variant, k)]
        assert np.array_equal(a, ref) and np.array_equal(np.signbit(a), np.signbit(ref)), k
    if markmod == 2:
        assert int((out[4] != me_in).sum()) > 1000


def test_oracle_ronurecalc_power_law_vs_reference_golden(oracle_mod):
    """ronurecalc with power-law rocks (viscalc, mark3mg.c:1463-1498): node
    fields bit-exact with the reference's own run (pl17.npz); types above 20
    stay constant even with markn0 != markn1."""
    from tests.golden.make_golden import power_law_model
    g = np.load(os.path.join(GOLDEN, "pl17.npz"))
    m, nu, mm, val1 = power_law_model()
    assert np.array_equal(val1, g["val1"]) and np.array_equal(m.markt, g["markt"])
    f = oracle_mod.ronurecalc(m, marknu=nu, markmm=mm, val1=val1)
    for k in f:
        assert np.array_equal(f[k], g["node_" + k]), k
    assert np.abs(oracle_mod.ronurecalc(m)["nu"] - f["nu"]).max() > 1.0


def _bulk_fields(g, nodes):
    f = {k: nodes["node_" + k] for k in ("nxx", "nxy", "nxz", "nyz")}
    f["ro"] = g["ro"]
    f.update({k: g["st_" + k] for k in ("exx", "eyy", "ezz", "exy", "exz", "eyz", "sxx", "syy", "szz", "sxy", "sxz",
                                        "syz")})
    return f


def bulk_line_values(out, counts):
    """The oracle's diagnostics in the order of the reference's printed line
    (after timesum, timestep): counts, matrix[12], incl[12], siin eiin eiivp
    hsn nubulk2 nubulk3 nubulk4."""
    return np.concatenate([[counts[2], counts[1], counts[0]], out[10:22], out[22:34],
                           [out[1], out[0], out[2], out[4], out[7], out[8], out[9]]])


def test_oracle_effbulk_vs_reference_golden(oracle_mod):
    """effbulkvisccalc(1) (mark3mg.c:2-150): the oracle's values equal the
    line the reference itself printed, to the 7 digits of its %e format."""
    g = np.load(os.path.join(GOLDEN, "bulk21.npz"))
    m, s = load_case("spheres21")
    out, counts = oracle_mod.effbulk(m, _bulk_fields(g, s))
    ref = g["line"][2:]
    mine = bulk_line_values(out, counts)
    assert np.all(np.abs(mine - ref) <= 6e-7 * np.abs(ref)), np.max(np.abs(mine - ref) / np.abs(ref))
    assert counts[2] > 1000 and counts[1] > 1000


# -- heat equation (titerate) -------------------------------------------------
def _heat_case():
    from tests.golden.make_golden import HEAT_COMMON, HEAT_VARIANTS, heat_inputs, heat_model
    g = np.load(os.path.join(GOLDEN, "heat17.npz"))
    m = heat_model()
    return m, g, heat_inputs(m), HEAT_COMMON, HEAT_VARIANTS


@pytest.mark.parametrize("variant", ["mg", "single"])
def test_oracle_titerate_vs_reference_golden(oracle_mod, variant):
    """heat3mg.c:292-829 restated (lexicographic Gauss-Seidel, the same
    V-cycle, sub-steps and marker update): the temperatures and marker
    temperatures of the reference's own titerate() bit for bit, and the same
    number of sub-steps and error checks."""
    m, g, (th, vel, se, pr, mk, markk), common, variants = _heat_case()
    np.testing.assert_array_equal(g["markk_in"], markk)
    v = variants[variant]
    hp = dict(common, **v, gx=m.params.gx, gy=m.params.gy, gz=m.params.gz, max_cycles=200)
    mx, my, mz, mt = mk
    tk, mko, info = oracle_mod.titerate(m.gx, m.gy, m.gz, v["multinumt"], m.bc.bondt, m.bc.bondv1, m.bc.bondn1, hp,
                                        th, vel=vel, pr=pr, se=se, markers=(mx[:-1], my[:-1], mz[:-1], mt[:-1]),
                                        markk=markk)
    assert not info["capped"]
    assert info["substeps"] == int(g["info_" + variant][0]) and info["substeps"] > 1
    np.testing.assert_array_equal(tk, g["tk_" + variant])
    np.testing.assert_array_equal(mko, g["markk_" + variant])
    # the step moved temperatures and every marker class
    assert np.abs(tk - th.tk).max() > 10
    assert np.abs(mko - markk)[mt[:-1] < 50].max() > 1
    assert np.abs(mko - markk)[(mt[:-1] >= 50) & (mt[:-1] < 100)].max() > 1
