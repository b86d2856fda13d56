"""Marker advection (movemark, pardiso/mark3mg.c:174) and the post-solve
stress / strain-rate pass of vpiterate on the GPU.

Bit-exact bar: the moved marker coordinates (float) equal the reference's
for every marker, through the host-array entry point (against the golden
vectors the reference itself produced, tests/golden/move17.npz) and through
the resident path after a resident solve (against the oracle restatement,
which the CPU suite pins to the same golden vectors).
"""
import os

import numpy as np
import pytest

import pardiso2_b200 as P
from pardiso2_b200.capi import P2Error
from pardiso2_b200 import model as M
from tests.golden.make_golden import MOVE_VARIANTS, move_markers

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def move17():
    g = np.load(os.path.join(GOLDEN, "move17.npz"))
    m = M.sphere_model(17, 2, (1, 1, 1), seed=3, eta_sphere=1e3)
    prob = P.StokesProblem(m)
    yield g, prob
    prob.close()


@pytest.mark.parametrize("variant", sorted(MOVE_VARIANTS))
def test_movemark_host_arrays_vs_reference_golden(move17, variant):
    g, prob = move17
    markmod, outgrid = MOVE_VARIANTS[variant]
    x, y, z = prob.ctx.movemark(float(g["dt"]), g["vx"], g["vy"], g["vz"], g["in_x"], g["in_y"], g["in_z"],
                                g["in_t"], markmod=markmod, outgrid=outgrid)
    for a, c in zip((x, y, z), "xyz"):
        ref = g["out_%s_%s" % (variant, c)]
        bad = np.flatnonzero(a.view(np.uint32) != ref.view(np.uint32))
        assert bad.size == 0, (variant, c, bad[:5], a[bad[:5]], ref[bad[:5]])


def test_movemark_zero_markers_and_bad_arguments(move17):
    g, prob = move17
    e = np.zeros(0, np.float32)
    assert [a.size for a in prob.ctx.movemark(1.0, g["vx"], g["vy"], g["vz"], e, e, e, np.zeros(0, np.int8))] == [0] * 3
    with pytest.raises(P2Error):
        prob.ctx.movemark(1.0, g["vx"], g["vy"], g["vz"], g["in_x"], g["in_y"], g["in_z"], g["in_t"], markmod=3)
    with pytest.raises(P2Error):
        prob.ctx.movemark(float("nan"), g["vx"], g["vy"], g["vz"], g["in_x"], g["in_y"], g["in_z"], g["in_t"])


@pytest.mark.parametrize("variant", ["rk4_og0", "rk4_og2"])
def test_movemark_resident_after_resident_solve_vs_oracle(oracle_mod, variant):
    """33^3, 4 spheres, 8 markers per cell (some outside, mixed types):
    upload, ronurecalc, solve and advect on the device; the oracle advects
    the same markers through the float cast of the FP64 solution."""
    markmod, outgrid = MOVE_VARIANTS[variant]
    m = M.random_spheres_model(33, 2, 4, (1e-2, 1e2), markers=(2, 2, 2), seed=5, name="move33")
    mx, my, mz, mt = move_markers(m)
    prob = P.StokesProblem(m, tol=1e-8)
    r = m.rocks
    prob.ctx.upload_markers(mx, my, mz, mt, r.n0, r.n1, r.ro)
    prob.ctx.ronurecalc_resident()
    info = prob.ctx.solve_resident()
    assert info.status == 0
    sol = prob.ctx.solution(m.nodenum)
    vel = tuple(np.asarray(sol[k], np.float32) for k in ("vx", "vy", "vz"))
    dt = 1.2 / 32 / max(float(np.abs(v).max()) for v in vel)
    prob.ctx.movemark_resident(dt, markmod=markmod, outgrid=outgrid)
    got = prob.ctx.get_markers(mx.size)
    prob.close()
    ref = oracle_mod.movemark(m, vel, dt, markmod, outgrid, markers=(mx, my, mz, mt))
    for a, b, c in zip(got, ref, "xyz"):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), c
    assert int(((got[0] != mx) | (got[1] != my) | (got[2] != mz)).sum()) > mx.size // 2


def test_stress_strain_after_solve_vs_oracle(oracle_mod):
    """Post-solve stresses and strain rates (move3mgNew.c:2908-3038) from the
    float velocities of a resident solve: bit-exact with the oracle's pass
    (pinned to the reference's own in the CPU suite); untouched positions
    keep the caller's values; velocity ranges over the valid positions."""
    from tests.test_oracle_golden import load_case
    m, g = load_case("sphere17")
    nodes = {k: g["node_" + k] for k in ("nu", "ro", "nxx", "nxy", "nxz", "nyz")}
    prob = P.StokesProblem(m, tol=1e-8)
    prob.set_nodes(nodes)
    assert prob.ctx.solve_resident().status == 0
    sol = prob.ctx.solution(m.nodenum)
    vel = tuple(np.asarray(sol[k], np.float32) for k in ("vx", "vy", "vz"))
    keys = oracle_mod.STRESS_KEYS
    got = {k: np.full(m.nodenum, -7.0, np.float32) for k in keys}
    vr = prob.ctx.stress_strain(got)
    part = {k: np.full(m.nodenum, -7.0, np.float32) for k in ("sxy", "ezz")}
    prob.ctx.stress_strain(part)
    prob.close()
    ref = oracle_mod.stress_strain(m, vel, nodes, init=-7.0)
    for k in keys:
        assert np.array_equal(got[k].view(np.uint32), ref[k].view(np.uint32)), k
    for k in part:
        assert np.array_equal(part[k], got[k]), k
    nx, ny, nz = m.shape
    kk, ii, jj = (a.ravel() for a in np.meshgrid(np.arange(nz), np.arange(nx), np.arange(ny), indexing="ij"))
    ok = [(jj < ny - 1) & (kk < nz - 1), (ii < nx - 1) & (kk < nz - 1), (ii < nx - 1) & (jj < ny - 1)]
    for c in range(3):
        assert vr[2 * c] == float(vel[c][ok[c]].min()) and vr[2 * c + 1] == float(vel[c][ok[c]].max()), c


def _ulps(a, b):
    """Distance in units in the last place between equal-signed floats."""
    it = np.int64 if a.dtype == np.float64 else np.int32
    return np.abs(a.view(it).astype(np.int64) - b.view(it).astype(np.int64))


@pytest.mark.parametrize("variant", ["rk4_og0", "simple_og0"])
def test_movemark_strain_outputs_vs_reference_golden(move17, variant):
    """p2_movemark_strain: positions bit-exact; val1 and marke within one unit
    in the last place of the reference's (it takes pow(x, 0.5) where the
    device takes a correctly rounded square root)."""
    g, prob = move17
    markmod, outgrid = MOVE_VARIANTS[variant]
    strain = [g["st_" + k] for k in ("exx", "eyy", "ezz", "exy", "exz", "eyz")]
    me_in = g["marke_in"] if markmod == 2 else np.zeros_like(g["marke_in"])
    x, y, z, v1, me = prob.ctx.movemark_strain(float(g["dt"]), (g["vx"], g["vy"], g["vz"]), strain,
                                               (g["in_x"], g["in_y"], g["in_z"], g["in_t"]),
                                               np.full(me_in.size, -1.0), me_in, markmod=markmod, outgrid=outgrid)
    for a, c in zip((x, y, z), "xyz"):
        assert np.array_equal(a.view(np.uint32), g["strain_%s_%s" % (variant, c)].view(np.uint32)), c
    rv, re_ = g["strain_%s_val1" % variant], g["strain_%s_marke" % variant]
    assert np.array_equal(v1 < 0, rv < 0)
    assert _ulps(v1, rv).max() <= 1 and _ulps(me, re_).max() <= 1
    if markmod == 2:
        assert int((me != me_in).sum()) > 1000
