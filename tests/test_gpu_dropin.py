"""The drop-in boundary end to end.

The reference's own state (its globals, pardiso/head3mg.c, set up by the
reference harness in oracle/ref/ref_harness.c) is driven through vpiterate()
ronurecalc() and movemark() taken from pardiso2_b200/csrc/move3mg_cuda.c, the
shim that replaces the reference's CPU functions and calls libp2cuda.so on
the GPU.  The arrays the shim writes back into the reference's globals
(nu..nyz; vx, vy, vz as float and pr as double; sxx..syz, exx..eyz and
timestep; markx, marky, markz, markk) must equal the golden vectors: node
fields bit for bit, solutions within 1e-6 relative L2; stresses, strain
rates, time step and moved markers bit for bit with the oracle on the
written velocities (the CPU suite pins the oracle to the reference's own).

Needs oracle/_ref/libp2ref_shim.so, built with the reference sources by
`make -C oracle refshim`; skipped when it is absent.
"""
import numpy as np
import pytest

from oracle import refdrv
from tests.golden.make_golden import move_markers
from tests.test_oracle_golden import load_case, rel, vmax_valid

pytestmark = pytest.mark.gpu
FIELDS = ("nu", "ro", "nxx", "nxy", "nxz", "nyz")


def test_vpiterate_ronurecalc_movemark_through_the_reference_globals(oracle_mod):
    if not refdrv.available(shim=True):
        pytest.skip("oracle/_ref/libp2ref_shim.so not built")
    m, g = load_case("spheres21")
    nl = m.multinum + 1
    r = refdrv.RefModel(m, npre=[4] * nl, npost=[4] * nl, shim=True)
    r.ronurecalc()                       # the shim's ronurecalc() -> p2_ronurecalc
    f = r.nodes()
    for k in FIELDS:
        assert np.array_equal(f[k], g["node_" + k]), k
    r.fill_stress(-7.0)
    r.set_step(0.01, 1e30)
    r.first_iteration()                  # the shim's vpiterate(0, 0) -> p2_stokes_solve
    w = r.written()
    assert w["vx"].dtype == np.float32 and w["pr"].dtype == np.float64
    for k in ("vx", "vy", "vz", "pr"):
        e = rel(w[k].astype(np.float64), g["sol_" + k])
        assert e < 1e-6, (k, e)
    # stresses, strain rates (p2_stress_strain) and the time-step limit
    vel = (w["vx"], w["vy"], w["vz"])
    st = r.written_stress()
    ref = oracle_mod.stress_strain(m, vel, f, init=-7.0)
    for k in st:
        assert np.array_equal(st[k].view(np.uint32), ref[k].view(np.uint32)), k
    assert r.timestep() == min(0.01 / vmax_valid(m, v, c) for c, v in enumerate(vel, 1))
    # effbulkvisccalc(1) through the shim (p2_effbulk_visc): the line it
    # appends equals the oracle's values on the same fields to 7 digits
    import tempfile
    from tests.test_oracle_golden import bulk_line_values
    ro = np.where(f["nu"] > 1.0, 4000.0, 3300.0).astype(np.float32)
    with tempfile.TemporaryDirectory() as d:
        line = r.effbulk(ro, d)
    bf = {"ro": ro, "nxx": f["nxx"], "nxy": f["nxy"], "nxz": f["nxz"], "nyz": f["nyz"]}
    bf.update(st)
    out, counts = oracle_mod.effbulk(m, bf)
    mine = bulk_line_values(out, counts)
    assert np.all(np.abs(mine - line[2:]) <= 6e-7 * np.abs(line[2:]))
    # the shim's movemark() -> p2_movemark on the velocities vpiterate wrote
    mx, my, mz, mt = move_markers(m)
    dt = 1.5 / 20 / max(float(np.abs(v).max()) for v in vel)
    r.set_markers(mx, my, mz, mt)
    r.fill_markk(300.0)
    r.fill_val1(-1.0)
    r.movemark(dt, 2, 0)
    got = r.markers()
    # val1: the strain-rate invariant at every moved marker, from the fields
    # vpiterate wrote (the device takes sqrt where the reference takes pow(., 0.5))
    v1, _ = r.val1_marke()
    strain = [st[k] for k in ("exx", "eyy", "ezz", "exy", "exz", "eyz")]
    ref_v1 = oracle_mod.movemark(m, vel, dt, 2, 0, markers=(mx, my, mz, mt), strain=strain,
                                 val1=np.full(mx.size, -1.0))[3]
    assert np.array_equal(v1 < 0, ref_v1 < 0)
    assert np.abs(v1.view(np.int64) - ref_v1.view(np.int64)).max() <= 1
    ref = oracle_mod.movemark(m, vel, dt, 2, 0, markers=(mx, my, mz, mt), markk=np.full(mx.size, 300.0, np.float32))
    for a, b, c in zip(got, ref, "xyzk"):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), c
    assert int((got[3] == 0).sum()) > 0
    # ronurecalc with a power-law rock: the shim's ronurecalc() ->
    # p2_ronurecalc_powerlaw with marknu, markmm and the val1 movemark left;
    # marke becomes 1e-20 where it was 0 for the markers it interpolates
    n0 = np.array(m.rocks.n0, np.float64)
    n1 = np.array(m.rocks.n1, np.float64)
    n1[1] = n0[1] * 1e3
    nu = np.array(n0) * 2.0
    mm = np.ones(n0.size)
    mm[1] = 3.0
    r.lib.p2ref_set_rocks(n0.size, n0, n1, np.ascontiguousarray(m.rocks.ro, np.float64))
    v1pl = np.where(v1 >= 0, v1, 1e-3)   # markers that did not move kept val1 = -1
    r.set_rheology(nu, mm, v1pl)
    r.set_markers(m.markx, m.marky, m.markz, m.markt)
    r.set_marke(np.zeros(m.markx.size, np.float32))
    r.ronurecalc()
    f = r.nodes()
    mpl = m
    mpl.rocks = type(m.rocks)(n0, n1, m.rocks.ro)
    ref = oracle_mod.ronurecalc(mpl, marknu=nu, markmm=mm, val1=v1pl, init={k: g["node_" + k] for k in FIELDS})
    for k in FIELDS:
        err = np.abs(f[k].astype(np.float64) - ref[k]) / np.maximum(np.abs(ref[k]), 1e-30)
        assert err.max() <= 1e-6, (k, float(err.max()))
    _, me = r.val1_marke()
    inside = (m.markx > 0) & (m.marky > 0) & (m.markz > 0) & (m.markx < 1) & (m.marky < 1) & (m.markz < 1) & (m.markt < 50)
    assert np.all(me[inside] == np.float32(1e-20)) and np.all(me[~inside] == 0)
