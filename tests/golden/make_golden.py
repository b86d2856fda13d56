"""Generate the golden vectors in tests/golden/*.npz from the reference itself.

Runs the reference's own C sources (oracle/_ref/libp2ref.so, built by
`make -C oracle ref` from the reference tree) single-threaded on small seeded
models and stores, per case:
  markers (x, y, z, type)          the exact inputs (float32 / int8)
  ronurecalc node fields            pardiso/mark3mg.c:630 (one thread)
  op_lev{l}                         y = A x of the reference's assembled rows
                                    (gausmat2 row store, move3mgNew.c:2329-2662)
                                    for x = probe_vector(level)
  restrict_lev{l}, prolong_lev{l}   vprestrict / vpprolong (move3mgNew.c:3965,
                                    3534) of probe vectors
  level_nu, level_ro                nu/ro of all levels after ronurestrict
  sol_{pr,vx,vy,vz}, rhs            the exact discrete solution of the
                                    reference's level-0 system (direct sparse
                                    LU of its assembled rows, pressure reset
                                    to pinit at the pinned cell)
and, in move17.npz, marker advection by the reference's movemark()
(pardiso/mark3mg.c:174) through the float sphere17 solution velocities:
  in_{x,y,z,t}, vx, vy, vz, dt      markers (some outside the box, types 0,
                                    1, 60, 110) and the inputs of the step
  out_<variant>_{x,y,z,k}           positions and markk after one step, for
                                    variants (markmod, outgrid) in MOVE_VARIANTS
  strain_<variant>_{x,y,z,val1,marke}  movemark with strain-rate fields set
                                    by that pass (rk4_og0, simple_og0):
                                    positions, val1 (filled with -1 before)
                                    and marke (in: marke_in, 0 for two
                                    thirds of the markers; all 0 for
                                    simple_og0)
and, in bulk21.npz, effbulkvisccalc(1) (pardiso/mark3mg.c:2-150) on the
spheres21 node fields and the stresses / strain rates of its solution:
  ro (a synthetic density above 1500 everywhere, above 3850 in the stiff
  spheres), st_{sxx..eyz}, and line: the 36 numbers it appends to
  effbulkvisc.txt (timesum timestep numinc nummat numtot, matrix exx..syz,
  inclusion exx..syz, siin eiin eiivp hsn nubulk2 nubulk3 nubulk4; %e)
and, in pl17.npz, ronurecalc with power-law rocks (viscalc,
pardiso/mark3mg.c:1463-1498): markers, rock tables (n0, n1, ro, nu, mm),
val1 per marker, the node fields, and marke after the call (the reference
sets it to 1e-20 where it was 0 for the markers it interpolates),
and, in heat17.npz, titerate (pardiso/heat3mg.c:292) per HEAT_VARIANTS on
the heat_inputs of heat_model: tk_<variant>, markk_<variant> (in: markk_in)
and info_<variant> (sub-steps, error checks, sub-step limit of the oracle).
  st_{sxx..syz, exx..eyz}           the post-solve stress / strain-rate pass
                                    of vpiterate (move3mgNew.c:2908-3038) on
                                    those velocities and sphere17's node
                                    fields (untouched positions hold -7)

Usage: OMP_NUM_THREADS=1 python tests/golden/make_golden.py
"""
import os
import sys

os.environ["OMP_NUM_THREADS"] = "1"
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import scipy.sparse as sp  # noqa: E402
import scipy.sparse.linalg as spl  # noqa: E402

from pardiso2_b200 import model as M  # noqa: E402

CASES = {
    "sphere17": lambda: M.sphere_model(17, 2, (2, 2, 2), seed=1, eta_sphere=1e3),
    "spheres21": lambda: M.random_spheres_model(21, 2, 4, (1e-2, 1e2), markers=(2, 2, 2), seed=7,
                                                name="spheres21"),
}


MOVE_VARIANTS = {"rk4_og0": (2, 0), "rk4_og1": (2, 1), "rk4_og2": (2, 2), "simple_og0": (1, 0)}


def move_markers(m):
    """Marker set for the movemark vectors: the model's markers, every 7th
    pushed outside the box along one axis, types 60 (moved only inside) and
    110 (immobile class, moved anywhere) mixed in."""
    x, y, z = (np.array(a, np.float32) for a in (m.markx, m.marky, m.markz))
    t = np.array(m.markt, np.int8)
    q = np.arange(x.size)
    for a, arr in enumerate((x, y, z)):
        sel = (q % 7 == 0) & ((q // 7) % 3 == a)
        lo = (q // 21) % 2 == 0
        arr[sel & lo] = np.float32(-0.03) * arr[sel & lo]
        arr[sel & ~lo] = np.float32(1.0) + np.float32(0.03) * arr[sel & ~lo]
    t[q % 5 == 1] = 60
    t[q % 11 == 2] = 110
    return x, y, z, t


def probe_vector(n_nodes: int, salt: int) -> np.ndarray:
    """Deterministic test vector (no RNG stream dependence)."""
    k = np.arange(n_nodes * 4, dtype=np.float64)
    return np.sin(0.37 * k + salt) + 0.5 * np.cos(0.011 * k * (salt + 1))


def pin_rows(m, lev):
    """Unknown indices (level-local, interleaved) of pure-constant pressure rows."""
    lv = m.levels
    off = lv.mgp[lev]
    out = []
    for u in range(lv.mgn[lev]):
        b = m.bc.bondm[(off + u) * 4]
        if b and m.bc.bondn1[b] == 0:
            out.append(u * 4)
    return np.array(out, dtype=np.int64)


def make_case(name, builder):
    from oracle import refdrv
    m = builder()
    nl = m.multinum
    r = refdrv.RefModel(m)
    r.ronurecalc()
    nodes = r.nodes()
    r.first_iteration()
    out = {"markx": m.markx, "marky": m.marky, "markz": m.markz, "markt": m.markt}
    out.update({"node_" + k: v for k, v in nodes.items()})
    lf = r.level_fields()
    out["level_nu"], out["level_ro"] = lf["nu"], lf["ro"]
    for lev in range(nl):
        row, col, val, rhs = r.rows(lev)
        N = int(r.mgn[lev]) * 4
        x = probe_vector(int(r.mgn[lev]), lev)
        y = np.zeros(N)
        np.add.at(y, row, val * x[col])
        has = np.zeros(N, bool)
        has[row] = True
        out["op_lev%d" % lev] = y
        out["op_rows_lev%d" % lev] = has
        if lev == 0:
            out["rhs"] = rhs
            g = np.where(~has)[0]
            A = sp.coo_matrix((np.concatenate([val, np.ones(g.size)]),
                               (np.concatenate([row, g]), np.concatenate([col, g]))), shape=(N, N)).tocsc()
            b = rhs.copy()
            b[g] = 0.0
            lu = spl.splu(A)
            x0 = lu.solve(b)
            for _ in range(3):  # iterative refinement
                x0 += lu.solve(b - A @ x0)
            res = np.linalg.norm(A @ x0 - b) / np.linalg.norm(b)
            assert res < 1e-11, res
            out["sol_rel_residual"] = np.array(res)
            p = m.params
            nx, ny, nz = m.shape
            pin = ((p.pin[2] * nx + p.pin[0]) * ny + p.pin[1]) * 4
            x0[0::4] += p.pinit - x0[pin]
            sol = x0.reshape(-1, 4)
            kk, ii, jj = np.meshgrid(np.arange(nz), np.arange(nx), np.arange(ny), indexing="ij")
            kk, ii, jj = kk.ravel(), ii.ravel(), jj.ravel()
            out["sol_pr"] = np.where((ii > 0) & (jj > 0) & (kk > 0), sol[:, 0], 0.0)
            out["sol_vx"] = np.where((jj < ny - 1) & (kk < nz - 1), sol[:, 1], 0.0)
            out["sol_vy"] = np.where((ii < nx - 1) & (kk < nz - 1), sol[:, 2], 0.0)
            out["sol_vz"] = np.where((ii < nx - 1) & (jj < ny - 1), sol[:, 3], 0.0)
    for lc in range(1, nl + 1):
        nf, nc = int(r.mgn[lc - 1]), int(r.mgn[lc])
        fr = probe_vector(nf, 10 + lc)
        fr[pin_rows(m, lc - 1)] = 0.0
        out["restrict_in_lev%d" % lc] = fr
        out["restrict_lev%d" % lc] = r.restrict(lc, fr)
        xc = probe_vector(nc, 20 + lc)
        xf = probe_vector(nf, 30 + lc)
        out["prolong_lev%d" % lc] = r.prolong(lc, xc, xf)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "written", {k: np.asarray(v).shape for k, v in out.items()})


def make_move_case():
    """move17.npz: movemark() of the reference on sphere17's solution."""
    from oracle import refdrv
    src = np.load(os.path.join(HERE, "sphere17.npz"))
    m = M.sphere_model(17, 2, (1, 1, 1), seed=3, eta_sphere=1e3)
    vel = [np.asarray(src["sol_" + k], np.float32) for k in ("vx", "vy", "vz")]
    h = 1.0 / 16
    dt = 1.5 * h / max(float(np.abs(v).max()) for v in vel)
    mx, my, mz, mt = move_markers(m)
    r = refdrv.RefModel(m)
    r.set_velocity(*vel)
    out = {"in_x": mx, "in_y": my, "in_z": mz, "in_t": mt, "vx": vel[0], "vy": vel[1], "vz": vel[2],
           "dt": np.array(dt)}
    for name, (mmod, og) in MOVE_VARIANTS.items():
        r.set_markers(mx, my, mz, mt)
        r.fill_markk(300.0)
        r.movemark(dt, mmod, og)
        for k, a in zip("xyzk", r.markers()):
            out["out_%s_%s" % (name, k)] = a
    r.set_nodes({k: src["node_" + k] for k in ("nu", "ro", "nxx", "nxy", "nxz", "nyz")})
    for k, a in r.stress_strain(init=-7.0).items():
        out["st_" + k] = a
    # movemark's strain-rate outputs, with the pass's fields in the globals
    r.fill_stress(-7.0)
    r.update_stress()
    q = np.arange(mx.size)
    marke_in = np.where(q % 3 == 0, np.float32(0.05) + np.float32(1e-4) * (q % 17), np.float32(0)).astype(np.float32)
    out["marke_in"] = marke_in
    for name in ("rk4_og0", "simple_og0"):
        mmod, og = MOVE_VARIANTS[name]
        r.set_markers(mx, my, mz, mt)
        # in the single-velocity branch the reference adds a Runge-Kutta average
        # left over from an earlier marker to marke: that case is not recorded
        r.set_marke(marke_in if mmod == 2 else np.zeros_like(marke_in))
        r.fill_val1(-1.0)
        r.movemark(dt, mmod, og)
        x, y, z, _ = r.markers()
        v1, me = r.val1_marke()
        for k, a in zip(("x", "y", "z", "val1", "marke"), (x, y, z, v1, me)):
            out["strain_%s_%s" % (name, k)] = a
    np.savez_compressed(os.path.join(HERE, "move17.npz"), **out)
    print("move17 written", {k: np.asarray(v).shape for k, v in out.items()})


def make_bulk_case():
    import tempfile
    from oracle import refdrv
    src = np.load(os.path.join(HERE, "spheres21.npz"))
    m = CASES["spheres21"]()
    m.markx, m.marky, m.markz, m.markt = src["markx"], src["marky"], src["markz"], src["markt"]
    r = refdrv.RefModel(m)
    r.set_nodes({k: src["node_" + k] for k in ("nu", "ro", "nxx", "nxy", "nxz", "nyz")})
    r.set_velocity(*[np.asarray(src["sol_" + k], np.float32) for k in ("vx", "vy", "vz")])
    r.fill_stress(0.0)
    r.update_stress()
    st = r.written_stress()
    ro = np.where(src["node_nu"] > 1.0, 4000.0, 3300.0).astype(np.float32)
    with tempfile.TemporaryDirectory() as d:
        line = r.effbulk(ro, d)
    out = {"ro": ro, "line": line}
    out.update({"st_" + k: v for k, v in st.items()})
    np.savez_compressed(os.path.join(HERE, "bulk21.npz"), **out)
    print("bulk21 written", line[:5])


def power_law_model():
    """sphere17 markers with a power-law sphere (type 1), a type-25 block
    (markn0 != markn1 but above type 20: constant markn0) and a constant
    background, plus seeded val1 per marker (log-uniform, some zeros)."""
    m = M.sphere_model(17, 2, (2, 2, 2), seed=11, eta_sphere=1e2)
    t = np.array(m.markt, np.int8)
    t[(m.markx > 0.8) & (m.marky < 0.5)] = 25
    m.markt = t
    n0 = np.ones(26); n1 = np.ones(26); ro = np.zeros(26); nu = np.ones(26); mm = np.ones(26)
    n0[1], n1[1], nu[1], mm[1], ro[1] = 1e-1, 1e3, 5.0, 3.0, 1.0
    n0[25], n1[25], ro[25] = 2.0, 50.0, -0.5
    m.rocks = M.Rocks(n0, n1, ro)
    rng = np.random.Generator(np.random.PCG64(17))
    val1 = 10.0 ** rng.uniform(-5, 1, m.markx.size)
    val1[::97] = 0.0
    return m, nu, mm, val1


def make_pl_case():
    from oracle import refdrv
    m, nu, mm, val1 = power_law_model()
    r = refdrv.RefModel(m)
    r.set_rheology(nu, mm, val1)
    r.ronurecalc()
    nodes = r.nodes()
    _, marke = r.val1_marke()
    out = {"markx": m.markx, "marky": m.marky, "markz": m.markz, "markt": m.markt, "n0": m.rocks.n0,
           "n1": m.rocks.n1, "ro": m.rocks.ro, "nu": nu, "mm": mm, "val1": val1, "marke_after": marke}
    out.update({"node_" + k: v for k, v in nodes.items()})
    np.savez_compressed(os.path.join(HERE, "pl17.npz"), **out)
    print("pl17 written", {k: np.asarray(v).shape for k, v in out.items()})


HEAT_VARIANTS = {
    # multinumt, multicyct, pre, post, frictyn, adiabyn, heatdif, timestep
    "mg": dict(multinumt=1, multicyct=2, pre=[3, 0], post=[0, 8], frictyn=1, adiabyn=1, heatdif=1.0, timestep=1e5),
    "single": dict(multinumt=0, multicyct=2, pre=[6], post=[0], frictyn=0, adiabyn=2, heatdif=0.0, timestep=3e4),
}
HEAT_COMMON = dict(maxtkstep=25.0, heatmin=5e-3, t0koef=1.0, t1koef=1.0, tdeep=1200.0, zdeep=0.6)


def heat_inputs(m):
    """Seeded inputs of the heat17 vectors (shared with the tests)."""
    th = M.thermal_fields(m, seed=11)
    n = m.nodenum
    rng = np.random.Generator(np.random.PCG64(12))
    f = lambda lo, hi: (lo + (hi - lo) * rng.random(n)).astype(np.float32)
    vel = [f(-1.0, 1.0) for _ in range(3)]
    se = [f(-100.0, 100.0) for _ in range(6)] + [f(-1.0, 1.0) for _ in range(6)]
    pr = (1e5 * rng.random(n)).astype(np.float64)
    mx, my, mz, mt = move_markers(m)
    q = np.arange(mx.size - 1)
    markk = np.where(q % 4 == 0, np.float32(0), np.float32(800) + np.float32(50) * (q % 13)).astype(np.float32)
    return th, vel, se, pr, (mx, my, mz, mt), markk


def heat_model():
    m = M.sphere_model(17, 2, (1, 1, 1), seed=11, eta_sphere=1e3)
    m.bc = M.with_thermal_bc(m)
    return m


def make_heat_case():
    """heat17.npz: titerate() of the reference (pardiso/heat3mg.c:292) on a
    17^3 box with fixed z planes and insulating walls, for HEAT_VARIANTS.
    The harness's last marker is the slot the reference reads past the
    marker arrays: the vectors cover the others."""
    from oracle import oracle as O
    from oracle import refdrv
    m = heat_model()
    th, vel, se, pr, mk, markk = heat_inputs(m)
    mx, my, mz, mt = mk
    r = refdrv.RefModel(m)
    r.set_tbc(m.bc)
    r.set_markers(mx, my, mz, mt)
    r.set_nodes({"nu": np.ones_like(th.ro), "ro": th.ro, "nxx": np.ones_like(th.ro), "nxy": np.ones_like(th.ro),
                 "nxz": np.ones_like(th.ro), "nyz": np.ones_like(th.ro)})
    r.set_velocity(*vel)
    r.set_stress(se)
    out = {"markk_in": markk}
    for name, v in HEAT_VARIANTS.items():
        hp = dict(HEAT_COMMON, **v, gx=m.params.gx, gy=m.params.gy, gz=m.params.gz, max_cycles=200)
        # the oracle first, with a cap: the reference itself loops until heatmin
        _, _, info = O.titerate(m.gx, m.gy, m.gz, v["multinumt"], m.bc.bondt, m.bc.bondv1, m.bc.bondn1, hp, th,
                                vel=vel, pr=pr, se=se, markers=(mx[:-1], my[:-1], mz[:-1], mt[:-1]), markk=markk)
        assert not info["capped"], (name, info)
        tk, mko = r.titerate(hp, v["multinumt"], th, markk, pr=pr)
        out["tk_" + name] = tk
        out["markk_" + name] = mko
        out["info_" + name] = np.array([info["substeps"], info["cycles"], info["tktimestep"]])
    np.savez_compressed(os.path.join(HERE, "heat17.npz"), **out)
    print("heat17 written", {k: np.asarray(v).shape for k, v in out.items()})


if __name__ == "__main__":
    # the reference keeps its state in globals: one case per process
    if len(sys.argv) > 1:
        if sys.argv[1] == "move17":
            make_move_case()
        elif sys.argv[1] == "pl17":
            make_pl_case()
        elif sys.argv[1] == "bulk21":
            make_bulk_case()
        elif sys.argv[1] == "heat17":
            make_heat_case()
        else:
            make_case(sys.argv[1], CASES[sys.argv[1]])
    else:
        import subprocess
        for c in list(CASES) + ["move17", "pl17", "bulk21", "heat17"]:
            subprocess.run([sys.executable, os.path.abspath(__file__), c], check=True)
