"""The reference's binary model file (.prn; loader() / saver() with file type
1, pardiso/load3mg.c:745-905 and 1298-1443) through the library's reader
and writer (p2_prn_read_header / p2_prn_read / p2_prn_write).

The reference's own saver() writes a model (node fields, gridlines, the
boundary rows of every level and the temperature rows, the rock table and
markers with their temperature / water / melt / strain values) from the
reference harness in a child process (its state lives in globals, one model
per process).  The library must read every value back exactly as the
reference's loader() would (floats as stored, the rock table in FP64), and
writing what it read must reproduce the file byte for byte.  A short file
and a file with other type sizes must be refused with a status, not a crash.
Skipped when oracle/_ref is not built (it needs the reference sources)."""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import refdrv

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from oracle import refdrv
from tests.test_prn import case
m, extra = case()
r = refdrv.RefModel(m)
r.set_tbc(m.bc)
r.ronurecalc()
rng = np.random.Generator(np.random.PCG64(5))
n = m.nodenum
r.set_velocity(*[(rng.random(n) - 0.5).astype(np.float32) for _ in range(3)])
r.save_prn(sys.argv[2], 7, *[extra[k] for k in ("tk", "cp", "et", "kt", "ht", "markk", "markw", "markd", "marke")])
nodes = r.nodes()
np.savez(sys.argv[3], **nodes)
"""


def case():
    from pardiso2_b200 import model as M
    from pardiso2_b200.prn import referenced_rows
    m = M.sphere_model(17, 2, (2, 2, 2), seed=3, eta_sphere=1e2)
    m.bc = referenced_rows(M.with_thermal_bc(m, 300.0, 1600.0))
    n, k = m.nodenum, m.markx.size
    rng = np.random.Generator(np.random.PCG64(4))
    extra = {key: (rng.random(n) * 1000).astype(np.float32) for key in ("tk", "cp", "et", "kt", "ht")}
    extra.update({key: (rng.random(k) * 10).astype(np.float32) for key in ("markk", "markw", "markd", "marke")})
    return m, extra


@pytest.fixture(scope="module")
def ref_file(tmp_path_factory):
    if not refdrv.available():
        pytest.skip("reference harness not built (needs the reference sources)")
    d = tmp_path_factory.mktemp("prn")
    path = os.path.join("/tmp", "p2prn_%d.prn" % os.getpid())  # the reference's file name buffer holds 59 characters
    nodes = str(d / "nodes.npz")
    env = dict(os.environ, OMP_NUM_THREADS="1")
    p = subprocess.run([sys.executable, "-c", CHILD, ROOT, path, nodes], env=env, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    yield path, np.load(nodes)
    os.remove(path)


def test_read_matches_what_the_reference_saved(ref_file):
    from pardiso2_b200 import prn
    path, nodes = ref_file
    m, extra = case()
    h, a = prn.read(path)
    assert (h.xnumx, h.ynumy, h.znumz) == m.shape
    assert h.cycle == 7 and h.marknum == m.markx.size and h.rocknum == len(m.rocks.n0)
    assert h.bondnum == m.bc.bondnum
    f = prn.node_fields(h, a)
    for k in ("tk", "cp", "et", "kt", "ht"):
        assert np.array_equal(f[k], extra[k]), k
    assert np.array_equal(f["nu"], nodes["nu"]) and np.array_equal(f["ro"], nodes["ro"])
    for g, gg in ((a["gx"], m.gx), (a["gy"], m.gy), (a["gz"], m.gz)):
        assert np.array_equal(g, gg.astype(np.float32))
    mk = a["markers"]
    assert np.array_equal(mk[:, 0], m.markx) and np.array_equal(mk[:, 1], m.marky) and np.array_equal(mk[:, 2], m.markz)
    for q, k in enumerate(("markk", "markw", "markd", "marke")):
        assert np.array_equal(mk[:, 3 + q], extra[k]), k
    assert np.array_equal(a["markt"], m.markt)
    r = a["rocks"]
    assert np.array_equal(r[0], m.rocks.n0) and np.array_equal(r[1], m.rocks.n1) and np.array_equal(r[16], m.rocks.ro)
    # the boundary tables rebuilt from the file are the ones the reference held
    bondm, bondv1, bondn1, bondt = prn.bc_tables(h, a, m.levels.total_nodes)
    assert np.array_equal(bondm, m.bc.bondm) and np.array_equal(bondt, m.bc.bondt)
    assert np.array_equal(bondv1, m.bc.bondv1) and np.array_equal(bondn1, m.bc.bondn1)


def test_write_reproduces_the_reference_file(ref_file, tmp_path):
    from pardiso2_b200 import prn
    path, _ = ref_file
    h, a = prn.read(path)
    out = str(tmp_path / "copy.prn")
    prn.write(out, h, a)
    assert open(out, "rb").read() == open(path, "rb").read()


def test_bad_files_are_refused(ref_file, tmp_path):
    from pardiso2_b200 import capi, prn
    path, _ = ref_file
    data = open(path, "rb").read()
    short = tmp_path / "short.prn"
    short.write_bytes(data[: len(data) // 2])
    with pytest.raises(capi.P2Error) as e:
        prn.read(str(short))
    assert e.value.code == 1 and "ends before" in str(e.value)
    sizes = tmp_path / "sizes.prn"
    sizes.write_bytes(bytes([4, 4]) + data[2:])  # a writer with a 4-byte long
    with pytest.raises(capi.P2Error) as e:
        prn.read(str(sizes))
    assert "LONG INT size" in str(e.value)
    with pytest.raises(capi.P2Error):
        prn.read(str(tmp_path / "missing.prn"))


def model_from_file(path, multinum):
    """A model (pardiso2_b200.model.Model) built from a binary model file:
    the file's gridlines (float, widened), boundary rows, rock table and
    markers; the multigrid depth comes from the caller (mode.t3c in the
    reference)."""
    from pardiso2_b200 import model as M
    from pardiso2_b200 import prn
    h, a = prn.read(path)
    gx, gy, gz = (a[k].astype(np.float64) for k in ("gx", "gy", "gz"))
    lv = M.make_levels(gx, gy, gz, multinum)
    bondm, bondv1, bondn1, bondt = prn.bc_tables(h, a, lv.total_nodes)
    r = a["rocks"]
    rocks = M.Rocks(r[0].copy(), r[1].copy(), r[16].copy())
    params = M.SolverParams(pinit=h.pinit, pin=(int(h.pxinit), int(h.pyinit), int(h.pzinit)), gx=h.gxkoef,
                            gy=h.gykoef, gz=h.gzkoef)
    mk = a["markers"]
    return M.Model("prn", gx, gy, gz, multinum, lv, M.BCTables(bondm, bondv1, bondn1, bondt),
                   np.ascontiguousarray(mk[:, 0]), np.ascontiguousarray(mk[:, 1]), np.ascontiguousarray(mk[:, 2]),
                   a["markt"].copy(), rocks, params)


@pytest.mark.gpu
def test_gpu_path_runs_from_a_reference_model_file(ref_file, oracle_mod):
    """Marker -> node fields on the GPU from the file's markers and grid,
    bit for bit with the oracle on the same inputs, and a converged solve."""
    import pardiso2_b200 as P
    path, _ = ref_file
    m = model_from_file(path, 2)
    prob = P.StokesProblem(m, tol=1e-8)
    f = prob.ronurecalc()
    fo = oracle_mod.ronurecalc(m)
    for k in f:
        assert np.array_equal(f[k], fo[k]), k
    _, info = prob.solve_fp64()
    prob.close()
    assert info.status == 0 and info.rel_residual <= 1e-8
