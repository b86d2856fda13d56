"""ctypes driver for oracle/_ref/libp2ref.so, the reference's own C sources
compiled by oracle/Makefile (TEST INFRASTRUCTURE ONLY: tests, smoke() and
bench.py's CPU-baseline leg use it as the checker; the product never does).

Each instance owns the reference's global state, so only one model can be
live per process (the reference keeps everything in globals, head3mg.c).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libp2ref.so")
# the same harness with vpiterate()/ronurecalc() from the drop-in shim
# (pardiso2_b200/csrc/move3mg_cuda.c, calling libp2cuda.so on the GPU)
SHIM_LIB_PATH = os.path.join(_HERE, "_ref", "libp2ref_shim.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_bp = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")

_libs = {}
_live = set()


def available(shim: bool = False) -> bool:
    return os.path.exists(SHIM_LIB_PATH if shim else LIB_PATH)


def _load(shim: bool = False) -> C.CDLL:
    path = SHIM_LIB_PATH if shim else LIB_PATH
    if path not in _libs:
        lib = C.CDLL(path)
        lib.p2ref_init.argtypes = [C.c_long, C.c_long, C.c_long, _dp, _dp, _dp, C.c_int, C.c_long]
        lib.p2ref_init.restype = C.c_int
        lib.p2ref_levels.argtypes = [_ip] * 5
        lib.p2ref_level_coords.argtypes = [C.c_int, _dp, _dp, _dp]
        lib.p2ref_set_params.argtypes = [_dp, _ip, _ip, _ip]
        lib.p2ref_set_bc.argtypes = [_ip, C.c_long, _fp, _ip]
        lib.p2ref_set_bc.restype = C.c_int
        lib.p2ref_set_rocks.argtypes = [C.c_int, _dp, _dp, _dp]
        lib.p2ref_set_markers.argtypes = [_fp, _fp, _fp, _bp]
        lib.p2ref_set_nodes.argtypes = [_fp] * 6
        lib.p2ref_get_nodes.argtypes = [_fp] * 6
        lib.p2ref_get_level_fields.argtypes = [_fp] * 3
        lib.p2ref_ronurecalc.restype = C.c_double
        lib.p2ref_true_residual.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.p2ref_true_residual.restype = C.c_double
        lib.p2ref_vpiterate_first.restype = C.c_double
        lib.p2ref_vcycle.argtypes = [C.c_int]
        lib.p2ref_get_solution.argtypes = [_dp] * 4
        lib.p2ref_get_written.argtypes = [_dp, _fp, _fp, _fp]
        lib.p2ref_get_vectors.argtypes = [_dp, _dp, _dp]
        lib.p2ref_set_sol0.argtypes = [_dp]
        lib.p2ref_rows_nnz.argtypes = [C.c_int]
        lib.p2ref_rows_nnz.restype = C.c_long
        lib.p2ref_get_rows.argtypes = [C.c_int, _ip, _ip, _dp, _dp]
        lib.p2ref_rows_apply.argtypes = [C.c_int, _dp, _dp]
        lib.p2ref_restrict.argtypes = [C.c_int, _dp, _dp]
        lib.p2ref_prolong.argtypes = [C.c_int, _dp, _dp]
        lib.p2ref_set_quiet.argtypes = [C.c_int]
        lib.p2ref_set_velocity.argtypes = [_fp] * 3
        lib.p2ref_movemark.argtypes = [C.c_double, C.c_int, C.c_int]
        lib.p2ref_movemark.restype = C.c_double
        lib.p2ref_fill_markk.argtypes = [C.c_float]
        lib.p2ref_stress_strain.argtypes = [C.POINTER(C.c_void_p)]
        lib.p2ref_fill_stress.argtypes = [C.c_float]
        lib.p2ref_get_stress.argtypes = [C.POINTER(C.c_void_p)]
        lib.p2ref_set_step.argtypes = [C.c_double, C.c_double]
        lib.p2ref_set_marke.argtypes = [_fp]
        lib.p2ref_set_rheology.argtypes = [C.c_int, _dp, _dp, _dp]
        lib.p2ref_effbulk.argtypes = [_fp]
        lib.p2ref_fill_val1.argtypes = [C.c_double]
        lib.p2ref_get_val1_marke.argtypes = [_dp, _fp]
        lib.p2ref_get_timestep.restype = C.c_double
        lib.p2ref_get_markers.argtypes = [_fp] * 4
        lib.p2ref_set_tbc.argtypes = [_ip]
        lib.p2ref_set_stress.argtypes = [C.POINTER(C.c_void_p)]
        lib.p2ref_titerate.argtypes = [_dp, _ip, _fp, _fp, _fp, _fp, _fp, C.c_void_p, _fp, _dp]
        lib.p2ref_save.argtypes = [C.c_char_p, C.c_int] + [_fp] * 9
        lib.p2ref_save.restype = C.c_int
        lib.p2ref_lu_count.restype = C.c_int
        lib.p2ref_num_threads.restype = C.c_int
        _libs[path] = lib
    return _libs[path]


class RefModel:
    """The reference's global state set up for one Model (pardiso2_b200.model)."""

    def __init__(self, model, npre=None, npost=None, shim: bool = False):
        key = SHIM_LIB_PATH if shim else LIB_PATH
        if key in _live:
            raise RuntimeError("the reference keeps its state in globals: one RefModel per library and process")
        lib = _load(shim)
        self.lib = lib
        self.m = model
        nx, ny, nz = model.shape
        nlev = lib.p2ref_init(nx, ny, nz, model.gx, model.gy, model.gz, model.multinum, model.markx.size)
        if nlev != model.multinum:
            raise RuntimeError("reference init failed")
        _live.add(key)
        L = nlev + 1
        self.mgx = np.zeros(L, np.int32)
        self.mgy = np.zeros(L, np.int32)
        self.mgz = np.zeros(L, np.int32)
        self.mgp = np.zeros(L, np.int32)
        self.mgn = np.zeros(L, np.int32)
        lib.p2ref_levels(self.mgx, self.mgy, self.mgz, self.mgp, self.mgn)
        p = model.params
        dpar = np.array([p.p0koef, p.p1koef, p.p2koef, p.v0koef, p.v1koef, p.nubeg, p.nuend, p.nukoef,
                         p.gx, p.gy, p.gz, p.pinit], dtype=np.float64)
        ipar = np.array([p.viscmod, p.pin[0], p.pin[1], p.pin[2], 1], dtype=np.int32)
        npre = np.array(npre if npre is not None else [2] * L, dtype=np.int32)
        npost = np.array(npost if npost is not None else [2] * L, dtype=np.int32)
        lib.p2ref_set_params(dpar, ipar, npre, npost)
        bc = model.bc
        if lib.p2ref_set_bc(np.ascontiguousarray(bc.bondm, np.int32), bc.bondnum,
                            np.ascontiguousarray(bc.bondv1.reshape(-1), np.float32),
                            np.ascontiguousarray(bc.bondn1, np.int32)):
            raise RuntimeError("too many boundary equations for the reference (MAXBON)")
        r = model.rocks
        lib.p2ref_set_rocks(len(r.n0), np.ascontiguousarray(r.n0, np.float64),
                            np.ascontiguousarray(r.n1, np.float64), np.ascontiguousarray(r.ro, np.float64))
        if model.markx.size:
            lib.p2ref_set_markers(model.markx, model.marky, model.markz, np.ascontiguousarray(model.markt, np.int8))

    # -- marker -> node ----------------------------------------------------
    def ronurecalc(self) -> float:
        return self.lib.p2ref_ronurecalc()

    def nodes(self):
        n = self.m.nodenum
        out = [np.zeros(n, np.float32) for _ in range(6)]
        self.lib.p2ref_get_nodes(*out)
        return dict(zip(("nu", "ro", "nxx", "nxy", "nxz", "nyz"), out))

    def set_nodes(self, f):
        self.lib.p2ref_set_nodes(*[np.ascontiguousarray(f[k], np.float32)
                                   for k in ("nu", "ro", "nxx", "nxy", "nxz", "nyz")])

    def level_fields(self):
        n = int(self.mgp[-1] + self.mgn[-1])
        out = [np.zeros(n, np.float32) for _ in range(3)]
        self.lib.p2ref_get_level_fields(*out)
        return dict(zip(("nu", "ro", "nd"), out))

    # -- solve -------------------------------------------------------------
    def residual(self):
        rn, bn = C.c_double(), C.c_double()
        rel = self.lib.p2ref_true_residual(C.byref(rn), C.byref(bn))
        return rel, rn.value, bn.value

    def first_iteration(self) -> float:
        return self.lib.p2ref_vpiterate_first()

    def vcycle(self, coarse: bool = True):
        self.lib.p2ref_vcycle(1 if coarse else 0)

    def solve(self, tol=1e-8, max_cycles=200, coarse=True, verbose=False):
        hist = []
        self.first_iteration()
        rel = self.residual()[0]
        hist.append(rel)
        it = 0
        while rel > tol and it < max_cycles:
            self.vcycle(coarse)
            rel = self.residual()[0]
            hist.append(rel)
            it += 1
            if verbose:
                print("ref cycle %d rel %.3e" % (it, rel))
        return hist

    def written(self):
        """The arrays vpiterate() writes back: pr (double), vx, vy, vz (float)."""
        n = self.m.nodenum
        pr = np.zeros(n, np.float64)
        v = [np.zeros(n, np.float32) for _ in range(3)]
        self.lib.p2ref_get_written(pr, *v)
        return {"pr": pr, "vx": v[0], "vy": v[1], "vz": v[2]}

    def set_markers(self, mx, my, mz, mt):
        """Replace the marker coordinates and types (same count as the model's)."""
        if np.asarray(mx).size != self.m.markx.size:
            raise ValueError("the reference's marker count is fixed at init")
        self.lib.p2ref_set_markers(*[np.ascontiguousarray(a, np.float32) for a in (mx, my, mz)],
                                   np.ascontiguousarray(mt, np.int8))

    def set_velocity(self, vx, vy, vz):
        self.lib.p2ref_set_velocity(*[np.ascontiguousarray(a, np.float32) for a in (vx, vy, vz)])

    def movemark(self, timestep, markmod=2, outgrid=0) -> float:
        """movemark() over one step; returns its wall time (s)."""
        return self.lib.p2ref_movemark(timestep, markmod, outgrid)

    STRESS_KEYS = ("sxx", "syy", "szz", "sxy", "sxz", "syz", "exx", "eyy", "ezz", "exy", "exz", "eyz")

    def stress_strain(self, init=0.0):
        """The reference's stress / strain-rate pass on its current vx, vy, vz
        and node viscosities; untouched positions hold init."""
        n = self.m.nodenum
        out = {k: np.full(n, init, np.float32) for k in self.STRESS_KEYS}
        arr = (C.c_void_p * 12)(*[out[k].ctypes.data for k in self.STRESS_KEYS])
        self.lib.p2ref_stress_strain(arr)
        return out

    def fill_stress(self, value):
        """Set vpiterate's stress / strain-rate globals to value everywhere."""
        self.lib.p2ref_fill_stress(value)

    def written_stress(self):
        """vpiterate's stress / strain-rate globals (dict of float32 arrays)."""
        n = self.m.nodenum
        out = {k: np.zeros(n, np.float32) for k in self.STRESS_KEYS}
        self.lib.p2ref_get_stress((C.c_void_p * 12)(*[out[k].ctypes.data for k in self.STRESS_KEYS]))
        return out

    def update_stress(self):
        """Run the stress / strain-rate pass into vpiterate's globals."""
        self.lib.p2ref_update_stress()

    def effbulk(self, ro, workdir):
        """effbulkvisccalc(1) with density ro on the current node fields and
        vpiterate's stress globals; returns the 36 numbers of the line it
        appends to workdir/effbulkvisc.txt (printed with %e)."""
        here = os.getcwd()
        os.chdir(workdir)
        try:
            self.lib.p2ref_effbulk(np.ascontiguousarray(ro, np.float32))
            with open(os.path.join(workdir, "effbulkvisc.txt")) as f:
                line = f.read().strip().splitlines()[-1]
        finally:
            os.chdir(here)
        return np.array([float(v) for v in line.split()])

    def set_rheology(self, marknu, markmm, val1):
        """Power-law parameters per rock type and val1 per marker."""
        self.lib.p2ref_set_rheology(len(marknu), np.ascontiguousarray(marknu, np.float64),
                                    np.ascontiguousarray(markmm, np.float64), np.ascontiguousarray(val1, np.float64))

    def set_marke(self, marke):
        self.lib.p2ref_set_marke(np.ascontiguousarray(marke, np.float32))

    def fill_val1(self, value):
        self.lib.p2ref_fill_val1(value)

    def val1_marke(self):
        n = self.m.markx.size
        v, e = np.zeros(n, np.float64), np.zeros(n, np.float32)
        self.lib.p2ref_get_val1_marke(v, e)
        return v, e

    def set_step(self, max_step, timestep):
        """maxxystep and timestep, the inputs of vpiterate's time-step limit."""
        self.lib.p2ref_set_step(max_step, timestep)

    def timestep(self) -> float:
        return self.lib.p2ref_get_timestep()

    def fill_markk(self, value):
        self.lib.p2ref_fill_markk(value)

    def markers(self):
        """markx, marky, markz, markk after the reference's marker routines."""
        n = self.m.markx.size
        out = [np.zeros(n, np.float32) for _ in range(4)]
        self.lib.p2ref_get_markers(*out)
        return out

    def solution(self):
        n = self.m.nodenum
        out = [np.zeros(n, np.float64) for _ in range(4)]
        self.lib.p2ref_get_solution(*out)
        return dict(zip(("pr", "vx", "vy", "vz"), out))

    def rows(self, lev=0):
        nnz = self.lib.p2ref_rows_nnz(lev)
        row = np.zeros(nnz, np.int32)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz, np.float64)
        rhs = np.zeros(int(self.mgn[lev]) * 4, np.float64)
        self.lib.p2ref_get_rows(lev, row, col, val, rhs)
        return row, col, val, rhs

    def vectors(self):
        n = int(self.mgp[-1] + self.mgn[-1]) * 4
        s0, f1, f0 = (np.zeros(n, np.float64) for _ in range(3))
        self.lib.p2ref_get_vectors(s0, f1, f0)
        return s0, f1, f0

    def restrict(self, lev_coarse, fine_res):
        out = np.zeros(int(self.mgn[lev_coarse]) * 4, np.float64)
        self.lib.p2ref_restrict(lev_coarse, np.ascontiguousarray(fine_res, np.float64), out)
        return out

    def prolong(self, lev_coarse, coarse_x, fine_x):
        f = np.ascontiguousarray(fine_x, np.float64).copy()
        self.lib.p2ref_prolong(lev_coarse, np.ascontiguousarray(coarse_x, np.float64), f)
        return f

    def num_threads(self):
        return self.lib.p2ref_num_threads()


    # -- heat equation ------------------------------------------------------
    def save_prn(self, path: str, cycle: int, tk, cp, et, kt, ht, markk, markw, markd, marke):
        """The reference's saver() in its binary branch (load3mg.c:1275) to
        path (under 60 characters): the harness's node fields with the given
        thermal fields (level 0) and marker properties."""
        f = lambda a: np.ascontiguousarray(a, np.float32)
        st = self.lib.p2ref_save(path.encode(), cycle, f(tk), f(cp), f(et), f(kt), f(ht), f(markk), f(markw), f(markd),
                                 f(marke))
        if st == -1:
            raise ValueError("path too long for the reference's file-name buffer: %s" % path)
        if st:
            raise MemoryError("could not extend the reference's bondm array")

    def set_tbc(self, bc):
        """Boundary tables including the temperature rows (model.BCTables with
        bondt): the Stokes rows and the shared row table, then the T section."""
        lib = self.lib
        if lib.p2ref_set_bc(np.ascontiguousarray(bc.bondm, np.int32), bc.bondnum,
                            np.ascontiguousarray(bc.bondv1.reshape(-1), np.float32),
                            np.ascontiguousarray(bc.bondn1, np.int32)):
            raise RuntimeError("too many boundary equations for the reference (MAXBON)")
        lib.p2ref_set_tbc(np.ascontiguousarray(bc.bondt, np.int32))

    def titerate(self, hp: dict, multinumt: int, thermal, markk, pr=None):
        """The reference's titerate(0) on the harness globals (markers from
        set_markers, velocities from set_velocity, stresses from
        fill_stress / update_stress).  The harness's last marker is the slot
        the reference reads past the marker arrays and stays outside the box;
        markk covers the others.  Returns (tk, markk)."""
        dpar = np.array([hp[k] for k in ("timestep", "maxtkstep", "heatmin", "t0koef", "t1koef", "heatdif", "tdeep",
                                         "zdeep")], np.float64)
        ip = np.zeros(36, np.int32)
        ip[0], ip[1], ip[2], ip[3] = multinumt, hp["multicyct"], hp["frictyn"], hp["adiabyn"]
        ip[4:4 + len(hp["pre"])] = hp["pre"]
        ip[20:20 + len(hp["post"])] = hp["post"]
        tk = np.array(thermal.tk, np.float32, copy=True)
        mk = np.zeros(self.m.markx.size, np.float32)
        mk[:len(markk)] = markk
        out = np.zeros(2, np.float64)
        f = lambda a: np.ascontiguousarray(a, np.float32)
        prp = None
        if pr is not None:
            prp = np.ascontiguousarray(pr, np.float64)
        self.lib.p2ref_titerate(dpar, ip, tk, f(thermal.kt), f(thermal.cp), f(thermal.ht), f(thermal.et),
                                None if prp is None else prp.ctypes.data_as(C.c_void_p), mk, out)
        return tk, mk[:len(markk)]

    def set_stress(self, arrays):
        """sxx syy szz sxy sxz syz exx eyy ezz exy exz eyz (float, node layout)."""
        arrs = [np.ascontiguousarray(a, np.float32) for a in arrays]
        ptrs = (C.c_void_p * 12)(*[a.ctypes.data_as(C.c_void_p) for a in arrs])
        self.lib.p2ref_set_stress(ptrs)
