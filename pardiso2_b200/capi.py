"""ctypes binding of libp2cuda.so (include/p2cuda.h).

Only plain host pointers and sizes cross this boundary.  There is no CPU
fallback: if the library or a CUDA device is missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libp2cuda.so")

P2_MAX_LEVELS = 12
STATUS = {0: "P2_OK", 1: "P2_ERR_ARG", 2: "P2_ERR_CUDA", 3: "P2_ERR_NOMEM", 4: "P2_ERR_NOT_CONVERGED",
          5: "P2_ERR_NAN", 6: "P2_ERR_SINGULAR", 7: "P2_ERR_STATE", 8: "P2_ERR_UNSUPPORTED"}
EXPORTED = ["p2_default_params", "p2_create", "p2_destroy", "p2_last_error", "p2_set_grid", "p2_set_bc",
            "p2_set_nodes", "p2_stokes_solve", "p2_stokes_solve_resident", "p2_get_solution", "p2_ronurecalc",
            "p2_upload_markers", "p2_ronurecalc_resident", "p2_get_nodes", "p2_debug_apply", "p2_debug_restrict",
            "p2_debug_prolong", "p2_debug_level_fields", "p2_debug_time_smoother", "p2_debug_smooth",
            "p2_debug_time_sweep", "p2_debug_time_stage", "p2_debug_rows_kernel", "p2_debug_vcycle", "p2_ronurecalc_noalloc", "p2_autotune",
            "p2_movemark", "p2_movemark_resident", "p2_get_markers", "p2_stress_strain",
            "p2_stokes_solve_batch", "p2_movemark_strain", "p2_ronurecalc_powerlaw", "p2_effbulk_visc",
            "p2_default_heat_params", "p2_heat_set_bc", "p2_titerate", "p2_prn_read_header", "p2_prn_read",
            "p2_prn_write"]


class Params(C.Structure):
    _fields_ = [("p0koef", C.c_double), ("p1koef", C.c_double), ("p2koef", C.c_double), ("v0koef", C.c_double),
                ("v1koef", C.c_double), ("nubeg", C.c_double), ("nuend", C.c_double), ("nukoef", C.c_double),
                ("gxkoef", C.c_double), ("gykoef", C.c_double), ("gzkoef", C.c_double), ("pinit", C.c_double),
                ("pxinit", C.c_int), ("pyinit", C.c_int), ("pzinit", C.c_int), ("viscmod", C.c_int),
                ("multinum", C.c_int), ("npre", C.c_int * P2_MAX_LEVELS), ("npost", C.c_int * P2_MAX_LEVELS),
                ("tol", C.c_double), ("max_iter", C.c_int), ("precision", C.c_int), ("restart", C.c_int),
                ("omega", C.c_double), ("use_graphs", C.c_int), ("smoother", C.c_int)]


class TuneInfo(C.Structure):
    _fields_ = [("smoother", C.c_int), ("sweep_growth", C.c_int), ("est_ms", C.c_double), ("rate", C.c_double),
                ("candidates", C.c_int), ("trial_iters", C.c_int), ("sweep_max", C.c_int),
                ("restart", C.c_int), ("sweeps0", C.c_int)]

    def as_dict(self) -> Dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class EffBulk(C.Structure):
    _fields_ = [("eiin", C.c_double), ("siin", C.c_double), ("eiivp", C.c_double), ("tau2", C.c_double),
                ("hsn", C.c_double), ("nubulkn", C.c_double), ("nubulk1", C.c_double), ("nubulk2", C.c_double),
                ("nubulk3", C.c_double), ("nubulk4", C.c_double), ("matrix", C.c_double * 12),
                ("incl", C.c_double * 12), ("numtot", C.c_long), ("nummat", C.c_long), ("numinc", C.c_long)]

    def as_dict(self) -> Dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["matrix"] = list(self.matrix)
        d["incl"] = list(self.incl)
        return d


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("rel_residual", C.c_double), ("rel_residual0", C.c_double),
                ("ms_total", C.c_double), ("ms_setup", C.c_double), ("ms_vcycles", C.c_double), ("status", C.c_int),
                ("kernels", C.c_longlong)]

    def as_dict(self) -> Dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class HeatParams(C.Structure):
    _fields_ = [("maxtkstep", C.c_double), ("heatmin", C.c_double), ("t0koef", C.c_double), ("t1koef", C.c_double),
                ("heatdif", C.c_double), ("tdeep", C.c_double), ("zdeep", C.c_double), ("multinumt", C.c_int),
                ("multicyct", C.c_int), ("multittt", (C.c_int * 12) * 2), ("frictyn", C.c_int),
                ("adiabyn", C.c_int), ("max_cycles", C.c_int)]


class HeatInfo(C.Structure):
    _fields_ = [("tktimestep", C.c_double), ("maxtkrate", C.c_double), ("substeps", C.c_int), ("cycles", C.c_int),
                ("converged", C.c_int), ("heatsum", C.c_double), ("mintk", C.c_double), ("maxtk", C.c_double),
                ("ms_total", C.c_double), ("kernels", C.c_longlong)]

    def as_dict(self) -> Dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


def heat_params(**kw) -> HeatParams:
    """p2_default_heat_params (mode.t3c values) with keyword overrides;
    pre / post set multittt[0] / multittt[1] per level."""
    hp = HeatParams()
    load().p2_default_heat_params(C.byref(hp))
    for k, v in kw.items():
        if k in ("pre", "post"):
            row = hp.multittt[0 if k == "pre" else 1]
            for i, n in enumerate(v):
                row[i] = int(n)
        elif k in ("gx", "gy", "gz", "timestep"):
            continue
        else:
            setattr(hp, k, v)
    return hp


class P2Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("%s: %s" % (STATUS.get(code, code), msg))
        self.code = code


_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_bp = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")
_lib: Optional[C.CDLL] = None


def load() -> C.CDLL:
    """Load the library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libp2cuda.so is not built (run python -m pardiso2_b200.build)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.p2_default_params.argtypes = [C.POINTER(Params)]
    L.p2_create.argtypes = [C.POINTER(vp), C.c_int]
    L.p2_destroy.argtypes = [vp]
    L.p2_last_error.argtypes = [vp]
    L.p2_last_error.restype = C.c_char_p
    L.p2_set_grid.argtypes = [vp, C.c_long, C.c_long, C.c_long, _dp, _dp, _dp, C.c_int, C.c_int, C.c_int,
                              C.POINTER(Params)]
    L.p2_set_bc.argtypes = [vp, _ip, C.c_long, _fp, _ip, C.c_long]
    L.p2_set_nodes.argtypes = [vp] + [_fp] * 6
    L.p2_stokes_solve.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(SolveInfo)]
    L.p2_stokes_solve_resident.argtypes = [vp, C.POINTER(SolveInfo)]
    L.p2_get_solution.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.p2_ronurecalc.argtypes = [vp, C.c_long, _fp, _fp, _fp, _bp, C.c_int, _dp, _dp, _dp] + [_fp] * 6
    L.p2_upload_markers.argtypes = [vp, C.c_long, _fp, _fp, _fp, _bp, C.c_int, _dp, _dp, _dp]
    L.p2_ronurecalc_resident.argtypes = [vp, C.POINTER(C.c_double)]
    L.p2_get_nodes.argtypes = [vp] + [C.c_void_p] * 6
    L.p2_autotune.argtypes = [vp, C.c_int, C.POINTER(TuneInfo)]
    L.p2_autotune.restype = C.c_int
    L.p2_movemark.argtypes = [vp, C.c_double, C.c_int, C.c_int, _fp, _fp, _fp, C.c_long, _fp, _fp, _fp, _bp]
    L.p2_movemark_resident.argtypes = [vp, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.p2_get_markers.argtypes = [vp, _fp, _fp, _fp]
    L.p2_stress_strain.argtypes = [vp] + [C.c_void_p] * 12 + [C.POINTER(C.c_double)]
    L.p2_stokes_solve_batch.argtypes = [C.POINTER(vp), C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_double)]
    L.p2_stokes_solve_batch.restype = C.c_int
    L.p2_movemark_strain.argtypes = [vp, C.c_double, C.c_int, C.c_int] + [_fp] * 9 + [C.c_long, _fp, _fp, _fp, _bp,
                                                                                          _dp, _fp]
    L.p2_movemark_strain.restype = C.c_int
    L.p2_ronurecalc_powerlaw.argtypes = [vp, C.c_long, _fp, _fp, _fp, _bp, C.c_int] + [_dp] * 6 + [_fp] * 6
    L.p2_ronurecalc_powerlaw.restype = C.c_int
    L.p2_effbulk_visc.argtypes = [vp] + [_fp] * 17 + [C.POINTER(EffBulk)]
    L.p2_effbulk_visc.restype = C.c_int
    L.p2_default_heat_params.argtypes = [C.POINTER(HeatParams)]
    L.p2_default_heat_params.restype = None
    L.p2_heat_set_bc.argtypes = [vp, _ip, C.c_long, _fp, _ip, C.c_long]
    L.p2_heat_set_bc.restype = C.c_int
    L.p2_titerate.argtypes = [vp, C.POINTER(HeatParams), C.c_double, _fp] + [_fp] * 5 + [C.c_void_p] * 5 + [
        C.c_long] + [C.c_void_p] * 5 + [C.POINTER(HeatInfo)]
    L.p2_titerate.restype = C.c_int
    for f in ("p2_movemark", "p2_movemark_resident", "p2_get_markers", "p2_stress_strain"):
        getattr(L, f).restype = C.c_int
    for f in ("p2_create", "p2_set_grid", "p2_set_bc", "p2_set_nodes", "p2_stokes_solve", "p2_stokes_solve_resident",
              "p2_get_solution", "p2_ronurecalc", "p2_upload_markers", "p2_ronurecalc_resident", "p2_get_nodes"):
        getattr(L, f).restype = C.c_int
    _lib = L
    return L


def default_params() -> Params:
    p = Params()
    load().p2_default_params(C.byref(p))
    return p


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Context:
    """One device context (p2_ctx): levels, boundary tables, node fields and
    solver state stay resident on the GPU across calls."""

    def __init__(self, device: int = 0):
        self.L = load()
        h = C.c_void_p()
        st = self.L.p2_create(C.byref(h), device)
        if st != 0:
            raise P2Error(st, "p2_create failed (is a CUDA device visible?)")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.p2_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, st: int, what: str):
        if st != 0:
            raise P2Error(st, "%s: %s" % (what, self.L.p2_last_error(self.h).decode()))

    def set_grid(self, gx, gy, gz, params: Params, periodic=(0, 0, 0)):
        gx, gy, gz = (np.ascontiguousarray(a, np.float64) for a in (gx, gy, gz))
        self._check(self.L.p2_set_grid(self.h, gx.size, gy.size, gz.size, gx, gy, gz, *periodic, C.byref(params)),
                    "p2_set_grid")

    def set_bc(self, bondm, bondv1, bondn1):
        bm = np.ascontiguousarray(bondm, np.int32)
        bv = np.ascontiguousarray(np.asarray(bondv1, np.float32).reshape(-1))
        bn = np.ascontiguousarray(bondn1, np.int32)
        self._check(self.L.p2_set_bc(self.h, bm, bm.size, bv, bn, bn.size - 1), "p2_set_bc")

    def set_nodes(self, f: Dict[str, np.ndarray]):
        self._check(self.L.p2_set_nodes(self.h, *[np.ascontiguousarray(f[k], np.float32)
                                                   for k in ("nu", "ro", "nxx", "nxy", "nxz", "nyz")]),
                    "p2_set_nodes")

    def stokes_solve(self, vx=None, vy=None, vz=None, pr=None, check=True):
        """vpiterate(): in/out arrays (float vx/vy/vz, double pr); returns SolveInfo."""
        info = SolveInfo()
        st = self.L.p2_stokes_solve(self.h, _ptr(vx), _ptr(vy), _ptr(vz), _ptr(pr), C.byref(info))
        if check:
            self._check(st, "p2_stokes_solve")
        return info

    def autotune(self, trial_iters: int = 16) -> TuneInfo:
        """Pick the smoother configuration on the resident fields (p2_autotune)."""
        info = TuneInfo()
        self._check(self.L.p2_autotune(self.h, trial_iters, C.byref(info)), "p2_autotune")
        return info

    def movemark(self, timestep: float, vx, vy, vz, mx, my, mz, mt, markmod: int = 2, outgrid: int = 0):
        """movemark(): returns the moved marker coordinates (new float32 arrays)."""
        out = [np.array(a, np.float32) for a in (mx, my, mz)]
        self._check(self.L.p2_movemark(self.h, timestep, markmod, outgrid, np.ascontiguousarray(vx, np.float32),
                                       np.ascontiguousarray(vy, np.float32), np.ascontiguousarray(vz, np.float32),
                                       out[0].size, out[0], out[1], out[2], np.ascontiguousarray(mt, np.int8)),
                    "p2_movemark")
        return out

    def movemark_strain(self, timestep: float, vel, strain, markers, val1, marke, markmod: int = 2, outgrid: int = 0):
        """movemark with its strain-rate outputs: vel = (vx, vy, vz), strain =
        (exx, eyy, ezz, exy, exz, eyz) float node fields, markers = (x, y, z,
        type).  Returns new (x, y, z, val1, marke) arrays."""
        out = [np.array(a, np.float32) for a in markers[:3]]
        v1 = np.array(val1, np.float64)
        me = np.array(marke, np.float32)
        f = [np.ascontiguousarray(a, np.float32) for a in list(vel) + list(strain)]
        self._check(self.L.p2_movemark_strain(self.h, timestep, markmod, outgrid, *f, out[0].size, out[0], out[1],
                                              out[2], np.ascontiguousarray(markers[3], np.int8), v1, me),
                    "p2_movemark_strain")
        return out[0], out[1], out[2], v1, me

    BULK_KEYS = ("ro", "nxx", "nxy", "nxz", "nyz", "exx", "eyy", "ezz", "exy", "exz", "eyz",
                 "sxx", "syy", "szz", "sxy", "sxz", "syz")

    def heat_set_bc(self, bc, nodenum: int):
        """Temperature boundary rows from model.BCTables (with bondt)."""
        bm = bc.reference_bondm(nodenum)
        bv = np.ascontiguousarray(np.asarray(bc.bondv1, np.float32).reshape(-1))
        bn = np.ascontiguousarray(bc.bondn1, np.int32)
        self._check(self.L.p2_heat_set_bc(self.h, bm, bm.size, bv, bn, bn.size - 1), "p2_heat_set_bc")

    def titerate(self, hp: HeatParams, timestep: float, thermal, vel=None, pr=None, se=None, markers=None,
                 markk=None):
        """One titerate() step: returns (tk, markk, HeatInfo); the inputs are
        not modified."""
        tk = np.array(thermal.tk, np.float32, copy=True)
        f = lambda a: np.ascontiguousarray(a, np.float32)
        keep = []

        def vp(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dt)
            keep.append(a)
            return a.ctypes.data_as(C.c_void_p)

        sep = None
        if se is not None:
            arrs = [np.ascontiguousarray(a, np.float32) for a in se]
            keep.extend(arrs)
            sep_arr = (C.c_void_p * 12)(*[a.ctypes.data_as(C.c_void_p) for a in arrs])
            keep.append(sep_arr)
            sep = C.cast(sep_arr, C.c_void_p)
        nm = 0 if markers is None else len(markers[0])
        mk = None if markk is None else np.array(markk, np.float32, copy=True)
        info = HeatInfo()
        v3 = vel if vel is not None else (None, None, None)
        m4 = markers if markers is not None else (None, None, None, None)
        self._check(self.L.p2_titerate(self.h, C.byref(hp), timestep, tk, f(thermal.kt), f(thermal.cp),
                                       f(thermal.ro), f(thermal.ht), f(thermal.et),
                                       *(vp(v, np.float32) for v in v3), vp(pr, np.float64), sep, nm,
                                       *(vp(a, np.float32) for a in m4[:3]), vp(m4[3], np.int8),
                                       None if mk is None else mk.ctypes.data_as(C.c_void_p), C.byref(info)),
                    "p2_titerate")
        return tk, mk, info

    def effbulk_visc(self, fields: Dict[str, np.ndarray]) -> EffBulk:
        """effbulkvisccalc(1) diagnostics of node fields (keys BULK_KEYS)."""
        out = EffBulk()
        self._check(self.L.p2_effbulk_visc(self.h, *[np.ascontiguousarray(fields[k], np.float32)
                                                     for k in self.BULK_KEYS], C.byref(out)), "p2_effbulk_visc")
        return out

    def movemark_resident(self, timestep: float, markmod: int = 2, outgrid: int = 0) -> float:
        ms = C.c_double()
        self._check(self.L.p2_movemark_resident(self.h, timestep, markmod, outgrid, C.byref(ms)), "p2_movemark_resident")
        return ms.value

    def get_markers(self, nmark: int):
        out = [np.zeros(nmark, np.float32) for _ in range(3)]
        self._check(self.L.p2_get_markers(self.h, *out), "p2_get_markers")
        return out

    STRESS_KEYS = ("sxx", "syy", "szz", "sxy", "sxz", "syz", "exx", "eyy", "ezz", "exy", "exz", "eyz")

    def stress_strain(self, fields: Dict[str, np.ndarray]):
        """Post-solve stresses and strain rates into float32 arrays (modified in
        place; keys of STRESS_KEYS, missing keys skipped); returns the velocity
        ranges (min vx, max vx, min vy, max vy, min vz, max vz)."""
        ptrs = []
        for k in self.STRESS_KEYS:
            a = fields.get(k)
            if a is not None and (a.dtype != np.float32 or not a.flags.c_contiguous):
                raise ValueError("field %s must be a contiguous float32 array" % k)
            ptrs.append(None if a is None else a.ctypes.data)
        vr = (C.c_double * 6)()
        self._check(self.L.p2_stress_strain(self.h, *ptrs, vr), "p2_stress_strain")
        return tuple(vr)

    def solve_resident(self, check=True) -> SolveInfo:
        info = SolveInfo()
        st = self.L.p2_stokes_solve_resident(self.h, C.byref(info))
        if check:
            self._check(st, "p2_stokes_solve_resident")
        return info

    def solution(self, n: int) -> Dict[str, np.ndarray]:
        out = {k: np.zeros(n, np.float64) for k in ("vx", "vy", "vz", "pr")}
        self._check(self.L.p2_get_solution(self.h, _ptr(out["vx"]), _ptr(out["vy"]), _ptr(out["vz"]),
                                           _ptr(out["pr"])), "p2_get_solution")
        return out

    def upload_markers(self, mx, my, mz, mt, n0, n1, ro):
        self._check(self.L.p2_upload_markers(self.h, mx.size, np.ascontiguousarray(mx, np.float32),
                                             np.ascontiguousarray(my, np.float32), np.ascontiguousarray(mz, np.float32),
                                             np.ascontiguousarray(mt, np.int8), len(n0),
                                             np.ascontiguousarray(n0, np.float64), np.ascontiguousarray(n1, np.float64),
                                             np.ascontiguousarray(ro, np.float64)), "p2_upload_markers")

    def ronurecalc_resident(self) -> float:
        ms = C.c_double()
        self._check(self.L.p2_ronurecalc_resident(self.h, C.byref(ms)), "p2_ronurecalc_resident")
        return ms.value

    def get_nodes(self, n: int) -> Dict[str, np.ndarray]:
        keys = ("nu", "ro", "nxx", "nxy", "nxz", "nyz")
        out = {k: np.zeros(n, np.float32) for k in keys}
        self._check(self.L.p2_get_nodes(self.h, *[_ptr(out[k]) for k in keys]), "p2_get_nodes")
        return out

    def ronurecalc_powerlaw(self, mx, my, mz, mt, n0, n1, ro, nu0, mm, val1, fields: Dict[str, np.ndarray]):
        """ronurecalc() with power-law rocks: in/out node fields (float32 arrays, modified in place)."""
        keys = ("nu", "ro", "nxx", "nxy", "nxz", "nyz")
        for k in keys:
            if fields[k].dtype != np.float32 or not fields[k].flags.c_contiguous:
                raise ValueError("node field %s must be a contiguous float32 array" % k)
        d = [np.ascontiguousarray(a, np.float64) for a in (n0, n1, ro, nu0, mm, val1)]
        self._check(self.L.p2_ronurecalc_powerlaw(self.h, np.asarray(mx).size, np.ascontiguousarray(mx, np.float32),
                                                  np.ascontiguousarray(my, np.float32),
                                                  np.ascontiguousarray(mz, np.float32),
                                                  np.ascontiguousarray(mt, np.int8), len(d[0]), *d,
                                                  *[fields[k] for k in keys]), "p2_ronurecalc_powerlaw")
        return fields

    def ronurecalc(self, mx, my, mz, mt, n0, n1, ro, fields: Dict[str, np.ndarray]):
        """ronurecalc(): in/out node fields (dict of float32 arrays, modified in place)."""
        keys = ("nu", "ro", "nxx", "nxy", "nxz", "nyz")
        for k in keys:
            if fields[k].dtype != np.float32 or not fields[k].flags.c_contiguous:
                raise ValueError("node field %s must be a contiguous float32 array" % k)
        self._check(self.L.p2_ronurecalc(self.h, mx.size, np.ascontiguousarray(mx, np.float32),
                                         np.ascontiguousarray(my, np.float32), np.ascontiguousarray(mz, np.float32),
                                         np.ascontiguousarray(mt, np.int8), len(n0), np.ascontiguousarray(n0, np.float64),
                                         np.ascontiguousarray(n1, np.float64), np.ascontiguousarray(ro, np.float64),
                                         *[fields[k] for k in keys]), "p2_ronurecalc")
        return fields


def solve_batch(contexts, host_threads: int = 0):
    """p2_stokes_solve_batch: resident solves of several contexts at once.
    Returns (list of SolveInfo, device ms of the whole batch); raises on the
    first failing status."""
    if not contexts:
        return [], 0.0
    L = contexts[0].L
    hs = (C.c_void_p * len(contexts))(*[c.h for c in contexts])
    infos = (SolveInfo * len(contexts))()
    ms = C.c_double()
    st = L.p2_stokes_solve_batch(hs, len(contexts), host_threads, C.cast(infos, C.c_void_p), C.byref(ms))
    if st != 0:
        bad = [i for i, x in enumerate(infos) if x.status != 0]
        raise P2Error(st, "p2_stokes_solve_batch: status %d (instances %s)" % (st, bad[:8]))
    return list(infos), ms.value


def _debug_sigs(L):
    _dpp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    _fpp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
    L.p2_debug_apply.argtypes = [C.c_void_p, C.c_int, _dpp, _dpp]
    L.p2_debug_restrict.argtypes = [C.c_void_p, C.c_int, _dpp, _dpp, C.c_int]
    L.p2_debug_prolong.argtypes = [C.c_void_p, C.c_int, _dpp, _dpp]
    L.p2_debug_level_fields.argtypes = [C.c_void_p, _fpp, _fpp]
    L.p2_debug_time_smoother.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.p2_debug_smooth.argtypes = [C.c_void_p, C.c_int, C.c_int, _dpp, _dpp]
    L.p2_debug_time_sweep.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.p2_debug_time_stage.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.p2_debug_rows_kernel.argtypes = [C.c_void_p, C.c_int]
    L.p2_debug_vcycle.argtypes = [C.c_void_p, _dpp, _dpp]
    for f in ("p2_debug_apply", "p2_debug_restrict", "p2_debug_prolong", "p2_debug_level_fields",
              "p2_debug_time_smoother", "p2_debug_smooth", "p2_debug_time_sweep", "p2_debug_time_stage",
              "p2_debug_rows_kernel", "p2_debug_vcycle"):
        getattr(L, f).restype = C.c_int


class DebugHooks:
    """Single-stage test hooks of the library (FP64, interleaved [P,Vx,Vy,Vz])."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        _debug_sigs(ctx.L)

    def apply(self, level: int, x: np.ndarray) -> np.ndarray:
        y = np.zeros_like(x, dtype=np.float64)
        self.ctx._check(self.ctx.L.p2_debug_apply(self.ctx.h, level, np.ascontiguousarray(x, np.float64), y),
                        "p2_debug_apply")
        return y

    def restrict(self, coarse_level: int, fine_res: np.ndarray, n_coarse: int, compat: bool = False) -> np.ndarray:
        out = np.zeros(n_coarse * 4, np.float64)
        self.ctx._check(self.ctx.L.p2_debug_restrict(self.ctx.h, coarse_level, np.ascontiguousarray(fine_res, np.float64),
                                                     out, 1 if compat else 0), "p2_debug_restrict")
        return out

    def prolong(self, coarse_level: int, coarse_x: np.ndarray, fine_x: np.ndarray) -> np.ndarray:
        f = np.array(fine_x, np.float64)
        self.ctx._check(self.ctx.L.p2_debug_prolong(self.ctx.h, coarse_level, np.ascontiguousarray(coarse_x, np.float64),
                                                    f), "p2_debug_prolong")
        return f

    def time_smoother(self, level: int = 0, passes: int = 20) -> float:
        ms = C.c_double()
        self.ctx._check(self.ctx.L.p2_debug_time_smoother(self.ctx.h, level, passes, C.byref(ms)),
                        "p2_debug_time_smoother")
        return ms.value

    def smooth(self, level: int, sweeps: int, b: np.ndarray, x: np.ndarray) -> np.ndarray:
        out = np.array(x, np.float64)
        self.ctx._check(self.ctx.L.p2_debug_smooth(self.ctx.h, level, sweeps, np.ascontiguousarray(b, np.float64),
                                                   out), "p2_debug_smooth")
        return out

    def time_sweep(self, level: int = 0, sweeps: int = 2) -> float:
        ms = C.c_double()
        self.ctx._check(self.ctx.L.p2_debug_time_sweep(self.ctx.h, level, sweeps, C.byref(ms)), "p2_debug_time_sweep")
        return ms.value

    STAGES = {"residual": 0, "true_residual": 1, "restrict": 2, "prolong": 3, "operator": 4}

    def time_stage(self, stage: str, level: int = 0, variant: int = 0, reps: int = 10) -> float:
        """Mean device time (ms) of one solve stage (p2_debug_time_stage)."""
        ms = C.c_double()
        self.ctx._check(self.ctx.L.p2_debug_time_stage(self.ctx.h, self.STAGES[stage], level, variant, reps,
                                                       C.byref(ms)), "p2_debug_time_stage")
        return ms.value

    def rows_kernel(self, variant: int):
        """Kernel of the operator rows for later calls (p2_debug_rows_kernel)."""
        self.ctx._check(self.ctx.L.p2_debug_rows_kernel(self.ctx.h, variant), "p2_debug_rows_kernel")

    def vcycle(self, b: np.ndarray) -> np.ndarray:
        """One preconditioning V-cycle from zero for the level-0 rhs b (p2_debug_vcycle)."""
        x = np.zeros(b.size, np.float64)
        self.ctx._check(self.ctx.L.p2_debug_vcycle(self.ctx.h, np.ascontiguousarray(b, np.float64), x),
                        "p2_debug_vcycle")
        return x

    def level_fields(self, total_nodes: int):
        nu = np.zeros(total_nodes, np.float32)
        ro = np.zeros(total_nodes, np.float32)
        self.ctx._check(self.ctx.L.p2_debug_level_fields(self.ctx.h, nu, ro), "p2_debug_level_fields")
        return nu, ro
