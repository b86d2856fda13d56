"""ctypes wrapper of the oracle restatement oracle/libp2oracle.so (built from
oracle/p2oracle.c by oracle/Makefile).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use it as the checker; nothing in pardiso2_b200 imports it.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libp2oracle.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_bp = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")
_lib: Optional[C.CDLL] = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        L.p2o_create.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_int, _ip, _fp, _ip]
        L.p2o_create.restype = C.c_void_p
        L.p2o_destroy.argtypes = [C.c_void_p]
        L.p2o_set_params.argtypes = [C.c_void_p, _dp, C.c_int, _ip, _ip]
        L.p2o_set_fields.argtypes = [C.c_void_p] + [_fp] * 6
        L.p2o_set_fields.restype = C.c_int
        L.p2o_solve.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, _dp]
        L.p2o_solve.restype = C.c_int
        L.p2o_get_solution.argtypes = [C.c_void_p] + [_dp] * 4
        L.p2o_set_solution.argtypes = [C.c_void_p] + [_dp] * 4
        L.p2o_apply.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        L.p2o_rhs.argtypes = [C.c_void_p, _dp]
        L.p2o_level_fields.argtypes = [C.c_void_p, C.c_int, _fp, _fp, _dp]
        L.p2o_rel_residual.argtypes = [C.c_void_p]
        L.p2o_rel_residual.restype = C.c_double
        L.p2o_ronurecalc.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_long, _fp, _fp, _fp, _bp,
                                     _dp, _dp, C.c_double, C.c_double, C.c_double, C.c_int] + [_fp] * 6 + [
                                         C.c_void_p] * 4
        L.p2o_movemark.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _fp, _fp, _fp, C.c_double, C.c_int,
                                   C.c_int, C.c_long, _fp, _fp, _fp, _bp, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
        L.p2o_stress_strain.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp] + [_fp] * 7 + [
            C.c_double, C.c_double, C.POINTER(C.c_void_p)]
        L.p2o_effbulk.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p), _dp,
                                  np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")]
        L.p2o_titerate.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_int, _ip, _fp, _ip, _dp, _ip,
                                   _fp, _fp, _fp, _fp, _fp, _fp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, _dp]
        L.p2o_titerate.restype = C.c_int
        _lib = L
    return _lib


BULK_KEYS = ("ro", "nxx", "nxy", "nxz", "nyz", "exx", "eyy", "ezz", "exy", "exz", "eyz",
             "sxx", "syy", "szz", "sxy", "sxz", "syz")


def effbulk(model, fields):
    """effbulkvisccalc(1) diagnostics by the oracle: (out[34], counts[3]) with
    out = eiin siin eiivp tau2 hsn nubulkn nubulk1..4, matrix[12], incl[12]
    and counts = numtot nummat numinc."""
    L = lib()
    nx, ny, nz = model.shape
    arrs = [np.ascontiguousarray(fields[k], np.float32) for k in BULK_KEYS]
    ptrs = (C.c_void_p * 17)(*[a.ctypes.data for a in arrs])
    out = np.zeros(34, np.float64)
    counts = np.zeros(3, np.int64)
    L.p2o_effbulk(nx, ny, nz, ptrs, out, counts)
    return out, counts


STRESS_KEYS = ("sxx", "syy", "szz", "sxy", "sxz", "syz", "exx", "eyy", "ezz", "exy", "exz", "eyz")


def stress_strain(model, vel, nodes, init=0.0):
    """Post-solve stresses and strain rates by the oracle (dict of float32
    arrays; positions the reference does not write hold init)."""
    L = lib()
    nx, ny, nz = model.shape
    out = {k: np.full(model.nodenum, init, np.float32) for k in STRESS_KEYS}
    arr = (C.c_void_p * 12)(*[out[k].ctypes.data for k in STRESS_KEYS])
    f = [np.ascontiguousarray(a, np.float32) for a in vel] + [np.ascontiguousarray(nodes[k], np.float32)
                                                             for k in ("nxx", "nxy", "nxz", "nyz")]
    p = model.params
    L.p2o_stress_strain(nx, ny, nz, model.gx, model.gy, model.gz, *f, p.nubeg, p.nuend, arr)
    return out


def ronurecalc(model, init=None, marknu=None, markmm=None, val1=None, markers=None):
    """Marker -> node fields (dict of float32 arrays) computed by the oracle;
    with marknu, markmm and val1 (per marker) rock types <= 20 with markn0 !=
    markn1 take the power-law viscosity.  markers = (x, y, z, type) defaults
    to the model's."""
    L = lib()
    n = model.nodenum
    keys = ("nu", "ro", "nxx", "nxy", "nxz", "nyz")
    out = {k: (np.array(init[k], np.float32) if init is not None else np.zeros(n, np.float32)) for k in keys}
    p = model.params
    nx, ny, nz = model.shape
    mx, my, mz, mt = markers if markers is not None else (model.markx, model.marky, model.markz, model.markt)
    extra = [None] * 4
    keep = []
    if val1 is not None:
        arrs = [np.ascontiguousarray(a, np.float64) for a in (model.rocks.n1, marknu, markmm, val1)]
        keep += arrs
        extra = [a.ctypes.data for a in arrs]
    L.p2o_ronurecalc(nx, ny, nz, model.gx, model.gy, model.gz, np.asarray(mx).size,
                     np.ascontiguousarray(mx, np.float32), np.ascontiguousarray(my, np.float32),
                     np.ascontiguousarray(mz, np.float32), np.ascontiguousarray(mt, np.int8),
                     np.ascontiguousarray(model.rocks.n0, np.float64), np.ascontiguousarray(model.rocks.ro, np.float64),
                     p.nubeg, p.nuend, p.nukoef, p.viscmod, *[out[k] for k in keys], *extra)
    return out


def movemark(model, vel, timestep, markmod=2, outgrid=0, markers=None, markk=None, strain=None, val1=None,
             marke=None):
    """Marker advection by the oracle: returns new (markx, marky, markz) and,
    when markk is given, the updated copy of it; with strain = (exx, eyy, ezz,
    exy, exz, eyz) node fields also the updated copies of val1 and marke.
    vel = (vx, vy, vz) float32 in the node layout; markers defaults to the
    model's."""
    L = lib()
    nx, ny, nz = model.shape
    mx, my, mz, mt = markers if markers is not None else (model.markx, model.marky, model.markz, model.markt)
    out = [np.array(a, np.float32) for a in (mx, my, mz)]
    kk = None if markk is None else np.array(markk, np.float32)
    n = out[0].size
    sp, v1, me = None, None, None
    keep = []
    if strain is not None:
        fields = [np.ascontiguousarray(a, np.float32) for a in strain]
        keep += fields
        sp = (C.c_void_p * 6)(*[a.ctypes.data for a in fields])
        v1 = np.zeros(n, np.float64) if val1 is None else np.array(val1, np.float64)
        me = np.zeros(n, np.float32) if marke is None else np.array(marke, np.float32)
    L.p2o_movemark(nx, ny, nz, model.gx, model.gy, model.gz, *[np.ascontiguousarray(a, np.float32) for a in vel],
                   timestep, markmod, outgrid, n, out[0], out[1], out[2],
                   np.ascontiguousarray(mt, np.int8), None if kk is None else kk.ctypes.data,
                   None if sp is None else C.cast(sp, C.c_void_p), None if v1 is None else v1.ctypes.data,
                   None if me is None else me.ctypes.data)
    res = tuple(out) + ((kk,) if kk is not None else ())
    return res + ((v1, me) if strain is not None else ())


class OracleSolver:
    """FP64 CPU multigrid on the reference's discrete Stokes problem."""

    def __init__(self, model, npre=None, npost=None):
        L = lib()
        self.L = L
        self.m = model
        nx, ny, nz = model.shape
        bc = model.bc
        # keep the tables alive: the C side stores the pointers
        self._bondm = np.ascontiguousarray(bc.bondm, np.int32)
        self._bondv1 = np.ascontiguousarray(bc.bondv1.reshape(-1), np.float32)
        self._bondn1 = np.ascontiguousarray(bc.bondn1, np.int32)
        self.h = L.p2o_create(nx, ny, nz, model.gx, model.gy, model.gz, model.multinum,
                              self._bondm, self._bondv1, self._bondn1)
        if not self.h:
            raise RuntimeError("oracle create failed")
        nlev = model.multinum + 1
        p = model.params
        if p.p2koef != 0:
            raise ValueError("the oracle restates p2koef == 0 only")
        dpar = np.array([p.p0koef, p.p1koef, p.v0koef, p.v1koef, p.nubeg, p.nuend, p.gx, p.gy, p.gz], np.float64)
        self.npre = np.array(npre if npre is not None else [2] * nlev, np.int32)
        self.npost = np.array(npost if npost is not None else [2] * nlev, np.int32)
        L.p2o_set_params(self.h, dpar, p.viscmod, self.npre, self.npost)

    def close(self):
        if self.h:
            self.L.p2o_destroy(self.h)
            self.h = None

    __del__ = close

    def set_fields(self, f):
        st = self.L.p2o_set_fields(self.h, *[np.ascontiguousarray(f[k], np.float32)
                                             for k in ("nu", "ro", "nxx", "nxy", "nxz", "nyz")])
        if st != 0:
            raise RuntimeError("coarsest LU failed (status %d)" % st)

    def solve(self, tol=1e-8, max_cycles=100, restart=8):
        hist = np.zeros(max_cycles + 1, np.float64)
        it = self.L.p2o_solve(self.h, tol, max_cycles, restart, hist)
        return hist[: it + 1]

    def solution(self):
        n = self.m.nodenum
        out = [np.zeros(n, np.float64) for _ in range(4)]
        self.L.p2o_get_solution(self.h, *out)
        return dict(zip(("pr", "vx", "vy", "vz"), out))

    def set_solution(self, s):
        self.L.p2o_set_solution(self.h, *[np.ascontiguousarray(s[k], np.float64) for k in ("pr", "vx", "vy", "vz")])

    def apply(self, lev, x):
        y = np.zeros_like(x)
        self.L.p2o_apply(self.h, lev, np.ascontiguousarray(x, np.float64), y)
        return y

    def rhs(self):
        b = np.zeros(self.m.nodenum * 4, np.float64)
        self.L.p2o_rhs(self.h, b)
        return b

    def rel_residual(self):
        return self.L.p2o_rel_residual(self.h)


def _transfer_sigs():
    L = lib()
    L.p2o_restrict.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_int]
    L.p2o_prolong.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
    return L


def restrict(solver: "OracleSolver", lc: int, fine_res, n_coarse: int, compat: bool = False):
    out = np.zeros(n_coarse * 4, np.float64)
    _transfer_sigs().p2o_restrict(solver.h, lc, np.ascontiguousarray(fine_res, np.float64), out, 1 if compat else 0)
    return out


def prolong(solver: "OracleSolver", lc: int, coarse_x, fine_x):
    f = np.array(fine_x, np.float64)
    _transfer_sigs().p2o_prolong(solver.h, lc, np.ascontiguousarray(coarse_x, np.float64), f)
    return f


HEAT_DPAR = ("timestep", "maxtkstep", "heatmin", "t0koef", "t1koef", "heatdif", "tdeep", "zdeep", "gx", "gy", "gz")


def heat_ipar(multinumt, multicyct, frictyn, adiabyn, max_cycles, pre, post):
    """ipar of p2o_titerate: multicyct, frictyn, adiabyn, max_cycles,
    multittt[0][0..15], multittt[1][0..15]."""
    ip = np.zeros(36, np.int32)
    ip[0], ip[1], ip[2], ip[3] = multicyct, frictyn, adiabyn, max_cycles
    ip[4:4 + len(pre)] = pre
    ip[20:20 + len(post)] = post
    return ip


def titerate(gx, gy, gz, multinumt, bondt, bondv1, bondn1, hp: dict, thermal, vel=None, pr=None, se=None,
             markers=None, markk=None):
    """titerate() restated (heat3mg.c:292-829): returns (tk, markk, info).
    hp holds HEAT_DPAR keys and multicyct, frictyn, adiabyn, max_cycles,
    pre (multittt[0]), post (multittt[1])."""
    L = lib()
    nx, ny, nz = len(gx), len(gy), len(gz)
    dpar = np.array([hp[k] for k in HEAT_DPAR], np.float64)
    ipar = heat_ipar(multinumt, hp["multicyct"], hp["frictyn"], hp["adiabyn"], hp.get("max_cycles", 0),
                     hp["pre"], hp["post"])
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
    info = np.zeros(8, np.float64)
    L.p2o_titerate(nx, ny, nz, np.ascontiguousarray(gx, np.float64), np.ascontiguousarray(gy, np.float64),
                   np.ascontiguousarray(gz, np.float64), multinumt, np.ascontiguousarray(bondt, np.int32),
                   np.ascontiguousarray(np.asarray(bondv1, np.float32).reshape(-1)),
                   np.ascontiguousarray(bondn1, np.int32), dpar, ipar, tk, f(thermal.kt), f(thermal.cp),
                   f(thermal.ro), f(thermal.ht), f(thermal.et),
                   *(vp(v, np.float32) for v in (vel if vel is not None else (None, None, None))),
                   vp(pr, np.float64), sep, nm,
                   *(vp(a, np.float32) for a in (markers[:3] if markers is not None else (None, None, None))),
                   vp(markers[3] if markers is not None else None, np.int8),
                   None if mk is None else mk.ctypes.data_as(C.c_void_p), info)
    return tk, mk, {"tktimestep": info[0], "substeps": int(info[1]), "cycles": int(info[2]), "heatsum": info[3],
                    "mintk": info[4], "maxtk": info[5], "capped": int(info[6]), "maxtkrate": info[7]}
