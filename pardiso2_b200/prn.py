"""The reference's binary model file (.prn) through the C ABI
(p2_prn_read_header / p2_prn_read / p2_prn_write, include/p2cuda.h), and the
conversion of a file into the inputs of the GPU path: gridlines, boundary
tables (bondm / bondv1 / bondn1 in the reference layout), node fields and
markers (pardiso/load3mg.c:745-905, the branch of loader() that needs no
HDF5)."""
from __future__ import annotations

import ctypes as C
from typing import Dict

import numpy as np

from . import capi

ROCK_TABLES = ("markn0", "markn1", "marks0", "marks1", "marknu", "markdh", "markdv", "markss", "markmm", "markll",
               "marka0", "marka1", "markb0", "markb1", "marke0", "marke1", "markro", "markbb", "markaa", "markcp",
               "markkt", "markkf", "markkp", "markht")
NODE_FIELDS = ("pr", "vx", "vy", "vz", "ro", "nu", "tk", "cp", "et", "kt", "ht")
MARKER_FIELDS = ("x", "y", "z", "markk", "markw", "markd", "marke")


class Header(C.Structure):
    _fields_ = [("xnumx", C.c_long), ("ynumy", C.c_long), ("znumz", C.c_long), ("mnumx", C.c_long),
                ("mnumy", C.c_long), ("mnumz", C.c_long), ("xsize", C.c_double), ("ysize", C.c_double),
                ("zsize", C.c_double), ("pxinit", C.c_long), ("pyinit", C.c_long), ("pzinit", C.c_long),
                ("pinit", C.c_double), ("gxkoef", C.c_double), ("gykoef", C.c_double), ("gzkoef", C.c_double),
                ("rocknum", C.c_int), ("bondnum", C.c_long), ("marknum", C.c_long), ("cycle", C.c_int),
                ("timesum_years", C.c_double), ("gridcur", C.c_double), ("gridtot", C.c_double)]

    def as_dict(self) -> Dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Data(C.Structure):
    _fields_ = [("rocks", C.c_void_p), ("nodes", C.c_void_p), ("gx", C.c_void_p), ("gy", C.c_void_p),
                ("gz", C.c_void_p), ("bond_index", C.c_void_p), ("bond_row", C.c_void_p),
                ("bond_value", C.c_void_p), ("bond_target", C.c_void_p), ("markers", C.c_void_p),
                ("markt", C.c_void_p)]


def _lib():
    L = capi.load()
    if not getattr(L, "_prn_sigs", False):
        L.p2_prn_read_header.argtypes = [C.c_char_p, C.POINTER(Header), C.c_char_p, C.c_long]
        L.p2_prn_read.argtypes = [C.c_char_p, C.POINTER(Header), C.POINTER(Data), C.c_char_p, C.c_long]
        L.p2_prn_write.argtypes = [C.c_char_p, C.POINTER(Header), C.POINTER(Data), C.c_char_p, C.c_long]
        for f in ("p2_prn_read_header", "p2_prn_read", "p2_prn_write"):
            getattr(L, f).restype = C.c_int
        L._prn_sigs = True
    return L


def _arrays(h: Header, arrays=None):
    n = h.xnumx * h.ynumy * h.znumz
    a = arrays or {
        "rocks": np.zeros((24, h.rocknum), np.float64), "nodes": np.zeros((n, 11), np.float32),
        "gx": np.zeros(h.xnumx, np.float32), "gy": np.zeros(h.ynumy, np.float32), "gz": np.zeros(h.znumz, np.float32),
        "bond_index": np.zeros(h.bondnum, np.int64), "bond_row": np.zeros(h.bondnum, np.int64),
        "bond_value": np.zeros((h.bondnum, 2), np.float32), "bond_target": np.zeros(h.bondnum, np.int64),
        "markers": np.zeros((h.marknum, 7), np.float32), "markt": np.zeros(h.marknum, np.int8)}
    d = Data(*[a[k].ctypes.data if a[k].size else None for k, _ in Data._fields_])
    return a, d


def read(path: str):
    """(header, arrays) of a binary model file; arrays in the file's layout."""
    L = _lib()
    h = Header()
    err = C.create_string_buffer(512)
    st = L.p2_prn_read_header(path.encode(), C.byref(h), err, len(err))
    if st:
        raise capi.P2Error(st, err.value.decode())
    a, d = _arrays(h)
    st = L.p2_prn_read(path.encode(), C.byref(h), C.byref(d), err, len(err))
    if st:
        raise capi.P2Error(st, err.value.decode())
    return h, a


def write(path: str, h: Header, arrays: Dict[str, np.ndarray]):
    """Write a binary model file the reference's loader() reads."""
    L = _lib()
    a = {k: np.ascontiguousarray(v) for k, v in arrays.items()}
    _, d = _arrays(h, a)
    err = C.create_string_buffer(512)
    st = L.p2_prn_write(path.encode(), C.byref(h), C.byref(d), err, len(err))
    if st:
        raise capi.P2Error(st, err.value.decode())


def bc_tables(h: Header, a: Dict[str, np.ndarray], total_nodes: int):
    """bondm (4 per node of every level), bondv1 (row -> const, koef) and
    bondn1 (row -> 1 + coupled unknown) as the reference holds them after
    loader(); temperature rows (bondm index from 8 * nodenum) are returned
    separately as bondt (per node of every level)."""
    nodenum = h.xnumx * h.ynumy * h.znumz
    nrow = int(a["bond_row"].max()) if a["bond_row"].size else 0
    bondm = np.zeros(4 * total_nodes, np.int32)
    bondt = np.zeros(total_nodes, np.int32)
    bondv1 = np.zeros((nrow + 1, 2), np.float32)
    bondn1 = np.zeros(nrow + 1, np.int32)
    for idx, row, val, tgt in zip(a["bond_index"], a["bond_row"], a["bond_value"], a["bond_target"]):
        if idx >= 8 * nodenum:
            bondt[idx - 8 * nodenum] = row
        else:
            bondm[idx] = row
        bondv1[row] = val
        bondn1[row] = tgt
    return bondm, bondv1, bondn1, bondt


def referenced_rows(bc):
    """The boundary tables with only the rows some bondm (or bondt) entry
    refers to, renumbered 1.. in order of first reference.  The reference's
    saver() writes one record per referenced row but stores bondnum as the
    row count (load3mg.c:1330, 1399-1410), and its loader() reads bondnum
    records, so a file is only consistent when no row is unreferenced (rows of
    overlapping boundary lines are overwritten in bondm)."""
    from .model import BCTables
    bondm = np.asarray(bc.bondm)
    bondt = np.asarray(bc.bondt) if bc.bondt is not None else None
    refs = np.concatenate([bondm[bondm > 0], bondt[bondt > 0] if bondt is not None else np.zeros(0, np.int64)])
    _, first = np.unique(refs, return_index=True)
    old = refs[np.sort(first)]
    new_id = np.zeros(bc.bondv1.shape[0], np.int32)
    new_id[old] = np.arange(1, old.size + 1, dtype=np.int32)
    v1 = np.zeros((old.size + 1, 2), np.float32)
    n1 = np.zeros(old.size + 1, np.int32)
    v1[1:] = bc.bondv1[old]
    n1[1:] = bc.bondn1[old]
    return BCTables(new_id[bondm].astype(np.int32), v1, n1,
                    new_id[bondt].astype(np.int32) if bondt is not None else None)


def node_fields(h: Header, a: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """Per-node fields as the reference's loader() leaves them (pr double,
    the rest float), by name."""
    out = {k: np.ascontiguousarray(a["nodes"][:, q]) for q, k in enumerate(NODE_FIELDS)}
    out["pr"] = out["pr"].astype(np.float64)
    return out
