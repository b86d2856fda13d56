"""Seeded synthetic Stokes models: grid, multigrid levels, boundary tables,
markers and rock tables, in the reference's own array layouts.

Everything here produces plain numpy arrays that are handed, unchanged, to
both the CUDA library (through its C ABI) and the CPU oracles, so that both
paths solve exactly the same discrete problem.

Reference semantics reproduced here:
  * level sizes and coarse gridlines: pardiso/load3mg.c:2064-2194 (gridcheck)
  * boundary-condition lines -> per-level tables bondm/bondv1/bondn1:
    pardiso/in3mg.c:237-390 (the per-level index mapping is at 304-323,
    the table entries at 331-349)
  * regular markers per cell: pardiso/in3mg.c:175-216 (the reference jitters
    them with libc rand(); here a seeded numpy PCG64 stream does it)
  * ellipsoid/sphere rock bodies: pardiso/in3mg.c:571-594
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

P, VX, VY, VZ, T = 0, 1, 2, 3, 4


# --------------------------------------------------------------------------
# Grid and levels
# --------------------------------------------------------------------------
@dataclasses.dataclass
class Levels:
    """Multigrid level tables mgx/mgy/mgz/mgxy/mgn/mgp/mgs and the per-level
    gridlines mggx/mggy/mggz (pardiso/load3mg.c:2056-2194)."""

    mgx: List[int]
    mgy: List[int]
    mgz: List[int]
    mgxy: List[int]
    mgn: List[int]
    mgp: List[int]
    mgs: List[int]
    cx: List[np.ndarray]
    cy: List[np.ndarray]
    cz: List[np.ndarray]

    @property
    def multinum(self) -> int:
        return len(self.mgx) - 1

    @property
    def total_nodes(self) -> int:
        return self.mgp[-1] + self.mgn[-1]


def _coarse_lines(g: np.ndarray, nl: int, s: int) -> np.ndarray:
    n = len(g)
    c = np.empty(nl, dtype=np.float64)
    c[0], c[1], c[2] = g[0], g[1], g[2]
    c[nl - 1], c[nl - 2], c[nl - 3] = g[n - 1], g[n - 2], g[n - 3]
    for n2 in range(3, nl - 3):
        c[n2] = g[(n2 - 2) * s + 2]
    return c


def make_levels(gx: np.ndarray, gy: np.ndarray, gz: np.ndarray, multinum: int) -> Levels:
    """Level sizes n_{l+1} = (n_l - 5)//2 + 5 and coarse lines: outer three
    lines on each side copied, interior line n2 = fine line (n2-2)*2^l + 2."""
    nx, ny, nz = len(gx), len(gy), len(gz)
    mgx, mgy, mgz, mgxy, mgn, mgp, mgs = [nx], [ny], [nz], [nx * ny], [nx * ny * nz], [0], [1]
    for _ in range(1, multinum + 1):
        mgp.append(mgp[-1] + mgn[-1])
        mgs.append(mgs[-1] * 2)
        mgx.append((mgx[-1] - 5) // 2 + 5)
        mgy.append((mgy[-1] - 5) // 2 + 5)
        mgz.append((mgz[-1] - 5) // 2 + 5)
        mgxy.append(mgx[-1] * mgy[-1])
        mgn.append(mgx[-1] * mgy[-1] * mgz[-1])
    for n in (mgx[-1], mgy[-1], mgz[-1]):
        if n < 6:
            raise ValueError("coarsest level too small: %d nodes per axis" % n)
    cx = [_coarse_lines(gx, mgx[l], mgs[l]) for l in range(multinum + 1)]
    cy = [_coarse_lines(gy, mgy[l], mgs[l]) for l in range(multinum + 1)]
    cz = [_coarse_lines(gz, mgz[l], mgs[l]) for l in range(multinum + 1)]
    return Levels(mgx, mgy, mgz, mgxy, mgn, mgp, mgs, cx, cy, cz)


def uniform_lines(n: int, size: float = 1.0) -> np.ndarray:
    """Gridlines gx[0]=0, gx[i]=gx[i-1]+size/(n-1) (pardiso/in3mg.c:106-111)."""
    g = np.zeros(n, dtype=np.float64)
    step = size / float(n - 1)
    for i in range(1, n):
        g[i] = g[i - 1] + step
    return g


# --------------------------------------------------------------------------
# Boundary-condition tables
# --------------------------------------------------------------------------
@dataclasses.dataclass
class BCLine:
    """One line of the reference's boundary description:
    VAR m10 m11 m20 m21 m30 m31 Const Koef [dm1 dm2 dm3]  (fine indices,
    negative values are relative to the last node: -1 == n-1, -2 == n-2)."""

    var: int
    m10: int
    m11: int
    m20: int
    m21: int
    m30: int
    m31: int
    const: float
    koef: float = 0.0
    shift: Tuple[int, int, int] = (0, 0, 0)


@dataclasses.dataclass
class BCTables:
    bondm: np.ndarray   # int32[4 * total_nodes]; 0 = no BC, else row in bondv1/bondn1
    bondv1: np.ndarray  # float32[bondnum + 1, 2] = (const, koef)
    bondn1: np.ndarray  # int32[bondnum + 1]; 1 + unknown index of the coupled unknown, 0 = none
    # temperature rows per node of every level (bondm[8*nodenum + u] in the
    # reference layout), None when the lines have no T entries
    bondt: Optional[np.ndarray] = None

    @property
    def bondnum(self) -> int:
        return int(self.bondv1.shape[0] - 1)

    def reference_bondm(self, nodenum: int) -> np.ndarray:
        """bondm as the reference lays it out: the four Stokes unknowns per
        node of every level from 0, the temperature rows from 8 * nodenum
        (pardiso/load3mg.c:2250, in3mg.c:367-383)."""
        total = self.bondm.size // 4
        out = np.zeros(max(self.bondm.size, 8 * nodenum + total), dtype=np.int32)
        out[:self.bondm.size] = self.bondm
        if self.bondt is not None:
            out[8 * nodenum:8 * nodenum + total] = self.bondt
        return out


def _map_index(m: int, nfine: int, nlev: int, s: int) -> int:
    # pardiso/in3mg.c:306-323 (C integer division truncates toward zero)
    r = int((m - 2) / s) + 2
    if m < 3:
        r = m
    if m > nfine - 4:
        r = nlev - (nfine - m)
    return r


def build_bc_tables(lv: Levels, lines: Sequence[BCLine]) -> BCTables:
    nx, ny, nz = lv.mgx[0], lv.mgy[0], lv.mgz[0]
    bondm = np.zeros(4 * lv.total_nodes, dtype=np.int32)
    bondt = np.zeros(lv.total_nodes, dtype=np.int32) if any(ln.var == T for ln in lines) else None
    consts: List[np.ndarray] = []
    koefs: List[np.ndarray] = []
    targets: List[np.ndarray] = []
    bondnum = 0

    def absidx(v: int, n: int) -> int:
        return v if v >= 0 else n + v

    for ln in lines:
        m10, m11 = absidx(ln.m10, nx), absidx(ln.m11, nx)
        m20, m21 = absidx(ln.m20, ny), absidx(ln.m21, ny)
        m30, m31 = absidx(ln.m30, nz), absidx(ln.m31, nz)
        has_shift = any(ln.shift)
        for l in range(lv.multinum + 1):
            s = lv.mgs[l]
            a1 = _map_index(m10, nx, lv.mgx[l], s)
            b1 = _map_index(m11, nx, lv.mgx[l], s)
            a2 = _map_index(m20, ny, lv.mgy[l], s)
            b2 = _map_index(m21, ny, lv.mgy[l], s)
            a3 = _map_index(m30, nz, lv.mgz[l], s)
            b3 = _map_index(m31, nz, lv.mgz[l], s)
            if b1 < a1 or b2 < a2 or b3 < a3:
                continue
            # node loop order m3, m1, m2 (pardiso/in3mg.c:328-330)
            m3, m1, m2 = np.meshgrid(np.arange(a3, b3 + 1), np.arange(a1, b1 + 1),
                                     np.arange(a2, b2 + 1), indexing="ij")
            m4 = (lv.mgp[l] + m3 * lv.mgxy[l] + m1 * lv.mgy[l] + m2).ravel()
            sx, sy, sz = ln.shift
            # |shift| > 1 means periodic wrap (pardiso/in3mg.c:335-337)
            if abs(sx) > 1:
                sx = -(lv.mgx[l] - 1)
            if abs(sy) > 1:
                sy = -(lv.mgy[l] - 1)
            if abs(sz) > 1:
                sz = -(lv.mgz[l] - 1)
            m6 = m4 + sz * lv.mgxy[l] + sx * lv.mgy[l] + sy
            cnt = m4.size
            ids = np.arange(bondnum + 1, bondnum + cnt + 1, dtype=np.int64)
            if ln.var == T:
                bondt[m4] = ids   # in3mg.c:367-383: node index, target m6 + 1
            else:
                bondm[m4 * 4 + ln.var] = ids
            consts.append(np.full(cnt, ln.const, dtype=np.float32))
            if has_shift:
                koefs.append(np.full(cnt, ln.koef, dtype=np.float32))
                targets.append((m6 + 1 if ln.var == T else m6 * 4 + ln.var + 1).astype(np.int64))
            else:
                koefs.append(np.zeros(cnt, dtype=np.float32))
                targets.append(np.zeros(cnt, dtype=np.int64))
            bondnum += cnt
    bondv1 = np.zeros((bondnum + 1, 2), dtype=np.float32)
    bondn1 = np.zeros(bondnum + 1, dtype=np.int32)
    if bondnum:
        bondv1[1:, 0] = np.concatenate(consts)
        bondv1[1:, 1] = np.concatenate(koefs)
        bondn1[1:] = np.concatenate(targets).astype(np.int32)
    return BCTables(bondm, bondv1, bondn1, bondt)


def thermal_lines(t_low: float = 273.0, t_high: float = 1573.0) -> List[BCLine]:
    """Temperature rows of a closed box: fixed temperatures on the z = 0 and
    z = max planes, insulating x and y walls (the wall node copies its inner
    neighbour, koef 1).  The x walls come after the y walls, so the vertical
    edges copy a y-wall node (a chain of two rows); the z planes come last."""
    return [BCLine(T, 0, -1, 0, 0, 0, -1, 0.0, 1.0, (0, +1, 0)),
            BCLine(T, 0, -1, -1, -1, 0, -1, 0.0, 1.0, (0, -1, 0)),
            BCLine(T, 0, 0, 0, -1, 0, -1, 0.0, 1.0, (+1, 0, 0)),
            BCLine(T, -1, -1, 0, -1, 0, -1, 0.0, 1.0, (-1, 0, 0)),
            BCLine(T, 0, -1, 0, -1, 0, 0, t_low),
            BCLine(T, 0, -1, 0, -1, -1, -1, t_high)]


@dataclasses.dataclass
class Thermal:
    """Level-0 node fields of the heat equation (float32, node layout)."""
    tk: np.ndarray
    kt: np.ndarray
    cp: np.ndarray
    ro: np.ndarray
    ht: np.ndarray
    et: np.ndarray


def thermal_fields(model: "Model", seed: int = 7, t_low: float = 273.0, t_high: float = 1573.0,
                   sphere_dt: float = 200.0, heat: Tuple[float, float] = (500.0, 2000.0)) -> Thermal:
    """Synthetic thermal state on the model's grid: a linear profile in z
    between the fixed planes plus a hot sphere, rock-like conductivity,
    heat capacity, density (above 2000, where the adiabatic and shear
    heating terms apply) and heat sources, with seeded +-5 % noise."""
    nx, ny, nz = model.shape
    Z, X, Y = np.meshgrid(model.gz, model.gx, model.gy, indexing="ij")
    zs = (Z - model.gz[0]) / (model.gz[-1] - model.gz[0])
    inside = ((X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2) < 0.2 ** 2
    rng = np.random.Generator(np.random.PCG64(seed))
    noise = lambda: 1.0 + 0.05 * (rng.random(Z.shape) - 0.5) * 2
    tk = t_low + (t_high - t_low) * zs + sphere_dt * inside
    kt = np.where(inside, 4.5, 2.5) * noise()
    cp = 1000.0 * noise()
    ro = np.where(inside, 3300.0, 3000.0) * noise()
    ht = np.where(inside, heat[1], heat[0]) * noise()
    et = 3e-5 * noise()
    f = lambda a: np.ascontiguousarray(a.reshape(-1), np.float32)
    return Thermal(f(tk), f(kt), f(cp), f(ro), f(ht), f(et))


def with_thermal_bc(model: "Model", t_low: float = 273.0, t_high: float = 1573.0) -> BCTables:
    """The model's free-slip tables with the thermal box rows added."""
    return build_bc_tables(model.levels, free_slip_lines(model.params.pin, model.params.pinit)
                           + thermal_lines(t_low, t_high))


def free_slip_lines(pin: Tuple[int, int, int] = (2, 2, 2), pin_value: float = 0.0) -> List[BCLine]:
    """Closed free-slip box in the reference's boundary language: the normal
    velocity is 0 on the wall line; the first/last interior half-cell of each
    tangential component copies its inner neighbour (koef 1, shift +-1);
    one pressure cell is pinned (the reference's 'P 2 2 2 2 2 2 0 0' line).
    Tangential lines come first so that the wall lines win at shared rows."""
    L: List[BCLine] = []
    # Vx: valid j<ny-1, k<nz-1
    L += [BCLine(VX, 0, -1, 0, 0, 0, -2, 0.0, 1.0, (0, +1, 0)),
          BCLine(VX, 0, -1, -2, -2, 0, -2, 0.0, 1.0, (0, -1, 0)),
          BCLine(VX, 0, -1, 0, -2, 0, 0, 0.0, 1.0, (0, 0, +1)),
          BCLine(VX, 0, -1, 0, -2, -2, -2, 0.0, 1.0, (0, 0, -1))]
    # Vy: valid i<nx-1, k<nz-1
    L += [BCLine(VY, 0, 0, 0, -1, 0, -2, 0.0, 1.0, (+1, 0, 0)),
          BCLine(VY, -2, -2, 0, -1, 0, -2, 0.0, 1.0, (-1, 0, 0)),
          BCLine(VY, 0, -2, 0, -1, 0, 0, 0.0, 1.0, (0, 0, +1)),
          BCLine(VY, 0, -2, 0, -1, -2, -2, 0.0, 1.0, (0, 0, -1))]
    # Vz: valid i<nx-1, j<ny-1
    L += [BCLine(VZ, 0, 0, 0, -2, 0, -1, 0.0, 1.0, (+1, 0, 0)),
          BCLine(VZ, -2, -2, 0, -2, 0, -1, 0.0, 1.0, (-1, 0, 0)),
          BCLine(VZ, 0, -2, 0, 0, 0, -1, 0.0, 1.0, (0, +1, 0)),
          BCLine(VZ, 0, -2, -2, -2, 0, -1, 0.0, 1.0, (0, -1, 0))]
    # normal components on the walls
    L += [BCLine(VX, 0, 0, 0, -2, 0, -2, 0.0), BCLine(VX, -1, -1, 0, -2, 0, -2, 0.0),
          BCLine(VY, 0, -2, 0, 0, 0, -2, 0.0), BCLine(VY, 0, -2, -1, -1, 0, -2, 0.0),
          BCLine(VZ, 0, -2, 0, -2, 0, 0, 0.0), BCLine(VZ, 0, -2, 0, -2, -1, -1, 0.0)]
    # Pressure in the 12 edge rows of cells enters no momentum equation once
    # the tangential velocities are copies; like the reference's own edge
    # lines (pardiso/init_inclusion.t3c:48-51) it copies its inner neighbour.
    L += [BCLine(P, 1, -1, 1, 1, 1, 1, 0.0, 1.0, (0, 0, +1)),
          BCLine(P, 1, -1, 1, 1, -1, -1, 0.0, 1.0, (0, 0, -1)),
          BCLine(P, 1, -1, -1, -1, 1, 1, 0.0, 1.0, (0, 0, +1)),
          BCLine(P, 1, -1, -1, -1, -1, -1, 0.0, 1.0, (0, 0, -1)),
          BCLine(P, 1, 1, 1, -1, 1, 1, 0.0, 1.0, (0, 0, +1)),
          BCLine(P, 1, 1, 1, -1, -1, -1, 0.0, 1.0, (0, 0, -1)),
          BCLine(P, -1, -1, 1, -1, 1, 1, 0.0, 1.0, (0, 0, +1)),
          BCLine(P, -1, -1, 1, -1, -1, -1, 0.0, 1.0, (0, 0, -1)),
          BCLine(P, 1, 1, 1, 1, 1, -1, 0.0, 1.0, (+1, 0, 0)),
          BCLine(P, 1, 1, -1, -1, 1, -1, 0.0, 1.0, (+1, 0, 0)),
          BCLine(P, -1, -1, 1, 1, 1, -1, 0.0, 1.0, (-1, 0, 0)),
          BCLine(P, -1, -1, -1, -1, 1, -1, 0.0, 1.0, (-1, 0, 0))]
    # Edge seal: the boundary-layer velocities that enter the edge cells are 0,
    # so every edge cell is divergence-free by construction.  Then the
    # volume-weighted divergence of all non-edge cells sums to zero and the
    # continuity row that the pressure pin replaces is redundant (without this
    # the pinned cell becomes a point source balancing the edge cells).
    def bl(first_interior):
        # boundary-layer index on the same side as first interior index 1 / n-2
        return 0 if first_interior == 1 else -2

    for a, b in ((1, 1), (-2, -2)):
        for c, d in ((0, 0), (-2, -2)):
            # edges along x
            L += [BCLine(VY, 0, -2, a, b, c, d, 0.0), BCLine(VZ, 0, -2, c, d, a, b, 0.0),
                  BCLine(VX, 0, -1, bl(a), bl(a), c, d, 0.0)]
    for a, b in ((1, 1), (-2, -2)):
        for c, d in ((0, 0), (-2, -2)):
            # edges along y (x wall and z wall)
            L += [BCLine(VX, a, b, 0, -2, c, d, 0.0), BCLine(VZ, c, d, 0, -2, a, b, 0.0),
                  BCLine(VY, bl(a), bl(a), 0, -1, c, d, 0.0)]
            # edges along z (x wall and y wall)
            L += [BCLine(VX, a, b, c, d, 0, -2, 0.0), BCLine(VY, c, d, a, b, 0, -2, 0.0),
                  BCLine(VZ, bl(a), bl(a), c, d, 0, -1, 0.0)]
    L.append(BCLine(P, pin[0], pin[0], pin[1], pin[1], pin[2], pin[2], pin_value))
    return L


# --------------------------------------------------------------------------
# Markers and rocks
# --------------------------------------------------------------------------
@dataclasses.dataclass
class Rocks:
    """Per-type constant viscosity (markn0 == markn1) and density."""

    n0: np.ndarray
    n1: np.ndarray
    ro: np.ndarray


def regular_markers(gx, gy, gz, mnx, mny, mnz, rng: Optional[np.random.Generator], jitter=1.0):
    """Marker coordinates in the reference's order (cell m3,m1,m2; then sub
    z,x,y), pardiso/in3mg.c:179-216, jittered by U(-jitter/2, +jitter/2)
    sub-cells.  Assumes uniform gridlines (as the generator does)."""
    nx1, ny1, nz1 = len(gx) - 1, len(gy) - 1, len(gz) - 1
    xs, ys, zs = gx[1] - gx[0], gy[1] - gy[0], gz[1] - gz[0]
    dx, dy, dz = xs / mnx, ys / mny, zs / mnz
    # index grids in marker order: (m3, m1, m2, m5(z), m6(x), m7(y))
    c3 = np.arange(nz1, dtype=np.float64)
    c1 = np.arange(nx1, dtype=np.float64)
    c2 = np.arange(ny1, dtype=np.float64)
    s5 = np.arange(mnz, dtype=np.float64)
    s6 = np.arange(mnx, dtype=np.float64)
    s7 = np.arange(mny, dtype=np.float64)
    z = (c3[:, None, None, None, None, None] * zs + dz / 2.0 + s5[None, None, None, :, None, None] * dz)
    x = (c1[None, :, None, None, None, None] * xs + dx / 2.0 + s6[None, None, None, None, :, None] * dx)
    y = (c2[None, None, :, None, None, None] * ys + dy / 2.0 + s7[None, None, None, None, None, :] * dy)
    shape = (nz1, nx1, ny1, mnz, mnx, mny)
    X = np.broadcast_to(x, shape).reshape(-1).astype(np.float64)
    Y = np.broadcast_to(y, shape).reshape(-1).astype(np.float64)
    Z = np.broadcast_to(z, shape).reshape(-1).astype(np.float64)
    if rng is not None and jitter > 0:
        n = X.size
        X = X + (rng.random(n) - 0.5) * jitter * dx
        Y = Y + (rng.random(n) - 0.5) * jitter * dy
        Z = Z + (rng.random(n) - 0.5) * jitter * dz
    return X.astype(np.float32), Y.astype(np.float32), Z.astype(np.float32)


def paint_ellipsoid(mx, my, mz, mt, x0, y0, z0, rx, ry, rz, typ):
    """markt = typ where (dx/rx)^2+(dy/ry)^2+(dz/rz)^2 <= 1 (in3mg.c:571-594)."""
    dx = np.abs(mx.astype(np.float64) - x0)
    dy = np.abs(my.astype(np.float64) - y0)
    dz = np.abs(mz.astype(np.float64) - z0)
    r1 = dx ** 2 / rx ** 2 + dy ** 2 / ry ** 2 + dz ** 2 / rz ** 2
    mt[r1 <= 1.0] = typ


def paint_box(mx, my, mz, mt, lo, hi, typ):
    sel = ((mx >= lo[0]) & (mx <= hi[0]) & (my >= lo[1]) & (my <= hi[1]) &
           (mz >= lo[2]) & (mz <= hi[2]))
    mt[sel] = typ


# --------------------------------------------------------------------------
# Whole problems
# --------------------------------------------------------------------------
@dataclasses.dataclass
class SolverParams:
    """The mode.t3c knobs vpiterate reads (pardiso/mode.t3c:83-97)."""

    p0koef: float = 0.3
    p1koef: float = 1.0
    p2koef: float = 0.0
    v0koef: float = 1.0
    v1koef: float = 1.0
    nubeg: float = 1e-6
    nuend: float = 1e8
    nukoef: float = 0.0
    viscmod: int = 0
    gx: float = 0.0
    gy: float = 0.0
    gz: float = -1.0
    pinit: float = 0.0
    pin: Tuple[int, int, int] = (2, 2, 2)


@dataclasses.dataclass
class Model:
    name: str
    gx: np.ndarray
    gy: np.ndarray
    gz: np.ndarray
    multinum: int
    levels: Levels
    bc: BCTables
    markx: np.ndarray
    marky: np.ndarray
    markz: np.ndarray
    markt: np.ndarray
    rocks: Rocks
    params: SolverParams

    @property
    def shape(self) -> Tuple[int, int, int]:
        return (len(self.gx), len(self.gy), len(self.gz))

    @property
    def nodenum(self) -> int:
        return len(self.gx) * len(self.gy) * len(self.gz)

    def real_dofs(self) -> int:
        """Unknowns that are equations of the level-0 system (P cells +
        staggered velocities), counted as in the level-size table."""
        nx, ny, nz = self.shape
        return ((nx - 1) * (ny - 1) * (nz - 1) + nx * (ny - 1) * (nz - 1)
                + (nx - 1) * ny * (nz - 1) + (nx - 1) * (ny - 1) * nz)


def _finish(name, n, multinum, mnx, mny, mnz, seed, rocks, paint, params=None, jitter=1.0, shape=None):
    if shape is None:
        shape = (n, n, n)
    gx, gy, gz = uniform_lines(shape[0]), uniform_lines(shape[1]), uniform_lines(shape[2])
    lv = make_levels(gx, gy, gz, multinum)
    params = params or SolverParams()
    bc = build_bc_tables(lv, free_slip_lines(params.pin, params.pinit))
    rng = np.random.Generator(np.random.PCG64(seed))
    mx, my, mz = regular_markers(gx, gy, gz, mnx, mny, mnz, rng, jitter)
    mt = np.zeros(mx.size, dtype=np.int8)
    paint(mx, my, mz, mt, rng)
    return Model(name, gx, gy, gz, multinum, lv, bc, mx, my, mz, mt, rocks, params)


def sphere_model(n=33, multinum=2, markers=(4, 4, 4), seed=1, eta_sphere=1e3, drho=1.0, radius=0.2):
    """One centred sphere in a unit cube (the 33^3 CPU-runnable case)."""
    rocks = Rocks(np.array([1.0, eta_sphere]), np.array([1.0, eta_sphere]), np.array([0.0, drho]))

    def paint(mx, my, mz, mt, rng):
        paint_ellipsoid(mx, my, mz, mt, 0.5, 0.5, 0.5, radius, radius, radius, 1)

    return _finish("sphere%d" % n, n, multinum, *markers, seed, rocks, paint)


def random_spheres_model(n, multinum, nsph, eta_range, rad_range=(0.05, 0.12), drho_range=(-1.0, 1.0),
                         markers=(2, 2, 2), seed=2, name=None, gap=None, shape=None):
    """nsph spheres: radius U[rad_range], centre U[0,1]^3, viscosity
    log-uniform in eta_range, density contrast U[drho_range]; background
    type 0 (viscosity 1, density 0).  Later spheres paint over earlier ones.
    With gap (a length), centres are redrawn until every pair of spheres is
    at least gap apart and every sphere lies inside the box: no sphere then
    touches another, so no thin sliver of one contrast welds onto another."""
    rng0 = np.random.Generator(np.random.PCG64(seed + 1000))
    rad = rng0.uniform(*rad_range, size=nsph)
    cen = rng0.uniform(0.0, 1.0, size=(nsph, 3))
    if gap is not None:
        for s in range(nsph):
            for _ in range(100000):
                c = cen[s]
                inside = np.all(c - rad[s] >= gap) and np.all(c + rad[s] <= 1.0 - gap)
                apart = all(np.linalg.norm(c - cen[t]) >= rad[s] + rad[t] + gap for t in range(s))
                if inside and apart:
                    break
                cen[s] = rng0.uniform(0.0, 1.0, size=3)
            else:
                raise ValueError("could not place %d separated spheres" % nsph)
    eta = np.exp(rng0.uniform(math.log(eta_range[0]), math.log(eta_range[1]), size=nsph))
    rho = rng0.uniform(*drho_range, size=nsph)
    n0 = np.concatenate([[1.0], eta])
    rocks = Rocks(n0, n0.copy(), np.concatenate([[0.0], rho]))
    lo = min(1.0, float(eta.min()))
    hi = max(1.0, float(eta.max()))
    params = SolverParams(nubeg=lo * 0.5, nuend=hi * 2.0)

    def paint(mx, my, mz, mt, rng):
        for s in range(nsph):
            paint_ellipsoid(mx, my, mz, mt, cen[s, 0], cen[s, 1], cen[s, 2], rad[s], rad[s], rad[s], s + 1)

    return _finish(name or ("spheres%d_%d" % (n, nsph)), n, multinum, *markers, seed, rocks, paint, params,
                   shape=shape)


def layered_model(n=257, multinum=6, markers=(2, 2, 2), seed=5, nlayers=45, name=None):
    """Layered lithosphere: viscosity exp(-ln(1e4) z) from 1e4 (z=0) to 1
    (z=1), quantised into `nlayers` constant-viscosity rock types (marker
    types must stay below 50: pardiso/mark3mg.c:692), an embedded dense slab
    block (density +1, viscosity 1e3) and a weak zone (viscosity 1e-2)."""
    zc = (np.arange(nlayers) + 0.5) / nlayers
    eta_l = 1e4 * np.exp(-math.log(1e4) * zc)
    n0 = np.concatenate([eta_l, [1e3, 1e-2]])
    rocks = Rocks(n0, n0.copy(), np.concatenate([np.zeros(nlayers), [1.0, 0.0]]))
    params = SolverParams(nubeg=5e-3, nuend=2e4)
    t_slab, t_weak = nlayers, nlayers + 1

    def paint(mx, my, mz, mt, rng):
        layer = np.minimum((mz.astype(np.float64) * nlayers).astype(np.int64), nlayers - 1)
        mt[:] = layer.astype(np.int8)
        paint_box(mx, my, mz, mt, (0.35, 0.2, 0.45), (0.55, 0.8, 0.8), t_slab)
        # an upper-crust weak zone beside the slab, separated from it by layered
        # material: a 1e-2 sheet welded to the 1e3 slab stalls every multigrid
        # variant tried (diagonal or full cell blocks, coarse averaging, Galerkin)
        paint_box(mx, my, mz, mt, (0.70, 0.2, 0.55), (0.85, 0.8, 1.0), t_weak)

    return _finish(name or ("layered%d" % n), n, multinum, *markers, seed, rocks, paint, params)


BATCH_SIZES = {33: 2, 49: 3, 65: 3, 81: 4, 97: 4}  # nodes per axis -> multinum (coarsest 9..12 nodes)


def batch_specs(count: int = 64, seed: int = 4):
    """The batched workload: per instance (nodes per axis, spheres, seed),
    sizes uniform in {33, 49, 65, 81, 97}, 1-10 spheres."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = rng.choice(sorted(BATCH_SIZES), size=count)
    nsph = rng.integers(1, 11, size=count)
    return [(int(n), int(s), seed * 1000 + i) for i, (n, s) in enumerate(zip(sizes, nsph))]


def batch_model(n: int, nsph: int, seed: int) -> Model:
    """One instance of the batched workload: nsph spheres with viscosity
    log-uniform in [1e-2, 1e2] in an n^3 box, 2x2x2 markers per cell."""
    return random_spheres_model(n, BATCH_SIZES[n], nsph, (1e-2, 1e2), markers=(2, 2, 2), seed=seed,
                                name="batch%d_%d" % (n, seed))


def config_model(idx: int, **kw) -> Model:
    """The five benchmark configurations (synthetic, seeded)."""
    if idx == 1:
        return sphere_model(33, 2, (4, 4, 4), seed=1, **kw)
    if idx == 2:
        return random_spheres_model(65, 3, 8, (1e-3, 1e3), markers=(2, 2, 2), seed=2, name="spheres65", **kw)
    if idx == 3:
        return random_spheres_model(129, 4, 20, (1e-2, 1e4), markers=(2, 2, 2), seed=3, name="spheres129", **kw)
    if idx == 5:
        return layered_model(257, 5, (2, 2, 2), seed=5, **kw)
    raise ValueError("unknown config %r" % idx)
