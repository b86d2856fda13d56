"""Seeded model generator: level tables, boundary tables and markers in the
reference's layouts (CPU)."""
import numpy as np
import pytest

from pardiso2_b200 import model as M


@pytest.mark.parametrize("n,ml,sizes", [
    (33, 2, [33, 19, 12]),
    (65, 3, [65, 35, 20, 12]),
    (129, 4, [129, 67, 36, 20, 12]),
    (257, 5, [257, 131, 68, 36, 20, 12]),
    (49, 3, [49, 27, 16, 10]),
    (81, 4, [81, 43, 24, 14, 9]),
])
def test_level_sizes(n, ml, sizes):
    # load3mg.c:2068-2070: n_{l+1} = (n_l - 5)/2 + 5
    g = M.uniform_lines(n)
    lv = M.make_levels(g, g, g, ml)
    assert lv.mgx == sizes
    assert lv.mgp[1] == n ** 3
    assert lv.total_nodes == sum(s ** 3 for s in sizes)


def test_coarse_gridlines_keep_outer_lines():
    # load3mg.c:2082-2098: lines 0-2 and the last 3 copied; interior n2 -> fine (n2-2)*2^l+2
    g = M.uniform_lines(33)
    lv = M.make_levels(g, g, g, 2)
    c1 = lv.cx[1]
    assert np.array_equal(c1[:3], g[:3]) and np.array_equal(c1[-3:], g[-3:])
    for n2 in range(3, len(c1) - 3):
        assert c1[n2] == g[(n2 - 2) * 2 + 2]


def _apply_bc(bc, x, nunk):
    idx = np.where(bc.bondm[:nunk] > 0)[0]
    for _ in range(4):
        b = bc.bondm[idx]
        t = bc.bondn1[b] - 1
        x[idx] = np.where(t >= 0, bc.bondv1[b, 0] + bc.bondv1[b, 1] * x[np.maximum(t, 0)], bc.bondv1[b, 0])
    return x


@pytest.mark.parametrize("n", [13, 17])
def test_free_slip_tables_seal_edges(n):
    """With the boundary rows applied, every edge cell is divergence-free for
    any velocity field, so the continuity row the pressure pin replaces is
    implied by the others (the sum of volume * div over all cells vanishes)."""
    m = M.sphere_model(n, 1, (1, 1, 1), seed=1)
    rng = np.random.default_rng(0)
    x = _apply_bc(m.bc, rng.standard_normal(n ** 3 * 4), n ** 3 * 4)
    v = x.reshape(n, n, n, 4)
    vx, vy, vz = v[..., 1], v[..., 2], v[..., 3]
    div = ((vx[:-1, 1:, :-1] - vx[:-1, :-1, :-1]) + (vy[:-1, :-1, 1:] - vy[:-1, :-1, :-1]) +
           (vz[1:, :-1, :-1] - vz[:-1, :-1, :-1]))  # cells (k,i,j) >= 1, unit spacing factor dropped
    cnt = np.zeros((n - 1, n - 1, n - 1), int)
    for ax in range(3):
        idx = np.arange(n - 1)
        on = (idx == 0) | (idx == n - 2)
        shape = [1, 1, 1]
        shape[ax] = n - 1
        cnt += on.reshape(shape)
    edge = cnt >= 2
    assert np.abs(div[edge]).max() < 1e-12
    assert abs(div.sum()) < 1e-9


def test_every_open_velocity_row_has_an_inner_stencil():
    """Non-boundary velocity rows keep their 17-point stencil inside the grid
    on every level (what the library validates in p2_set_bc)."""
    m = M.sphere_model(17, 2, (1, 1, 1), seed=1)
    lv = m.levels
    for l in range(lv.multinum + 1):
        nx = ny = nz = lv.mgx[l]
        off = lv.mgp[l]
        bm = m.bc.bondm[off * 4:(off + lv.mgn[l]) * 4].reshape(nz, nx, ny, 4)
        k, i, j = np.meshgrid(np.arange(nz), np.arange(nx), np.arange(ny), indexing="ij")
        okx = (i >= 1) & (i <= nx - 2) & (j >= 1) & (j <= ny - 3) & (k >= 1) & (k <= nz - 3)
        validx = (j < ny - 1) & (k < nz - 1)
        assert not np.any(validx & (bm[..., 1] == 0) & ~okx)


def test_pressure_pin_and_tables_reference_layout():
    m = M.sphere_model(17, 2, (1, 1, 1), seed=1)
    bc = m.bc
    assert bc.bondm.dtype == np.int32 and bc.bondv1.dtype == np.float32 and bc.bondn1.dtype == np.int32
    assert bc.bondv1.shape == (bc.bondnum + 1, 2)
    # one pure-constant pressure row per level, at cell (2,2,2)
    lv = m.levels
    for l in range(lv.multinum + 1):
        nx = lv.mgx[l]
        u = lv.mgp[l] + (2 * nx + 2) * nx + 2
        b = bc.bondm[u * 4]
        assert b > 0 and bc.bondn1[b] == 0
    # copy targets stay on their own level and component
    src = np.where(bc.bondm > 0)[0]
    t = bc.bondn1[bc.bondm[src]] - 1
    has = t >= 0
    assert np.all(t[has] % 4 == src[has] % 4)
    lev_of = np.searchsorted(np.array(lv.mgp), src // 4, side="right")
    assert np.array_equal(lev_of[has], np.searchsorted(np.array(lv.mgp), t[has] // 4, side="right"))
    # later lines overwrite earlier ones: live rows never exceed the table size
    assert src.size <= bc.bondnum


def test_markers_seeded_and_inside():
    a = M.sphere_model(9, 1, (2, 2, 2), seed=3)
    b = M.sphere_model(9, 1, (2, 2, 2), seed=3)
    assert a.markx.size == 8 ** 3 * 8
    assert np.array_equal(a.markx, b.markx) and np.array_equal(a.markt, b.markt)
    for arr in (a.markx, a.marky, a.markz):
        assert arr.min() > 0 and arr.max() < 1
    assert set(np.unique(a.markt)) <= {0, 1}


def test_thermal_rows_cover_every_wall_node():
    """The heat equation needs a T boundary row on every wall node of every
    level (heaterr reads all six neighbours of a heat row); copy targets stay
    on their level and chains end within two rows at a heat row or a fixed
    temperature."""
    import numpy as np
    from pardiso2_b200 import model as M
    m = M.sphere_model(33, 3, (1, 1, 1), seed=5)
    bc = M.with_thermal_bc(m, 300.0, 1600.0)
    lv = m.levels
    assert bc.bondt is not None and bc.bondt.size == lv.total_nodes
    for l in range(lv.multinum + 1):
        nx, ny, nz, off = lv.mgx[l], lv.mgy[l], lv.mgz[l], lv.mgp[l]
        k, i, j = np.meshgrid(np.arange(nz), np.arange(nx), np.arange(ny), indexing="ij")
        wall = ((i == 0) | (j == 0) | (k == 0) | (i == nx - 1) | (j == ny - 1) | (k == nz - 1)).ravel()
        rows = bc.bondt[off:off + lv.mgn[l]]
        assert np.all(rows[wall] > 0) and np.all(rows[~wall] == 0), l
        for u in np.nonzero(wall)[0]:
            r, depth = rows[u], 0
            while bc.bondn1[r]:
                t = bc.bondn1[r] - 1
                assert off <= t < off + lv.mgn[l]
                r = bc.bondt[t]
                depth += 1
                if not r:
                    break
            assert depth <= 2
    # z planes fixed, walls insulating copies
    z0 = bc.bondt[lv.mgp[0] + (lv.mgn[0] - 1)]  # top corner node: fixed plane wins
    assert bc.bondn1[z0] == 0 and bc.bondv1[z0, 0] == np.float32(1600.0)
    ref = bc.reference_bondm(m.nodenum)
    assert ref.size >= 8 * m.nodenum + lv.total_nodes
    np.testing.assert_array_equal(ref[8 * m.nodenum:8 * m.nodenum + lv.total_nodes], bc.bondt)
    np.testing.assert_array_equal(ref[:bc.bondm.size], bc.bondm)
