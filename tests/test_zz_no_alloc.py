"""p2_ronurecalc_noalloc: the marker -> node interpolation for callers that
cannot allocate device memory (their device memory comes from their own pool,
or cudaMalloc's device-wide synchronisation is not allowed inside their time
loop).  Its scratch is a fixed array inside the library, so it takes device
arrays from the caller and allocates nothing itself.

The test calls it through the C ABI twice in a row (a larger case, then a
smaller one on a different grid, so stale scratch from the first call would
show) and requires node fields bit-identical to p2_ronurecalc's, the
tolerance every ronurecalc test here uses.  The test allocates its own device
arrays with torch; the entry point under test does not.  This file sorts last
so that a run stopping at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

KEYS = ("nu", "ro", "nxx", "nxy", "nxz", "nyz")
MAX_MARKERS = 1 << 18


def _bind():
    from pardiso2_b200 import capi
    L = capi.load()
    f = L.p2_ronurecalc_noalloc
    vp = C.c_void_p
    f.argtypes = ([C.c_int] * 3 + [vp] * 3 + [C.POINTER(capi.Params), C.c_int] + [vp] * 3 + [C.c_long]
                  + [vp] * 4 + [vp] * 6 + [vp, C.c_char_p, C.c_long])
    f.restype = C.c_int
    return f


def _host(a, dt):
    a = np.ascontiguousarray(a, dt)
    return a, a.ctypes.data_as(C.c_void_p)


def _noalloc(f, m, params, init):
    """One call with device markers and node fields; returns host fields."""
    import torch
    dev = torch.device("cuda", 0)
    r = m.rocks
    gx, pgx = _host(m.gx, np.float64)
    gy, pgy = _host(m.gy, np.float64)
    gz, pgz = _host(m.gz, np.float64)
    n0, p0 = _host(r.n0, np.float64)
    n1, p1 = _host(r.n1, np.float64)
    ro, pro = _host(r.ro, np.float64)
    mk = [torch.from_numpy(np.ascontiguousarray(a, dt)).to(dev)
          for a, dt in ((m.markx, np.float32), (m.marky, np.float32), (m.markz, np.float32), (m.markt, np.int8))]
    out = [torch.from_numpy(np.array(init[k], np.float32)).to(dev) for k in KEYS]
    torch.cuda.synchronize()
    err = C.create_string_buffer(512)
    st = f(len(gx), len(gy), len(gz), pgx, pgy, pgz, C.byref(params), len(n0), p0, p1, pro, m.markx.size,
           *[t.data_ptr() for t in mk], *[t.data_ptr() for t in out], None, err, len(err))
    assert st == 0, err.value.decode()
    torch.cuda.synchronize()
    return {k: t.cpu().numpy() for k, t in zip(KEYS, out)}


def _existing(m, init):
    import pardiso2_b200 as P
    prob = P.StokesProblem(m, device=0)
    try:
        return prob.ronurecalc(init)
    finally:
        prob.close()


def _init(m, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    return {k: rng.uniform(0.5, 2.0, m.nodenum).astype(np.float32) for k in KEYS}


@pytest.mark.gpu
def test_noalloc_matches_ronurecalc_on_two_calls_in_a_row():
    import pardiso2_b200 as P
    from pardiso2_b200 import model as M
    f = _bind()
    big = M.random_spheres_model(21, 2, 6, (1e-2, 1e2), markers=(3, 3, 3), seed=5, name="spheres21")
    small = M.sphere_model(17, 2, (2, 2, 2), seed=1, eta_sphere=1e3)
    assert big.markx.size <= MAX_MARKERS
    for m, seed in ((big, 11), (small, 12)):
        init = _init(m, seed)
        want = _existing(m, {k: v.copy() for k, v in init.items()})
        got = _noalloc(f, m, P.params_for(m), init)
        for k in KEYS:
            assert np.array_equal(got[k], want[k]), (m.name, k)


@pytest.mark.gpu
def test_noalloc_rejects_sizes_beyond_its_scratch():
    import pardiso2_b200 as P
    from pardiso2_b200 import model as M
    f = _bind()
    m = M.sphere_model(17, 2, (2, 2, 2), seed=1)
    params = P.params_for(m)
    g, pg = _host(m.gx, np.float64)
    rk, pr = _host(m.rocks.n0, np.float64)
    err = C.create_string_buffer(256)
    st = f(len(g), len(g), len(g), pg, pg, pg, C.byref(params), len(rk), pr, pr, pr, MAX_MARKERS + 1,
           *([None] * 10), None, err, len(err))
    assert st == 1 and b"262144" in err.value
    big = np.linspace(0.0, 1.0, 60)  # 59^3 cells > 131072
    bg, pbg = _host(big, np.float64)
    st = f(60, 60, 60, pbg, pbg, pbg, C.byref(params), len(rk), pr, pr, pr, 0, *([None] * 10), None, err, len(err))
    assert st == 1 and b"131072" in err.value
    # host arrays where device arrays are required are refused before any launch
    host = np.zeros(m.nodenum, np.float32)
    st = f(len(g), len(g), len(g), pg, pg, pg, C.byref(params), len(rk), pr, pr, pr, 0, *([None] * 4),
           *([host.ctypes.data_as(C.c_void_p)] * 6), None, err, len(err))
    assert st == 1 and b"device" in err.value


def _with_high_type_law(m):
    """The model with its rock table extended to type 30 holding markn0 !=
    markn1 (a power-law pair above type 20, which the reference reads as the
    constant markn0) and a tenth of its markers moved to that type."""
    import copy
    mm = copy.copy(m)
    r = copy.copy(m.rocks)
    n0 = np.concatenate([r.n0, np.full(31 - r.n0.size, 1.0)])
    n1 = n0.copy()
    ro = np.concatenate([r.ro, np.zeros(31 - r.ro.size)])
    n0[30], n1[30], ro[30] = 5.0, 50.0, 0.5
    r.n0, r.n1, r.ro = n0, n1, ro
    mm.rocks = r
    mt = np.array(m.markt, np.int8)
    mt[::10] = 30
    mm.markt = mt
    return mm


@pytest.mark.gpu
def test_noalloc_type_above_20_with_distinct_markn1_matches_ronurecalc():
    import pardiso2_b200 as P
    from pardiso2_b200 import model as M
    f = _bind()
    m = _with_high_type_law(M.sphere_model(17, 2, (2, 2, 2), seed=1, eta_sphere=1e3))
    init = _init(m, 13)
    want = _existing(m, {k: v.copy() for k, v in init.items()})
    got = _noalloc(f, m, P.params_for(m), init)
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), k


@pytest.mark.gpu
def test_noalloc_without_markers_matches_ronurecalc():
    import copy
    import pardiso2_b200 as P
    from pardiso2_b200 import model as M
    f = _bind()
    m = copy.copy(M.sphere_model(17, 2, (2, 2, 2), seed=1))
    for k in ("markx", "marky", "markz"):
        setattr(m, k, np.zeros(0, np.float32))
    m.markt = np.zeros(0, np.int8)
    init = _init(m, 14)
    want = _existing(m, {k: v.copy() for k, v in init.items()})
    got = _noalloc(f, m, P.params_for(m), init)
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), k


@pytest.mark.gpu
def test_noalloc_refuses_marker_types_without_a_rock_entry():
    import copy
    import pardiso2_b200 as P
    from pardiso2_b200 import model as M
    f = _bind()
    m = copy.copy(M.sphere_model(17, 2, (2, 2, 2), seed=1))
    mt = np.array(m.markt, np.int8)
    mt[5] = 40  # below 50, past the two-entry rock table
    m.markt = mt
    with pytest.raises(AssertionError, match="without a rock entry"):
        _noalloc(f, m, P.params_for(m), _init(m, 15))
