"""The bench line's solution errors (bench.py): the relative L2 error of
every field, of the velocity as one vector field, and against a fixture's
sub-lattice and full-field norms."""
import numpy as np

import bench


class _M:
    shape = (5, 4, 3)


def _fields(rng, n):
    return {k: rng.standard_normal(n) for k in ("vx", "vy", "vz", "pr")}


def test_velocity_error_weights_components_by_their_norms():
    rng = np.random.Generator(np.random.PCG64(1))
    ref = _fields(rng, 60)
    ref["vy"] *= 1e-3  # a small component
    sol = {k: v.copy() for k, v in ref.items()}
    sol["vy"] += 1e-6  # large relative to vy, small relative to the velocity
    assert bench.rel_l2(sol["vy"], ref["vy"]) > 1e-4
    assert bench.velocity_rel_l2(sol, ref) < 1e-5
    assert bench.velocity_rel_l2(ref, ref) == 0.0


def test_errors_against_a_fixture_subsample_and_norms():
    rng = np.random.Generator(np.random.PCG64(2))
    m = _M()
    nx, ny, nz = m.shape
    ref = _fields(rng, nx * ny * nz)
    st = 2
    fx = {"stride": np.array(st)}
    for k, v in ref.items():
        fx["sub_" + k] = v.reshape(nz, nx, ny)[::st, ::st, ::st].reshape(-1)
        fx["norm_" + k] = np.array(np.linalg.norm(v))
    e = bench.errors_vs_fixture(ref, m, fx)
    assert all(e[k] == 0.0 for k in ("vx", "vy", "vz", "pr", "velocity"))
    sol = {k: v * (1 + 1e-7) for k, v in ref.items()}
    e = bench.errors_vs_fixture(sol, m, fx)
    for k in ("vx", "vy", "vz", "pr", "velocity"):
        assert abs(e[k] - 1e-7) < 1e-9, (k, e[k])
        if k != "velocity":
            assert abs(e[k + "_norm"] - 1e-7) < 1e-9
