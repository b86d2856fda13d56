"""Heat equation step on the GPU (p2_titerate, titerate of
pardiso/heat3mg.c:292) against the reference's own titerate() (golden
vectors, tests/golden/heat17.npz) and the oracle restatement, which the CPU
suite pins bit for bit to those vectors.

The GPU smoother is Gauss-Seidel in two colours, the reference's sweeps the
rows in order: both stop once the RMS error of the heat rows times the
sub-step is below heatmin, so the temperatures agree to within what heatmin
leaves.  Each sub-step's error e solves (I + dt/(ro cp) L) e = r with
||r||_rms <= heatmin and the operator's inverse bounded by 1, so per
sub-step the difference is of order heatmin; over the sub-steps of a call
the bar is max |dT| <= 0.1 K and RMS <= 0.02 K (heatmin 5e-3 K, 4 and 11
sub-steps), with temperatures of 273..1573 K (about 1e-4 relative).  The
right-hand side, the sub-step limit and the sub-step count follow the
reference's float/double operations exactly."""
import os

import numpy as np
import pytest

import pardiso2_b200 as P
from pardiso2_b200 import capi
from pardiso2_b200 import model as M
from tests.golden.make_golden import HEAT_COMMON, HEAT_VARIANTS, heat_inputs, heat_model

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TK_MAX, TK_RMS = 0.1, 0.02


def _problem(m):
    prob = P.StokesProblem(m)
    prob.ctx.heat_set_bc(m.bc, m.nodenum)
    return prob


def _hp(m, v, **over):
    d = dict(HEAT_COMMON, **v, max_cycles=200)
    d.update(over)
    return capi.heat_params(**{k: d[k] for k in ("maxtkstep", "heatmin", "t0koef", "t1koef", "heatdif", "tdeep",
                                                 "zdeep", "multinumt", "multicyct", "frictyn", "adiabyn",
                                                 "max_cycles", "pre", "post")})


@pytest.mark.parametrize("variant", ["mg", "single"])
def test_titerate_vs_reference_golden(variant):
    m = heat_model()
    g = np.load(os.path.join(GOLDEN, "heat17.npz"))
    th, vel, se, pr, (mx, my, mz, mt), markk = heat_inputs(m)
    v = HEAT_VARIANTS[variant]
    prob = _problem(m)
    for _ in range(2):  # a second call on the same context gives the same step
        tk, mk, info = prob.ctx.titerate(_hp(m, v), v["timestep"], th, vel=vel, pr=pr, se=se,
                                         markers=(mx[:-1], my[:-1], mz[:-1], mt[:-1]), markk=markk)
        assert info.converged == 1 and info.heatsum <= HEAT_COMMON["heatmin"]
        assert info.substeps == int(g["info_" + variant][0])
        assert info.tktimestep == pytest.approx(float(g["info_" + variant][2]), rel=1e-12)
        ref = g["tk_" + variant]
        d = tk.astype(np.float64) - ref
        assert np.abs(d).max() <= TK_MAX and np.sqrt(np.mean(d * d)) <= TK_RMS, (np.abs(d).max(), np.sqrt(np.mean(d * d)))
        dm = mk.astype(np.float64) - g["markk_" + variant]
        assert np.abs(dm).max() <= TK_MAX, np.abs(dm).max()
        # boundary planes exactly at their fixed temperatures
        nx, ny, nz = m.shape
        t3 = tk.reshape(nz, nx, ny)
        assert np.all(t3[0] == np.float32(273.0)) and np.all(t3[-1] == np.float32(1573.0))
        assert info.kernels > 0 and info.ms_total > 0
    prob.close()


def test_titerate_vs_oracle_33(oracle_mod):
    """33^3, three heat levels, all heating terms: the GPU against the oracle
    (same heatmin; different smoother order)."""
    m = M.sphere_model(33, 3, (1, 1, 1), seed=21, eta_sphere=1e3)
    m.bc = M.with_thermal_bc(m, 300.0, 1600.0)
    th = M.thermal_fields(m, seed=22, t_low=300.0, t_high=1600.0)
    n = m.nodenum
    rng = np.random.Generator(np.random.PCG64(23))
    vel = [(rng.random(n) * 2 - 1).astype(np.float32) for _ in range(3)]
    se = [(rng.random(n) * 200 - 100).astype(np.float32) for _ in range(6)] + [
        (rng.random(n) * 2 - 1).astype(np.float32) for _ in range(6)]
    v = dict(multinumt=2, multicyct=1, pre=[3, 3, 0], post=[0, 3, 10], frictyn=1, adiabyn=1, heatdif=1.0)
    hpd = dict(HEAT_COMMON, **v, heatmin=5e-3, gx=m.params.gx, gy=m.params.gy, gz=m.params.gz, max_cycles=500,
               timestep=2e4)
    mx, my, mz = m.markx, m.marky, m.markz
    mt = np.where(np.arange(mx.size) % 9 == 4, 70, m.markt).astype(np.int8)
    markk = np.where(np.arange(mx.size) % 3 == 0, 0.0, 900.0).astype(np.float32)
    tko, mko, oi = oracle_mod.titerate(m.gx, m.gy, m.gz, 2, m.bc.bondt, m.bc.bondv1, m.bc.bondn1, hpd, th, vel=vel,
                                       se=se, markers=(mx, my, mz, mt), markk=markk)
    assert not oi["capped"]
    prob = _problem(m)
    tk, mk, info = prob.ctx.titerate(_hp(m, v, heatmin=5e-3, max_cycles=500), hpd["timestep"], th, vel=vel, se=se,
                                     markers=(mx, my, mz, mt), markk=markk)
    assert info.converged == 1 and info.substeps == oi["substeps"]
    assert info.tktimestep == pytest.approx(oi["tktimestep"], rel=1e-12)
    d = tk.astype(np.float64) - tko
    assert np.abs(d).max() <= TK_MAX and np.sqrt(np.mean(d * d)) <= TK_RMS
    assert np.abs(mk.astype(np.float64) - mko).max() <= TK_MAX
    assert np.abs(tk - th.tk).max() > 10
    prob.close()


def test_titerate_zero_step_and_cap():
    m = heat_model()
    th, vel, se, pr, (mx, my, mz, mt), markk = heat_inputs(m)
    v = HEAT_VARIANTS["mg"]
    prob = _problem(m)
    # timestep 0: the reference returns after the step limit, nothing moves
    tk, mk, info = prob.ctx.titerate(_hp(m, v), 0.0, th, vel=vel, se=se, markers=(mx[:-1], my[:-1], mz[:-1], mt[:-1]),
                                     markk=markk)
    np.testing.assert_array_equal(tk, th.tk)
    np.testing.assert_array_equal(mk, markk)
    assert info.substeps == 0 and info.tktimestep > 0
    # an unreachable heatmin with a cap of 3 error checks: reported, not looped
    tk, _, info = prob.ctx.titerate(_hp(m, v, heatmin=1e-12, max_cycles=3), v["timestep"], th, vel=vel, se=se)
    assert info.converged == 0 and info.cycles == 3 and np.isfinite(tk).all()
    prob.close()


def test_titerate_argument_errors():
    m = heat_model()
    th = heat_inputs(m)[0]
    prob = P.StokesProblem(m)
    with pytest.raises(capi.P2Error) as e:  # no T rows yet
        prob.ctx.titerate(_hp(m, HEAT_VARIANTS["mg"]), 1e4, th)
    assert e.value.code == 7
    bc = m.bc
    # bondm without the temperature section (length 4 * total nodes only)
    st = prob.ctx.L.p2_heat_set_bc(prob.ctx.h, np.ascontiguousarray(bc.bondm), bc.bondm.size,
                                   np.ascontiguousarray(bc.bondv1.reshape(-1)), np.ascontiguousarray(bc.bondn1),
                                   bc.bondnum)
    assert st == 1
    # a wall node without a T row
    bad = M.BCTables(bc.bondm, bc.bondv1, bc.bondn1, bc.bondt.copy())
    bad.bondt[0] = 0
    with pytest.raises(capi.P2Error) as e:
        prob.ctx.heat_set_bc(bad, m.nodenum)
    assert e.value.code == 8
    prob.ctx.heat_set_bc(bc, m.nodenum)
    with pytest.raises(capi.P2Error) as e:  # frictyn without the stress fields
        prob.ctx.titerate(_hp(m, HEAT_VARIANTS["mg"]), 1e4, th)
    assert e.value.code == 1
    prob.close()


def test_titerate_vs_oracle_65_all_levels(oracle_mod):
    """The bench's heat step (spheres65 grid, all four levels, 2.1 M markers,
    2000 s in sub-steps of at most 25 K, heatmin 1e-3 K) against the oracle:
    same sub-steps, temperatures within the heatmin bar."""
    m = M.config_model(2)
    n = m.nodenum
    bc = M.with_thermal_bc(m)
    th = M.thermal_fields(m, seed=31, heat=(2e4, 8e4))
    rng = np.random.Generator(np.random.PCG64(32))
    vel = [(rng.random(n) * 0.02 - 0.01).astype(np.float32) for _ in range(3)]
    se = [(rng.random(n) * 2 - 1).astype(np.float32) for _ in range(12)]
    nt = m.multinum
    v = dict(multinumt=nt, multicyct=1, pre=[3] * nt + [0], post=[0] + [3] * (nt - 1) + [10], frictyn=1, adiabyn=1,
             heatdif=1.0)
    q = np.arange(m.markx.size)
    mt = np.where(q % 9 == 4, 70, m.markt).astype(np.int8)
    markk = np.where(q % 3 == 0, 0.0, 900.0).astype(np.float32)
    markers = (m.markx, m.marky, m.markz, mt)
    hpd = dict(HEAT_COMMON, **v, heatmin=1e-3, gx=m.params.gx, gy=m.params.gy, gz=m.params.gz, max_cycles=200,
               timestep=2000.0)
    tko, mko, oi = oracle_mod.titerate(m.gx, m.gy, m.gz, nt, bc.bondt, bc.bondv1, bc.bondn1, hpd, th, vel=vel, se=se,
                                       markers=markers, markk=markk)
    assert not oi["capped"] and oi["substeps"] == 3
    m.bc = bc
    prob = _problem(m)
    tk, mk, info = prob.ctx.titerate(_hp(m, v, heatmin=1e-3), 2000.0, th, vel=vel, se=se, markers=markers,
                                     markk=markk)
    assert info.converged == 1 and info.substeps == oi["substeps"]
    d = tk.astype(np.float64) - tko
    assert np.abs(d).max() <= TK_MAX and np.sqrt(np.mean(d * d)) <= TK_RMS
    assert np.abs(mk.astype(np.float64) - mko).max() <= TK_MAX
    # the marker sums into the nodes do not depend on the order the markers
    # arrive in: a second identical call gives the same markk bit for bit
    tk2, mk2, _ = prob.ctx.titerate(_hp(m, v, heatmin=1e-3), 2000.0, th, vel=vel, se=se, markers=markers,
                                    markk=markk)
    assert np.array_equal(tk2, tk) and np.array_equal(mk2, mk)
    prob.close()
