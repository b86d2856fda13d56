"""The heat-step restatement (oracle/p2oracle.c, p2o_titerate) against the
reference's own titerate() (pardiso/heat3mg.c:292), run live on the CPU
through the reference harness (oracle/_ref/libp2ref.so) at 33^3 with three
heat levels, adiabatic and shear heating, numerical diffusion and the
three marker classes: temperatures and marker temperatures bit for bit.
The golden vectors (tests/golden/heat17.npz) pin one and two levels; this
case adds the intermediate level of a three-level cycle.

The harness keeps the reference's state in globals, one model per process,
so the reference runs in a child process.  Skipped when oracle/_ref is not
built (it needs the reference sources)."""
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
from tests.test_oracle_heat_live import case
m, th, vel, se, (mx, my, mz, mt), markk, hp, nt = case()
r = refdrv.RefModel(m)
r.set_tbc(m.bc)
r.set_markers(mx, my, mz, mt)
one = np.ones_like(th.ro)
r.set_nodes({"nu": one, "ro": th.ro, "nxx": one, "nxy": one, "nxz": one, "nyz": one})
r.set_velocity(*vel)
r.set_stress(se)
tk, mk = r.titerate(hp, nt, th, markk)
np.savez(sys.argv[2], tk=tk, markk=mk)
"""


def case():
    """33^3, three heat levels; the last marker is the harness's
    out-of-box slot (the reference reads one past its marker arrays)."""
    from pardiso2_b200 import model as M
    from tests.golden.make_golden import HEAT_COMMON, move_markers
    m = M.sphere_model(33, 3, (1, 1, 1), seed=21, eta_sphere=1e3)
    m.bc = M.with_thermal_bc(m, 300.0, 1600.0)
    th = M.thermal_fields(m, seed=22, t_low=300.0, t_high=1600.0, heat=(2e4, 8e4))
    n = m.nodenum
    rng = np.random.Generator(np.random.PCG64(23))
    vel = [(rng.random(n) * 2 - 1).astype(np.float32) for _ in range(3)]
    se = [(rng.random(n) * 200 - 100).astype(np.float32) for _ in range(6)] + [
        (rng.random(n) * 2 - 1).astype(np.float32) for _ in range(6)]
    mx, my, mz, mt = move_markers(m)
    q = np.arange(mx.size - 1)
    markk = np.where(q % 3 == 0, np.float32(0), np.float32(900)).astype(np.float32)
    nt = 2
    hp = dict(HEAT_COMMON, timestep=8000.0, heatmin=2e-3, multicyct=1, pre=[3, 3, 0], post=[0, 3, 10], frictyn=1,
              adiabyn=1, heatdif=1.0, gx=m.params.gx, gy=m.params.gy, gz=m.params.gz, max_cycles=500)
    return m, th, vel, se, (mx, my, mz, mt), markk, hp, nt


def test_oracle_titerate_vs_live_reference_33(oracle_mod, tmp_path):
    if not refdrv.available():
        pytest.skip("oracle/_ref/libp2ref.so not built")
    m, th, vel, se, (mx, my, mz, mt), markk, hp, nt = case()
    tko, mko, info = oracle_mod.titerate(m.gx, m.gy, m.gz, nt, m.bc.bondt, m.bc.bondv1, m.bc.bondn1, hp, th,
                                         vel=vel, se=se, markers=(mx[:-1], my[:-1], mz[:-1], mt[:-1]), markk=markk)
    assert not info["capped"] and info["substeps"] > 1
    out = str(tmp_path / "ref_heat33.npz")
    env = dict(os.environ, OMP_NUM_THREADS="1")
    p = subprocess.run([sys.executable, "-c", CHILD, ROOT, out], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    ref = np.load(out)
    np.testing.assert_array_equal(tko, ref["tk"])
    np.testing.assert_array_equal(mko, ref["markk"])
    assert np.abs(tko - th.tk).max() > 10
