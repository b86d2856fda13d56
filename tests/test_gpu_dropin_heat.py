"""titerate() through the drop-in boundary.

The reference harness compiled with the shim (oracle/_ref/libp2ref_shim.so)
keeps its state in globals, one model per process, so the heat model runs in
a child process: its titerate() is the shim's (pardiso2_b200/csrc/
move3mg_cuda.c), which reads tk, kt, cp, ro, ht, et, the T rows of bondm,
the heat parameters, velocities, pressure, stresses and markers from the
reference's globals and writes tk and markk back through p2_titerate.  The
written arrays must match the reference's own titerate() (golden vectors,
tests/golden/heat17.npz) within the heatmin tolerance of
tests/test_gpu_heat.py.

Needs oracle/_ref/libp2ref_shim.so (`make -C oracle refshim`); skipped when
it is absent.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import refdrv
from tests.test_gpu_heat import TK_MAX, TK_RMS

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")

CHILD = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from oracle import refdrv
from tests.golden.make_golden import HEAT_COMMON, HEAT_VARIANTS, heat_inputs, heat_model
m = heat_model()
th, vel, se, pr, (mx, my, mz, mt), markk = heat_inputs(m)
r = refdrv.RefModel(m, shim=True)
r.set_tbc(m.bc)
r.set_markers(mx, my, mz, mt)
one = np.ones_like(th.ro)
r.set_nodes({"nu": one, "ro": th.ro, "nxx": one, "nxy": one, "nxz": one, "nyz": one})
r.set_velocity(*vel)
r.set_stress(se)
out = {}
for name, v in HEAT_VARIANTS.items():
    hp = dict(HEAT_COMMON, **v)
    tk, mk = r.titerate(hp, v["multinumt"], th, markk, pr=pr)
    out["tk_" + name] = tk
    out["markk_" + name] = mk
np.savez(sys.argv[2], **out)
"""


def test_titerate_through_the_reference_globals(tmp_path):
    if not refdrv.available(shim=True):
        pytest.skip("oracle/_ref/libp2ref_shim.so not built")
    out = str(tmp_path / "heat_shim.npz")
    env = dict(os.environ, OMP_NUM_THREADS="1")
    p = subprocess.run([sys.executable, "-c", CHILD, ROOT, out], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    got = np.load(out)
    g = np.load(os.path.join(GOLDEN, "heat17.npz"))
    for name in ("mg", "single"):
        d = got["tk_" + name].astype(np.float64) - g["tk_" + name]
        assert np.abs(d).max() <= TK_MAX and np.sqrt(np.mean(d * d)) <= TK_RMS, name
        assert np.abs(got["markk_" + name].astype(np.float64) - g["markk_" + name]).max() <= TK_MAX, name
