"""ronurecalc with power-law rocks on the GPU (p2_ronurecalc_powerlaw)
against the reference's own run (tests/golden/pl17.npz).

Tolerance: node fields within 1e-6 relative.  The power marknu *
val1^((1-n)/n) is the device's pow, whose last-place rounding can differ
from the host C library's; the float accumulation then differs by a few
units in the last place at most.  Everything else is as in p2_ronurecalc.
"""
import os

import numpy as np
import pytest

import pardiso2_b200 as P
from pardiso2_b200.capi import P2Error
from tests.golden.make_golden import power_law_model

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIELDS = ("nu", "ro", "nxx", "nxy", "nxz", "nyz")


def test_power_law_ronurecalc_vs_reference():
    g = np.load(os.path.join(GOLDEN, "pl17.npz"))
    m, nu, mm, val1 = power_law_model()
    prob = P.StokesProblem(m)
    for _ in range(2):
        f = {k: np.zeros(m.nodenum, np.float32) for k in FIELDS}
        r = m.rocks
        prob.ctx.ronurecalc_powerlaw(m.markx, m.marky, m.markz, m.markt, r.n0, r.n1, r.ro, nu, mm, val1, f)
        for k in FIELDS:
            ref = g["node_" + k]
            err = np.abs(f[k].astype(np.float64) - ref) / np.maximum(np.abs(ref), 1e-30)
            assert err.max() <= 1e-6, (k, float(err.max()))
    # without the power-law tables the same rocks are refused
    with pytest.raises(P2Error):
        prob.ronurecalc()
    prob.close()
