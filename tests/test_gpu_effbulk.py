"""Effective bulk viscosity diagnostics on the GPU (p2_effbulk_visc,
effbulkvisccalc mode 1) against the oracle, which the CPU suite pins to the
reference's own printed output.  Per-node values follow the reference's
float/double operations; the sums run in another order, so the results
agree to 1e-9 relative (component averages: to 1e-9 of the largest of their
twelve)."""
import os

import numpy as np
import pytest

import pardiso2_b200 as P
from tests.test_oracle_golden import _bulk_fields, load_case

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_effbulk_vs_oracle(oracle_mod):
    g = np.load(os.path.join(GOLDEN, "bulk21.npz"))
    m, s = load_case("spheres21")
    f = _bulk_fields(g, s)
    prob = P.StokesProblem(m)
    for _ in range(2):
        r = prob.ctx.effbulk_visc(f)
        out, counts = oracle_mod.effbulk(m, f)
        assert (r.numtot, r.nummat, r.numinc) == tuple(int(c) for c in counts)
        got = [r.eiin, r.siin, r.eiivp, r.tau2, r.hsn, r.nubulkn, r.nubulk1, r.nubulk2, r.nubulk3, r.nubulk4]
        assert np.allclose(got, out[:10], rtol=1e-9, atol=0)
        for a, b in ((list(r.matrix), out[10:22]), (list(r.incl), out[22:34])):
            assert np.max(np.abs(np.array(a) - b)) <= 1e-9 * np.max(np.abs(b))
    prob.close()
