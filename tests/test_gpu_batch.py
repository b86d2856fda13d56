"""Batched solves (p2_stokes_solve_batch): several independent instances on
concurrent streams give exactly the results of solving them one after
another (every instance is deterministic and owns its buffers, streams and
graphs), and every one converges."""
import numpy as np
import pytest

import pardiso2_b200 as P
from pardiso2_b200 import capi
from pardiso2_b200 import model as M

pytestmark = pytest.mark.gpu


def _problems():
    specs = [(33, 3, 41), (33, 1, 42), (49, 6, 43), (33, 9, 44), (49, 2, 45)]
    out = []
    for n, s, seed in specs:
        m = M.batch_model(n, s, seed)
        p = P.StokesProblem(m, tol=1e-8)
        p.ctx.upload_markers(m.markx, m.marky, m.markz, m.markt, m.rocks.n0, m.rocks.n1, m.rocks.ro)
        p.ctx.ronurecalc_resident()
        out.append((m, p))
    return out


def test_batch_equals_sequential():
    probs = _problems()
    seq = []
    for m, p in probs:
        info = p.ctx.solve_resident()
        assert info.status == 0 and info.rel_residual <= 1e-8
        seq.append((info.iterations, p.ctx.solution(m.nodenum)))
    for threads in (0, 2):
        infos, ms = capi.solve_batch([p.ctx for _, p in probs], host_threads=threads)
        assert ms > 0
        for (m, p), info, (its, sol) in zip(probs, infos, seq):
            assert info.status == 0 and info.iterations == its
            got = p.ctx.solution(m.nodenum)
            for k in sol:
                assert np.array_equal(got[k], sol[k]), (m.name, k)
    for _, p in probs:
        p.close()


def test_batch_arguments():
    assert capi.solve_batch([]) == ([], 0.0)
    L = capi.load()
    assert L.p2_stokes_solve_batch(None, 2, 0, None, None) != 0
    m = M.batch_model(33, 1, 7)
    p = P.StokesProblem(m)
    with pytest.raises(capi.P2Error):   # no node fields yet
        capi.solve_batch([p.ctx])
    p.close()
