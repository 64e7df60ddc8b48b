"""Batched cases (cfs_batch_*): one persistent launch per stage over all cases,
per-case CFL dt.  Each cell's arithmetic is the single-grid kernel's, and the
CFL maximum is exact, so every case of a batch must equal, bit for bit, the
same case advanced alone by a single context."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [0, 1])
def test_batch_equals_single_contexts(cfsb, workloads, prec):
    cases, states = workloads.batch_cases(8, seed=5, sizes=[48, 64, 96, 112, 160])
    with cfsb.Batch(cases, precision=prec) as b:
        for k, U in enumerate(states):
            b.set_state(k, U)
        t = b.advance(7, cfl=0.5)
        got = [b.get_state(k) for k in range(len(cases))]
    for k, (c, U) in enumerate(zip(cases, states)):
        with cfsb.Solver(c["nx"], c["ny"], c["lx"], c["ly"], precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                         bc=c["bc"], bc_prim=c.get("bc_prim")) as s:
            if "circle" in c:
                s.build_circle(*c["circle"], 400, cfsb.IB_BILINEAR_SLIP)
            s.set_state(U)
            ts, _ = s.advance(7, cfl=0.5)
            ref = s.get_state()
        assert np.array_equal(got[k], ref), f"case {k}: max diff {np.abs(got[k] - ref).max()}"
        assert t[k] == ts
        assert np.all(np.isfinite(ref))


def test_batch_rejects_exact_form(cfsb, workloads):
    cases, _ = workloads.batch_cases(2, seed=1, sizes=[32])
    with pytest.raises(cfsb.CfsError):
        cfsb.Batch(cases, precision=cfsb.FP64_EXACT)
