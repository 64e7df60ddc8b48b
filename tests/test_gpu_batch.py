"""Batched cases (cfs_batch_*): one persistent launch per stage over all cases,
per-case CFL dt.  Each cell's arithmetic is the single-grid kernel's; the two
are separate kernel instantiations, so the compiler may contract multiply-adds
differently and the results may differ in the last bits.  Every case of a
batch must equal the same case advanced alone by a single context to 1e-12
(FP64) / 1e-5 (FP32-mixed) relative to the state's magnitude."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mixed_cases(workloads):
    """Quadrant and cylinder cases (edge code) beside periodic body-free
    smooth-advection cases (no edge code): the batch runs them as separate
    feature groups."""
    cases, states = workloads.batch_cases(8, seed=5, sizes=[48, 64, 96, 112, 160])
    for n in (64, 96, 150):
        w = workloads.smooth_advection(n)
        cases.append({"nx": n, "ny": n, "lx": 1.0, "ly": 1.0, "bc": (2, 2, 2, 2)})
        states.append(w.U0)
    return cases, states


@pytest.mark.parametrize("prec", [0, 1])
def test_batch_equals_single_contexts(cfsb, workloads, prec):
    cases, states = _mixed_cases(workloads)
    with cfsb.Batch(cases, precision=prec, positivity=cfsb.POSITIVITY_BODY) as b:
        for k, U in enumerate(states):
            b.set_state(k, U)
        t = b.advance(7, cfl=0.5)
        got = [b.get_state(k) for k in range(len(cases))]
    for k, (c, U) in enumerate(zip(cases, states)):
        with cfsb.Solver(c["nx"], c["ny"], c["lx"], c["ly"], precision=prec, rk=cfsb.RK_SSP3, hll=cfsb.HLL_DAVIS,
                         bc=c["bc"], bc_prim=c.get("bc_prim"), positivity=cfsb.POSITIVITY_BODY) as s:
            if "circle" in c:
                s.build_circle(*c["circle"], 400, cfsb.IB_BILINEAR_SLIP)
            s.set_state(U)
            ts, _ = s.advance(7, cfl=0.5)
            ref = s.get_state()
        tol = 1e-12 if prec == cfsb.FP64 else 1e-5
        assert np.all(np.isfinite(ref))
        err = np.abs(got[k] - ref).max() / np.abs(ref).max()
        assert err <= tol, f"case {k}: relative max diff {err}"
        assert abs(t[k] - ts) <= tol * ts


def test_batch_rejects_exact_form(cfsb, workloads):
    cases, _ = workloads.batch_cases(2, seed=1, sizes=[32])
    with pytest.raises(cfsb.CfsError):
        cfsb.Batch(cases, precision=cfsb.FP64_EXACT)


def test_batch_replays_a_dt_sequence_per_case(cfsb, workloads):
    """cfs_batch_dt_last records each case's CFL step; cfs_batch_advance_dt
    replays those steps on a second batch of the same cases and form: the
    states are equal bit for bit and every case reaches the same time."""
    cases, states = workloads.batch_cases(12, seed=3, sizes=[64, 96, 128])
    kw = dict(precision=cfsb.FP64, positivity=cfsb.POSITIVITY_FLOOR)
    with cfsb.Batch(cases, **kw) as b:
        for k, U in enumerate(states):
            b.set_state(k, U)
        seq, t_ref = [], np.zeros(len(cases))
        for _ in range(5):
            t_ref += b.advance(1, cfl=0.5)
            seq.append(b.dt_last())
        ref = [b.get_state(k) for k in range(len(cases))]
    assert np.all(np.array(seq) > 0)
    assert np.any(np.array(seq)[0] != np.array(seq)[0][0])  # the cases keep their own dt
    with cfsb.Batch(cases, **kw) as b:
        for k, U in enumerate(states):
            b.set_state(k, U)
        t = np.zeros(len(cases))
        for d in seq:
            t += b.advance(1, dt=d)
        for k in range(len(cases)):
            assert np.array_equal(b.get_state(k), ref[k])
    assert np.array_equal(t, t_ref)


@pytest.mark.parametrize("prec", [0, 1])
def test_edge_code_on_request_changes_nothing(cfsb, workloads, prec):
    """cfs_case.edge_code = 1 puts periodic body-free cases into the edge-code
    launch (one feature group instead of two); their physics is unchanged --
    the edge code finds no physical side and no cell flags -- so they end
    within the instantiation tolerance of the same batch without the request."""
    cases, states = _mixed_cases(workloads)
    forced = [dict(c, edge_code=True) for c in cases]
    out = []
    for cs in (cases, forced):
        with cfsb.Batch(cs, precision=prec, positivity=cfsb.POSITIVITY_BODY) as b:
            for k, U in enumerate(states):
                b.set_state(k, U)
            t = b.advance(5, cfl=0.5)
            out.append(([b.get_state(k) for k in range(len(cs))], t))
    tol = 1e-12 if prec == cfsb.FP64 else 1e-5
    for k in range(len(cases)):
        a, b_ = out[0][0][k], out[1][0][k]
        assert np.all(np.isfinite(b_))
        assert np.abs(a - b_).max() / np.abs(a).max() <= tol, k
        assert abs(out[0][1][k] - out[1][1][k]) <= tol * out[0][1][k]
