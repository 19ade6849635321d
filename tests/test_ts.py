"""The RK time stepper's CPU restatement (oracle/port/oracle_ts.c): tableau
orders, error control, rejection and non-finite handling.  The device
stepper is compared with it in test_gpu_ts.py.

The reference steps with PETSc's TSRK/TSADAPTDSP, which is not vendored, so
trajectories are checked against this restatement and against the
methods' known convergence orders, not against PETSc.
"""
import numpy as np
import pytest

import cipher_b200 as cb
from cipher_b200 import _lib as L
import oracle


def _gg(res=(24, 20), ng=8, cap=8, seed=3):
    P = cb.Problem.grain_growth(2, list(res), ng, cap, seed)
    M = cb.Mesh(P)
    return P, M, cb.diffuse_state_aos(P, M, 4.0)


def _smooth_two_phase(res=(24, 20)):
    """two phases present everywhere with 0.2 < phi < 0.8: every slot stays
    active, so the RHS is smooth (no active-set switching)"""
    P = cb.Problem.grain_growth(2, list(res), 2, 2, 1)
    M = cb.Mesh(P)
    A = P.aos
    X = cb.initial_state_aos(P, M)
    x = np.arange(M.ncells) % res[0]
    y = np.arange(M.ncells) // res[0]
    p0 = 0.5 + 0.2 * np.sin(2 * np.pi * x / res[0]) * np.cos(2 * np.pi * y / res[1])
    X[:, 0] = 2
    X[:, 1], X[:, 2] = 0, 1
    X[:, A.pf_offset], X[:, A.pf_offset + 1] = p0, 1.0 - p0
    return P, M, X


@pytest.mark.parametrize("scheme,order", [("1fe", 1), ("2a", 2), ("3bs", 3)])
def test_fixed_step_convergence_order(scheme, order):
    """fixed steps, no PostStep: the error at t=T falls as dt^order"""
    P, M, X0 = _smooth_two_phase()
    T = 0.5

    def run(sch, dt):
        o = cb.ts_options(P, sch, dt0=dt, dtmin=dt, dtmax=dt, reltol=1e30, abstol=1e30, poststep=0)
        ts = oracle.PortTS(P, M, o)
        X = X0.copy()
        ts.solve(X, 0.0, T, L.TSStats())
        return X

    ref = run("3bs", T / 512)
    errs = [np.abs(run(scheme, T / k) - ref).max() for k in (16, 32)]
    rate = np.log2(errs[0] / errs[1])
    assert abs(rate - order) < 0.35, (errs, rate)


def test_adaptive_run_keeps_states_valid():
    P, M, X = _gg()
    A = P.aos
    o = cb.ts_options(P, "2a", dt0=1e-3, dtmin=1e-8, dtmax=1.0, reltol=1e-4, abstol=1e-4)
    ts = oracle.PortTS(P, M, o)
    st = ts.solve(X, 0.0, 2.0, L.TSStats())
    assert st.t == 2.0 and st.steps > 3
    assert st.rhs_calls == 2 * (st.steps + st.rejected)
    n = X[:, 0].astype(int)
    assert n.min() >= 1 and n.max() <= A.pf_size
    phi = X[:, A.pf_offset:A.pf_offset + A.pf_size]
    s = np.array([phi[c, :n[c]].sum() for c in range(len(n))])
    assert np.abs(s - 1.0).max() < 1e-12
    assert st.last_norm <= 1.0 + 1e-12


def test_tight_tolerance_rejects_and_shrinks():
    P, M, X = _gg()
    o = cb.ts_options(P, "2a", dt0=0.5, dtmin=1e-9, dtmax=1.0, reltol=1e-9, abstol=1e-9)
    ts = oracle.PortTS(P, M, o)
    acc = ts.step(X, 10.0)
    st = ts.stats(L.TSStats())
    assert not acc and st.rejected == 1 and st.dt < 0.5
    assert st.last_norm > 1.0


def test_nonfinite_state_is_rejected_then_fails_at_dtmin():
    """a NaN planted in the state: every attempt is rejected and dt is cut
    by 10 until the minimum step, where the stepper reports the failure"""
    P, M, X = _gg()
    A = P.aos
    X[5, A.pf_offset] = np.nan
    o = cb.ts_options(P, "2a", dt0=1e-2, dtmin=1e-5, dtmax=1.0, reltol=1e-4, abstol=1e-4)
    ts = oracle.PortTS(P, M, o)
    dts = []
    for _ in range(3):
        assert not ts.step(X, 1.0)
        dts.append(ts.stats(L.TSStats()).dt)
    assert np.allclose(dts, [1e-3, 1e-4, 1e-5])
    with pytest.raises(RuntimeError):
        ts.step(X, 1.0)


def test_final_step_matches_end_time():
    P, M, X = _gg()
    o = cb.ts_options(P, "3bs", dt0=0.03, dtmin=1e-8, dtmax=0.03, reltol=1e-2, abstol=1e-2)
    ts = oracle.PortTS(P, M, o)
    st = ts.solve(X, 0.0, 0.1, L.TSStats())
    assert st.t == 0.1
    st2 = ts.solve(X, 0.1, 0.25, L.TSStats())
    assert st2.t == 0.25 and st2.steps > st.steps
