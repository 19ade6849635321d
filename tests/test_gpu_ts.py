"""Device time stepper (cipher_ts_*) against its CPU restatement over the
oracle RHS (needs a B200: -m gpu).

FP64: the RHS, the stage combinations, PostStep and the error norm (whose
device reduction order the restatement replicates) are bit-exact, so whole
adaptive trajectories agree bit for bit: the same accepted and rejected
steps, the same step sizes, the same states.  Problems whose models call exp
or log agree to the last bits of those functions, so their trajectories are
compared within a tolerance.
"""
import numpy as np
import pytest

import cipher_b200 as cb
from cipher_b200 import _lib as L
import oracle

pytestmark = pytest.mark.gpu


def _device_run(P, M, X0, opts, t_end, precision="fp64"):
    ctx = cb.Context(P, M, precision)
    ts = cb.TimeStepper(ctx, opts)
    dX = ctx.alloc_state()
    ctx.from_aos(X0, dX)
    st = ts.solve(dX, 0.0, t_end)
    return ctx.to_aos(dX), st


def _port_run(P, M, X0, opts, t_end):
    X = X0.copy()
    ts = oracle.PortTS(P, M, opts)
    st = ts.solve(X, 0.0, t_end, L.TSStats())
    return X, st


def _defined(P, X):
    """(counts, ids and phi of the active slots) of an AoS state"""
    A = P.aos
    n = X[:, 0].astype(int)
    ids = np.where(np.arange(A.pf_size)[None, :] < n[:, None], X[:, 1:1 + A.pf_size], -1)
    phi = np.where(np.arange(A.pf_size)[None, :] < n[:, None], X[:, A.pf_offset:A.pf_offset + A.pf_size], 0.0)
    return n, ids, phi


@pytest.mark.parametrize("scheme", ["2a", "3bs"])
def test_trajectory_fp64_bit_exact(scheme):
    P = cb.Problem.grain_growth(2, [40, 32], 12, 8, 5)
    M = cb.Mesh(P)
    X0 = cb.diffuse_state_aos(P, M, 4.0)
    o = cb.ts_options(P, scheme, dt0=1e-3, dtmin=1e-9, dtmax=1.0, reltol=1e-4, abstol=1e-4)
    Xd, sd = _device_run(P, M, X0, o, 1.5)
    Xo, so = _port_run(P, M, X0, o, 1.5)
    assert (sd.steps, sd.rejected, sd.rhs_calls) == (so.steps, so.rejected, so.rhs_calls)
    assert sd.dt == so.dt and sd.last_norm == so.last_norm
    nd, idd, pd = _defined(P, Xd)
    no, ido, po = _defined(P, Xo)
    assert np.array_equal(nd, no) and np.array_equal(idd, ido)
    assert np.array_equal(pd, po)


def test_config0_to_t100_and_prefix_bit_exact():
    """2D grain growth 128^2, 64 grains, P=8, sharp start, 2a at
    rtol=abstol=1e-4 to t=100 on the device; its first steps (to t=1) are
    checked bit for bit against the CPU restatement"""
    P = cb.Problem.grain_growth(2, [128, 128], 64, 8, 2024)
    M = cb.Mesh(P)
    A = P.aos
    X0 = cb.initial_state_aos(P, M)
    o = cb.ts_options(P, "2a")
    assert o.reltol == 1e-4 and o.abstol == 1e-4
    Xd1, sd1 = _device_run(P, M, X0, o, 1.0)
    Xo1, so1 = _port_run(P, M, X0, o, 1.0)
    assert (sd1.steps, sd1.rejected) == (so1.steps, so1.rejected)
    assert np.array_equal(_defined(P, Xd1)[2], _defined(P, Xo1)[2])
    X, st = _device_run(P, M, X0, o, 100.0)
    assert st.t == 100.0 and st.steps > 10
    n, ids, phi = _defined(P, X)
    assert n.min() >= 1 and n.max() <= A.pf_size
    assert np.abs(phi.sum(axis=1) - 1.0).max() < 1e-12
    # grains coarsen: fewer grains own a cell at t=100 than at t=0
    owner = ids[np.arange(len(n)), phi.argmax(axis=1)]
    assert 0 < len(np.unique(owner)) < 64


def test_alloy_trajectory_within_tolerance():
    P = cb.Problem.alloy(2, [32, 24], "calphad2sl", 4, 6, 8, 61, 0x01)
    M = cb.Mesh(P)
    A = P.aos
    X0 = oracle.port_initial_state(P, M)
    o = cb.ts_options(P, "2a", dt0=1e-6, dtmin=1e-12, dtmax=1e-2, reltol=1e-3, abstol=1e-3, max_steps=12)
    Xd, sd = _device_run(P, M, X0, o, 1.0)
    Xo, so = _port_run(P, M, X0, o, 1.0)
    assert sd.steps == so.steps == 12
    assert abs(sd.t - so.t) <= 1e-9 * so.t
    nd, idd, pd = _defined(P, Xd)
    no, ido, po = _defined(P, Xo)
    assert np.array_equal(nd, no) and np.array_equal(idd, ido)
    assert np.abs(pd - po).max() <= 1e-8
    dp = slice(A.dp_offset, A.dp_offset + A.dp_size)
    assert np.abs(Xd[:, dp] - Xo[:, dp]).max() <= 1e-8 * np.abs(Xo[:, dp]).max()


def test_mixed_trajectory_close_to_fp64():
    P = cb.Problem.grain_growth(2, [48, 40], 14, 8, 9)
    M = cb.Mesh(P)
    X0 = cb.diffuse_state_aos(P, M, 4.0)
    o = cb.ts_options(P, "2a", dt0=1e-3, dtmin=1e-9, dtmax=1.0, reltol=1e-4, abstol=1e-4)
    X64, s64 = _device_run(P, M, X0, o, 1.0)
    Xm, sm = _device_run(P, M, X0, o, 1.0, "mixed")
    assert sm.t == 1.0
    assert abs(sm.steps - s64.steps) <= max(2, s64.steps // 10)
    assert np.abs(_defined(P, Xm)[2].sum(axis=1) - 1.0).max() < 1e-5
    # phase fractions of cells whose sets agree
    n64, i64, p64 = _defined(P, X64)
    nm, im, pm = _defined(P, Xm)
    same = np.all(i64 == im, axis=1)
    assert same.mean() > 0.99
    assert np.abs(p64[same] - pm[same]).max() < 1e-3


def test_nonfinite_state_rejected_on_device():
    P = cb.Problem.grain_growth(2, [24, 20], 8, 8, 3)
    M = cb.Mesh(P)
    A = P.aos
    X0 = cb.diffuse_state_aos(P, M, 4.0)
    X0[5, A.pf_offset] = np.nan
    ctx = cb.Context(P, M, "fp64")
    o = cb.ts_options(P, "2a", dt0=1e-2, dtmin=1e-5, dtmax=1.0, reltol=1e-4, abstol=1e-4)
    ts = cb.TimeStepper(ctx, o)
    dX = ctx.alloc_state()
    ctx.from_aos(X0, dX)
    dts = []
    for _ in range(3):
        assert not ts.step(dX, 1.0)
        dts.append(ts.stats().dt)
    assert np.allclose(dts, [1e-3, 1e-4, 1e-5])
    with pytest.raises(L.CipherError) as e:
        ts.step(dX, 1.0)
    assert e.value.code == L.E_NONFINITE
