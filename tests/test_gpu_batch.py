"""Many domains stepped together (cipher_batch_*) against each domain
stepped alone with cipher_ts (needs a B200: -m gpu).

A domain's arithmetic in the batch is the single stepper's (the same cell
bodies, the same per-domain combination blocks and norm reduction order,
the same host step control), so every domain's trajectory must be identical
bit for bit to its run alone — in FP64 and in the mixed layout, with graphs
on or off, and when domains join or leave mid-run.
"""
import numpy as np
import pytest

import cipher_b200 as cb
from cipher_b200 import _lib as L
import oracle

pytestmark = pytest.mark.gpu

# (res, grains, cap, seed): uneven sizes and caps, config-0 physics
DOMAINS = [([32, 32], 4, 4, 1), ([48, 40], 12, 8, 2), ([64, 64], 20, 8, 3), ([40, 24], 6, 6, 4),
           ([96, 64], 30, 12, 5), ([56, 56], 16, 8, 6)]


def _gg(res, ng, cap, seed):
    P = cb.Problem.grain_growth(2, res, ng, cap, seed)
    M = cb.Mesh(P)
    return P, M, cb.diffuse_state_aos(P, M, 4.0)


def _opts(P, **kw):
    base = dict(dt0=1e-3, dtmin=1e-9, dtmax=1.0, reltol=1e-4, abstol=1e-4)
    base.update(kw)
    return cb.ts_options(P, "2a", **base)


def _alone(P, M, X0, opts, t_end, precision):
    ctx = cb.Context(P, M, precision)
    ts = cb.TimeStepper(ctx, opts)
    dX = ctx.alloc_state()
    ctx.from_aos(X0, dX)
    st = ts.solve(dX, 0.0, t_end)
    return ctx.to_aos(dX), st


def _same(P, Xa, Xb):
    A = P.aos
    n = Xa[:, 0].astype(int)
    if not np.array_equal(n, Xb[:, 0].astype(int)):
        return False
    k = np.arange(A.pf_size)[None, :] < n[:, None]
    ids_a = np.where(k, Xa[:, 1:1 + A.pf_size], -1)
    ids_b = np.where(k, Xb[:, 1:1 + A.pf_size], -1)
    ph_a = np.where(k, Xa[:, A.pf_offset:A.pf_offset + A.pf_size], 0)
    ph_b = np.where(k, Xb[:, A.pf_offset:A.pf_offset + A.pf_size], 0)
    rest = slice(A.dp_offset, A.ndof)
    return (np.array_equal(ids_a, ids_b) and np.array_equal(ph_a, ph_b)
            and np.array_equal(Xa[:, rest], Xb[:, rest]))


def _run_batch(doms, t_ends, precision, graphs=True):
    opts = _opts(doms[0][0])
    b = cb.Batch(opts, precision, graphs=graphs)
    live = []
    for (P, M, X0), te in zip(doms, t_ends):
        ctx = cb.Context(P, M, precision)
        dX = ctx.alloc_state()
        ctx.from_aos(X0, dX)
        live.append((ctx, dX, b.attach(ctx, dX, 0.0, te)))
    steps = 0
    while b.step() > 0:
        steps += 1
        assert steps < 100000
    b.flush()
    out = []
    for ctx, dX, slot in live:
        st, status, err = b.stats(slot)
        assert status == L.BATCH_FINISHED, (status, err)
        out.append((ctx.to_aos(dX), st))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_each_domain_alone(precision):
    doms = [_gg(*d) for d in DOMAINS]
    t_ends = [0.6, 1.0, 0.8, 1.2, 0.5, 0.9]
    res = _run_batch(doms, t_ends, precision)
    for (P, M, X0), te, (Xb, sb) in zip(doms, t_ends, res):
        Xa, sa = _alone(P, M, X0, _opts(P), te, precision)
        assert (sb.steps, sb.rejected, sb.rhs_calls) == (sa.steps, sa.rejected, sa.rhs_calls)
        assert sb.t == sa.t == te and sb.dt == sa.dt
        assert _same(P, Xb, Xa)


def test_graphs_on_and_off_agree():
    doms = [_gg(*d) for d in DOMAINS[:3]]
    t_ends = [0.5, 0.7, 0.4]
    on = _run_batch(doms, t_ends, "fp64", graphs=True)
    off = _run_batch(doms, t_ends, "fp64", graphs=False)
    for (P, _, _), (Xa, sa), (Xb, sb) in zip(doms, on, off):
        assert sa.steps == sb.steps and _same(P, Xa, Xb)


def test_general_path_domain_in_batch():
    """an alloy domain (general kernels, launched per domain) among
    phase-field domains: each still matches its run alone"""
    Pa = cb.Problem.alloy(2, [32, 24], "calphad2sl", 4, 6, 8, 61, 0x01)
    Ma = cb.Mesh(Pa)
    Xa0 = oracle.port_initial_state(Pa, Ma)
    opts = cb.ts_options(Pa, "2a", dt0=1e-6, dtmin=1e-12, dtmax=1e-2, reltol=1e-3, abstol=1e-3)
    doms = [(Pa, Ma, Xa0)] + [_gg(*d) for d in DOMAINS[:2]]
    b = cb.Batch(opts, "fp64")
    live = []
    for (P, M, X0), te in zip(doms, [0.004, 0.3, 0.3]):
        ctx = cb.Context(P, M, "fp64")
        dX = ctx.alloc_state()
        ctx.from_aos(X0, dX)
        live.append((P, M, X0, te, ctx, dX, b.attach(ctx, dX, 0.0, te)))
    while b.step() > 0:
        pass
    b.flush()
    for P, M, X0, te, ctx, dX, slot in live:
        st, status, _ = b.stats(slot)
        assert status == L.BATCH_FINISHED
        Xa, sa = _alone(P, M, X0, opts, te, "fp64")
        assert st.steps == sa.steps and st.rejected == sa.rejected
        assert _same(P, ctx.to_aos(dX), Xa)


def test_join_and_leave_mid_run():
    """continuous batching: a domain that joins after others have stepped,
    and one that leaves early, still match their runs alone"""
    doms = [_gg(*d) for d in DOMAINS[:4]]
    opts = _opts(doms[0][0])
    b = cb.Batch(opts, "fp64")
    ctxs = []
    for P, M, X0 in doms:
        ctx = cb.Context(P, M, "fp64")
        dX = ctx.alloc_state()
        ctx.from_aos(X0, dX)
        ctxs.append((ctx, dX))
    s0 = b.attach(ctxs[0][0], ctxs[0][1], 0.0, 0.8)
    s1 = b.attach(ctxs[1][0], ctxs[1][1], 0.0, 0.8)
    for _ in range(5):
        b.step()
    s2 = b.attach(ctxs[2][0], ctxs[2][1], 0.0, 0.6)
    for _ in range(3):
        b.step()
    # leave early: its state is the one after the steps it took
    st1, _, _ = b.stats(s1)
    b.detach(s1)
    s3 = b.attach(ctxs[3][0], ctxs[3][1], 0.0, 0.5)
    while b.step() > 0:
        pass
    b.flush()
    for (P, M, X0), (ctx, dX), slot, te in zip([doms[0], doms[2], doms[3]], [ctxs[0], ctxs[2], ctxs[3]],
                                               [s0, s2, s3], [0.8, 0.6, 0.5]):
        st, status, _ = b.stats(slot)
        assert status == L.BATCH_FINISHED
        Xa, sa = _alone(P, M, X0, opts, te, "fp64")
        assert st.steps == sa.steps and _same(P, ctx.to_aos(dX), Xa)
    # the domain that left: equal to its run alone to the time it reached
    P, M, X0 = doms[1]
    Xa, sa = _alone(P, M, X0, _opts(P, max_steps=int(st1.steps)), 0.8, "fp64")
    assert sa.steps == st1.steps and sa.t == st1.t
    assert _same(P, ctxs[1][0].to_aos(ctxs[1][1]), Xa)


def test_failed_domain_is_isolated():
    doms = [_gg(*d) for d in DOMAINS[:3]]
    P, M, X0 = doms[1]
    A = P.aos
    Xbad = X0.copy()
    Xbad[7, A.pf_offset] = np.nan
    doms[1] = (P, M, Xbad)
    opts = _opts(doms[0][0], dtmin=1e-5)
    b = cb.Batch(opts, "fp64")
    live = []
    for (P, M, X0), te in zip(doms, [0.4, 0.4, 0.4]):
        ctx = cb.Context(P, M, "fp64")
        dX = ctx.alloc_state()
        ctx.from_aos(X0, dX)
        live.append((P, M, X0, ctx, dX, b.attach(ctx, dX, 0.0, te)))
    while b.step() > 0:
        pass
    b.flush()
    statuses = [b.stats(s)[1:] for *_, s in live]
    assert statuses[1] == (L.BATCH_FAILED, L.E_NONFINITE)
    for k in (0, 2):
        P, M, X0, ctx, dX, slot = live[k]
        assert statuses[k][0] == L.BATCH_FINISHED
        Xa, sa = _alone(P, M, X0, opts, 0.4, "fp64")
        assert _same(P, ctx.to_aos(dX), Xa)
