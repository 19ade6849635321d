"""Serving with continuous batching (cipher_server_*) (needs a B200: -m gpu).

Each request's result must equal the same request solved alone with the
single stepper, bit for bit, however the requests overlap on the device;
admission must respect the HBM budget; a request that can never fit must
fail without blocking the ones behind it.
"""
import numpy as np
import pytest

import cipher_b200 as cb
from cipher_b200 import _lib as L

pytestmark = pytest.mark.gpu

# (kind, builder args, init, t_end)
REQUESTS = [
    ("gg", ([48, 48], 10, 8, 11), "diffuse", 0.6),
    ("gg", ([64, 32], 12, 8, 12), "diffuse", 0.4),
    ("alloy", ([32, 24], "calphad2sl", 4, 6, 8, 61, 0x01), "sharp", 0.003),
    ("gg", ([96, 96], 30, 8, 13), "diffuse", 0.3),
    ("gg", ([32, 32], 6, 6, 14), "diffuse", 0.8),
    ("gg", ([128, 64], 40, 8, 15), "diffuse", 0.2),
]


def _problem(kind, args):
    if kind == "gg":
        res, ng, cap, seed = args
        return cb.Problem.grain_growth(2, res, ng, cap, seed)
    res, model, ncp, npr, cap, seed, feats = args
    return cb.Problem.alloy(2, res, model, ncp, npr, cap, seed, feats)


def _opts():
    P = cb.Problem.grain_growth(2, [8, 8], 2, 2, 1)
    return cb.ts_options(P, "2a", dt0=1e-6, dtmin=1e-12, dtmax=1.0, reltol=1e-4, abstol=1e-4)


def _alone(kind, args, init, t_end, opts):
    P = _problem(kind, args)
    M = cb.Mesh(P)
    X0 = cb.initial_state_aos(P, M) if init == "sharp" else cb.diffuse_state_aos(P, M, 4.0)
    ctx = cb.Context(P, M, "fp64")
    dX = ctx.alloc_state()
    ctx.from_aos(X0, dX)
    ctx.chem_init(dX)
    ts = cb.TimeStepper(ctx, opts)
    st = ts.solve(dX, 0.0, t_end)
    return ctx.to_aos(dX), st


def _serve(opts, budget, max_active=64, extra=()):
    srv = cb.Server(opts, "fp64", hbm_budget=budget, max_active=max_active)
    ids = []
    for kind, args, init, t_end in list(REQUESTS) + list(extra):
        ids.append(srv.submit(_problem(kind, args), t_end, init))
    for _ in range(200000):
        q, a, d = srv.poll()
        if d == len(ids):
            break
    return srv, ids


def _check_equal_alone(srv, ids, opts):
    for rid, (kind, args, init, t_end) in zip(ids, REQUESTS):
        r, X = srv.result(rid, with_state=True)
        assert r.state == 2 and r.status == L.BATCH_FINISHED, (rid, r.status, r.error)
        Xa, sa = _alone(kind, args, init, t_end, opts)
        assert (r.stats.steps, r.stats.rejected) == (sa.steps, sa.rejected)
        assert r.stats.t == t_end
        assert np.array_equal(np.nan_to_num(X, nan=-7.0), np.nan_to_num(Xa, nan=-7.0))
        assert r.t_submit <= r.t_admit <= r.t_finish


def test_requests_in_the_mix_equal_alone():
    opts = _opts()
    srv, ids = _serve(opts, budget=8 << 30)
    _check_equal_alone(srv, ids, opts)
    used, peak = srv.usage()
    assert used == 0 and peak > 0


def test_budget_limits_admission():
    opts = _opts()
    # room for about two of the smaller requests at a time
    srv, ids = _serve(opts, budget=6 << 20)
    _check_equal_alone(srv, ids, opts)
    used, peak = srv.usage()
    assert peak <= 6 << 20
    admits = sorted(srv.result(i)[0].t_admit for i in ids)
    finishes = sorted(srv.result(i)[0].t_finish for i in ids)
    # not everything was admitted at once
    assert admits[-1] > finishes[0]


def test_oversized_request_fails_without_blocking():
    opts = _opts()
    big = ("gg", ([1024, 1024], 64, 8, 99), "diffuse", 0.1)
    srv = cb.Server(opts, "fp64", hbm_budget=4 << 20, max_active=8)
    rb = srv.submit(_problem(big[0], big[1]), big[3], big[2])
    rs = srv.submit(_problem(*REQUESTS[0][:2]), REQUESTS[0][3], REQUESTS[0][2])
    for _ in range(100000):
        if srv.poll()[2] == 2:
            break
    r, _ = srv.result(rb)
    assert r.state == 2 and r.status == L.BATCH_FAILED and r.error == L.E_NOMEM
    r, _ = srv.result(rs)
    assert r.state == 2 and r.status == L.BATCH_FINISHED
