"""Several-interface grain growth on the device (needs a B200: -m gpu).

Grain growth whose grain pairs meet through different interfaces (per-pair
energy and mobility, some with activation energies, some with other widths)
takes the phase-field kernels' several-interface form: the reference-order
cell terms of pf_cell.cuh, with per-pair interface properties looked up
through interfacelist (src/cipher.c:420-472) and the triple-junction maximum
over the three pairs (src/cipher.c:482-489).

Tolerances:
    FP64 path   bit-exact against the reference (oracle/_ref, or the golden
                fixtures the reference produced) when no interface has an
                activation energy; with one, the factor exp(Q(T)/RT) comes from
                CUDA's exp, which may differ from the host libm in the last
                bit, so max|F - F_ref| / max|F_ref| <= 1e-10 (as for the
                chemistry kernels)
    mixed path  max|F_mixed - F_64| / max|F_64| <= 1e-6 against the FP64
                oracle on the same FP32-rounded input
Active sets after PostStep are bit-exact; phase fractions are bit-exact in
FP64 and equal to the oracle's rounded to FP32 in the mixed layout.  The quadratic interpolant
(src/utility.c:470-565) takes the same kernels; the batched stepper and the
mixed server must give each domain the result it gets alone.
"""
import glob
import os

import numpy as np
import pytest

import cipher_b200 as cb
from cipher_b200 import _lib as L
import oracle

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
MULTI_GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "ggmulti*.npz")))
TOLMIX = 1e-6
TOL64 = 1e-10

# (name, dim, res, ngrains, cap, seed, ninterfaces, activation, widths)
CASES = [
    ("2d_P4_3itf", 2, [40, 24], 6, 4, 5, 3, False, False),
    ("2d_P8_5itf_act_widths", 2, [48, 40], 24, 8, 9, 5, True, True),
    ("3d_P12_4itf_widths", 3, [16, 16, 16], 30, 12, 3, 4, False, True),
    ("3d_P15_6itf_act", 3, [12, 14, 10], 40, 15, 21, 6, True, False),
]


def _build(dim, res, ng, cap, seed, nitf, act, wid, interp=None):
    P = cb.Problem.grain_growth_multi(dim, res, ng, cap, seed, nitf, activation=act, widths=wid)
    if interp is not None:
        P.s.interpolation = interp
    M = cb.Mesh(P)
    return P, M, cb.diffuse_state_aos(P, M, 4.0)


def _oracle_rhs(P, M, X):
    if oracle.ref_available():
        with oracle.RefOracle(P, M) as R:
            return R.rhs(X)
    return oracle.port_rhs(P, M, X)


def _device_rhs(ctx, X):
    dX, dF = ctx.alloc_state(), ctx.alloc_state()
    ctx.from_aos(X, dX)
    ctx.rhs(0.0, dX, dF)
    ctx.check()
    return ctx.to_aos(dF)


def _round32(P, X):
    A = P.aos
    Y = X.copy()
    for off, size in ((A.pf_offset, A.pf_size), (A.tm_offset, 1)):
        Y[:, off:off + size] = Y[:, off:off + size].astype(np.float32).astype(np.float64)
    return Y


def _rel_err(P, F, Fo):
    A = P.aos
    sl = slice(A.pf_offset, A.pf_offset + A.pf_size)
    return np.abs(F[:, sl] - Fo[:, sl]).max() / np.abs(Fo[:, sl]).max()


def _check_fp64(P, F, Fo, activation):
    if activation:
        assert _rel_err(P, F, Fo) <= TOL64, _rel_err(P, F, Fo)
        A = P.aos
        rest = np.ones(F.shape[1], dtype=bool)
        rest[A.pf_offset:A.pf_offset + A.pf_size] = False
        assert np.array_equal(F[:, rest], Fo[:, rest])
    else:
        assert np.array_equal(F, Fo), np.abs(F - Fo).max()


def test_multi_fixtures_present():
    assert len(MULTI_GOLDEN) >= 2


def test_problems_take_the_several_interface_form():
    """the builder gives pairs different interfaces, so the context cannot
    take the single-interface closed forms"""
    P, M, X = _build(*CASES[1][1:])
    s = P.s
    ids = {s.interfacelist[a * s.npf + b] for a in range(s.npf) for b in range(a + 1, s.npf)}
    assert len(ids) > 1


@pytest.mark.parametrize("path", MULTI_GOLDEN, ids=[os.path.basename(p) for p in MULTI_GOLDEN])
def test_rhs_fp64_matches_reference_fixture(path):
    g = np.load(path)
    dim, *r = (int(v) for v in g["meta"][:4])
    ng, cap, seed, nitf, feats = (int(v) for v in g["meta"][4:9])
    P, M, X = _build(dim, r[:dim], ng, cap, seed, nitf, bool(feats & 1), bool(feats & 2))
    assert np.array_equal(X, g["X"])
    ctx = cb.Context(P, M, "fp64")
    F = _device_rhs(ctx, X)
    _check_fp64(P, F, g["F"], activation=bool(feats & 1))


@pytest.mark.parametrize("interp", [None, L.INTERP_QUADRATIC], ids=["cubic", "quadratic"])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_rhs_fp64_bit_exact(case, interp):
    P, M, X = _build(*case[1:], interp=interp)
    ctx = cb.Context(P, M, "fp64")
    F = _device_rhs(ctx, X)
    Fo = _oracle_rhs(P, M, X)
    _check_fp64(P, F, Fo, activation=case[7])


@pytest.mark.parametrize("interp", [None, L.INTERP_QUADRATIC], ids=["cubic", "quadratic"])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_rhs_mixed_within_1e6(case, interp):
    P, M, X = _build(*case[1:], interp=interp)
    X32 = _round32(P, X)
    ctx = cb.Context(P, M, "mixed")
    F = _device_rhs(ctx, X32)
    Fo = _oracle_rhs(P, M, X32)
    err = _rel_err(P, F, Fo)
    assert err <= TOLMIX, err


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", CASES[1:], ids=[c[0] for c in CASES[1:]])
def test_poststep_bit_exact(case, precision):
    P, M, X = _build(*case[1:])
    if precision == "mixed":
        X = _round32(P, X)
    ctx = cb.Context(P, M, precision)
    dX = ctx.alloc_state()
    ctx.from_aos(X, dX)
    ctx.poststep(dX)
    Xd = ctx.to_aos(dX)
    Xo = X.copy()
    assert oracle.port_poststep(P, M, Xo) == 0
    A = P.aos
    if precision == "mixed":           # the projection runs in FP64; the layout stores FP32
        Xo[:, A.pf_offset:A.pf_offset + A.pf_size] = Xo[:, A.pf_offset:A.pf_offset + A.pf_size].astype(np.float32)
    n = Xo[:, 0].astype(int)
    assert np.array_equal(Xd[:, 0], Xo[:, 0])
    for g in range(A.pf_size):
        m = n > g
        assert np.array_equal(Xd[m, 1 + g], Xo[m, 1 + g])
        assert np.array_equal(Xd[m, A.pf_offset + g], Xo[m, A.pf_offset + g])


def test_trajectory_fp64_bit_exact():
    """15 forward-Euler steps (device AXPY + RHS + PostStep) stay
    bit-identical to the oracle driven the same way (P = 15, five
    interfaces of different widths, no activation energies)"""
    P, M, X = _build(3, [14, 12, 10], 12, 15, 7, 5, False, True)
    ctx = cb.Context(P, M, "fp64")
    dX, dF = ctx.alloc_state(), ctx.alloc_state()
    ctx.from_aos(X, dX)
    dt = 0.02
    Xo = X.copy()
    for _ in range(15):
        ctx.rhs(0.0, dX, dF)
        ctx.waxpy(dX, dX, dt, dF)
        Xo = Xo + dt * oracle.port_rhs(P, M, Xo)
        assert oracle.port_poststep(P, M, Xo) == 0
        ctx.poststep(dX)
    Xd = ctx.to_aos(dX)
    A = P.aos
    n = Xo[:, 0].astype(int)
    assert np.array_equal(Xd[:, 0], Xo[:, 0])
    for g in range(A.pf_size):
        m = n > g
        assert np.array_equal(Xd[m, 1 + g], Xo[m, 1 + g])
        assert np.array_equal(Xd[m, A.pf_offset + g], Xo[m, A.pf_offset + g])


# ------------------------------------------------------------------ batch ----

def _opts(P):
    return cb.ts_options(P, "2a", dt0=1e-3, dtmin=1e-9, dtmax=1.0, reltol=1e-4, abstol=1e-4)


def _same(P, Xa, Xb):
    A = P.aos
    n = Xa[:, 0].astype(int)
    if not np.array_equal(n, Xb[:, 0].astype(int)):
        return False
    k = np.arange(A.pf_size)[None, :] < n[:, None]
    return (np.array_equal(np.where(k, Xa[:, 1:1 + A.pf_size], -1), np.where(k, Xb[:, 1:1 + A.pf_size], -1))
            and np.array_equal(np.where(k, Xa[:, A.pf_offset:A.pf_offset + A.pf_size], 0),
                               np.where(k, Xb[:, A.pf_offset:A.pf_offset + A.pf_size], 0))
            and np.array_equal(Xa[:, A.dp_offset:], Xb[:, A.dp_offset:]))


def _alone(P, M, X0, opts, t_end, precision):
    ctx = cb.Context(P, M, precision)
    ts = cb.TimeStepper(ctx, opts)
    dX = ctx.alloc_state()
    ctx.from_aos(X0, dX)
    st = ts.solve(dX, 0.0, t_end)
    return ctx.to_aos(dX), st


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_with_several_interface_domains_matches_alone(precision):
    """several-interface domains (their own kernel group) beside
    single-interface ones: every domain's trajectory equals its run alone"""
    doms = []
    for (res, ng, cap, seed, nitf, act, wid) in [([48, 40], 12, 8, 2, 4, True, False),
                                                  ([32, 32], 6, 6, 3, 3, False, True),
                                                  ([64, 48], 20, 8, 4, 5, True, True)]:
        P = cb.Problem.grain_growth_multi(2, res, ng, cap, seed, nitf, activation=act, widths=wid)
        M = cb.Mesh(P)
        doms.append((P, M, cb.diffuse_state_aos(P, M, 4.0)))
    for (res, ng, cap, seed) in [([40, 40], 10, 8, 5), ([56, 32], 8, 6, 6)]:
        P = cb.Problem.grain_growth(2, res, ng, cap, seed)
        M = cb.Mesh(P)
        doms.append((P, M, cb.diffuse_state_aos(P, M, 4.0)))
    t_ends = [0.5, 0.7, 0.4, 0.6, 0.3]
    opts = _opts(doms[0][0])
    b = cb.Batch(opts, precision)
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
    for (P, M, X0), te, (ctx, dX, slot) in zip(doms, t_ends, live):
        st, status, err = b.stats(slot)
        assert status == L.BATCH_FINISHED, (status, err)
        Xa, sa = _alone(P, M, X0, opts, te, precision)
        assert (st.steps, st.rejected, st.rhs_calls) == (sa.steps, sa.rejected, sa.rhs_calls)
        assert _same(P, ctx.to_aos(dX), Xa)


# ----------------------------------------------------------------- server ----

def test_mixed_server_requests_equal_alone():
    """continuous batching in the mixed precision: each request's final state
    equals the same request solved alone in the mixed precision, within the
    mixed path's tolerance (1e-6 of the largest phase fraction change); in
    practice bit for bit, since a domain's arithmetic is the same in the mix"""
    P0 = cb.Problem.grain_growth(2, [8, 8], 2, 2, 1)
    opts = cb.ts_options(P0, "2a", dt0=1e-6, dtmin=1e-12, dtmax=1.0, reltol=1e-4, abstol=1e-4)
    reqs = [(([48, 48], 10, 8, 11), None, 0.5), (([64, 32], 12, 8, 12), (4, True), 0.4),
            (([96, 64], 24, 8, 13), None, 0.3), (([32, 32], 6, 6, 14), (3, False), 0.6)]

    def problem(args, multi):
        res, ng, cap, seed = args
        if multi is None:
            return cb.Problem.grain_growth(2, res, ng, cap, seed)
        return cb.Problem.grain_growth_multi(2, res, ng, cap, seed, multi[0], activation=multi[1])

    srv = cb.Server(opts, "mixed", hbm_budget=8 << 30, max_active=64)
    ids = [srv.submit(problem(a, m), te, "diffuse") for a, m, te in reqs]
    for _ in range(200000):
        if srv.poll()[2] == len(ids):
            break
    for rid, (a, m, te) in zip(ids, reqs):
        r, X = srv.result(rid, with_state=True)
        assert r.state == 2 and r.status == L.BATCH_FINISHED, (r.status, r.error)
        P = problem(a, m)
        M = cb.Mesh(P)
        Xa, sa = _alone(P, M, cb.diffuse_state_aos(P, M, 4.0), opts, te, "mixed")
        assert r.stats.t == te
        A = P.aos
        assert np.array_equal(X[:, 0], Xa[:, 0])
        sl = slice(A.pf_offset, A.pf_offset + A.pf_size)
        d = np.abs(np.nan_to_num(X[:, sl], nan=-7.0) - np.nan_to_num(Xa[:, sl], nan=-7.0))
        assert d.max() <= TOLMIX
