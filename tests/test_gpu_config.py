"""Runs set up from configuration files on the device (needs a B200: -m gpu).

Each committed configuration is read by the library's loader; the device
builds the SetUpProblem state (sets, phi, T on the device from the voxel
map, then mu and the explicit site potentials from c0) and evaluates the RHS
there.  The reference's own SetUpProblem state and RHSFunction on the same
file are the fixtures (tests/golden/configs/*.state.npz).  Tolerances as for
the other device tests: grain growth bit-exact in FP64; chemistry
max|dF|/max|F| <= 1e-10 per field (CUDA's exp/log against the host libm).
"""
import glob
import os

import numpy as np
import pytest

import cipher_b200 as cb

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
STATE_CONFIGS = sorted(p for p in glob.glob(os.path.join(HERE, "golden", "configs", "*.yaml"))
                       if not os.path.basename(p).startswith("parse_"))
TOL64 = 1e-10


def _fields(P):
    A = P.aos
    return [(n, o, s) for n, o, s in (("as", A.as_offset, A.as_size), ("pf", A.pf_offset, A.pf_size),
                                      ("dp", A.dp_offset, A.dp_size), ("ex", A.ex_offset, A.ex_size),
                                      ("tm", A.tm_offset, 1)) if s]


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_state_configs_present():
    assert len(STATE_CONFIGS) >= 3


@pytest.mark.parametrize("path", STATE_CONFIGS, ids=[os.path.basename(p) for p in STATE_CONFIGS])
def test_device_setup_and_rhs_match_reference(path):
    cfg = cb.Config.load(path)
    P = cfg.problem
    M = cb.Mesh(P)
    g = np.load(path[:-5] + ".state.npz")
    ctx = cb.Context(P, M, "fp64")
    dX, dF = ctx.alloc_state(), ctx.alloc_state()
    ctx.init_sharp(dX)
    if P.s.ndp:
        ctx.chem_init(dX)
    X0 = ctx.to_aos(dX)
    chem = P.s.ndp > 0
    for name, off, size in _fields(P):
        a, b = X0[:, off:off + size], g["X0"][:, off:off + size]
        if chem and name in ("dp", "ex"):
            assert _rel(a, b) <= TOL64, (name, _rel(a, b))
        else:
            assert np.array_equal(a, b), name
    ctx.from_aos(g["X0"], dX)
    ctx.rhs(0.0, dX, dF)
    ctx.check()
    F = ctx.to_aos(dF)
    for name, off, size in _fields(P):
        if name == "as":
            continue
        a, b = F[:, off:off + size], g["F"][:, off:off + size]
        if chem:
            assert _rel(a, b) <= TOL64, (name, _rel(a, b))
        else:
            assert np.array_equal(a, b), name


ANISO = [p for p in STATE_CONFIGS if os.path.basename(p).startswith("aniso")]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("path", ANISO, ids=[os.path.basename(p) for p in ANISO])
def test_device_anisotropy_matches_reference(path, precision):
    """gradient-based anisotropy on the device (least-squares gradient pass,
    then the general RHS with per-pair normals) on a state evolved by the
    reference: FP64 grain growth bit-exact, chemistry within 1e-10; the
    mixed path (FP32 phi storage) within 1e-6 of the FP64 oracle on the
    FP32-rounded state"""
    import oracle
    cfg = cb.Config.load(path)
    P = cfg.problem
    M = cb.Mesh(P)
    g = np.load(path[:-5] + ".state.npz")
    X = g["X1"]
    A = P.aos
    if precision == "mixed":
        X = X.copy()
        for off, size in ((A.pf_offset, A.pf_size), (A.tm_offset, 1)):
            X[:, off:off + size] = X[:, off:off + size].astype(np.float32).astype(np.float64)
        Fo = oracle.port_rhs(P, M, X)
    else:
        Fo = g["F1"]
    ctx = cb.Context(P, M, precision)
    dX, dF = ctx.alloc_state(), ctx.alloc_state()
    ctx.from_aos(X, dX)
    ctx.rhs(0.0, dX, dF)
    ctx.check()
    F = ctx.to_aos(dF)
    sl = slice(A.pf_offset, A.pf_offset + A.pf_size)
    if precision == "mixed":
        assert _rel(F[:, sl], Fo[:, sl]) <= 1e-6
    elif P.s.ndp:
        for name, off, size in _fields(P):
            if name != "as":
                assert _rel(F[:, off:off + size], Fo[:, off:off + size]) <= TOL64, name
    else:
        assert np.array_equal(F, Fo)


def test_config_runs_through_the_stepper():
    """the grain-growth file stepped with the stepper its petscoptions name
    (3bs) and its tolerances (cap lifted to all phases): finite state with
    valid sets"""
    cfg = cb.Config.load(os.path.join(HERE, "golden", "configs", "gg_small.yaml"))
    P = cfg.problem
    # the file caps sets at 4 phases; its voxel map has all 5 meeting: lift the cap
    cb.load().cipher_problem_set_cap(P.ptr, 5)
    M = cb.Mesh(P)
    ctx = cb.Context(P, M, "fp64")
    dX = ctx.alloc_state()
    ctx.init_sharp(dX)
    ts = cb.TimeStepper(ctx, cfg.ts_options(max_steps=20))
    st = ts.solve(dX, 0.0, P.s.time[0])
    X = ctx.to_aos(dX)
    assert st.steps >= 1 and np.isfinite(X).all()
    n = X[:, 0].astype(int)
    assert n.min() >= 1 and n.max() <= P.s.pf_size
