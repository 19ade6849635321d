"""Device RHS and PostStep against the oracle (needs a B200: -m gpu).

FP64 path: bit-identical to the reference (fields and sets), because the
kernel keeps the reference's operation order including the face-flux
summation order and compiles without multiply-add contraction.

Mixed path (FP32 phase-field storage and stencil): per-field error against
the FP64 oracle on the same (FP32-representable) input state,
    max|F_mixed - F_64| / max|F_64| <= 1e-6,
and bit-exact phase sets after PostStep.
"""
import numpy as np
import pytest

import cipher_b200 as cb
import oracle

pytestmark = pytest.mark.gpu

CASES = [
    ("2d_sharp_P8", 2, [32, 32], 10, 8, 1234, "sharp"),
    ("2d_diffuse_P4", 2, [40, 24], 6, 4, 5, "diffuse"),
    ("2d_diffuse_P8", 2, [64, 48], 30, 8, 9, "diffuse"),
    ("3d_diffuse_P12", 3, [16, 16, 16], 30, 12, 3, "diffuse"),
    ("3d_diffuse_P15", 3, [12, 14, 10], 40, 15, 21, "diffuse"),
    ("3d_sharp_P6", 3, [8, 9, 10], 12, 6, 2, "sharp"),
]


def _build(dim, res, ng, cap, seed, kind):
    P = cb.Problem.grain_growth(dim, res, ng, cap, seed)
    M = cb.Mesh(P)
    X = cb.initial_state_aos(P, M) if kind == "sharp" else cb.diffuse_state_aos(P, M, 4.0)
    return P, M, X


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


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_rhs_fp64_bit_exact(case):
    P, M, X = _build(*case[1:])
    ctx = cb.Context(P, M, "fp64")
    F = _device_rhs(ctx, X)
    Fo = _oracle_rhs(P, M, X)
    assert np.array_equal(F, Fo), np.abs(F - Fo).max()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_poststep_fp64_bit_exact(case):
    P, M, X = _build(*case[1:])
    ctx = cb.Context(P, M, "fp64")
    dX = ctx.alloc_state()
    ctx.from_aos(X, dX)
    ctx.poststep(dX)
    Xd = ctx.to_aos(dX)
    Xo = X.copy()
    assert oracle.port_poststep(P, M, Xo) == 0
    # compare the defined part: AS count + ids, phi of active slots
    L = P.aos
    n = Xo[:, 0].astype(int)
    assert np.array_equal(Xd[:, 0], Xo[:, 0])
    for g in range(P.s.pf_size):
        m = n > g
        assert np.array_equal(Xd[m, 1 + g], Xo[m, 1 + g])
        assert np.array_equal(Xd[m, L.pf_offset + g], Xo[m, L.pf_offset + g])


def test_trajectory_fp64_bit_exact():
    """20 forward-Euler steps (device AXPY + RHS + PostStep) stay bit-identical
    to the oracle driven the same way."""
    P, M, X = _build(3, [20, 18, 16], 12, 12, 17, "sharp")
    ctx = cb.Context(P, M, "fp64")
    dX, dF = ctx.alloc_state(), ctx.alloc_state()
    ctx.from_aos(X, dX)
    dt = 0.03
    Xo = X.copy()
    for step in range(20):
        ctx.rhs(0.0, dX, dF)
        ctx.waxpy(dX, dX, dt, dF)
        Fo = oracle.port_rhs(P, M, Xo)
        Xo = Xo + dt * Fo
        rc = oracle.port_poststep(P, M, Xo)
        if rc:
            # a cap overflow must be reported by the device at the same step
            with pytest.raises(cb.CipherError) as e:
                ctx.poststep(dX)
            assert e.value.code == 3 and rc == 3
            return
        ctx.poststep(dX)
    Xd = ctx.to_aos(dX)
    n = Xo[:, 0].astype(int)
    assert np.array_equal(Xd[:, 0], Xo[:, 0])
    L = P.aos
    for g in range(P.s.pf_size):
        m = n > g
        assert np.array_equal(Xd[m, 1 + g], Xo[m, 1 + g])
        assert np.array_equal(Xd[m, L.pf_offset + g], Xo[m, L.pf_offset + g])


@pytest.mark.parametrize("case", CASES[1:5], ids=[c[0] for c in CASES[1:5]])
def test_rhs_mixed_within_1e6(case):
    P, M, X = _build(*case[1:])
    L = P.aos
    # the mixed path stores phi and T in FP32: feed both paths the same values
    X32 = X.copy()
    X32[:, L.pf_offset:L.pf_offset + P.s.pf_size] = X32[:, L.pf_offset:L.pf_offset + P.s.pf_size].astype(np.float32)
    X32[:, L.tm_offset] = X32[:, L.tm_offset].astype(np.float32)
    ctx = cb.Context(P, M, "mixed")
    F = _device_rhs(ctx, X32)
    Fo = _oracle_rhs(P, M, X32)
    sl = slice(L.pf_offset, L.pf_offset + P.s.pf_size)
    err = np.abs(F[:, sl] - Fo[:, sl]).max() / np.abs(Fo[:, sl]).max()
    assert err <= 1e-6, err


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("res,periodic_z", [([12, 12, 12], 1), ([12, 12, 12], 0), ([16, 8, 5], 1), ([10, 6, 3], 1)])
def test_rhs_host_aos_entry_point_matches_device_path(precision, res, periodic_z):
    """the host-buffer call (3D grids of 4 or more planes run as a z-slab
    pipeline; fewer planes take one pass) equals the device-buffer call bit
    for bit, on repeated calls"""
    P = cb.Problem.grain_growth(3, res, 20, 12, 8)
    P.s.periodic[2] = periodic_z
    M = cb.Mesh(P)
    X = cb.diffuse_state_aos(P, M, 4.0)
    if precision == "mixed":
        L = P.aos
        X[:, L.pf_offset:L.pf_offset + P.s.pf_size] = X[:, L.pf_offset:L.pf_offset + P.s.pf_size].astype(np.float32)
        X[:, L.tm_offset] = X[:, L.tm_offset].astype(np.float32)
    ctx = cb.Context(P, M, precision)
    F2 = _device_rhs(ctx, X)
    for _ in range(2):
        F1 = ctx.rhs_aos_host(0.0, X)
        assert np.array_equal(F1, F2)


def test_bad_active_count_is_reported_not_trapped():
    P, M, X = _build(2, [16, 16], 6, 4, 1, "sharp")
    X[7, 0] = 9          # n > P
    ctx = cb.Context(P, M, "fp64")
    dX, dF = ctx.alloc_state(), ctx.alloc_state()
    ctx.from_aos(X, dX)
    ctx.rhs(0.0, dX, dF)
    with pytest.raises(cb.CipherError) as e:
        ctx.check()
    assert e.value.code == 1
    ctx.check()          # flags were cleared


def test_cap_overflow_is_reported():
    P, M, X = _build(2, [16, 16], 40, 8, 8, "sharp")
    L = P.aos
    c = 5 * 16 + 5
    near = set()
    for nb in (c, c - 1, c + 1, c - 16, c + 16):
        near |= set(X[nb, 1:1 + int(X[nb, 0])].astype(int))
    ids = sorted(set(range(40)) - near)[:8]
    X[c, L.as_offset] = 8
    X[c, L.as_offset + 1:L.as_offset + 9] = ids
    X[c, L.pf_offset:L.pf_offset + 8] = 0.125
    ctx = cb.Context(P, M, "fp64")
    dX = ctx.alloc_state()
    ctx.from_aos(X, dX)
    with pytest.raises(cb.CipherError) as e:
        ctx.poststep(dX)
    assert e.value.code == 3


def test_full_size_config_properties():
    """128^3, 2000 grains, P = 12 (the 3D benchmark configuration): per-cell
    sum of dphi/dt is zero, single-phase cells have zero rate, and a strided
    sample of cells matches the oracle bit for bit."""
    P = cb.Problem.grain_growth(3, [128, 128, 128], 2000, 12, 12345)
    M = cb.Mesh(P)
    X = cb.diffuse_state_aos(P, M, 4.0)
    ctx = cb.Context(P, M, "fp64")
    F = _device_rhs(ctx, X)
    L = P.aos
    n = X[:, 0].astype(int)
    phi_rate = F[:, L.pf_offset:L.pf_offset + 12]
    scale = np.abs(phi_rate).max()
    assert scale > 0
    assert np.abs(phi_rate.sum(1)).max() <= 1e-12 * scale
    assert np.all(phi_rate[n == 1] == 0)
    Fo = oracle.port_rhs(P, M, X)
    assert np.array_equal(F, Fo)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_rhs_fp64_closed_form_within_1e10(case):
    """the closed-form single-interface kernel on an FP64 state: the pair and
    triple sums of the reference summed in another order, so equal to the
    reference within FP64 rounding: max|dF|/max|F| <= 1e-10"""
    P, M, X = _build(*case[1:])
    ctx = cb.Context(P, M, "fp64")
    ctx.set_rhs_form("closed")
    F = _device_rhs(ctx, X)
    Fo = _oracle_rhs(P, M, X)
    L = P.aos
    sl = slice(L.pf_offset, L.pf_offset + P.s.pf_size)
    err = np.abs(F[:, sl] - Fo[:, sl]).max() / np.abs(Fo[:, sl]).max()
    assert err <= 1e-10, err
    assert np.array_equal(F[:, L.tm_offset], Fo[:, L.tm_offset])
