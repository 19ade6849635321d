"""The device RHS, PostStep and state transfer on adapted meshes (needs a
B200: -m gpu).

A context built over a forest's mesh takes the general kernels with per-cell
face lists (conforming and hanging faces in the mesh's face order, each face
with the reference's face factor from the two cell sizes, src/cipher.c:
273-275).  Tolerances as for uniform grids: grain growth (no transcendental
functions on its path) bit-exact in FP64; chemistry max|dF|/max|F| <= 1e-10
per field in FP64 (CUDA's exp/log against the host libm); mixed <= 1e-6
against the FP64 oracle on FP32-rounded input.  The reference fixtures were
made by the reference's own RHSFunction/PostStep on the same adapted meshes.
"""
import glob
import os

import numpy as np
import pytest

import cipher_b200 as cb
import oracle

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
AMR_GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "amr*.npz")))
TOL64, TOLMIX = 1e-10, 1e-6


def _fixture(path):
    from golden.make_golden import build_amr
    g = np.load(path)
    meta = [int(v) for v in g["meta"]]
    P, F, M = build_amr(*meta)
    return P, F, M, g, meta[0]


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


def _field_errors(P, F, Fo):
    A = P.aos
    out = {}
    for name, off, size in (("pf", A.pf_offset, A.pf_size), ("dp", A.dp_offset, A.dp_size), ("tm", A.tm_offset, 1)):
        if size:
            a, b = F[:, off:off + size], Fo[:, off:off + size]
            out[name] = float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    return out


def test_amr_fixtures_present():
    assert len(AMR_GOLDEN) >= 3


@pytest.mark.parametrize("path", AMR_GOLDEN, ids=[os.path.basename(p) for p in AMR_GOLDEN])
def test_rhs_fp64_on_adapted_mesh(path):
    P, F, M, g, kind = _fixture(path)
    assert M.s.uniform == 0
    ctx = cb.Context(P, M, "fp64")
    Fd = _device_rhs(ctx, g["X"])
    if kind == 0:
        assert np.array_equal(Fd, g["F"]), np.abs(Fd - g["F"]).max()
    else:
        err = _field_errors(P, Fd, g["F"])
        assert max(err.values()) <= TOL64, err


@pytest.mark.parametrize("path", AMR_GOLDEN, ids=[os.path.basename(p) for p in AMR_GOLDEN])
def test_rhs_mixed_on_adapted_mesh(path):
    P, F, M, g, kind = _fixture(path)
    X32 = _round32(P, g["X"])
    ctx = cb.Context(P, M, "mixed")
    Fd = _device_rhs(ctx, X32)
    Fo = oracle.port_rhs(P, M, X32)
    err = _field_errors(P, Fd, Fo)
    assert err["pf"] <= TOLMIX, err


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("path", AMR_GOLDEN, ids=[os.path.basename(p) for p in AMR_GOLDEN])
def test_specialised_kernels_same_bits_on_adapted_mesh(path, prec, monkeypatch):
    """on face lists (hanging faces included) the single-phase and item
    kernels give the general kernels' bits"""
    P, F, M, g, kind = _fixture(path)
    X = g["X"] if prec == "fp64" else _round32(P, g["X"])
    monkeypatch.setenv("CIPHER_B200_SPECIALISED_KERNELS", "1")
    Fs = _device_rhs(cb.Context(P, M, prec), X)
    monkeypatch.setenv("CIPHER_B200_SPECIALISED_KERNELS", "0")
    assert np.array_equal(Fs, _device_rhs(cb.Context(P, M, prec), X))


@pytest.mark.parametrize("path", AMR_GOLDEN, ids=[os.path.basename(p) for p in AMR_GOLDEN])
def test_poststep_on_adapted_mesh(path):
    P, F, M, g, kind = _fixture(path)
    ctx = cb.Context(P, M, "fp64")
    dX = ctx.alloc_state()
    ctx.from_aos(g["X"], dX)
    ctx.poststep(dX)
    Xd = ctx.to_aos(dX)
    Xo = g["Xpost"]
    A = P.aos
    n = Xo[:, 0].astype(int)
    assert np.array_equal(Xd[:, 0], Xo[:, 0])
    for k in range(A.pf_size):
        m = n > k
        assert np.array_equal(Xd[m, 1 + k], Xo[m, 1 + k])
        assert np.array_equal(Xd[m, A.pf_offset + k], Xo[m, A.pf_offset + k])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_transfer_equals_host_transfer(precision):
    """after an adaptation the state moves to the new mesh on the device;
    the result equals the forest's host transfer (FP64: bit for bit)"""
    P = cb.Problem.grain_growth(2, [32, 32], 6, 8, 3)
    F = cb.Forest(2, [1, 1], 2, 5)
    M0 = F.mesh(P)
    X0 = cb.diffuse_state_aos(P, M0, 4.0)
    if precision == "mixed":
        X0 = _round32(P, X0)
    c0 = cb.Context(P, M0, precision)
    d0 = c0.alloc_state()
    c0.from_aos(X0, d0)
    F.adapt(F.mark_active(X0), X0, P.aos.pf_offset)
    M1 = F.mesh(P)
    c1 = cb.Context(P, M1, precision)
    d1 = c1.alloc_state()
    c1.transfer_from(d1, c0, d0, F)
    Xd = c1.to_aos(d1)
    Xh = F.transfer_aos(X0)
    A = P.aos
    n = Xh[:, 0].astype(int)
    assert np.array_equal(Xd[:, 0], Xh[:, 0])
    tol = 0.0 if precision == "fp64" else 1e-7
    for k in range(A.pf_size):
        m = n > k
        assert np.array_equal(Xd[m, 1 + k], Xh[m, 1 + k])
        assert np.abs(Xd[m, A.pf_offset + k] - Xh[m, A.pf_offset + k]).max(initial=0.0) <= tol


def test_adapt_loop_matches_cpu_restatement():
    """forward-Euler steps with PostStep, adapting every 3 steps by the
    reference's marks and moving the state on the device, equal the same loop
    run with the CPU restatement and the host transfer (FP64, bit for bit)"""
    P = cb.Problem.grain_growth(2, [32, 32], 6, 8, 9)
    F = cb.Forest(2, [1, 1], 2, 5)
    M = F.mesh(P)
    X = cb.diffuse_state_aos(P, M, 4.0)
    Xo = X.copy()
    ctx = cb.Context(P, M, "fp64")
    dX, dF = ctx.alloc_state(), ctx.alloc_state()
    ctx.from_aos(X, dX)
    dt = 0.05
    for step in range(1, 13):
        ctx.rhs(0.0, dX, dF)
        ctx.waxpy(dX, dX, dt, dF)
        ctx.poststep(dX)
        Xo = Xo + dt * oracle.port_rhs(P, M, Xo)
        assert oracle.port_poststep(P, M, Xo) == 0
        if step % 3 == 0:
            Xh = ctx.to_aos(dX)
            assert np.array_equal(Xh[:, 0], Xo[:, 0])
            F.adapt(F.mark_active(Xo), Xo, P.aos.pf_offset)
            M = F.mesh(P)
            c1 = cb.Context(P, M, "fp64")
            d1, f1 = c1.alloc_state(), c1.alloc_state()
            c1.transfer_from(d1, ctx, dX, F)
            Xo = F.transfer_aos(Xo)
            ctx, dX, dF = c1, d1, f1
    Xd = ctx.to_aos(dX)
    A = P.aos
    n = Xo[:, 0].astype(int)
    assert np.array_equal(Xd[:, 0], Xo[:, 0])
    for k in range(A.pf_size):
        m = n > k
        assert np.array_equal(Xd[m, 1 + k], Xo[m, 1 + k])
        assert np.array_equal(Xd[m, A.pf_offset + k], Xo[m, A.pf_offset + k])


def _cpu_amr_loop(P, nblocks, lmin, lmax, initcoarsen, interval, opts, t_end):
    """the same loop with the CPU restatement of the stepper and the host
    forest: initial coarsening, then `interval` accepted steps between
    adaptations, the step size carried over"""
    from cipher_b200 import _lib as L
    F = cb.Forest(P.s.dim, nblocks, lmin, lmax, periodic=tuple(P.s.periodic[d] for d in range(3)))
    M = F.mesh(P)
    X = cb.initial_state_aos(P, M)
    for _ in range(initcoarsen):
        F.adapt(F.mark_active(X), X, P.aos.pf_offset)
        X = F.transfer_aos(X)
        M = F.mesh(P)
    X = np.ascontiguousarray(X)
    t, steps, dt, nad = 0.0, 0, None, 0
    while t < t_end:
        o = L.TSOpts.from_buffer_copy(opts)
        o.max_steps = interval
        if dt is not None:
            o.dt0 = dt
        ts = oracle.PortTS(P, M, o)
        st = ts.solve(X, t, t_end, L.TSStats())
        t, dt = st.t, st.dt
        steps += st.steps
        ts.close()
        if t < t_end and st.steps >= interval:
            A = P.aos
            sets = X[:, :A.pf_offset].copy()
            n = sets[:, 0].astype(int)
            for k in range(1, A.pf_offset):
                sets[n < k, k] = 0.0
            F.adapt(F.mark_active(sets), sets, A.pf_offset)
            X = np.ascontiguousarray(F.transfer_aos(X))
            M = F.mesh(P)
            nad += 1
    return X, steps, nad, F


def test_amr_driver_matches_cpu_restatement():
    """the device AMR loop (cipher_amr_*) equals the same loop run with the
    CPU restatement of the stepper and the host forest, bit for bit (FP64,
    grain growth: the same steps, adaptations and final state)"""
    P = cb.Problem.grain_growth(2, [32, 32], 6, 8, 9)
    o = cb.ts_options(P, "2a", dt0=1e-3, dtmin=1e-9, dtmax=1.0, reltol=1e-4, abstol=1e-4)
    amr = cb.AMR(P, [1, 1], 2, 5, 3, 4, o, "fp64")
    st = amr.solve(0.6)
    _, _, m, nad = amr.state()
    Xd = amr.state_aos()
    Xo, steps, nad_o, F = _cpu_amr_loop(P, [1, 1], 2, 5, 3, 4, o, 0.6)
    assert st.steps == steps and nad == nad_o and nad >= 2
    assert Xd.shape == Xo.shape
    A = P.aos
    n = Xo[:, 0].astype(int)
    assert np.array_equal(Xd[:, 0], Xo[:, 0])
    for k in range(A.pf_size):
        msk = n > k
        assert np.array_equal(Xd[msk, 1 + k], Xo[msk, 1 + k])
        assert np.array_equal(Xd[msk, A.pf_offset + k], Xo[msk, A.pf_offset + k])


def test_amr_driver_alloy_runs_and_adapts():
    """a chemistry problem (calphad2sl, walls) through the AMR driver: the
    initial coarsening leaves fewer leaves than voxels, adaptations happen,
    and the state stays finite with valid sets"""
    P = cb.Problem.alloy(2, [64, 64], "calphad2sl", 3, 4, 8, 5, cb._lib.ALLOY_WALLS)
    o = cb.ts_options(P, "2a", dt0=1e-6, dtmin=1e-12, dtmax=1e-2, reltol=1e-3, abstol=1e-3)
    amr = cb.AMR(P, [1, 1], 3, 6, 3, 5, o, "fp64")
    _, _, m0, _ = amr.state()
    n0 = int(m0.ncells)
    assert n0 < 64 * 64
    st = amr.solve(1.0, max_steps=15)
    _, _, m, nad = amr.state()
    X = amr.state_aos()
    assert st.steps == 15 and nad >= 2
    assert np.isfinite(X).all()
    n = X[:, 0].astype(int)
    assert n.min() >= 1 and n.max() <= P.s.pf_size
