"""Device RHS, PostStep and initial chemistry on alloy problems (needs a B200: -m gpu).

The general kernels (chemistry, heat, boundary faces) evaluate the same IEEE
operations in the reference's order, except that CUDA's exp and log may
differ from the host libm in the last bit.  Tolerances, per field
(phi rates, mu rates, EX rates, T rate), as max|dev - ref| / max|ref|:
    FP64 path   <= 1e-10
    mixed path  <= 1e-6 against the FP64 oracle on the same FP32-rounded
                   phi and T (the mixed layout stores them in FP32)
Active sets and phase fractions after PostStep are bit-exact.

Explicit site-potential slots past a phase's own sublattices are never read
by the model; they are masked out of the EX comparisons.
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
ALLOY_GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "alloy*.npz")))
MODELS = {0: "quadratic", 1: "calphaddis", 2: "calphad2sl"}
TOL64, TOLMIX = 1e-10, 1e-6


def _fixture(path):
    g = np.load(path)
    meta = [int(v) for v in g["meta"]]
    dim = meta[0]
    res = meta[1:1 + dim]
    model, ncp, npr, cap, seed, feats = meta[4:10]
    P = cb.Problem.alloy(dim, res, MODELS[model], ncp, npr, cap, seed, feats)
    if len(meta) == 12:             # fixtures of the linear / quadratic interpolants
        P.s.interpolation = meta[11]
    return P, cb.Mesh(P), g


def _ex_mask(P, X):
    """[ncells, P*SP] True where an EX slot belongs to a sublattice of the
    phase in that slot"""
    A, s = P.aos, P.s
    ndp, SP = s.ndp, A.sp_size
    pmm = np.ctypeslib.as_array(s.phasematerialmapping, shape=(s.npf,))
    nsites = np.array([s.material[m].nsites for m in range(s.nmat)])
    mask = np.zeros((X.shape[0], A.ex_size), dtype=bool)
    n = X[:, 0].astype(int)
    for g in range(A.pf_size):
        live = n > g
        ids = np.where(live, X[:, 1 + g], 0).astype(int)
        ns = nsites[pmm[ids]]
        for q in range(SP):
            mask[:, g * SP + q] = live & (q < ns * ndp)
    return mask


def _field_errors(P, F, Fo, X):
    """per-field relative max-norm errors"""
    A = P.aos
    out = {}
    for name, off, size in (("pf", A.pf_offset, A.pf_size), ("dp", A.dp_offset, A.dp_size),
                            ("tm", A.tm_offset, 1)):
        a, b = F[:, off:off + size], Fo[:, off:off + size]
        out[name] = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300) if size else 0.0
    if A.ex_size:
        m = _ex_mask(P, X)
        a, b = F[:, A.ex_offset:A.ex_offset + A.ex_size][m], Fo[:, A.ex_offset:A.ex_offset + A.ex_size][m]
        out["ex"] = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300) if a.size else 0.0
    return out


def _device_rhs(ctx, X):
    dX, dF = ctx.alloc_state(), ctx.alloc_state()
    ctx.from_aos(X, dX)
    ctx.rhs(0.0, dX, dF)
    ctx.check()
    return ctx.to_aos(dF)


def _round32(P, X):
    """phi and T rounded to FP32, as the mixed layout stores them"""
    A = P.aos
    Y = X.copy()
    for off, size in ((A.pf_offset, A.pf_size), (A.tm_offset, 1)):
        Y[:, off:off + size] = Y[:, off:off + size].astype(np.float32).astype(np.float64)
    return Y


def _evolve_port(P, M, X, steps):
    A = P.aos
    for _ in range(steps):
        F = oracle.port_rhs(P, M, X)
        fphi = np.abs(F[:, A.pf_offset:A.pf_offset + A.pf_size]).max()
        fdp = np.abs(F[:, A.dp_offset:A.dp_offset + A.dp_size]).max()
        mu = np.abs(X[:, A.dp_offset:A.dp_offset + A.dp_size]).max()
        X = X + min(0.05 / max(fphi, 1e-300), 0.02 * mu / max(fdp, 1e-300)) * F
        assert oracle.port_poststep(P, M, X) == 0
    return X


def test_alloy_fixtures_present():
    assert len(ALLOY_GOLDEN) >= 3


@pytest.mark.parametrize("path", ALLOY_GOLDEN, ids=[os.path.basename(p) for p in ALLOY_GOLDEN])
def test_rhs_fp64_matches_reference_fixture(path):
    P, M, g = _fixture(path)
    ctx = cb.Context(P, M, "fp64")
    F = _device_rhs(ctx, g["X"])
    err = _field_errors(P, F, g["F"], g["X"])
    assert max(err.values()) <= TOL64, err


@pytest.mark.parametrize("path", ALLOY_GOLDEN, ids=[os.path.basename(p) for p in ALLOY_GOLDEN])
def test_rhs_mixed_within_tolerance(path):
    P, M, g = _fixture(path)
    X = _round32(P, g["X"])
    Fo = oracle.port_rhs(P, M, X)
    ctx = cb.Context(P, M, "mixed")
    F = _device_rhs(ctx, X)
    err = _field_errors(P, F, Fo, X)
    assert max(err.values()) <= TOLMIX, err


@pytest.mark.parametrize("path", ALLOY_GOLDEN, ids=[os.path.basename(p) for p in ALLOY_GOLDEN])
def test_poststep_matches_reference_fixture(path):
    P, M, g = _fixture(path)
    A = P.aos
    ctx = cb.Context(P, M, "fp64")
    dX = ctx.alloc_state()
    ctx.from_aos(g["X"], dX)
    ctx.poststep(dX)
    Xd = ctx.to_aos(dX)
    Xo = g["Xpost"]
    n = Xo[:, 0].astype(int)
    assert np.array_equal(Xd[:, 0], Xo[:, 0])
    for k in range(A.pf_size):
        live = n > k
        assert np.array_equal(Xd[live, 1 + k], Xo[live, 1 + k])
        assert np.array_equal(Xd[live, A.pf_offset + k], Xo[live, A.pf_offset + k])
    assert np.array_equal(Xd[:, A.dp_offset:A.dp_offset + A.dp_size], Xo[:, A.dp_offset:A.dp_offset + A.dp_size])
    assert np.array_equal(Xd[:, A.tm_offset], Xo[:, A.tm_offset])
    m = _ex_mask(P, Xo)
    a = Xd[:, A.ex_offset:A.ex_offset + A.ex_size][m]
    b = Xo[:, A.ex_offset:A.ex_offset + A.ex_size][m]
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


@pytest.mark.parametrize("model,feats", [("calphad2sl", 0), ("calphaddis", 0xFF), ("quadratic", 0x7F)])
def test_chem_init_matches_port(model, feats):
    P = cb.Problem.alloy(2, [24, 20], model, 4, 6, 8, 7, feats)
    M = cb.Mesh(P)
    A = P.aos
    Xo = oracle.port_initial_state(P, M)
    ctx = cb.Context(P, M, "fp64")
    dX = ctx.alloc_state()
    ctx.from_aos(cb.initial_state_aos(P, M), dX)
    ctx.chem_init(dX)
    ctx.check()
    Xd = ctx.to_aos(dX)
    head = A.dp_offset
    assert np.array_equal(Xd[:, :head], Xo[:, :head])
    assert np.array_equal(Xd[:, A.tm_offset], Xo[:, A.tm_offset])
    for off, size in ((A.dp_offset, A.dp_size), (A.ex_offset, A.ex_size)):
        a, b = Xd[:, off:off + size], Xo[:, off:off + size]
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


LIVE = [
    ("3d_2sl_ncp4_P15", 3, [20, 18, 16], "calphad2sl", 4, 12, 15, 41, 0),
    ("2d_all_mixedmodels", 2, [64, 48], "calphaddis", 4, 16, 12, 42, 0xFF),
    ("3d_quad_all", 3, [12, 12, 12], "quadratic", 3, 6, 8, 43, 0x7F),
    ("2d_dis_ncp5_seg", 2, [40, 40], "calphaddis", 5, 10, 8, 44, 0x03),
]


@pytest.mark.parametrize("case", LIVE, ids=[c[0] for c in LIVE])
def test_rhs_live_vs_port(case):
    _, dim, res, model, ncp, npr, cap, seed, feats = case
    P = cb.Problem.alloy(dim, res, model, ncp, npr, cap, seed, feats)
    M = cb.Mesh(P)
    X = _evolve_port(P, M, oracle.port_initial_state(P, M), 2)
    F64 = _device_rhs(cb.Context(P, M, "fp64"), X)
    err = _field_errors(P, F64, oracle.port_rhs(P, M, X), X)
    assert max(err.values()) <= TOL64, err
    X32 = _round32(P, X)
    Fm = _device_rhs(cb.Context(P, M, "mixed"), X32)
    errm = _field_errors(P, Fm, oracle.port_rhs(P, M, X32), X32)
    assert max(errm.values()) <= TOLMIX, errm


SPECIALISED_CASES = LIVE + [("3d_2sl_ncp5", 3, [16, 14, 12], "calphad2sl", 5, 8, 8, 45, 0x7F),
                            ("2d_quad_ncp2", 2, [36, 30], "quadratic", 2, 8, 8, 46, 0x7F),
                            ("2d_2sl_ncp3_mixedmodels", 2, [40, 36], "calphad2sl", 3, 10, 8, 47, 0xFF)]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("case", SPECIALISED_CASES, ids=[c[0] for c in SPECIALISED_CASES])
def test_specialised_kernels_same_bits(case, prec, monkeypatch):
    """cells evaluated by the kernels compiled for one component count and
    model (single-phase cells; cells of 2 and 3 phases when every material
    shares the model) give the same bits as the general kernels"""
    _, dim, res, model, ncp, npr, cap, seed, feats = case
    P = cb.Problem.alloy(dim, res, model, ncp, npr, cap, seed, feats)
    M = cb.Mesh(P)
    X = _evolve_port(P, M, oracle.port_initial_state(P, M), 2)
    if prec == "mixed":
        X = _round32(P, X)
    assert (X[:, 0] == 1).mean() > 0.3
    monkeypatch.setenv("CIPHER_B200_SPECIALISED_KERNELS", "1")     # at any domain size
    F_single = _device_rhs(cb.Context(P, M, prec), X)
    monkeypatch.setenv("CIPHER_B200_SPECIALISED_KERNELS", "0")
    F_general = _device_rhs(cb.Context(P, M, prec), X)
    assert np.array_equal(F_single, F_general)


@pytest.mark.parametrize("path", ALLOY_GOLDEN, ids=[os.path.basename(p) for p in ALLOY_GOLDEN])
def test_specialised_kernels_same_bits_fixtures(path, monkeypatch):
    P, M, g = _fixture(path)
    monkeypatch.setenv("CIPHER_B200_SPECIALISED_KERNELS", "1")
    F_single = _device_rhs(cb.Context(P, M, "fp64"), g["X"])
    monkeypatch.setenv("CIPHER_B200_SPECIALISED_KERNELS", "0")
    F_general = _device_rhs(cb.Context(P, M, "fp64"), g["X"])
    assert np.array_equal(F_single, F_general)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_item_capacity_overflow_same_bits(prec, monkeypatch):
    """with room for only some items (the rest of the cells of several phases
    evaluated whole, a cell's items straddling the capacity included) and a
    second listing over a different state in the same context (entries of
    the first listing left in the item table), the RHS keeps the general
    kernels' bits"""
    P = cb.Problem.alloy(2, [48, 40], "calphad2sl", 4, 12, 8, 52, 0)
    M = cb.Mesh(P)
    X1 = _evolve_port(P, M, oracle.port_initial_state(P, M), 2)
    X2 = _evolve_port(P, M, X1, 2)
    if prec == "mixed":
        X1, X2 = _round32(P, X1), _round32(P, X2)
    n1 = X1[:, 0].astype(int)
    assert ((n1 >= 2) * n1).sum() > 101
    monkeypatch.setenv("CIPHER_B200_SPECIALISED_KERNELS", "1")
    monkeypatch.setenv("CIPHER_B200_ITEM_CAPACITY", "101")
    ctx = cb.Context(P, M, prec)
    Fs = [_device_rhs(ctx, X) for X in (X2, X1)]
    monkeypatch.setenv("CIPHER_B200_SPECIALISED_KERNELS", "0")
    monkeypatch.delenv("CIPHER_B200_ITEM_CAPACITY")
    ctxg = cb.Context(P, M, prec)
    for X, F in zip((X2, X1), Fs):
        assert np.array_equal(F, _device_rhs(ctxg, X))


def test_trajectory_fp64_vs_port():
    """explicit steps on the device (waxpy + PostStep) against the oracle:
    identical sets at every step, fields within the accumulated tolerance"""
    P = cb.Problem.alloy(2, [32, 24], "calphad2sl", 4, 6, 8, 51, 0x01)
    M = cb.Mesh(P)
    A = P.aos
    X = oracle.port_initial_state(P, M)
    ctx = cb.Context(P, M, "fp64")
    dX, dF = ctx.alloc_state(), ctx.alloc_state()
    ctx.from_aos(X, dX)
    for _ in range(5):
        F = oracle.port_rhs(P, M, X)
        fphi = np.abs(F[:, A.pf_offset:A.pf_offset + A.pf_size]).max()
        fdp = np.abs(F[:, A.dp_offset:A.dp_offset + A.dp_size]).max()
        mu = np.abs(X[:, A.dp_offset:A.dp_offset + A.dp_size]).max()
        dt = min(0.05 / max(fphi, 1e-300), 0.02 * mu / max(fdp, 1e-300))
        X = X + dt * F
        assert oracle.port_poststep(P, M, X) == 0
        ctx.rhs(0.0, dX, dF)
        ctx.waxpy(dX, dX, dt, dF)
        ctx.poststep(dX)
        Xd = ctx.to_aos(dX)
        assert np.array_equal(Xd[:, :1 + A.pf_size][:, 0], X[:, 0])
        n = X[:, 0].astype(int)
        for k in range(A.pf_size):
            live = n > k
            assert np.array_equal(Xd[live, 1 + k], X[live, 1 + k])
        for off, size in ((A.pf_offset, A.pf_size), (A.dp_offset, A.dp_size)):
            a, b = Xd[:, off:off + size], X[:, off:off + size]
            assert np.abs(a - b).max() <= 1e-9 * max(np.abs(b).max(), 1.0)


def test_unsupported_configurations_rejected():
    P = cb.Problem.alloy(2, [8, 8], "calphad2sl", 3, 2, 4, 1, 0)
    M = cb.Mesh(P)
    # gradient-based anisotropy runs on whole-domain uniform grids only
    P.s.gradient_calculation = 1
    P.s.interface[0].energy_naniso = 1
    P.s.interface[0].energy_aniso_val[0] = 0.1
    P.s.interface[0].energy_aniso_dir[0] = 1.0
    Mf = cb.Forest(2, [1, 1], 2, 3).mesh(P)
    with pytest.raises(L.CipherError) as e:
        cb.Context(P, Mf, "fp64")
    assert e.value.code == L.E_UNSUPPORTED
    P.s.gradient_calculation = 0
    P.s.material[1].nsources = 1
    P.s.material[1].sources[0].model = L.SOURCE_RANDOM
    with pytest.raises(L.CipherError) as e:
        cb.Context(P, M, "fp64")
    assert e.value.code == L.E_UNSUPPORTED


@pytest.mark.parametrize("kind", ["gg2d", "gg3d", "alloy"])
def test_device_initial_state_matches_host(kind):
    """cipher_state_init_sharp (device, from the voxel map) equals the host
    SetUpProblem state converted to the device, chemistry included"""
    if kind == "gg2d":
        P = cb.Problem.grain_growth(2, [40, 32], 12, 8, 3)
    elif kind == "gg3d":
        P = cb.Problem.grain_growth(3, [12, 14, 10], 20, 12, 4)
    else:
        P = cb.Problem.alloy(2, [24, 20], "calphad2sl", 4, 6, 8, 7, 0xFF)
    M = cb.Mesh(P)
    ctx = cb.Context(P, M, "fp64")
    Xh = ctx.alloc_state()
    ctx.from_aos(cb.initial_state_aos(P, M), Xh)
    ctx.chem_init(Xh)
    Mg = cb.Mesh(P, grid_only=True)
    ctxg = cb.Context(P, Mg, "fp64")
    Xd = ctxg.alloc_state()
    ctxg.init_sharp(Xd)
    assert np.array_equal(ctx.to_aos(Xh), ctxg.to_aos(Xd))
    # and the same RHS (face maps included)
    Fh, Fd = ctx.alloc_state(), ctxg.alloc_state()
    ctx.rhs(0.0, Xh, Fh)
    ctxg.rhs(0.0, Xd, Fd)
    assert np.array_equal(ctx.to_aos(Fh), ctxg.to_aos(Fd))
