"""The CPU oracle pinned to the reference (CPU only).

* The project's C restatement (oracle/port) must reproduce the reference's own
  RHSFunction / PostStep bit for bit on the committed golden fixtures, which
  the reference code produced (tests/golden/make_golden.py).
* Where the reference build is present (oracle/_ref), the restatement is also
  compared live on fresh states, including states evolved over many steps.
"""
import glob
import os

import numpy as np
import pytest

import cipher_b200 as cb
import oracle

# fixtures on adapted meshes carry a forest description: tests/test_forest.py
GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith(("amr", "nuc_ref", "out_ref")))


MODELS = {0: "quadratic", 1: "calphaddis", 2: "calphad2sl"}


def _case(meta, X_fixture=None):
    """Rebuild a fixture's problem and mesh.  Grain-growth fixtures (8 meta
    entries) and several-interface grain growth (9: + ninterfaces, features)
    also rebuild their state; alloy fixtures (11, or 12 with the
    interpolation) carry theirs."""
    dim = int(meta[0])
    res = [int(v) for v in meta[1:1 + dim]]
    if len(meta) == 8:
        ng, cap, seed, sharp = (int(v) for v in meta[4:8])
        P = cb.Problem.grain_growth(dim, res, ng, cap, seed)
        M = cb.Mesh(P)
        X = cb.initial_state_aos(P, M) if sharp else cb.diffuse_state_aos(P, M, 4.0)
        return P, M, X
    if len(meta) == 9:
        ng, cap, seed, nitf, feats = (int(v) for v in meta[4:9])
        P = cb.Problem.grain_growth_multi(dim, res, ng, cap, seed, nitf, activation=bool(feats & 1),
                                          widths=bool(feats & 2))
        M = cb.Mesh(P)
        return P, M, cb.diffuse_state_aos(P, M, 4.0)
    model, ncp, npr, cap, seed, feats = (int(v) for v in meta[4:10])
    P = cb.Problem.alloy(dim, res, MODELS[model], ncp, npr, cap, seed, feats)
    if len(meta) == 12:
        P.s.interpolation = int(meta[11])
    M = cb.Mesh(P)
    return P, M, X_fixture


def test_golden_fixtures_exist():
    assert len(GOLDEN) >= 11
    assert sum(1 for p in GOLDEN if os.path.basename(p).startswith("alloy")) >= 5
    assert sum(1 for p in GOLDEN if os.path.basename(p).startswith("ggmulti")) >= 2


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_port_matches_reference_golden(path):
    g = np.load(path)
    P, M, X = _case(g["meta"], g["X"])
    # the host builders are deterministic: the same problem (and, for grain
    # growth, the same input state) is rebuilt
    assert P.ndof == g["X"].shape[1]
    assert np.array_equal(X, g["X"])
    F = oracle.port_rhs(P, M, X)
    assert np.array_equal(F, g["F"]), np.abs(F - g["F"]).max()
    Xp = X.copy()
    assert oracle.port_poststep(P, M, Xp) == 0
    assert np.array_equal(Xp, g["Xpost"])


def test_initial_state_matches_port():
    P = cb.Problem.grain_growth(3, [10, 12, 14], 17, 12, 99)
    M = cb.Mesh(P)
    assert np.array_equal(cb.initial_state_aos(P, M), oracle.port_initial_state(P, M))


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) absent")


@needs_ref
@pytest.mark.parametrize("dim,res,ng,cap,seed", [(2, [32, 32], 10, 8, 1234), (3, [12, 12, 12], 12, 12, 4),
                                                  (2, [20, 36], 40, 4, 77)])
def test_port_matches_reference_evolution(dim, res, ng, cap, seed):
    """Forward-Euler trajectory: RHS and PostStep of port and reference agree
    bit for bit at every step (sets and fields)."""
    P = cb.Problem.grain_growth(dim, res, ng, cap, seed)
    M = cb.Mesh(P)
    X = cb.initial_state_aos(P, M)
    dt = 0.05 if dim == 2 else 0.03
    with oracle.RefOracle(P, M) as R:
        for step in range(15):
            Fr = R.rhs(X)
            Fp = oracle.port_rhs(P, M, X)
            assert np.array_equal(Fr, Fp), (step, np.abs(Fr - Fp).max())
            X = X + dt * Fr
            Xr, Xp = X.copy(), X.copy()
            # a superset above the cap aborts the reference (assert at
            # src/cipher.c:968, after SetUnion has overrun its arrays), so the
            # reference only sees states the port accepts
            rp = oracle.port_poststep(P, M, Xp)
            if rp:
                assert rp == 3
                return
            assert R.poststep(Xr) == 0
            assert np.array_equal(Xr, Xp), step
            X = Xr


@needs_ref
def test_slab_with_halo_matches_whole_domain():
    """The halo (ghost-cell) path of the reference's RHS, as an MPI rank sees
    it, reproduces the whole-domain RHS on the owned slab."""
    P = cb.Problem.grain_growth(3, [12, 12, 16], 20, 12, 5)
    Mfull = cb.Mesh(P)
    Xfull = cb.diffuse_state_aos(P, Mfull, 4.0)
    with oracle.RefOracle(P, Mfull) as R:
        Ffull = R.rhs(Xfull)
    Ms = cb.Mesh(P, slab=(4, 9))
    gl = Ms.cell_global()
    Xs = Xfull[gl]
    with oracle.RefOracle(P, Ms) as R:
        Fs = R.rhs(Xs)
    own = gl[:Ms.nowned]
    # halo cells are numbered after the owned ones, so faces to the halo come
    # later in face order than in the whole domain: same terms, another
    # summation order (as between MPI decompositions of the reference)
    scale = np.abs(Ffull).max()
    assert np.abs(Fs - Ffull[own]).max() <= 1e-13 * scale
    Fp = oracle.port_rhs(P, Ms, Xs)
    assert np.array_equal(Fp, Fs)


def test_simplex_projection_properties():
    rng = np.random.default_rng(3)
    for n in range(2, 16):
        for _ in range(20):
            v = rng.normal(0.3, 0.5, n)
            w = oracle.simplex_projection(v)
            assert np.all(w >= 0)
            assert abs(w.sum() - 1.0) < 1e-12
            # idempotent on the simplex
            assert np.allclose(oracle.simplex_projection(w), w, atol=1e-15)


def test_poststep_cap_overflow_detected():
    """A neighbourhood with more phases than the cap is an error, as the
    reference's assert(superset[0] < AS_SIZE) (src/cipher.c:968) makes it."""
    P = cb.Problem.grain_growth(2, [16, 16], 40, 8, 8)
    M = cb.Mesh(P)
    X = cb.initial_state_aos(P, M)
    # give one cell eight surviving phases that its neighbours do not have
    L = P.aos
    c = 5 * 16 + 5
    near = set()
    for nb in (c, c - 1, c + 1, c - 16, c + 16):
        near |= set(X[nb, 1:1 + int(X[nb, 0])].astype(int))
    ids = sorted(set(range(40)) - near)[:8]
    X[c, L.as_offset] = 8
    X[c, L.as_offset + 1:L.as_offset + 9] = ids
    X[c, L.pf_offset:L.pf_offset + 8] = 0.125
    assert oracle.port_poststep(P, M, X) == 3


@needs_ref
@pytest.mark.parametrize("model,feats,dim,res", [
    ("calphad2sl", 0, 2, [20, 16]),
    ("calphaddis", 0xFF, 2, [16, 16]),
    ("quadratic", 0x7F, 3, [8, 8, 8]),
    ("calphad2sl", 0x0B, 3, [8, 10, 6]),
])
def test_port_matches_reference_alloy_evolution(model, feats, dim, res):
    """chemistry, heat, sources, walls: RHS and PostStep bit-exact over steps"""
    P = cb.Problem.alloy(dim, res, model, 4, 5, 8, 31, feats)
    M = cb.Mesh(P)
    A = P.aos
    X = oracle.port_initial_state(P, M)
    with oracle.RefOracle(P, M) as R:
        for _ in range(4):
            F = oracle.port_rhs(P, M, X)
            assert np.array_equal(F, R.rhs(X))
            fphi = np.abs(F[:, A.pf_offset:A.pf_offset + A.pf_size]).max()
            fdp = np.abs(F[:, A.dp_offset:A.dp_offset + A.dp_size]).max()
            mu = np.abs(X[:, A.dp_offset:A.dp_offset + A.dp_size]).max()
            X = X + min(0.05 / max(fphi, 1e-300), 0.02 * mu / max(fdp, 1e-300)) * F
            Xr = X.copy()
            assert oracle.port_poststep(P, M, X) == 0
            assert R.poststep(Xr) == 0
            assert np.array_equal(X, Xr)
