"""Adaptive quadtree / octree meshes (cipher_forest_*), CPU only.

The forest plays the role of the reference's p4est forest.  Its adaptation
follows the reference's marks (refine where a leaf holds more than one
phase, coarsen elsewhere: src/cipher.c:1380-1386), keeps 2:1 balance across
faces, and transfers states as finite volumes (children copy, families
average).  The mesh lists every interior face once, hanging faces included;
on such meshes the CPU restatement must equal the reference's own
RHSFunction and PostStep bit for bit (the reference compiled through the
PETSc shim takes the same explicit face list).
"""
import glob
import os

import numpy as np
import pytest

import cipher_b200 as cb
import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
AMR_GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "amr*.npz")))
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) absent")


def adapted(problem, dim, nblocks, lmin, lmax, iters, state="sharp"):
    """a forest adapted `iters` times from the finest level by the reference's
    marks on the problem's initial state (the reference's initcoarsen loop)"""
    F = cb.Forest(dim, nblocks, lmin, lmax, periodic=tuple(problem.s.periodic[d] for d in range(3)))
    M = F.mesh(problem)
    X = cb.initial_state_aos(problem, M) if state == "sharp" else cb.diffuse_state_aos(problem, M, 4.0)
    for _ in range(iters):
        F.adapt(F.mark_active(X), X, problem.aos.pf_offset)
        X = F.transfer_aos(X)
        M = F.mesh(problem)
    return F, M, X


def _check_forest(F, lmin, lmax, dim):
    lev, cor = F.leaves()
    res = F.resolution()
    assert lev.min() >= lmin and lev.max() <= lmax
    own = -np.ones(res[::-1], dtype=np.int64)           # [z][y][x]
    for i, (l, c) in enumerate(zip(lev, cor)):
        s = 1 << (lmax - l)
        sz = [s if d < dim else 1 for d in range(3)]
        blk = own[c[2]:c[2] + sz[2], c[1]:c[1] + sz[1], c[0]:c[0] + sz[0]]
        assert (blk == -1).all(), "leaves overlap"
        blk[...] = i
    assert (own >= 0).all(), "leaves leave a gap"
    return lev, cor, own


@pytest.mark.parametrize("dim", [2, 3])
def test_adapted_forest_covers_domain_and_is_balanced(dim):
    res = [32, 32] if dim == 2 else [16, 16, 16]
    lmax = 5 if dim == 2 else 4
    P = cb.Problem.grain_growth(dim, res, 6, 8 if dim == 2 else 12, 3)
    F, M, X = adapted(P, dim, [1] * dim, 2, lmax, 3)
    lev, cor, own = _check_forest(F, 2, lmax, dim)
    assert F.nleaves < np.prod(res)                       # something coarsened
    assert len(np.unique(lev)) > 1
    # 2:1 balance: face neighbours differ by at most one level
    fc = np.ctypeslib.as_array(M.s.face_cells, shape=(M.s.nfaces, 2))
    assert np.abs(lev[fc[:, 0]] - lev[fc[:, 1]]).max() <= 1


@pytest.mark.parametrize("dim", [2, 3])
def test_faces_cover_every_leaf_side(dim):
    """each leaf side is covered exactly by its faces: the areas of the faces
    on the +d side (leaf is L) and on the -d side (leaf is R) sum to s^(dim-1)"""
    res = [32, 32] if dim == 2 else [16, 16, 16]
    lmax = 5 if dim == 2 else 4
    P = cb.Problem.grain_growth(dim, res, 6, 8 if dim == 2 else 12, 5)
    F, M, X = adapted(P, dim, [1] * dim, 1, lmax, 3)
    lev, cor = F.leaves()
    side = (1 << (lmax - lev)).astype(np.float64)
    fc = np.ctypeslib.as_array(M.s.face_cells, shape=(M.s.nfaces, 2))
    area = np.minimum(side[fc[:, 0]], side[fc[:, 1]]) ** (dim - 1)
    as_l = np.bincount(fc[:, 0], weights=area, minlength=F.nleaves)
    as_r = np.bincount(fc[:, 1], weights=area, minlength=F.nleaves)
    np.testing.assert_array_equal(as_l, dim * side ** (dim - 1))
    np.testing.assert_array_equal(as_r, dim * side ** (dim - 1))
    geom = np.ctypeslib.as_array(M.s.cellgeom, shape=(F.nleaves,))
    np.testing.assert_array_equal(geom, side)


def test_boundary_faces_and_labels():
    P = cb.Problem.alloy(2, [32, 32], "calphad2sl", 3, 3, 8, 4, cb._lib.ALLOY_WALLS)
    F, M, X = adapted(P, 2, [1, 1], 2, 5, 2)
    lev, cor = F.leaves()
    side = 1 << (5 - lev)
    nb = M.s.nbfaces
    cells = np.ctypeslib.as_array(M.s.bface_cell, shape=(nb,))
    labels = np.ctypeslib.as_array(M.s.bface_label, shape=(nb,))
    assert set(labels) == {1, 2}                          # x walls only (y periodic)
    assert (cor[cells[labels == 1], 0] == 0).all()
    assert (cor[cells[labels == 2], 0] + side[cells[labels == 2]] == 32).all()
    # the wall length is covered exactly
    assert side[cells[labels == 1]].sum() == 32 and side[cells[labels == 2]].sum() == 32


def test_transfer_copies_children_and_averages_families():
    P = cb.Problem.grain_growth(2, [16, 16], 4, 8, 7)
    F = cb.Forest(2, [1, 1], 0, 4)
    M = F.mesh(P)
    X = np.random.default_rng(1).random((F.nleaves, P.ndof))
    X[:, :P.aos.pf_offset] = 0.0                           # one phase everywhere: every family may coarsen
    X[:, 0] = 1.0
    lev0, _ = F.leaves()
    F.adapt(-np.ones(F.nleaves, dtype=np.int8), X, P.aos.pf_offset)
    Y = F.transfer_aos(X)
    s0, ns = F.transfer_plan()
    assert (ns == 4).all() and F.nleaves == 64
    for i in range(F.nleaves):
        np.testing.assert_array_equal(Y[i], X[s0[i]:s0[i] + 4].sum(0) / 4.0)
    # integral conservation of every field
    vol0 = np.ones(256)
    vol1 = np.full(64, 4.0)
    np.testing.assert_allclose(vol1 @ Y[:, 2:], vol0 @ X[:, 2:], rtol=1e-13)
    # refine back: children copy the parent
    F.adapt(np.ones(F.nleaves, dtype=np.int8))
    Z = F.transfer_aos(Y)
    s0, ns = F.transfer_plan()
    assert (ns == 1).all() and F.nleaves == 256
    np.testing.assert_array_equal(Z, Y[s0])


def test_families_with_different_sets_are_kept():
    P = cb.Problem.grain_growth(2, [8, 8], 4, 8, 7)
    F = cb.Forest(2, [1, 1], 0, 3)
    X = np.zeros((F.nleaves, P.ndof))
    X[:, 0] = 1.0
    X[:, 1] = np.arange(F.nleaves) % 2                    # siblings hold different phases
    F.adapt(-np.ones(F.nleaves, dtype=np.int8), X, P.aos.pf_offset)
    assert F.nleaves == 64


@needs_ref
@pytest.mark.parametrize("kind", ["gg2d", "gg3d", "alloy2d_walls"])
def test_port_matches_reference_on_adapted_meshes(kind):
    if kind == "gg2d":
        P = cb.Problem.grain_growth(2, [32, 32], 6, 8, 3)
        F, M, X = adapted(P, 2, [1, 1], 2, 5, 3, "diffuse")
    elif kind == "gg3d":
        P = cb.Problem.grain_growth(3, [16, 16, 16], 8, 12, 4)
        F, M, X = adapted(P, 3, [1, 1, 1], 1, 4, 2, "diffuse")
    else:
        P = cb.Problem.alloy(2, [32, 32], "calphad2sl", 3, 3, 8, 4, cb._lib.ALLOY_WALLS | cb._lib.ALLOY_THERMAL)
        F, M, X = adapted(P, 2, [1, 1], 2, 5, 2)
        X = np.ascontiguousarray(X)
    with oracle.RefOracle(P, M) as R:
        Fr = R.rhs(X)
        Xr = X.copy()
        rr = R.poststep(Xr)
    Fp = oracle.port_rhs(P, M, X)
    Xp = X.copy()
    rp = oracle.port_poststep(P, M, Xp)
    assert np.array_equal(Fp, Fr), np.abs(Fp - Fr).max()
    assert rr == rp == 0
    assert np.array_equal(Xp[:, 0], Xr[:, 0])


def test_amr_fixtures_present():
    assert len(AMR_GOLDEN) >= 2


@pytest.mark.parametrize("path", AMR_GOLDEN, ids=[os.path.basename(p) for p in AMR_GOLDEN])
def test_port_matches_reference_amr_golden(path):
    """the forest rebuilds the fixture's adapted mesh; the CPU restatement
    reproduces the reference's RHS and PostStep on it"""
    from golden.make_golden import build_amr
    g = np.load(path)
    P, F, M = build_amr(*[int(v) for v in g["meta"]])
    assert F.nleaves == g["X"].shape[0]
    lev, cor = F.leaves()
    np.testing.assert_array_equal(lev, g["levels"])
    Fp = oracle.port_rhs(P, M, g["X"])
    assert np.array_equal(Fp, g["F"]), np.abs(Fp - g["F"]).max()
    Xp = g["X"].copy()
    assert oracle.port_poststep(P, M, Xp) == 0
    assert np.array_equal(Xp, g["Xpost"])
