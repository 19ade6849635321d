"""Host-side builders: Voronoi maps, meshes, initial and diffuse states (CPU)."""
import ctypes as C

import numpy as np

import cipher_b200 as cb
import cipher_b200._lib as L


def test_voronoi_deterministic_and_nearest():
    lib = L.load()
    res = (C.c_int32 * 3)(20, 16, 1)
    a = np.zeros(320, dtype=np.int32)
    b = np.zeros(320, dtype=np.int32)
    cen = np.zeros(9 * 3)
    ip = C.POINTER(C.c_int32)
    assert lib.cipher_voronoi(2, res, 9, 42, a.ctypes.data_as(ip), cen.ctypes.data_as(C.POINTER(C.c_double))) == 0
    assert lib.cipher_voronoi(2, res, 9, 42, b.ctypes.data_as(ip), None) == 0
    assert np.array_equal(a, b)
    # brute-force nearest centre under the periodic metric
    c = cen.reshape(9, 3)[:, :2]
    for idx in range(320):
        p = np.array([idx % 20 + 0.5, idx // 20 + 0.5])
        d = np.abs(c - p)
        d = np.minimum(d, np.array([20, 16]) - d)
        assert a[idx] == int(np.argmin((d ** 2).sum(1)))


def test_uniform_mesh_faces_periodic():
    P = cb.Problem.grain_growth(3, [5, 4, 3], 4, 4, 1)
    M = cb.Mesh(P)
    s = M.s
    assert s.ncells == 60 and s.nowned == 60
    assert s.nfaces == 3 * 60 and s.nbfaces == 0
    f = np.ctypeslib.as_array(s.face_cells, shape=(s.nfaces, 2))
    # faces listed by L cell, then direction
    assert np.all(np.diff(f[:, 0]) >= 0)
    # every cell appears in exactly 2*dim faces
    assert np.all(np.bincount(f.ravel(), minlength=60) == 6)


def test_slab_mesh_has_halo_planes():
    P = cb.Problem.grain_growth(2, [8, 10], 4, 4, 1)
    M = cb.Mesh(P, slab=(3, 6))
    assert M.nowned == 3 * 8
    assert M.ncells == 5 * 8
    gl = M.cell_global()
    assert set(gl[M.nowned:] // 8) == {2, 6}


def test_initial_state_sets_are_own_phase_and_neighbours():
    P = cb.Problem.grain_growth(2, [16, 12], 7, 8, 3)
    M = cb.Mesh(P)
    X = cb.initial_state_aos(P, M)
    vp = P.voxelphase().reshape(12, 16)
    Lay = P.aos
    for c in range(16 * 12):
        y, x = divmod(c, 16)
        want = {vp[y, x], vp[(y + 1) % 12, x], vp[(y - 1) % 12, x], vp[y, (x + 1) % 16], vp[y, (x - 1) % 16]}
        n = int(X[c, 0])
        ids = X[c, 1:1 + n].astype(int)
        assert list(ids) == sorted(want)
        assert X[c, Lay.pf_offset + list(ids).index(vp[y, x])] == 1.0
        assert X[c, Lay.pf_offset:Lay.pf_offset + n].sum() == 1.0


def test_diffuse_state_is_on_simplex_and_within_cap():
    P = cb.Problem.grain_growth(3, [16, 16, 16], 30, 12, 9)
    M = cb.Mesh(P)
    X = cb.diffuse_state_aos(P, M, 4.0)
    Lay = P.aos
    n = X[:, 0].astype(int)
    assert n.min() >= 1 and n.max() <= 12
    phi = X[:, Lay.pf_offset:Lay.pf_offset + 12]
    mask = np.arange(12)[None, :] < n[:, None]
    sums = np.where(mask, phi, 0).sum(1)
    assert np.allclose(sums, 1.0, atol=1e-14)
    assert np.all(phi[mask] >= 0)
    # ids sorted and unique within each set
    for c in range(0, M.ncells, 97):
        ids = X[c, 1:1 + n[c]]
        assert np.all(np.diff(ids) > 0)
