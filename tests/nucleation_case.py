"""A small nucleation scenario shared by the CPU and GPU nucleation tests:
a calphad2sl alloy (two matrix grains, four precipitate phases) with six
3x3 sites and one nucleus of each model."""
import numpy as np

import cipher_b200 as cb
from cipher_b200 import _lib as L


def build(seed: int = 5, sitenucleus=None):
    P = cb.Problem.alloy(2, [32, 24], "calphad2sl", 4, 4, 8, seed, 0x01)
    vox = P.voxelphase()
    res = (32, 24)
    voxelsite = np.full(res[0] * res[1], -1, dtype=np.int32)
    v2 = vox.reshape(res[1], res[0])

    def matrix_only(x0, y0):            # the 3x3 box and its face neighbours hold matrix phases
        ys = [(y0 + k) % res[1] for k in range(-1, 4)]
        xs = [(x0 + k) % res[0] for k in range(-1, 4)]
        return bool(np.all(v2[np.ix_(ys, xs)] <= 1))

    clean = [(x, y) for y in range(1, res[1] - 3, 4) for x in range(1, res[0] - 3, 4) if matrix_only(x, y)]
    dirty = [(x, y) for y in range(1, res[1] - 3, 4) for x in range(1, res[0] - 3, 4)
             if np.any(v2[y:y + 3, x:x + 3] > 1)]
    corners = clean[:5] + dirty[:1]     # five valid sites and one that holds a precipitate
    assert len(corners) == 6, (len(clean), len(dirty))
    for s, (x0, y0) in enumerate(corners):
        for y in range(y0, y0 + 3):
            for x in range(x0, x0 + 3):
                voxelsite[x + res[0] * y] = s
    sitephase = np.array([2, 3, 4, 5, 2, 3], dtype=np.int32)
    sitenucleus = np.array([0, 1, 2, 3, 1, 0] if sitenucleus is None else sitenucleus, dtype=np.int32)
    common = dict(matrix=[0, 1], active_solutes=[1, 1, 1, 0], gamma=0.3, shapefactor=0.5, minsize=1e-3,
                  atomicvolume=1e-5, lengthscale=10.0, incubationtimemin=0.0, liquidus=2000.0)
    nuclei = cb.nuclei_array([
        dict(model=L.NUC_CNT, **common),
        dict(model=L.NUC_CONSTANT, nucleation_rate=1e30, **common),
        dict(common, model=L.NUC_THERMAL, solvus_temperature_0=900.0, enthalpy_fusion_0=4e9, has_solvus_c=1,
             solvus_temperature_c=[50.0, -20.0, 10.0, 0.0]),
        dict(model=L.NUC_CONSTANT, nucleation_rate=0.0, **common),
    ])
    return P, voxelsite, sitephase, sitenucleus, nuclei, vox
