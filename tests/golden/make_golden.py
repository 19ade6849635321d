"""Generate the golden fixtures from the reference's own code.

Each fixture is a small seeded grain-growth problem built with the library's
host builders; the reference's RHSFunction and PostStep (compiled unmodified
through the PETSc shim into oracle/_ref/libcipher_ref.so) produce the outputs:

  X      state in the reference AoS layout (owned cells)
  F      RHSFunction(X)
  Xpost  PostStep(X) (projection, pruning, neighbour union, reorder)

Run from the repository root where the reference sources exist:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import cipher_b200 as cb  # noqa: E402
import oracle  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# (name, dim, res, ngrains, cap, seed, state kind)
CASES = [
    ("gg2d_sharp", 2, [24, 24], 12, 8, 11, "sharp"),
    ("gg2d_diffuse", 2, [24, 24], 12, 8, 11, "diffuse"),
    ("gg3d_diffuse", 3, [12, 12, 12], 16, 12, 5, "diffuse"),
    ("gg3d_cap15", 3, [10, 10, 10], 30, 15, 3, "diffuse"),
]


def build_case(dim, res, ngrains, cap, seed, kind):
    P = cb.Problem.grain_growth(dim, res, ngrains, cap, seed)
    M = cb.Mesh(P)
    X = cb.initial_state_aos(P, M) if kind == "sharp" else cb.diffuse_state_aos(P, M, 4.0)
    return P, M, X


def main():
    oracle.build(ref=True)
    for name, dim, res, ng, cap, seed, kind in CASES:
        P, M, X = build_case(dim, res, ng, cap, seed, kind)
        with oracle.RefOracle(P, M) as R:
            F = R.rhs(X)
            Xp = X.copy()
            rc = R.poststep(Xp)
            assert rc == 0, rc
        np.savez_compressed(os.path.join(HERE, name + ".npz"), X=X, F=F, Xpost=Xp,
                            meta=np.array([dim] + list(res) + [0] * (3 - len(res)) + [ng, cap, seed,
                                                                                        int(kind == "sharp")]))
        print(name, X.shape, "max|F|", np.abs(F).max())


if __name__ == "__main__":
    main()
