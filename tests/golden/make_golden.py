"""Generate the golden fixtures from the reference's own code.

Each fixture is a small seeded grain-growth or alloy problem built with the
library's host builders; the reference's RHSFunction and PostStep (compiled unmodified
through the PETSc shim into oracle/_ref/libcipher_ref.so) produce the outputs:

  X      state in the reference AoS layout (owned cells)
  F      RHSFunction(X)
  Xpost  PostStep(X) (projection, pruning, neighbour union, reorder)

Run from the repository root where the reference sources exist:
    python tests/golden/make_golden.py [fixture names...]
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


# alloy cases: (name, dim, res, model, ncp, nprecip, cap, seed, features, steps).  The
# state is the SetUpProblem state of the restatement (the reference's init.c
# needs libyaml), then `steps` explicit steps taken with the reference's own
# RHSFunction and PostStep; F and Xpost come from the reference.
ALLOY_CASES = [
    ("alloy2sl_2d", 2, [16, 12], "calphad2sl", 4, 4, 8, 21, 0, 3),
    ("alloydis_all_2d", 2, [16, 12], "calphaddis", 3, 4, 8, 22, 0xFF, 2),
    ("alloyquad_all_3d", 3, [8, 8, 6], "quadratic", 3, 3, 8, 23, 0x7F, 2),
]
MODEL_ID = {"quadratic": 0, "calphaddis": 1, "calphad2sl": 2}

# grain growth with several interfaces (cipher_problem_grain_growth_multi):
# (name, dim, res, ngrains, cap, seed, ninterfaces, features), diffuse state
MULTI_CASES = [
    ("ggmulti2d_act_widths", 2, [24, 24], 12, 8, 11, 5, 0x3),
    ("ggmulti3d_act_cap15", 3, [10, 10, 10], 30, 15, 3, 6, 0x1),
]

# alloy cases with another interpolant: an ALLOY_CASES entry plus the
# interpolation (0 linear, 1 quadratic; the other fixtures are cubic)
ALLOY_INTERP_CASES = [
    ("alloy2sl_linear_2d", 2, [16, 12], "calphad2sl", 4, 4, 8, 21, 0, 3, 0),
    ("alloydis_quadinterp_2d", 2, [16, 12], "calphaddis", 3, 4, 8, 22, 0xFF, 2, 1),
]


def build_alloy(dim, res, model, ncp, nprecip, cap, seed, features):
    P = cb.Problem.alloy(dim, res, model, ncp, nprecip, cap, seed, features)
    M = cb.Mesh(P)
    return P, M


def evolve_with_reference(P, M, R, X, steps):
    """explicit steps with the reference's RHS and PostStep; dt keeps the
    largest phase-fraction change at 0.05 and mu changes at 2 %"""
    A = P.aos
    for _ in range(steps):
        F = R.rhs(X)
        fphi = np.abs(F[:, A.pf_offset:A.pf_offset + A.pf_size]).max()
        fdp = np.abs(F[:, A.dp_offset:A.dp_offset + A.dp_size]).max()
        mu = np.abs(X[:, A.dp_offset:A.dp_offset + A.dp_size]).max()
        dt = min(0.05 / max(fphi, 1e-300), 0.02 * mu / max(fdp, 1e-300))
        X = X + dt * F
        assert R.poststep(X) == 0
    return X


def build_case(dim, res, ngrains, cap, seed, kind):
    P = cb.Problem.grain_growth(dim, res, ngrains, cap, seed)
    M = cb.Mesh(P)
    X = cb.initial_state_aos(P, M) if kind == "sharp" else cb.diffuse_state_aos(P, M, 4.0)
    return P, M, X


def build_multi(dim, res, ng, cap, seed, nitf, feats):
    P = cb.Problem.grain_growth_multi(dim, res, ng, cap, seed, nitf, activation=bool(feats & 1),
                                      widths=bool(feats & 2))
    M = cb.Mesh(P)
    return P, M, cb.diffuse_state_aos(P, M, 4.0)


def main(only=None):
    """regenerate every fixture, or only the named ones"""
    oracle.build(ref=True)

    def wanted(name):
        return not only or name in only

    for name, dim, res, ng, nitf_cap, seed, nitf, feats in MULTI_CASES:
        if not wanted(name):
            continue
        P, M, X = build_multi(dim, res, ng, nitf_cap, seed, nitf, feats)
        with oracle.RefOracle(P, M) as R:
            F = R.rhs(X)
            Xp = X.copy()
            assert R.poststep(Xp) == 0
        meta = [dim] + list(res) + [0] * (3 - len(res)) + [ng, nitf_cap, seed, nitf, feats]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), X=X, F=F, Xpost=Xp, meta=np.array(meta))
        print(name, X.shape, "max|F|", np.abs(F).max(), "mean n", X[:, 0].mean())
    for name, dim, res, model, ncp, npr, cap, seed, feats, steps, interp in ALLOY_INTERP_CASES:
        if not wanted(name):
            continue
        P, M = build_alloy(dim, res, model, ncp, npr, cap, seed, feats)
        P.s.interpolation = interp
        X0 = oracle.port_initial_state(P, M)
        with oracle.RefOracle(P, M) as R:
            X = evolve_with_reference(P, M, R, X0, steps)
            F = R.rhs(X)
            Xp = X.copy()
            assert R.poststep(Xp) == 0
        meta = [dim] + list(res) + [0] * (3 - len(res)) + [MODEL_ID[model], ncp, npr, cap, seed, feats, steps,
                                                            interp]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), X=X, F=F, Xpost=Xp, meta=np.array(meta))
        print(name, X.shape, "max|F|", np.abs(F).max(), "mean n", X[:, 0].mean())
    for name, dim, res, ng, cap, seed, kind in CASES:
        if not wanted(name):
            continue
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
    for name, dim, res, model, ncp, npr, cap, seed, feats, steps in ALLOY_CASES:
        if not wanted(name):
            continue
        P, M = build_alloy(dim, res, model, ncp, npr, cap, seed, feats)
        X0 = oracle.port_initial_state(P, M)
        with oracle.RefOracle(P, M) as R:
            X = evolve_with_reference(P, M, R, X0, steps)
            F = R.rhs(X)
            Xp = X.copy()
            assert R.poststep(Xp) == 0
        meta = [dim] + list(res) + [0] * (3 - len(res)) + [MODEL_ID[model], ncp, npr, cap, seed, feats, steps]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), X=X, F=F, Xpost=Xp, meta=np.array(meta))
        print(name, X.shape, "max|F|", np.abs(F).max(), "mean n", X[:, 0].mean())


if __name__ == "__main__":
    main(sys.argv[1:])
