"""Generate the golden fixtures from the reference's own code.

Each fixture is a small seeded grain-growth or alloy problem built with the
library's host builders; the reference's RHSFunction and PostStep (compiled unmodified
through the PETSc shim into oracle/_ref/libcipher_ref.so) produce the outputs:

  X      state in the reference AoS layout (owned cells)
  F      RHSFunction(X)
  Xpost  PostStep(X) (projection, pruning, neighbour union, reorder)

Two more kinds pin the parts of PostStep around the active-set update:

  nuc_ref.npz        the reference's per-site nucleation averages
                     (NucleationBarrier, src/material.c:137-290, summed as
                     src/cipher.c:733-815) and its event decisions
                     (NucleationEvent, src/material.c:47-135) for seeded
                     draws of the C library's generator
  out_ref_*.npz      the fields of the reference's output step
                     (src/cipher.c:976-1081) after its PostStep
  configs/*.ref.npz  the reference's SetUpConfig (src/init.c:104-1716) on
                     the configuration files configs/*.yaml (YAML events from
                     PyYAML, see oracle/config_dump.py)
  configs/*.state.npz its SetUpProblem state (src/init.c:1721-1830) and
                     RHSFunction there (not for parse_* files, whose random
                     sources the reference draws with rand()); aniso_* files
                     also hold a state evolved by 3 reference steps (X1, F1)

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


# adapted meshes: (name, kind, dim, res, a, ncp, nprecip, cap, seed, features,
# lmin, lmax, adapt iterations, diffuse start, reference steps).  kind 0:
# grain growth with a = ngrains; kind 1: alloy with a = model id.  The forest
# starts at the finest level (res), the state is adapted `iterations` times
# by the reference's marks (the initcoarsen loop of src/cipher.c:1365), then
# evolved by `steps` explicit reference steps on the adapted mesh.
AMR_CASES = [
    ("amr2d_gg_diffuse", 0, 2, [32, 32], 6, 1, 0, 8, 3, 0, 2, 5, 3, 1, 0),
    ("amr3d_gg_sharp", 0, 3, [16, 16, 16], 4, 1, 0, 12, 4, 0, 1, 4, 2, 0, 0),
    ("amr2d_alloy2sl_walls", 1, 2, [32, 32], 2, 3, 3, 8, 4, 0x28, 2, 5, 2, 0, 2),
]


def build_amr(kind, dim, r0, r1, r2, a, ncp, npr, cap, seed, feats, lmin, lmax, iters, diffuse, steps=0):
    """the problem, forest and mesh of an adapted-mesh case (the forest is
    rebuilt deterministically from the problem's initial state)"""
    res = [r0, r1, r2][:dim]
    if kind == 0:
        P = cb.Problem.grain_growth(dim, res, a, cap, seed)
    else:
        P = cb.Problem.alloy(dim, res, {0: "quadratic", 1: "calphaddis", 2: "calphad2sl"}[a], ncp, npr, cap, seed,
                             feats)
    nb = [r // (1 << lmax) for r in res]
    F = cb.Forest(dim, nb, lmin, lmax, periodic=tuple(P.s.periodic[d] for d in range(3)))
    M = F.mesh(P)
    if kind == 0:
        X = cb.diffuse_state_aos(P, M, 4.0) if diffuse else cb.initial_state_aos(P, M)
    else:
        X = oracle.port_initial_state(P, M)
    for _ in range(iters):
        F.adapt(F.mark_active(X), X, P.aos.pf_offset)
        X = F.transfer_aos(X)
        M = F.mesh(P)
    build_amr.state = X
    return P, F, M


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
        dt = 0.05 / max(fphi, 1e-300)
        if A.dp_size:
            fdp = np.abs(F[:, A.dp_offset:A.dp_offset + A.dp_size]).max()
            mu = np.abs(X[:, A.dp_offset:A.dp_offset + A.dp_size]).max()
            dt = min(dt, 0.02 * mu / max(fdp, 1e-300))
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


# nucleation fixture: the shared nucleation scenario with a CNT nucleus on
# the two-phase site 3 and a thermal one on site 4, evolved by the
# reference's own steps, with a temperature field that varies by cell
NUC_SITENUCLEUS = [0, 1, 2, 0, 2, 3]
NUC_STEPS = 4
NUC_SEEDS = 48

# output fixtures: (name, builder kind, args, steps, field names, component names)
OUT_CASES = [
    ("out_ref_alloy2d", "alloy", (2, [40, 32], "calphad2sl", 4, 6, 8, 9, 0x01), 3,
     ["phaseid", "matid", "interfaceid", "al_chempot", "cu_chempot", "va_chempot", "al_c", "cu_c", "mg_c", "va_c",
      "2_phi", "0_phi", "7_phi", "temperature"], ["al", "cu", "mg", "va"]),
    ("out_ref_gg3d", "gg", (3, [12, 10, 8], 20, 8, 4), 0,
     ["phaseid", "matid", "interfaceid", "3_phi", "11_phi", "temperature"], []),
]


def nucleation_fixture():
    """the reference's nucleation averages on an evolved state, and its
    event decisions at a step size that puts each site's threshold near one
    half, for seeds 1..NUC_SEEDS"""
    sys.path.insert(0, os.path.dirname(HERE))
    from nucleation_case import build
    P, voxelsite, sitephase, sitenucleus, nuclei, vox = build(sitenucleus=NUC_SITENUCLEUS)
    M = cb.Mesh(P)
    A = P.aos
    X0 = oracle.port_initial_state(P, M)
    with oracle.RefOracle(P, M, nucleation=(sitephase, sitenucleus, nuclei)) as R:
        X = evolve_with_reference(P, M, R, X0, NUC_STEPS)
        x = np.arange(M.nowned) % P.s.resolution[0]
        X[:, A.tm_offset] = 690.0 + 0.75 * x
        sites, active = R.nucleation_sites(X, voxelsite)
        rows = []
        for s in range(len(sitephase)):
            if not active[s]:
                continue
            gv, diff, T, vol = sites[s]
            nz = nuclei[sitenucleus[s]]
            draws, thr1 = oracle.port_nucleation_threshold(nz, P.s.dim, 1.0, 1.0, T, vol, gv, diff)
            dt = 0.5 / thr1 if draws and thr1 > 0 else 1e-3
            for seed in range(1, NUC_SEEDS + 1):
                fired, u = R.nucleation_event(s, 1.0, dt, T, vol, gv, diff, seed)
                rows.append([s, 1.0, dt, seed, u, float(fired)])
    np.savez_compressed(os.path.join(HERE, "nuc_ref.npz"), X=X, sites=sites, active=active,
                        events=np.array(rows), sitenucleus=np.array(NUC_SITENUCLEUS))
    n = X[:, 0].astype(int)
    print("nuc_ref", X.shape, "active", active, "two-phase cells in sites",
          int(((voxelsite >= 0) & (n > 1)).sum()), "fired", int(np.array(rows)[:, 5].sum()), "of", len(rows))


def output_case(kind, args):
    if kind == "alloy":
        P, M = build_alloy(*args)
    else:
        dim, res, ng, cap, seed = args
        P = cb.Problem.grain_growth(dim, res, ng, cap, seed)
        M = cb.Mesh(P)
    return P, M


def output_fixture(name, kind, args, steps, names, comps):
    """the reference's PostStep with its output step on an evolved state"""
    P, M = output_case(kind, args)
    with oracle.RefOracle(P, M) as R:
        X0 = oracle.port_initial_state(P, M) if kind == "alloy" else cb.diffuse_state_aos(P, M, 4.0)
        X = evolve_with_reference(P, M, R, X0, steps) if steps else X0
        Xp = np.ascontiguousarray(X.copy())
        O = R.output_fields(Xp, names, comps)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), X=X, Xpost=Xp, out=O, names=np.array(names),
                        comps=np.array(comps if comps else [""]))
    print(name, X.shape, "fields", O.shape, "two-phase cells", int((Xp[:, 0] > 1).sum()))


CONFIG_DIR = os.path.join(HERE, "configs")


def config_fixtures(name):
    """for configs/<name>.yaml: the reference's SetUpConfig result
    (<name>.ref.npz, by oracle.config_dump in its own process, since the
    reference aborts on a file it rejects) and its SetUpProblem state with the
    RHS there (<name>.state.npz)"""
    import subprocess
    path = os.path.join(CONFIG_DIR, name + ".yaml")
    out = os.path.join(CONFIG_DIR, name + ".ref.npz")
    r = subprocess.run([sys.executable, "-m", "oracle.config_dump", path, out], cwd=ROOT, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    if name.startswith("parse_"):
        print(name, "config")
        return
    cfg = cb.Config.load(path)
    P = cfg.problem
    M = cb.Mesh(P)
    cellphase = P.voxelphase()[np.ctypeslib.as_array(M.s.cell_global, shape=(M.nowned,))]
    extra = {}
    with oracle.RefOracle(P, M) as R:
        X0 = R.setup_problem(cellphase)
        F = R.rhs(X0)
        if name.startswith("aniso"):
            # a state with diffuse interfaces for the gradient-based anisotropy
            X1 = evolve_with_reference(P, M, R, X0, 3)
            extra = dict(X1=X1, F1=R.rhs(X1))
    np.savez_compressed(os.path.join(CONFIG_DIR, name + ".state.npz"), X0=X0, F=F, **extra)
    print(name, "config and state", X0.shape, "max|F|", np.abs(F).max())


def main(only=None):
    """regenerate every fixture, or only the named ones"""
    oracle.build(ref=True)

    def wanted(name):
        return not only or name in only

    for f in sorted(os.listdir(CONFIG_DIR)):
        if f.endswith(".yaml") and wanted("config_" + f[:-5]):
            config_fixtures(f[:-5])
    if wanted("nuc_ref"):
        nucleation_fixture()
    for name, kind, args, steps, names, comps in OUT_CASES:
        if wanted(name):
            output_fixture(name, kind, args, steps, names, comps)
    for name, kind, dim, res, a, ncp, npr, cap, seed, feats, lmin, lmax, iters, diffuse, steps in AMR_CASES:
        if not wanted(name):
            continue
        r = list(res) + [1] * (3 - len(res))
        meta = [kind, dim] + r + [a, ncp, npr, cap, seed, feats, lmin, lmax, iters, diffuse]
        P, F, M = build_amr(*meta)
        X = build_amr.state
        with oracle.RefOracle(P, M) as R:
            if steps:
                X = evolve_with_reference(P, M, R, X, steps)
            F_ = R.rhs(X)
            Xp = X.copy()
            assert R.poststep(Xp) == 0
        lev, _ = F.leaves()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), X=X, F=F_, Xpost=Xp, meta=np.array(meta),
                            levels=lev)
        print(name, X.shape, "levels", np.bincount(lev), "max|F|", np.abs(F_).max(), "mean n", X[:, 0].mean())
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
