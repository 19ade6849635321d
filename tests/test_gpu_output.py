"""Output fields on the device (cipher_output_fields) against the CPU
restatement (needs a B200: -m gpu).  Ids, phase fractions, chemical
potentials and temperature are copies and compare exactly; compositions go
through the site fractions (exp on the device) and compare within 1e-12."""
import numpy as np
import pytest

import cipher_b200 as cb
import oracle

pytestmark = pytest.mark.gpu

SPEC = [("phaseid", "phaseid", 0), ("matid", "matid", 0), ("interfaceid", "interfaceid", 0),
        ("al_chempot", "chempot", 0), ("cu_chempot", "chempot", 1), ("al_c", "c", 0), ("cu_c", "c", 1),
        ("va_c", "c", 3), ("2_phi", "phi", 2), ("0_phi", "phi", 0), ("temperature", "temperature", 0)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_output_fields_match_restatement(precision, tmp_path):
    P = cb.Problem.alloy(2, [40, 32], "calphad2sl", 4, 6, 8, 9, 0x01)
    M = cb.Mesh(P)
    X = oracle.port_initial_state(P, M)
    for _ in range(2):                      # a few steps: diffuse interfaces
        F = oracle.port_rhs(P, M, X)
        X = X + 2e-3 * F
        assert oracle.port_poststep(P, M, X) == 0
    A = P.aos
    if precision == "mixed":
        for off, size in ((A.pf_offset, A.pf_size), (A.tm_offset, 1)):
            X[:, off:off + size] = X[:, off:off + size].astype(np.float32)
    ctx = cb.Context(P, M, precision)
    dX = ctx.alloc_state()
    ctx.from_aos(X, dX)
    D = cb.compute_output(ctx, dX, SPEC)
    kinds = [cb.api.OUTPUT_KINDS[k] for _, k, _ in SPEC]
    idx = [i for _, _, i in SPEC]
    O = oracle.port_output_fields(P, M, X, kinds, idx)
    comp = [k for k, (_, kind, _) in enumerate(SPEC) if kind == "c"]
    for k in range(len(SPEC)):
        if k in comp:
            assert np.abs(D[k] - O[k]).max() <= 1e-12, SPEC[k]
        else:
            assert np.array_equal(D[k], O[k]), SPEC[k]
    path = str(tmp_path / "alloy_0.vtu")
    cb.write_vtu(path, P, SPEC, D)
    assert open(path, "rb").read(5) == b"<?xml"


def test_output_fields_match_reference_fixtures():
    """the device's fields on the reference's post-step state against the
    fields the reference's own output step wrote (fixtures): ids, phase
    fractions, potentials and temperature exactly, compositions 1e-12"""
    import glob
    import os
    from golden.make_golden import OUT_CASES, output_case
    paths = sorted(glob.glob(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "out_ref_*.npz")))
    assert len(paths) >= 2
    for path in paths:
        case = next(c for c in OUT_CASES if c[0] == os.path.basename(path)[:-4])
        P, M = output_case(case[1], case[2])
        g = np.load(path)
        spec = cb.api.output_spec([str(n) for n in g["names"]], [str(c) for c in g["comps"] if str(c)])
        ctx = cb.Context(P, M, "fp64")
        dX = ctx.alloc_state()
        ctx.from_aos(g["Xpost"], dX)
        D = cb.compute_output(ctx, dX, spec)
        for k, (name, kind, _) in enumerate(spec):
            if kind == "c":
                assert np.abs(D[k] - g["out"][k]).max() <= 1e-12, (path, name)
            else:
                assert np.array_equal(D[k], g["out"][k]), (path, name)
