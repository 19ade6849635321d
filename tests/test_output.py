"""Output fields (the reference's output step, src/cipher.c:976-1093) and the
VTU writer, on the CPU: the restatement's fields have the properties the
reference's definitions imply, and a written file parses back to the same
grid and arrays."""
import glob
import os
import re
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import cipher_b200 as cb
from cipher_b200 import _lib as L
import oracle

SPEC = [("phaseid", "phaseid", 0), ("matid", "matid", 0), ("interfaceid", "interfaceid", 0),
        ("al_chempot", "chempot", 0), ("al_c", "c", 0), ("cu_c", "c", 1), ("mg_c", "c", 2), ("va_c", "c", 3),
        ("2_phi", "phi", 2), ("temperature", "temperature", 0)]


def _kinds(spec):
    return [cb.api.OUTPUT_KINDS[k] for _, k, _ in spec], [i for _, _, i in spec]


def read_vtu(path):
    raw = open(path, "rb").read()
    head, _, rest = raw.partition(b'<AppendedData encoding="raw">')
    blob = rest[rest.index(b"_") + 1:]
    root = ET.fromstring(head + b"</VTKFile>" if b"</VTKFile>" not in head else head)
    piece = root.find("UnstructuredGrid/Piece")
    out = {"npts": int(piece.get("NumberOfPoints")), "ncells": int(piece.get("NumberOfCells"))}
    dt = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}
    for arr in root.iter("DataArray"):
        off = int(arr.get("offset"))
        nb = int(np.frombuffer(blob[off:off + 8], dtype=np.uint64)[0])
        out[arr.get("Name") or "points"] = np.frombuffer(blob[off + 8:off + 8 + nb], dtype=dt[arr.get("type")])
    return out


def test_fields_of_sharp_alloy_state():
    P = cb.Problem.alloy(2, [20, 16], "calphad2sl", 4, 5, 8, 3, 0x01)
    M = cb.Mesh(P)
    X = oracle.port_initial_state(P, M)
    k, i = _kinds(SPEC)
    F = oracle.port_output_fields(P, M, X, k, i)
    vox = P.voxelphase()
    assert np.array_equal(F[0], vox)                      # the own phase has h = 1
    pmm = np.ctypeslib.as_array(P.s.phasematerialmapping, shape=(P.s.npf,))
    assert np.array_equal(F[1], pmm[vox])
    assert np.allclose(F[4:8].sum(axis=0), 1.0, atol=1e-12)   # compositions sum to one
    assert np.array_equal(F[8], (vox == 2).astype(float))
    assert np.all(F[9] == 700.0)
    n = X[:, 0]
    assert np.all((F[2] == -1.0) == (n == 1))


@pytest.mark.parametrize("dim,res", [(2, [6, 5]), (3, [4, 3, 5])])
def test_vtu_round_trip(tmp_path, dim, res):
    P = cb.Problem.grain_growth(dim, res, 3, 3, 1)
    M = cb.Mesh(P)
    X = cb.diffuse_state_aos(P, M, 2.0)
    spec = [("phaseid", "phaseid", 0), ("0_phi", "phi", 0), ("temperature", "temperature", 0)]
    k, i = _kinds(spec)
    F = oracle.port_output_fields(P, M, X, k, i)
    path = str(tmp_path / "out_0.vtu")
    cb.write_vtu(path, P, spec, F)
    d = read_vtu(path)
    ncell = int(np.prod(res))
    assert d["ncells"] == ncell and d["npts"] == int(np.prod([r + 1 for r in res]))
    nv = 4 if dim == 2 else 8
    assert np.array_equal(d["offsets"], nv * np.arange(1, ncell + 1))
    assert np.all(d["types"] == (9 if dim == 2 else 12))
    pts = d["points"].reshape(-1, 3)
    conn = d["connectivity"].reshape(ncell, nv)
    # each cell's nodes span one cell of size 1 around its centre
    c = 7
    x, y = c % res[0], (c // res[0]) % res[1]
    lo = pts[conn[c]].min(axis=0)
    hi = pts[conn[c]].max(axis=0)
    assert lo[0] == x and lo[1] == y and hi[0] == x + 1 and hi[1] == y + 1
    for name, row in zip([s[0] for s in spec], F):
        assert np.array_equal(d[name], row)


# ---- pinned against the reference's own output step ----

OUT_REF = sorted(glob.glob(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "out_ref_*.npz")))


def _out_case(path):
    from golden.make_golden import OUT_CASES, output_case
    name = os.path.basename(path)[:-4]
    case = next(c for c in OUT_CASES if c[0] == name)
    P, M = output_case(case[1], case[2])
    g = np.load(path)
    names = [str(n) for n in g["names"]]
    comps = [str(c) for c in g["comps"] if str(c)]
    return P, M, g, cb.api.output_spec(names, comps)


def test_reference_output_fixtures_present():
    assert len(OUT_REF) >= 2


@pytest.mark.parametrize("path", OUT_REF, ids=[os.path.basename(p) for p in OUT_REF])
def test_restatement_equals_reference_output(path):
    """the fields the reference's output step wrote after its PostStep
    (fixture) equal the restatement's on the same post-step state: ids,
    phase fractions, potentials and temperature exactly, compositions (site
    fractions through exp) to 1e-14"""
    P, M, g, spec = _out_case(path)
    k, i = _kinds(spec)
    O = oracle.port_output_fields(P, M, g["Xpost"], k, i)
    for f, (name, kind, _) in enumerate(spec):
        if kind == "c":
            assert np.abs(O[f] - g["out"][f]).max() <= 1e-14, name
        else:
            assert np.array_equal(O[f], g["out"][f]), name


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")
@pytest.mark.parametrize("path", OUT_REF, ids=[os.path.basename(p) for p in OUT_REF])
def test_reference_output_step_reproduces_fixture(path):
    """the reference run again here gives the fixture bit for bit (state
    after PostStep and every field)"""
    P, M, g, spec = _out_case(path)
    X = np.ascontiguousarray(g["X"].copy())
    names = [str(n) for n in g["names"]]
    comps = [str(c) for c in g["comps"] if str(c)]
    with oracle.RefOracle(P, M) as R:
        O = R.output_fields(X, names, comps)
    assert np.array_equal(X, g["Xpost"])
    assert np.array_equal(O, g["out"])
