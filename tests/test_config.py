"""Configuration files (cipher_config_*, the reference's YAML input read by
SetUpConfig, src/init.c:24-1716) on the CPU.

* The YAML subset parser reads every file as PyYAML does (all scalars as
  strings): the committed configurations, edge cases of the syntax, and the
  reference's own example configurations where its sources are present.
* The loader's tables equal the reference's own SetUpConfig result, byte for
  byte: committed dumps for the committed configurations (made by
  oracle/config_dump.py, tests/golden/make_golden.py), and, where the
  reference is built here, live on all of its example configurations,
  including the ones it rejects (the loader must reject them too).
* The SetUpProblem state of each committed configuration (the reference's,
  fixture) equals the restatement's, chemistry included.
"""
import glob
import os
import subprocess
import sys

import numpy as np
import pytest
import yaml

import cipher_b200 as cb
import oracle
from config_compare import compare

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CONFIGS = sorted(glob.glob(os.path.join(HERE, "golden", "configs", "*.yaml")))
# configurations with a SetUpProblem / RHS fixture (parse_* files hold random
# sources, which the reference draws with rand() inside its RHS)
STATE_CONFIGS = [p for p in CONFIGS if not os.path.basename(p).startswith("parse_")]
EXAMPLES = sorted(glob.glob(os.path.join(oracle.REF_ROOT, "examples", "*", "*.yaml"))) if oracle.REF_ROOT else []


def _ids(paths):
    return [os.path.basename(p) for p in paths]


def test_committed_configs_present():
    assert len(CONFIGS) >= 7 and len(STATE_CONFIGS) >= 6


@pytest.mark.parametrize("path", CONFIGS + EXAMPLES, ids=_ids(CONFIGS + EXAMPLES))
def test_parser_reads_files_as_pyyaml(path):
    text = open(path, encoding="utf-8").read()
    assert cb.api.yaml_to_json(text) == yaml.load(text, Loader=yaml.BaseLoader)


EDGE_CASES = [
    "a: 1\r\nb: [x, 'y, z', \"q\\\"r\"]\r\n",
    "---\nk : v   # comment\n# full-line comment\nm:\n  n: |-\n    line 1\n      indented\n\n    line 3\n  o: |\n    kept\n\n",
    "(al:cu) :\n  t: [1, 2]\n(al,cu:zn): x\n",
    "top:\n  - one\n  - two: 2\n    three: 3\n  - [4, 5]\nnext: {a: 1, b: [2, 3]}\n",
    "f: >\n  folded\n  text\n\n  para\nplain: multi\n  line words\nempty:\nlast: '' \n",
    "seq:\n- a\n- b\nq: \"x # not a comment\"\n",
    "nested: [[1, 2], [3, [4]]]\nmultiline: [1,\n   2, 3]\n",
]


@pytest.mark.parametrize("text", EDGE_CASES, ids=[f"edge{i}" for i in range(len(EDGE_CASES))])
def test_parser_edge_cases_as_pyyaml(text):
    assert cb.api.yaml_to_json(text) == yaml.load(text, Loader=yaml.BaseLoader)


@pytest.mark.parametrize("text", ["a: [1, 2\n", "a: 1\n  b: 2\n", "a: &x 1\n", "a:\n\tb: 1\n", "---\na: 1\n---\nb: 2\n"])
def test_parser_rejects_what_it_does_not_read(text):
    with pytest.raises(cb.CipherError) as e:
        cb.api.yaml_to_json(text)
    assert "line" in str(e.value)


@pytest.mark.parametrize("path", CONFIGS, ids=_ids(CONFIGS))
def test_loader_equals_reference_setupconfig_fixture(path):
    g = np.load(path[:-5] + ".ref.npz")
    cfg = cb.Config.load(path)
    assert compare(cfg, g) == []


@pytest.mark.parametrize("path", STATE_CONFIGS, ids=_ids(STATE_CONFIGS))
def test_restatement_initial_state_equals_reference_setupproblem(path):
    """the SetUpProblem state (sets, phi, T, and for chemistry mu and the
    explicit site potentials from c0) of the restatement equals the
    reference's (fixture) bit for bit"""
    cfg = cb.Config.load(path)
    M = cb.Mesh(cfg.problem)
    X0 = oracle.port_initial_state(cfg.problem, M)
    assert np.array_equal(X0, np.load(path[:-5] + ".state.npz")["X0"])


@pytest.mark.parametrize("path", STATE_CONFIGS, ids=_ids(STATE_CONFIGS))
def test_restatement_rhs_on_config_equals_reference(path):
    cfg = cb.Config.load(path)
    M = cb.Mesh(cfg.problem)
    g = np.load(path[:-5] + ".state.npz")
    assert np.array_equal(oracle.port_rhs(cfg.problem, M, g["X0"]), g["F"])


ANISO = [p for p in STATE_CONFIGS if os.path.basename(p).startswith("aniso")]


@pytest.mark.parametrize("path", ANISO, ids=_ids(ANISO))
def test_restatement_anisotropy_equals_reference_on_evolved_state(path):
    """gradient-based anisotropy (least-squares gradients, normals of each
    pair, (u . dir)^4 terms on energy and mobility): the restatement equals
    the reference's RHS bit for bit on a state evolved by the reference, and
    the anisotropy changes the result"""
    cfg = cb.Config.load(path)
    M = cb.Mesh(cfg.problem)
    g = np.load(path[:-5] + ".state.npz")
    F = oracle.port_rhs(cfg.problem, M, g["X1"])
    assert np.array_equal(F, g["F1"])
    cfg.problem.s.gradient_calculation = 0
    F0 = oracle.port_rhs(cfg.problem, M, g["X1"])
    A = cfg.problem.aos
    sl = slice(A.pf_offset, A.pf_offset + A.pf_size)
    assert np.abs(F0[:, sl] - F[:, sl]).max() > 1e-3 * np.abs(F[:, sl]).max()


def test_config_values():
    """a few values of the committed grain-growth file read back"""
    cfg = cb.Config.load(os.path.join(HERE, "golden", "configs", "gg_small.yaml"))
    P = cfg.problem.s
    assert (P.dim, P.npf, P.ncp, P.nmat, P.nf, P.pf_size) == (2, 5, 1, 1, 2, 4)
    assert list(P.time)[:2] == [1.0, 2.5] and P.has_temperature_rate and P.temperature_rate[1] == -2.0
    assert P.interpolation == cb._lib.INTERP_QUADRATIC and P.periodic[0] == 1 and P.periodic[1] == 1
    assert cfg.s.rk_type == b"3bs" and cfg.s.outputfreq == 5 and cfg.s.random_seed == 12345
    assert [o[1] for o in cfg.output_spec()] == ["phaseid", "matid", "interfaceid", "phi", "phi"]
    vox = cfg.problem.voxelphase()
    assert vox[:20].tolist() == [0] * 20 and vox[20:25].tolist() == [0, 1, 2, 3, 4]
    o = cfg.ts_options()
    assert o.scheme == cb._lib.TS_RK3BS and o.dt0 == 1e-4 and o.dtmax == 0.05


def test_nucleation_tables_of_config():
    cfg = cb.Config.load(os.path.join(HERE, "golden", "configs", "nuc_small.yaml"))
    vs, sp, sn, nz = cfg.nucleation_tables()
    assert sp.tolist() == [2, 2, 3] and sn.tolist() == [0, 1, 2]
    assert np.bincount(vs[vs >= 0]).tolist() == [4, 4, 3] and (vs == -1).sum() == 85
    assert list(nz[0].matrix[:2]) == [0, 1]          # read as [1, 0], kept sorted
    assert list(nz[0].active_solutes[:2]) == [0, 1]


@pytest.mark.parametrize("bad,what", [
    ("n_phases : 5", "n_phases : 0"),
    ("    5 of 1\n  interface_mapping", "    4 of 1\n  interface_mapping"),
    ("    59 of 5", "    60 of 5"),
    ("      t_exponent : [0, 1]\n\ninterface", "      t_exponent : [0]\n\ninterface"),
    ("  initrefine : 2", "  initrefine : 3"),
    ("  interpolation : quadratic", "  interpolation : spline"),
    ("      m0 : 1.0e-2\n", "      m1 : 1.0e-2\n"),
])
def test_loader_rejects_what_the_reference_asserts(bad, what):
    text = open(os.path.join(HERE, "golden", "configs", "gg_small.yaml")).read()
    assert bad in text
    with pytest.raises(cb.CipherError) as e:
        cb.Config.parse(text.replace(bad, what, 1))
    assert e.value.code == cb._lib.E_ARG


def test_mapping_read_from_a_file(tmp_path):
    """a mapping whose first line names a .txt file is read from that file
    (next to the configuration, then the working directory)"""
    src = open(os.path.join(HERE, "golden", "configs", "gg_small.yaml")).read()
    body = src.split("voxel_phase_mapping : |-\n", 1)[1]
    (tmp_path / "voxels.txt").write_text("\n".join(line.strip() for line in body.splitlines()) + "\n")
    text = src.split("voxel_phase_mapping : |-\n", 1)[0] + "voxel_phase_mapping : |-\n    voxels.txt\n"
    cfg_path = tmp_path / "gg.yaml"
    cfg_path.write_text(text)
    a = cb.Config.load(str(cfg_path)).problem.voxelphase()
    b = cb.Config.load(os.path.join(HERE, "golden", "configs", "gg_small.yaml")).problem.voxelphase()
    assert np.array_equal(a, b)


def _reference_dump(path, out):
    r = subprocess.run([sys.executable, "-m", "oracle.config_dump", path, out], cwd=ROOT, capture_output=True,
                       text=True, timeout=600)
    return r.returncode


@pytest.mark.skipif(not (oracle.ref_available() and EXAMPLES), reason="reference sources / oracle not present")
@pytest.mark.parametrize("path", EXAMPLES, ids=_ids(EXAMPLES))
def test_loader_equals_reference_on_its_examples(path, tmp_path):
    """the reference's own example configurations: the loader's tables equal
    the reference's SetUpConfig result, and a file the reference rejects (an
    assert aborts it) is rejected by the loader too"""
    out = str(tmp_path / "ref.npz")
    rc = _reference_dump(path, out)
    if rc != 0:
        with pytest.raises(cb.CipherError):
            cb.Config.load(path)
        return
    assert compare(cb.Config.load(path), np.load(out)) == []
