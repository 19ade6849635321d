"""Nucleation restatement (oracle/port/oracle_nuc.c) on the CPU: site
retirement, events of the constant model, the reset of fired sites."""
import numpy as np

import cipher_b200 as cb
import oracle
from nucleation_case import build


def test_sites_fire_retire_and_reset():
    P, voxelsite, sitephase, sitenucleus, nuclei, vox = build()
    M = cb.Mesh(P)
    A = P.aos
    X = oracle.port_initial_state(P, M)
    X0 = X.copy()
    nu = oracle.PortNucleation(P, M, voxelsite, sitephase, sitenucleus, nuclei, seed=3)
    cells = [np.flatnonzero(voxelsite == s) for s in range(6)]
    nf = nu.step(X, 0.1, 1e-3)
    # site 5 holds a precipitate phase: retired without an event
    assert nu.active[5] == 0 and np.isnan(nu.last[5, 0])
    assert np.array_equal(X[cells[5]], X0[cells[5]])
    # site 1 (constant model, enormous rate) fires: its cells become its phase
    assert nu.active[1] == 0
    assert np.all(X[cells[1], 0] == 1) and np.all(X[cells[1], 1] == sitephase[1])
    assert np.all(X[cells[1], A.pf_offset] == 1.0)
    # site 3 (constant model, zero rate) stays active and unchanged
    assert nu.active[3] == 1 and np.array_equal(X[cells[3]], X0[cells[3]])
    # the cnt and thermal sites were evaluated: finite averages over 9 cells
    for s in (0, 2, 4):
        assert np.isfinite(nu.last[s]).all() and nu.last[s, 3] == 9.0 and nu.last[s, 2] == 700.0
    fired = [s for s in range(6) if nu.active[s] == 0 and s != 5]
    assert nf == len(fired) >= 1


def test_stream_is_reproducible():
    P, voxelsite, sitephase, sitenucleus, nuclei, vox = build()
    M = cb.Mesh(P)
    runs = []
    for _ in range(2):
        X = oracle.port_initial_state(P, M)
        nu = oracle.PortNucleation(P, M, voxelsite, sitephase, sitenucleus, nuclei, seed=11)
        nf = [nu.step(X, 0.1 * k, 1e-3) for k in range(1, 4)]
        runs.append((nf, X.copy(), nu.active.copy()))
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1], runs[1][1]) and np.array_equal(runs[0][2], runs[1][2])


# ---- pinned against the reference's own nucleation helpers ----

import os  # noqa: E402

import pytest  # noqa: E402

NUC_REF = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "nuc_ref.npz")


def _ref_case():
    g = np.load(NUC_REF)
    P, voxelsite, sitephase, sitenucleus, nuclei, vox = build(sitenucleus=list(g["sitenucleus"]))
    return g, P, cb.Mesh(P), voxelsite, sitephase, sitenucleus, nuclei


def test_restatement_averages_equal_reference():
    """per-site barrier, diffusivity, temperature and volume of the
    restatement equal the reference's (NucleationBarrier summed as its
    PostStep sums them; fixture) bit for bit, on a state with two-phase
    cells inside CNT and thermal sites and a temperature that varies by cell;
    the site holding a precipitate is retired by both"""
    g, P, M, voxelsite, sitephase, sitenucleus, nuclei = _ref_case()
    n = g["X"][:, 0].astype(int)
    assert ((voxelsite >= 0) & (n > 1)).sum() >= 10
    nu = oracle.PortNucleation(P, M, voxelsite, sitephase, sitenucleus, nuclei, seed=1)
    X = g["X"].copy()
    nu.step(X, 0.0, 0.0)                 # dt = 0: every threshold is zero, nothing fires
    ref = g["sites"]
    ev = ~np.isnan(ref[:, 0])
    assert np.array_equal(np.isnan(nu.last[:, 0]), ~ev)
    assert np.array_equal(nu.last[ev], ref[ev])
    assert np.array_equal(nu.active, g["active"])
    assert not g["active"][5] and np.isnan(nu.last[5, 0])


def test_restatement_event_rule_replays_reference_decisions():
    """for every evaluated site and 48 seeds of the C library's generator,
    the reference's NucleationEvent fired exactly when the restatement's rule
    (a draw happens and the number drawn is below its threshold) says so; the
    step size puts each threshold near one half"""
    g, P, M, voxelsite, sitephase, sitenucleus, nuclei = _ref_case()
    rows = g["events"]
    fired_sites = set()
    for s, t, dt, seed, u, fired in rows:
        s = int(s)
        gv, diff, T, vol = g["sites"][s]
        draws, thr = oracle.port_nucleation_threshold(nuclei[sitenucleus[s]], P.s.dim, t, dt, T, vol, gv, diff)
        assert bool(fired) == (draws and u < thr), (s, seed, u, thr)
        if fired:
            fired_sites.add(s)
    models = {int(nuclei[sitenucleus[s]].model) for s in fired_sites}
    assert models == {cb._lib.NUC_CNT, cb._lib.NUC_CONSTANT, cb._lib.NUC_THERMAL}
    assert 0.2 < rows[:, 5].mean() < 0.8


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")
def test_reference_helpers_reproduce_fixture_and_agree_on_fresh_states():
    """the reference run again here gives the fixture; on the sharp initial
    state and on a state with a shifted temperature the restatement and the
    reference agree bit for bit"""
    g, P, M, voxelsite, sitephase, sitenucleus, nuclei = _ref_case()
    A = P.aos
    with oracle.RefOracle(P, M, nucleation=(sitephase, sitenucleus, nuclei)) as R:
        out, act = R.nucleation_sites(g["X"], voxelsite)
        assert np.array_equal(np.isnan(out), np.isnan(g["sites"]))
        ok = ~np.isnan(out)
        assert np.array_equal(out[ok], g["sites"][ok]) and np.array_equal(act, g["active"])
        X0 = oracle.port_initial_state(P, M)
        for shift in (0.0, -40.0):
            X = X0.copy()
            X[:, A.tm_offset] += shift
            out, act = R.nucleation_sites(X, voxelsite)
            nu = oracle.PortNucleation(P, M, voxelsite, sitephase, sitenucleus, nuclei, seed=1)
            nu.step(X.copy(), 0.0, 0.0)
            ev = ~np.isnan(out[:, 0])
            assert np.array_equal(nu.last[ev], out[ev])
