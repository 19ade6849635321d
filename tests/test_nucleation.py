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
