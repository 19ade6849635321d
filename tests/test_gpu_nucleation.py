"""Nucleation on the device (cipher_nucleation_*) against its CPU
restatement (needs a B200: -m gpu): the same sites retire and fire with the
same event stream, per-site averages agree to 1e-12 (they pass through exp
and log), and the reset cells are identical."""
import numpy as np
import pytest

import cipher_b200 as cb
import oracle
from nucleation_case import build

pytestmark = pytest.mark.gpu


def test_device_matches_restatement():
    P, voxelsite, sitephase, sitenucleus, nuclei, vox = build()
    M = cb.Mesh(P)
    A = P.aos
    X = oracle.port_initial_state(P, M)
    ctx = cb.Context(P, M, "fp64")
    dX = ctx.alloc_state()
    ctx.from_aos(X, dX)
    dev = cb.Nucleation(ctx, voxelsite, sitephase, sitenucleus, nuclei, seed=7)
    ref = oracle.PortNucleation(P, M, voxelsite, sitephase, sitenucleus, nuclei, seed=7)
    for k in range(1, 4):
        nd = dev.step(dX, 0.1 * k, 1e-3)
        nr = ref.step(X, 0.1 * k, 1e-3)
        assert nd == nr
        sd = dev.sites()
        assert np.array_equal(sd["active"], ref.active)
        got = np.stack([sd["barrier"], sd["diffusivity"], sd["temperature"], sd["volume"]], axis=1)
        ev = ~np.isnan(ref.last[:, 0])
        assert np.array_equal(np.isnan(got[:, 0]), ~ev)
        scale = np.maximum(np.abs(ref.last[ev]), 1e-300)
        assert (np.abs(got[ev] - ref.last[ev]) <= 1e-12 * scale + 1e-300).all()
    Xd = ctx.to_aos(dX)
    n = X[:, 0].astype(int)
    assert np.array_equal(Xd[:, 0], X[:, 0])
    for g in range(A.pf_size):
        live = n > g
        assert np.array_equal(Xd[live, 1 + g], X[live, 1 + g])
        assert np.array_equal(Xd[live, A.pf_offset + g], X[live, A.pf_offset + g])
    ex = slice(A.ex_offset, A.ex_offset + A.sp_size)          # slot 0: the reset potentials
    assert np.abs(Xd[:, ex] - X[:, ex]).max() <= 1e-12 * np.abs(X[:, ex]).max()


def test_stepper_restarts_from_dtmin_after_a_nucleus():
    P, voxelsite, sitephase, sitenucleus, nuclei, vox = build()
    M = cb.Mesh(P)
    ctx = cb.Context(P, M, "fp64")
    dX = ctx.alloc_state()
    ctx.from_aos(oracle.port_initial_state(P, M), dX)
    nu = cb.Nucleation(ctx, voxelsite, sitephase, sitenucleus, nuclei, seed=7)
    o = cb.ts_options(P, "2a", dt0=1e-4, dtmin=1e-9, dtmax=1e-2, reltol=1e-3, abstol=1e-3)
    ts = cb.TimeStepper(ctx, o)
    ts.set_nucleation(nu)
    assert ts.step(dX, 1.0)
    st = ts.stats()
    assert st.dt == 1e-9                    # a constant-model site fired in the first update
    assert nu.sites()["active"][1] == 0


def test_device_averages_match_reference_fixture():
    """per-site averages on the device against the reference's own
    NucleationBarrier sums (fixture made by the reference): 1e-12 (the site
    fractions pass through exp and log on the device), the same sites
    evaluated and retired"""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "nuc_ref.npz"))
    P, voxelsite, sitephase, sitenucleus, nuclei, vox = build(sitenucleus=list(g["sitenucleus"]))
    M = cb.Mesh(P)
    ctx = cb.Context(P, M, "fp64")
    dX = ctx.alloc_state()
    ctx.from_aos(g["X"], dX)
    dev = cb.Nucleation(ctx, voxelsite, sitephase, sitenucleus, nuclei, seed=1)
    assert dev.step(dX, 0.0, 0.0) == 0            # dt = 0: every threshold is zero
    sd = dev.sites()
    got = np.stack([sd["barrier"], sd["diffusivity"], sd["temperature"], sd["volume"]], axis=1)
    ref = g["sites"]
    ev = ~np.isnan(ref[:, 0])
    assert np.array_equal(sd["active"], g["active"])
    assert np.array_equal(np.isnan(got[:, 0]), ~ev)
    scale = np.maximum(np.abs(ref[ev]), 1e-300)
    assert (np.abs(got[ev] - ref[ev]) <= 1e-12 * scale).all()
