"""The allocation-free active-set update, through the C ABI (needs a GPU).

cipher_poststep_noalloc serves callers that cannot allocate device memory:
it takes no context and keeps its scratch in a fixed array inside the
library.  Its result must equal cipher_poststep's (the context entry point)
bit for bit, on two calls in a row, since the second call reuses the scratch
the first one left behind.  With chemistry (S > 0) a phase that joins a cell
gets its explicit site potentials from the material tables the caller passes;
the test checks that some cells do gain a phase, so that branch runs.  This
file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import cipher_b200 as cb
import cipher_b200._lib as L

pytestmark = pytest.mark.gpu


def _material_tables(problem):
    """device copies of the problem's material table and phase-material
    mapping (the test allocates them; the entry point does not)"""
    import torch
    lib = L.load()
    sizes = (C.c_int64 * 9)()
    lib.cipher_abi_sizes(sizes, 9)
    s = problem.s
    mat_bytes = int(sizes[4]) * s.nmat
    mat = np.ctypeslib.as_array(C.cast(s.material, C.POINTER(C.c_uint8)), shape=(mat_bytes,)).copy()
    pmm = np.ctypeslib.as_array(s.phasematerialmapping, shape=(s.npf,)).astype(np.int32)
    return torch.from_numpy(mat).cuda(), torch.from_numpy(pmm).cuda()


def _desc(problem, ctx, tables=None):
    s = problem.s
    d = L.GridDesc()
    d.dim = s.dim
    for k in range(3):
        d.res[k] = s.resolution[k] if k < s.dim else 1
        d.periodic[k] = s.periodic[k] if k < s.dim else 0
    d.layout = ctx.layout
    d.ex_per_phase = ctx.layout.ex_size // ctx.layout.pf_size
    d.npf, d.ncp, d.nmat = s.npf, s.ncp, s.nmat
    if tables is not None:
        d.materials = tables[0].data_ptr()
        d.phasematerialmapping = tables[1].data_ptr()
    return d


def _noalloc(desc, X):
    lib = L.load()
    return lib.cipher_poststep_noalloc(C.byref(desc), C.c_void_p(X.data_ptr()), C.c_void_p(0))


def _explicit_step(ctx, X, F, dt):
    ctx.rhs(0.0, X, F)
    ctx.waxpy(X, X, dt, F)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_matches_context_poststep_twice(precision):
    import torch
    P = cb.Problem.grain_growth(3, [24, 20, 16], 12, 12, 31)
    M = cb.Mesh(P)
    X = cb.diffuse_state_aos(P, M, 4.0)
    ctx = cb.Context(P, M, precision)
    desc = _desc(P, ctx)
    assert desc.ex_per_phase == 0
    Xa, Xb, F = ctx.alloc_state(), ctx.alloc_state(), ctx.alloc_state()
    ctx.from_aos(X, Xa)
    ctx.from_aos(X, Xb)
    torch.cuda.synchronize()
    for call in range(2):
        ctx.poststep(Xa)
        assert _noalloc(desc, Xb) == L.OK
        assert torch.equal(Xa, Xb), f"call {call}: states differ"
        # move both states on by the same explicit step before the next call
        _explicit_step(ctx, Xa, F, 0.02)
        _explicit_step(ctx, Xb, F, 0.02)
        torch.cuda.synchronize()


def _alloy_dt(ctx, P, X, F):
    """a step that moves phase fractions by at most 0.05 and mu by 2 %"""
    A = P.aos
    Fh, Xh = ctx.to_aos(F), ctx.to_aos(X)
    fphi = np.abs(Fh[:, A.pf_offset:A.pf_offset + A.pf_size]).max()
    fdp = np.abs(Fh[:, A.dp_offset:A.dp_offset + A.dp_size]).max()
    mu = np.abs(Xh[:, A.dp_offset:A.dp_offset + A.dp_size]).max()
    return min(0.05 / max(fphi, 1e-300), 0.02 * mu / max(fdp, 1e-300))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_with_chemistry_matches_context_poststep_twice(precision):
    """S > 0 (calphad2sl, 4 components): new phases get SitepotentialExplicit
    of c0 at the cell's temperature from the caller's material tables"""
    import torch
    P = cb.Problem.alloy(2, [24, 20], "calphad2sl", 4, 4, 8, 21, 0)
    M = cb.Mesh(P)
    ctx = cb.Context(P, M, precision)
    tables = _material_tables(P)
    desc = _desc(P, ctx, tables)
    assert desc.ex_per_phase > 0
    Xa, Xb, F = ctx.alloc_state(), ctx.alloc_state(), ctx.alloc_state()
    ctx.init_sharp(Xa)
    ctx.rhs(0.0, Xa, F)
    dt = _alloy_dt(ctx, P, Xa, F)
    gained = 0
    for call in range(2):
        _explicit_step(ctx, Xa, F, dt)
        Xb.copy_(Xa)
        as_before = ctx.planes(Xa)[0].clone()
        ctx.poststep(Xa)
        assert _noalloc(desc, Xb) == L.OK
        assert torch.equal(Xa, Xb), f"call {call}: states differ"
        as_after = ctx.planes(Xa)[0]
        n0, n1 = as_before[0].long(), as_after[0].long()
        gained += int((n1 > n0).sum())
        ctx.check()
    assert gained > 0, "no cell gained a phase: the new-phase branch did not run"


def test_noalloc_rejects_grids_above_its_scratch():
    P = cb.Problem.grain_growth(2, [16, 16], 6, 4, 1)
    M = cb.Mesh(P)
    ctx = cb.Context(P, M, "fp64")
    desc = _desc(P, ctx)
    desc.layout.stride = 1 << 24          # (P+1)*stride above the 4 Mi-entry scratch
    assert L.load().cipher_poststep_noalloc(C.byref(desc), C.c_void_p(1), C.c_void_p(0)) == L.E_ARG


def test_noalloc_rejects_inconsistent_descriptions():
    """bad descriptions are refused before any launch (X is never touched)"""
    lib = L.load()
    P = cb.Problem.alloy(2, [12, 10], "calphad2sl", 4, 2, 8, 3, 0)
    M = cb.Mesh(P)
    ctx = cb.Context(P, M, "fp64")

    def rc(**changes):
        d = _desc(P, ctx)
        d.materials, d.phasematerialmapping = 256, 512      # never dereferenced: refused first
        for k, v in changes.items():
            if k.startswith("layout_"):
                setattr(d.layout, k[7:], v)
            else:
                setattr(d, k, v)
        return lib.cipher_poststep_noalloc(C.byref(d), C.c_void_p(1), C.c_void_p(0))

    S = ctx.layout.ex_size // ctx.layout.pf_size
    assert rc(ex_per_phase=-1) == L.E_ARG
    assert rc(ex_per_phase=2 * 5 + 1) == L.E_ARG
    assert rc(ex_per_phase=S + 1) == L.E_ARG            # ex_size != P*S
    assert rc(materials=None) == L.E_ARG                 # S > 0 needs the tables
    assert rc(phasematerialmapping=None) == L.E_ARG
    assert rc(npf=0) == L.E_ARG
    assert rc(ncp=1) == L.E_ARG
    assert rc(layout_map_planes=3) == L.E_ARG            # neither 0 nor P
