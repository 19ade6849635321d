"""The allocation-free active-set update, through the C ABI (needs a GPU).

cipher_poststep_noalloc serves callers that cannot allocate device memory:
it takes no context and keeps its scratch in a fixed array inside the
library.  Its result must equal cipher_poststep's (the context entry point)
bit for bit, on two calls in a row, since the second call reuses the scratch
the first one left behind.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import cipher_b200 as cb
import cipher_b200._lib as L

pytestmark = pytest.mark.gpu


def _desc(problem, ctx):
    s = problem.s
    d = L.GridDesc()
    d.dim = s.dim
    for k in range(3):
        d.res[k] = s.resolution[k] if k < s.dim else 1
        d.periodic[k] = s.periodic[k] if k < s.dim else 0
    d.ex_per_phase = 0
    d.layout = ctx.layout
    d.ex_init = None
    return d


def _noalloc(desc, X):
    lib = L.load()
    return lib.cipher_poststep_noalloc(C.byref(desc), C.c_void_p(X.data_ptr()), C.c_void_p(0))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_matches_context_poststep_twice(precision):
    import torch
    P = cb.Problem.grain_growth(3, [24, 20, 16], 12, 12, 31)
    M = cb.Mesh(P)
    X = cb.diffuse_state_aos(P, M, 4.0)
    ctx = cb.Context(P, M, precision)
    desc = _desc(P, ctx)
    Xa, Xb, F = ctx.alloc_state(), ctx.alloc_state(), ctx.alloc_state()
    ctx.from_aos(X, Xa)
    ctx.from_aos(X, Xb)
    torch.cuda.synchronize()
    for call in range(2):
        ctx.poststep(Xa)
        assert _noalloc(desc, Xb) == L.OK
        assert torch.equal(Xa, Xb), f"call {call}: states differ"
        # move both states on by the same explicit step before the next call
        ctx.rhs(0.0, Xa, F)
        ctx.waxpy(Xa, Xa, 0.02, F)
        ctx.rhs(0.0, Xb, F)
        ctx.waxpy(Xb, Xb, 0.02, F)
        torch.cuda.synchronize()


def test_noalloc_rejects_grids_above_its_scratch():
    P = cb.Problem.grain_growth(2, [16, 16], 6, 4, 1)
    M = cb.Mesh(P)
    ctx = cb.Context(P, M, "fp64")
    desc = _desc(P, ctx)
    desc.layout.stride = 1 << 24          # (P+1)*stride above the 4 Mi-entry scratch
    assert L.load().cipher_poststep_noalloc(C.byref(desc), C.c_void_p(1), C.c_void_p(0)) == L.E_ARG
