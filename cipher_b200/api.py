"""Python face of the C ABI: problems, meshes, device contexts.

Mirrors the reference's callback pair: ``Context.RHSFunction(ts, t, X, F)``
is the RHSFunction of src/cipher.c:27 and ``Context.PostStep(ts)`` its
PostStep (src/cipher.c:686); both call the CUDA library.  Device buffers are
torch uint8 tensors of ``layout.bytes`` (torch provides memory and streams;
the arithmetic is the library's).
"""
from __future__ import annotations

import ctypes as C
import re
from dataclasses import dataclass

import numpy as np

from . import _lib as L


class Problem:
    """Owns a ``cipher_problem`` (model parameters + initial voxel map)."""

    def __init__(self, ptr, owner=None):
        """owner: an object that owns the problem (a Config); the problem is
        then freed with it, not by this wrapper"""
        self._lib = L.load()
        self.ptr = ptr
        self._owner = owner

    @classmethod
    def grain_growth(cls, dim: int, res, ngrains: int, cap: int, seed: int, energy: float = 1.0,
                     mobility: float = 1.0, width: float = 4.0, molarvolume: float = 1e-5,
                     temperature0: float = 500.0) -> "Problem":
        lib = L.load()
        r = (C.c_int32 * 3)(*(list(res) + [1] * (3 - len(res))))
        out = L.PP()
        L.check(lib.cipher_problem_grain_growth(dim, r, ngrains, cap, seed, energy, mobility, width,
                                                molarvolume, temperature0, C.byref(out)),
                "cipher_problem_grain_growth")
        return cls(out)

    @classmethod
    def grain_growth_multi(cls, dim: int, res, ngrains: int, cap: int, seed: int, ninterfaces: int = 4,
                           activation: bool = False, widths: bool = False) -> "Problem":
        """Grain growth with several seeded interfaces (per-pair energy and
        mobility; optionally T-dependent, optionally of different widths)."""
        lib = L.load()
        r = (C.c_int32 * 3)(*(list(res) + [1] * (3 - len(res))))
        feats = (L.GG_ACTIVATION if activation else 0) | (L.GG_WIDTHS if widths else 0)
        out = L.PP()
        L.check(lib.cipher_problem_grain_growth_multi(dim, r, ngrains, cap, seed, ninterfaces, feats,
                                                      C.byref(out)), "cipher_problem_grain_growth_multi")
        return cls(out)

    @classmethod
    def alloy(cls, dim: int, res, model: str = "calphad2sl", ncp: int = 4, nprecip: int = 20, cap: int = 15,
              seed: int = 1, features: int = 0) -> "Problem":
        """Seeded alloy problem (cipher_problem_alloy): two matrix grains with
        `nprecip` precipitates; `features` is a mask of the ALLOY_* bits."""
        lib = L.load()
        mid = {"quadratic": L.CHEM_QUADRATIC, "calphaddis": L.CHEM_CALPHADDIS, "calphad2sl": L.CHEM_CALPHAD2SL}[model]
        r = (C.c_int32 * 3)(*(list(res) + [1] * (3 - len(res))))
        out = L.PP()
        L.check(lib.cipher_problem_alloy(dim, r, mid, ncp, nprecip, cap, seed, features, C.byref(out)),
                "cipher_problem_alloy")
        return cls(out)

    @property
    def s(self) -> L.ProblemStruct:
        return self.ptr.contents

    @property
    def aos(self) -> L.AosLayout:
        return self._lib.cipher_problem_aos_layout(self.ptr)

    @property
    def ndof(self) -> int:
        return self.aos.ndof

    def voxelphase(self) -> np.ndarray:
        s = self.s
        n = int(np.prod([s.resolution[d] for d in range(s.dim)]))
        return np.ctypeslib.as_array(s.voxelphase, shape=(n,)).copy()

    def close(self):
        if self.ptr and self._owner is None:
            self._lib.cipher_problem_free(self.ptr)
        self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Config:
    """A run read from the reference's YAML configuration format
    (cipher_config_load / cipher_config_parse, SetUpConfig src/init.c:104-1716):
    the problem, nucleation sites and nuclei, output fields and the solver,
    AMR and output parameters."""

    def __init__(self, ptr):
        self._lib = L.load()
        self.ptr = ptr
        self.problem = Problem(self.s.problem, owner=self)

    @classmethod
    def load(cls, path: str) -> "Config":
        lib = L.load()
        out = C.POINTER(L.ConfigStruct)()
        L.check(lib.cipher_config_load(path.encode(), C.byref(out)), f"cipher_config_load({path})")
        return cls(out)

    @classmethod
    def parse(cls, text: str, basedir: str | None = None) -> "Config":
        lib = L.load()
        b = text.encode()
        out = C.POINTER(L.ConfigStruct)()
        L.check(lib.cipher_config_parse(b, len(b), basedir.encode() if basedir else None, C.byref(out)),
                "cipher_config_parse")
        return cls(out)

    @property
    def s(self) -> L.ConfigStruct:
        return self.ptr.contents

    @property
    def components(self) -> list:
        s = self.s
        return [s.componentname[i].value.decode() for i in range(s.ncomponents)]

    def nucleation_tables(self):
        """(voxelsite, sitephase, sitenucleus, nuclei) or None without sites"""
        s = self.s
        if s.nsites == 0:
            return None
        P = self.problem.s
        n = int(np.prod([P.resolution[d] for d in range(P.dim)]))
        vs = np.ctypeslib.as_array(s.voxelsite, shape=(n,)).copy()
        sp = np.ctypeslib.as_array(s.sitephase, shape=(s.nsites,)).copy()
        sn = np.ctypeslib.as_array(s.sitenucleus, shape=(s.nsites,)).copy()
        nz = (L.Nucleus * max(s.nnuclei, 1))()
        C.memmove(nz, s.nuclei, C.sizeof(L.Nucleus) * s.nnuclei)
        return vs, sp, sn, nz

    def output_spec(self):
        """the header's output fields as [(name, kind, index)]"""
        s = self.s
        inv = {v: k for k, v in OUTPUT_KINDS.items()}
        return [(s.outputs[i].name.decode(), inv[s.outputs[i].kind], s.outputs[i].index) for i in range(s.noutputs)]

    def ts_options(self, **over):
        """stepper options of the configuration: the -ts_rk_type of its
        petscoptions (PETSc's default 3bs), tolerances and step limits"""
        rk = self.s.rk_type.decode()
        if rk not in ("1fe", "2a", "3bs"):
            raise ValueError(f"-ts_rk_type {rk}: the stepper has the 1fe, 2a and 3bs tableaux")
        return ts_options(self.problem, rk, **over)

    def close(self):
        if self.ptr:
            self.problem.ptr = None
            self._lib.cipher_config_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def yaml_to_json(text: str):
    """the configuration parser's reading of a YAML text, as Python objects
    (dicts, lists, strings)"""
    import json
    lib = L.load()
    b = text.encode()
    need = C.c_size_t(0)
    L.check(lib.cipher_yaml_to_json(b, len(b), None, 0, C.byref(need)), "cipher_yaml_to_json")
    buf = C.create_string_buffer(need.value)
    L.check(lib.cipher_yaml_to_json(b, len(b), buf, need.value, C.byref(need)), "cipher_yaml_to_json")
    return json.loads(buf.value.decode())


class Mesh:
    """Owns a ``cipher_mesh`` (uniform grid, whole domain or a slab + halo)."""

    def __init__(self, problem: Problem, slab=None, grid_only: bool = False):
        """grid_only: the face-list-free grid (cipher_mesh_grid), enough for
        a device context but not for the host builders or the oracle"""
        self._lib = L.load()
        s = problem.s
        out = L.MP()
        if grid_only:
            L.check(self._lib.cipher_mesh_grid(problem.ptr, C.byref(out)), "cipher_mesh_grid")
        else:
            lo, hi = (0, s.resolution[s.dim - 1]) if slab is None else slab
            L.check(self._lib.cipher_mesh_uniform(problem.ptr, lo, hi, C.byref(out)), "cipher_mesh_uniform")
        self.ptr = out
        self.problem = problem

    @classmethod
    def adopt(cls, problem: Problem, ptr) -> "Mesh":
        """take ownership of a cipher_mesh built elsewhere (e.g. by a forest)"""
        m = cls.__new__(cls)
        m._lib = L.load()
        m.ptr = ptr
        m.problem = problem
        return m

    @property
    def s(self) -> L.MeshStruct:
        return self.ptr.contents

    @property
    def ncells(self) -> int:
        return self.s.ncells

    @property
    def nowned(self) -> int:
        return self.s.nowned

    def cell_global(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.s.cell_global, shape=(self.ncells,)).copy()

    def close(self):
        if self.ptr:
            self._lib.cipher_mesh_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Forest:
    """An adaptive quadtree / octree mesh (cipher_forest_*): the role the
    reference's p4est forest plays.  Leaves are the cells of `mesh()`."""

    def __init__(self, dim: int, nblocks, lmin: int, lmax: int, linit: int = None, periodic=(1, 1, 1), size=None):
        self._lib = L.load()
        nb = (C.c_int32 * 3)(*(list(nblocks) + [1] * (3 - len(nblocks))))
        per = (C.c_int32 * 3)(*(list(periodic) + [0] * (3 - len(periodic))))
        sz = None if size is None else (C.c_double * 3)(*(list(size) + [1.0] * (3 - len(size))))
        out = C.c_void_p()
        L.check(self._lib.cipher_forest_create(dim, nb, lmin, lmax, lmax if linit is None else linit, per, sz,
                                               C.byref(out)), "cipher_forest_create")
        self.ptr = out
        self.dim = dim

    @property
    def nleaves(self) -> int:
        return int(self._lib.cipher_forest_nleaves(self.ptr))

    def leaves(self):
        """(level[n], corner[n, 3]) on the finest grid"""
        n = self.nleaves
        lev = np.zeros(n, dtype=np.int32)
        cor = np.zeros((n, 3), dtype=np.int32)
        L.check(self._lib.cipher_forest_leaves(self.ptr, lev.ctypes.data_as(C.POINTER(C.c_int32)),
                                               cor.ctypes.data_as(C.POINTER(C.c_int32))), "cipher_forest_leaves")
        return lev, cor

    def resolution(self):
        r = (C.c_int32 * 3)()
        L.check(self._lib.cipher_forest_resolution(self.ptr, r), "cipher_forest_resolution")
        return list(r)

    def mark_active(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float64)
        mark = np.zeros(self.nleaves, dtype=np.int8)
        L.check(self._lib.cipher_forest_mark_active(self.ptr, X.ctypes.data_as(C.POINTER(C.c_double)), X.shape[1],
                                                    mark.ctypes.data_as(C.POINTER(C.c_int8))),
                "cipher_forest_mark_active")
        return mark

    def adapt(self, mark, X: np.ndarray = None, as_size: int = 0):
        """refine / coarsen by marks (+1 / -1 / 0) and balance; with X the
        families whose active sets (first as_size dofs) differ are kept"""
        mark = np.ascontiguousarray(mark, dtype=np.int8)
        xp, nd = None, 0
        if X is not None:
            X = np.ascontiguousarray(X, dtype=np.float64)
            xp, nd = X.ctypes.data_as(C.POINTER(C.c_double)), X.shape[1]
        L.check(self._lib.cipher_forest_adapt(self.ptr, mark.ctypes.data_as(C.POINTER(C.c_int8)), xp, nd, as_size),
                "cipher_forest_adapt")

    def transfer_plan(self):
        n = self.nleaves
        s0 = np.zeros(n, dtype=np.int64)
        ns = np.zeros(n, dtype=np.int32)
        L.check(self._lib.cipher_forest_transfer_plan(self.ptr, s0.ctypes.data_as(C.POINTER(C.c_int64)),
                                                      ns.ctypes.data_as(C.POINTER(C.c_int32))),
                "cipher_forest_transfer_plan")
        return s0, ns

    def transfer_aos(self, Xold: np.ndarray) -> np.ndarray:
        Xold = np.ascontiguousarray(Xold, dtype=np.float64)
        Xnew = np.zeros((self.nleaves, Xold.shape[1]), dtype=np.float64)
        L.check(self._lib.cipher_forest_transfer_aos(self.ptr, Xold.ctypes.data_as(C.POINTER(C.c_double)),
                                                     Xold.shape[1], Xnew.ctypes.data_as(C.POINTER(C.c_double))),
                "cipher_forest_transfer_aos")
        return Xnew

    def mesh(self, problem: "Problem") -> "Mesh":
        out = L.MP()
        L.check(self._lib.cipher_forest_mesh(self.ptr, C.byref(out)), "cipher_forest_mesh")
        return Mesh.adopt(problem, out)

    def close(self):
        if self.ptr:
            self._lib.cipher_forest_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class AMR:
    """Time stepping with adaptive refinement (cipher_amr_*): the reference's
    main loop with its forest - initial coarsening of the SetUpProblem state,
    then an adaptation every `interval` accepted steps, the state moved on the
    device."""

    def __init__(self, problem: Problem, nblocks, lmin: int, lmax: int, initcoarsen: int, interval: int,
                 opts: L.TSOpts, precision: str = "fp64", device: int = 0):
        self._lib = L.load()
        o = L.AMROpts()
        for d, v in enumerate(list(nblocks) + [1] * (3 - len(nblocks))):
            o.nblocks[d] = v
        o.lmin, o.lmax, o.initcoarsen, o.interval = lmin, lmax, initcoarsen, interval
        o.precision = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED}[precision]
        o.device = device
        o.ts = opts
        out = C.c_void_p()
        L.check(self._lib.cipher_amr_create(problem.ptr, C.byref(o), C.byref(out)), "cipher_amr_create")
        self.ptr = out
        self.problem = problem
        self.device = device

    def solve(self, t_end: float, max_steps: int = 0) -> L.TSStats:
        st = L.TSStats()
        L.check(self._lib.cipher_amr_solve(self.ptr, float(t_end), int(max_steps), C.byref(st)), "cipher_amr_solve")
        return st

    def state(self):
        """(context pointer, device state pointer, mesh struct, adaptations)"""
        ctx, X, m, n = C.c_void_p(), C.c_void_p(), L.MP(), C.c_int64()
        L.check(self._lib.cipher_amr_state(self.ptr, C.byref(ctx), C.byref(X), C.byref(m), C.byref(n)),
                "cipher_amr_state")
        return ctx, X, m.contents, n.value

    def state_aos(self) -> np.ndarray:
        """the current state in the reference AoS layout (host)"""
        import torch
        ctx, X, m, _ = self.state()
        out = torch.empty((int(m.ncells), self.problem.ndof), dtype=torch.float64, device=f"cuda:{self.device}")
        L.check(self._lib.cipher_state_to_aos(ctx, X, C.c_void_p(out.data_ptr()), None), "cipher_state_to_aos")
        torch.cuda.synchronize(self.device)
        return out.cpu().numpy()

    def close(self):
        if self.ptr:
            self._lib.cipher_amr_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def initial_state_aos(problem: Problem, mesh: Mesh) -> np.ndarray:
    """SetUpProblem's state (src/init.c:1721-1830) in the reference AoS layout."""
    lib = L.load()
    X = np.zeros((mesh.ncells, problem.ndof), dtype=np.float64)
    L.check(lib.cipher_initial_state_aos(problem.ptr, mesh.ptr, X.ctypes.data_as(C.POINTER(C.c_double))),
            "cipher_initial_state_aos")
    return X


def diffuse_state_aos(problem: Problem, mesh: Mesh, width: float = 4.0) -> np.ndarray:
    """Diffuse-interface Voronoi state (see cipher_initial_state_diffuse_aos)."""
    lib = L.load()
    X = np.zeros((mesh.ncells, problem.ndof), dtype=np.float64)
    L.check(lib.cipher_initial_state_diffuse_aos(problem.ptr, mesh.ptr, float(width),
                                                 X.ctypes.data_as(C.POINTER(C.c_double))),
            "cipher_initial_state_diffuse_aos")
    return X


@dataclass
class TSView:
    """The slice of a PETSc TS the callbacks read: solution, time, step."""
    X: object = None
    t: float = 0.0
    dt: float = 0.0
    step: int = 0


def _ptr(t) -> int:
    return int(t.data_ptr()) if hasattr(t, "data_ptr") else int(t)


def _stream_handle(stream) -> C.c_void_p:
    if stream is None:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if hasattr(stream, "cuda_stream"):
        return C.c_void_p(stream.cuda_stream)
    return C.c_void_p(int(stream))


class Context:
    """A device context (``cipher_ctx``) for one problem on one GPU."""

    def __init__(self, problem: Problem, mesh: Mesh, precision: str = "fp64", device: int = 0):
        self._lib = L.load()
        prec = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED}[precision]
        out = C.c_void_p()
        L.check(self._lib.cipher_ctx_create(problem.ptr, mesh.ptr, prec, device, C.byref(out)),
                "cipher_ctx_create")
        self.ptr = out
        self.problem, self.mesh, self.precision, self.device = problem, mesh, precision, device
        lay = L.StateLayout()
        L.check(self._lib.cipher_ctx_layout(self.ptr, C.byref(lay)), "cipher_ctx_layout")
        self.layout = lay

    # -- buffers -------------------------------------------------------------
    def alloc_state(self):
        import torch
        return torch.zeros(int(self.layout.bytes), dtype=torch.uint8, device=f"cuda:{self.device}")

    def planes(self, X):
        """Typed views (as, phi, dp, ex, tm) of a device state tensor."""
        import torch
        lay = self.layout
        S, P = int(lay.stride), int(lay.pf_size)
        rt = torch.float64 if self.precision == "fp64" else torch.float32
        rb = 8 if self.precision == "fp64" else 4

        def view(off, n, dt, nb):
            return X[off:off + n * S * nb].view(dt).view(n, S) if n else X[0:0].view(dt).view(0, S)
        return (view(int(lay.as_offset), P + 1, torch.int16, 2), view(int(lay.pf_offset), P, rt, rb),
                view(int(lay.dp_offset), int(lay.dp_size), torch.float64, 8),
                view(int(lay.ex_offset), int(lay.ex_size), torch.float64, 8),
                view(int(lay.tm_offset), 1, rt, rb))

    # -- conversions -----------------------------------------------------------
    def from_aos(self, aos, X, stream=None):
        """Device state X <- reference AoS array (numpy host or torch device)."""
        import torch
        if isinstance(aos, np.ndarray):
            aos = torch.from_numpy(np.ascontiguousarray(aos, dtype=np.float64)).to(f"cuda:{self.device}")
        L.check(self._lib.cipher_state_from_aos(self.ptr, C.c_void_p(_ptr(aos)), C.c_void_p(_ptr(X)),
                                                 _stream_handle(stream)), "cipher_state_from_aos")
        return X

    def to_aos(self, X, stream=None) -> np.ndarray:
        import torch
        out = torch.empty((int(self.layout.ncells), self.problem.ndof), dtype=torch.float64,
                          device=f"cuda:{self.device}")
        L.check(self._lib.cipher_state_to_aos(self.ptr, C.c_void_p(_ptr(X)), C.c_void_p(_ptr(out)),
                                               _stream_handle(stream)), "cipher_state_to_aos")
        torch.cuda.synchronize(self.device)
        return out.cpu().numpy()

    # -- the two callbacks -------------------------------------------------------
    def rhs(self, t: float, X, F, stream=None):
        L.check(self._lib.cipher_rhs(self.ptr, float(t), C.c_void_p(_ptr(X)), C.c_void_p(_ptr(F)),
                                     _stream_handle(stream)), "cipher_rhs")

    def poststep(self, X, stream=None):
        L.check(self._lib.cipher_poststep(self.ptr, C.c_void_p(_ptr(X)), _stream_handle(stream)),
                "cipher_poststep")

    def waxpy(self, Y, X, a: float, F, stream=None):
        """Y = X + a*F on the real planes (AS copied from X)."""
        L.check(self._lib.cipher_waxpy(self.ptr, C.c_void_p(_ptr(Y)), C.c_void_p(_ptr(X)), float(a),
                                       C.c_void_p(_ptr(F)), _stream_handle(stream)), "cipher_waxpy")

    def set_rhs_form(self, form: str):
        """FP64 single-interface kernel: "reference" (bit-identical to the
        reference, the default) or "closed" (the closed form in FP64)"""
        f = {"reference": L.RHS_REFERENCE_ORDER, "closed": L.RHS_CLOSED_FORM}[form]
        L.check(self._lib.cipher_ctx_set_rhs_form(self.ptr, f), "cipher_ctx_set_rhs_form")

    def check(self, stream=None):
        L.check(self._lib.cipher_ctx_check(self.ptr, _stream_handle(stream)), "cipher_ctx_check")

    def init_sharp(self, X, stream=None):
        """the SetUpProblem state built on the device from the problem's voxel map"""
        vox = np.ascontiguousarray(self.problem.voxelphase(), dtype=np.int32)
        L.check(self._lib.cipher_state_init_sharp(self.ptr, vox.ctypes.data_as(C.POINTER(C.c_int32)),
                                                  C.c_void_p(_ptr(X)), _stream_handle(stream)),
                "cipher_state_init_sharp")
        return X

    def chem_init(self, X, stream=None):
        """EX and mu of an initial state from the materials' c0 (SetUpProblem)."""
        L.check(self._lib.cipher_chem_init(self.ptr, C.c_void_p(_ptr(X)), _stream_handle(stream)),
                "cipher_chem_init")

    def transfer_from(self, X, src: "Context", Xsrc, forest: "Forest", stream=None):
        """X (this context's adapted mesh) <- Xsrc (src's mesh before the
        forest's last adaptation), by the forest's transfer plan"""
        s0, ns = forest.transfer_plan()
        L.check(self._lib.cipher_state_transfer(self.ptr, C.c_void_p(_ptr(X)), src.ptr, C.c_void_p(_ptr(Xsrc)),
                                                s0.ctypes.data_as(C.POINTER(C.c_int64)),
                                                ns.ctypes.data_as(C.POINTER(C.c_int32)), _stream_handle(stream)),
                "cipher_state_transfer")
        return X

    def RHSFunction(self, ts: TSView, ftime: float, X, F) -> int:
        """Reference-shaped callback: F = RHS(ftime, X); returns 0 like PetscErrorCode."""
        self.rhs(ftime, X, F)
        return 0

    def PostStep(self, ts: TSView) -> int:
        """Reference-shaped callback: active-set update of ts.X in place."""
        self.poststep(ts.X)
        return 0

    def rhs_aos_host(self, t: float, X, F=None, stream=None):
        """Drop-in call on host buffers in the reference AoS layout (numpy
        arrays, or pinned CPU torch tensors for full-speed copies)."""
        if hasattr(X, "data_ptr"):
            xp = C.cast(C.c_void_p(X.data_ptr()), C.POINTER(C.c_double))
            fp = C.cast(C.c_void_p(F.data_ptr()), C.POINTER(C.c_double))
        else:
            X = np.ascontiguousarray(X, dtype=np.float64)
            if F is None:
                F = np.empty_like(X)
            xp = X.ctypes.data_as(C.POINTER(C.c_double))
            fp = F.ctypes.data_as(C.POINTER(C.c_double))
        L.check(self._lib.cipher_rhs_aos_host(self.ptr, float(t), xp, fp, _stream_handle(stream)),
                "cipher_rhs_aos_host")
        return F

    def close(self):
        if self.ptr:
            self._lib.cipher_ctx_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ts_options(problem: Problem, scheme: str = "2a", **kw) -> L.TSOpts:
    """Stepper options from the problem (timestep0, step limits, tolerances),
    overridden by keyword (dt0, dtmin, dtmax, reltol, abstol, max_steps, poststep)."""
    lib = L.load()
    o = L.TSOpts()
    L.check(lib.cipher_ts_default_opts(problem.ptr, C.byref(o)), "cipher_ts_default_opts")
    o.scheme = {"1fe": L.TS_RK1FE, "2a": L.TS_RK2A, "3bs": L.TS_RK3BS}[scheme]
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class TimeStepper:
    """Explicit RK stepper with embedded error control on device states
    (cipher_ts_*): the role PETSc's TSRK + TSADAPTDSP play for the reference."""

    def __init__(self, ctx: Context, opts: L.TSOpts):
        self._lib = L.load()
        self.ctx, self.opts = ctx, opts
        out = C.c_void_p()
        L.check(self._lib.cipher_ts_create(ctx.ptr, C.byref(opts), C.byref(out)), "cipher_ts_create")
        self.ptr = out

    def step(self, X, t_end: float, stream=None) -> bool:
        acc = C.c_int(0)
        L.check(self._lib.cipher_ts_step(self.ptr, C.c_void_p(_ptr(X)), float(t_end), C.byref(acc),
                                         _stream_handle(stream)), "cipher_ts_step")
        return bool(acc.value)

    def solve(self, X, t0: float, t_end: float, stream=None) -> L.TSStats:
        st = L.TSStats()
        L.check(self._lib.cipher_ts_solve(self.ptr, C.c_void_p(_ptr(X)), float(t0), float(t_end), C.byref(st),
                                          _stream_handle(stream)), "cipher_ts_solve")
        return st

    def stats(self) -> L.TSStats:
        st = L.TSStats()
        L.check(self._lib.cipher_ts_get_stats(self.ptr, C.byref(st)), "cipher_ts_get_stats")
        return st

    def set_dt(self, dt: float):
        L.check(self._lib.cipher_ts_set_dt(self.ptr, float(dt)), "cipher_ts_set_dt")

    def set_nucleation(self, nu):
        L.check(self._lib.cipher_ts_set_nucleation(self.ptr, nu.ptr if nu is not None else None),
                "cipher_ts_set_nucleation")
        self._nu = nu

    def close(self):
        if self.ptr:
            self._lib.cipher_ts_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent domains stepped together (cipher_batch_*): each with
    its own step size and error control, all in one graph launch per step."""

    def __init__(self, opts: L.TSOpts, precision: str = "fp64", device: int = 0, graphs: bool = True):
        self._lib = L.load()
        out = C.c_void_p()
        prec = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED}[precision]
        L.check(self._lib.cipher_batch_create(device, prec, C.byref(opts), C.byref(out)), "cipher_batch_create")
        self.ptr = out
        self._keep = {}
        if not graphs:
            L.check(self._lib.cipher_batch_set_graphs(self.ptr, 0), "cipher_batch_set_graphs")

    def footprint(self, ctx: Context) -> int:
        v = C.c_int64()
        L.check(self._lib.cipher_batch_footprint(self.ptr, ctx.ptr, C.byref(v)), "cipher_batch_footprint")
        return int(v.value)

    def attach(self, ctx: Context, X, t0: float, t_end: float) -> int:
        slot = C.c_int()
        L.check(self._lib.cipher_batch_attach(self.ptr, ctx.ptr, C.c_void_p(_ptr(X)), float(t0), float(t_end),
                                              C.byref(slot)), "cipher_batch_attach")
        self._keep[slot.value] = (ctx, X)
        return slot.value

    def detach(self, slot: int):
        L.check(self._lib.cipher_batch_detach(self.ptr, int(slot)), "cipher_batch_detach")
        self._keep.pop(slot, None)

    def step(self) -> int:
        running = C.c_int()
        L.check(self._lib.cipher_batch_step(self.ptr, C.byref(running)), "cipher_batch_step")
        return running.value

    def flush(self):
        L.check(self._lib.cipher_batch_flush(self.ptr), "cipher_batch_flush")

    def stats(self, slot: int):
        st, status, err = L.TSStats(), C.c_int(), C.c_int()
        L.check(self._lib.cipher_batch_slot_stats(self.ptr, int(slot), C.byref(st), C.byref(status), C.byref(err)),
                "cipher_batch_slot_stats")
        return st, status.value, err.value

    def close(self):
        if self.ptr:
            self._lib.cipher_batch_destroy(self.ptr)
            self.ptr = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request loop (cipher_server_*): requests are
    admitted in arrival order while they fit the HBM budget and stepped
    together; each result equals the request solved alone."""

    def __init__(self, opts: L.TSOpts, precision: str = "fp64", device: int = 0, hbm_budget: int = 8 << 30,
                 max_active: int = 256):
        self._lib = L.load()
        so = L.ServerOpts()
        so.device = device
        so.precision = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED}[precision]
        so.max_active = max_active
        so.hbm_budget = hbm_budget
        so.ts = opts
        out = C.c_void_p()
        L.check(self._lib.cipher_server_create(C.byref(so), C.byref(out)), "cipher_server_create")
        self.ptr = out

    def submit(self, problem: Problem, t_end: float, init: str = "diffuse", width: float = 4.0) -> int:
        """queue a request; the server takes ownership of the problem"""
        rid = C.c_int64()
        kind = {"sharp": L.INIT_SHARP, "diffuse": L.INIT_DIFFUSE}[init]
        L.check(self._lib.cipher_server_submit(self.ptr, problem.ptr, kind, float(width), float(t_end),
                                               C.byref(rid)), "cipher_server_submit")
        problem.ptr = None          # owned by the server now
        return rid.value

    def poll(self):
        q, a, d = C.c_int(), C.c_int(), C.c_int()
        L.check(self._lib.cipher_server_poll(self.ptr, C.byref(q), C.byref(a), C.byref(d)), "cipher_server_poll")
        return q.value, a.value, d.value

    def result(self, rid: int, with_state: bool = False):
        r = L.ServerResult()
        L.check(self._lib.cipher_server_result(self.ptr, int(rid), C.byref(r), None), "cipher_server_result")
        X = None
        if with_state and r.state == 2:
            X = np.empty((int(r.ncells), int(r.ndof)), dtype=np.float64)
            L.check(self._lib.cipher_server_result(self.ptr, int(rid), C.byref(r),
                                                   X.ctypes.data_as(C.POINTER(C.c_double))), "cipher_server_result")
        return r, X

    def release(self, rid: int):
        L.check(self._lib.cipher_server_release(self.ptr, int(rid)), "cipher_server_release")

    def counters(self) -> dict:
        c = L.ServerCounters()
        L.check(self._lib.cipher_server_get_counters(self.ptr, C.byref(c)), "cipher_server_get_counters")
        return {k: getattr(c, k) for k, _ in L.ServerCounters._fields_}

    def usage(self):
        u, p = C.c_int64(), C.c_int64()
        L.check(self._lib.cipher_server_usage(self.ptr, C.byref(u), C.byref(p)), "cipher_server_usage")
        return u.value, p.value

    def close(self):
        if self.ptr:
            self._lib.cipher_server_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


CIPHER_MAXCP_PY = 1 << 20     # an index past every component: the field is zero

OUTPUT_KINDS = {"phaseid": L.OUT_PHASEID, "matid": L.OUT_MATID, "interfaceid": L.OUT_INTERFACEID,
                "chempot": L.OUT_CHEMPOT, "c": L.OUT_COMP, "phi": L.OUT_PHI, "temperature": L.OUT_TEMPERATURE}


def output_fields(spec):
    """[(name, kind, index)] -> ctypes array of cipher_output_field; kind is a
    key of OUTPUT_KINDS (the reference's output names: phaseid, matid,
    interfaceid, <comp>_chempot, <comp>_c, <phase>_phi, temperature)"""
    arr = (L.OutputField * len(spec))()
    for k, (name, kind, index) in enumerate(spec):
        arr[k].kind = OUTPUT_KINDS[kind]
        arr[k].index = int(index)
        arr[k].name = name.encode()[:47]
    return arr


def _atoi(tok: str) -> int:
    """C atoi: optional sign and leading digits, 0 when there are none"""
    m = re.match(r"\s*([+-]?\d+)", tok)
    return int(m.group(1)) if m else 0


def output_spec(names, components):
    """[(name, kind, index)] for the reference's output names, read as its
    output step reads them (src/cipher.c:1005-1080): "phaseid", "matid",
    "interfaceid" and "temperature" by name; a name holding "_chempot",
    else "_c", else "_phi" takes the text before its first "_" as the
    component (looked up in `components`; no match gives a zero field, as the
    reference leaves the field at zero) or the phase id (C atoi)"""
    spec = []
    for name in names:
        tok = name.lstrip("_").split("_", 1)[0]          # strtok_r(name, "_")
        if name in ("phaseid", "matid", "interfaceid", "temperature"):
            spec.append((name, name, 0))
        elif "_chempot" in name or "_c" in name:
            # the potentials hold the first ncp-1 components: the last one's
            # position is past them and gives zero, as in the reference
            idx = components.index(tok) if tok in components else CIPHER_MAXCP_PY
            spec.append((name, "chempot" if "_chempot" in name else "c", idx))
        elif "_phi" in name:
            spec.append((name, "phi", _atoi(tok)))
        else:
            raise ValueError(f"unknown output field {name!r}")
    return spec


def compute_output(ctx: Context, X, spec, stream=None) -> np.ndarray:
    """the derived fields of device state X: [nfields, ncells] (host)"""
    import torch
    fields = output_fields(spec)
    out = torch.empty((len(spec), int(ctx.layout.ncells)), dtype=torch.float64, device=f"cuda:{ctx.device}")
    L.check(ctx._lib.cipher_output_fields(ctx.ptr, C.c_void_p(_ptr(X)), C.cast(fields, C.c_void_p), len(spec),
                                          C.c_void_p(_ptr(out)), _stream_handle(stream)), "cipher_output_fields")
    return out.cpu().numpy()


def write_vtu(path: str, problem: Problem, spec, values: np.ndarray):
    """a .vtu file of the problem's grid with cell data values[nfields, ncells]"""
    fields = output_fields(spec)
    v = np.ascontiguousarray(values, dtype=np.float64)
    L.check(L.load().cipher_write_vtu(path.encode(), problem.ptr, C.cast(fields, C.c_void_p), len(spec),
                                      v.ctypes.data_as(C.POINTER(C.c_double))), "cipher_write_vtu")


def nuclei_array(specs) -> "C.Array":
    """ctypes array of cipher_nucleus from dicts of its fields (matrix and
    active_solutes as lists)"""
    arr = (L.Nucleus * len(specs))()
    for k, d in enumerate(specs):
        for key, val in d.items():
            if key == "matrix":
                arr[k].nmatrix = len(val)
                for j, v in enumerate(sorted(val)):
                    arr[k].matrix[j] = int(v)
            elif key in ("active_solutes", "solvus_temperature_c", "enthalpy_fusion_c"):
                for j, v in enumerate(val):
                    getattr(arr[k], key)[j] = v
            else:
                setattr(arr[k], key, val)
    return arr


class Nucleation:
    """Nucleation sites of a context (cipher_nucleation_*)."""

    def __init__(self, ctx: Context, voxelsite, sitephase, sitenucleus, nuclei, seed: int = 1):
        self._lib = L.load()
        self.ctx = ctx
        self.voxelsite = np.ascontiguousarray(voxelsite, dtype=np.int32)
        self.sitephase = np.ascontiguousarray(sitephase, dtype=np.int32)
        self.sitenucleus = np.ascontiguousarray(sitenucleus, dtype=np.int32)
        self.nuclei = nuclei if isinstance(nuclei, C.Array) else nuclei_array(nuclei)
        self.nsites = len(self.sitephase)
        out = C.c_void_p()
        i32 = C.POINTER(C.c_int32)
        L.check(self._lib.cipher_nucleation_create(ctx.ptr, self.nsites, self.voxelsite.ctypes.data_as(i32),
                                                   self.sitephase.ctypes.data_as(i32),
                                                   self.sitenucleus.ctypes.data_as(i32), len(self.nuclei),
                                                   C.cast(self.nuclei, C.c_void_p), int(seed), C.byref(out)),
                "cipher_nucleation_create")
        self.ptr = out

    def step(self, X, t: float, dt: float, stream=None) -> int:
        nf = C.c_int()
        L.check(self._lib.cipher_nucleation_step(self.ptr, C.c_void_p(_ptr(X)), float(t), float(dt), C.byref(nf),
                                                 _stream_handle(stream)), "cipher_nucleation_step")
        return nf.value

    def sites(self) -> dict:
        n = self.nsites
        act = np.zeros(n, dtype=np.int8)
        arrs = [np.zeros(n) for _ in range(4)]
        d = C.POINTER(C.c_double)
        L.check(self._lib.cipher_nucleation_sites(self.ptr, act.ctypes.data_as(C.POINTER(C.c_int8)),
                                                  *[a.ctypes.data_as(d) for a in arrs]), "cipher_nucleation_sites")
        return {"active": act, "barrier": arrs[0], "diffusivity": arrs[1], "temperature": arrs[2],
                "volume": arrs[3]}

    def close(self):
        if self.ptr:
            self._lib.cipher_nucleation_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
