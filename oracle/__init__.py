"""CPU oracles for CIPHER's RHS and per-step active-set update.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py``; the product never imports it.

Two oracles:

* ``port``: this project's C restatement (oracle/port/*.c), built into
  ``oracle/liboracle_port.so``.
* ``ref``: the reference's own src/{typedef,utility,material,init,cipher}.c
  compiled unmodified against the PETSc shim (oracle/shim, with a replay of
  libyaml's event API for init.c) into ``oracle/_ref/libcipher_ref.so``;
  built where the reference sources exist and shipped as a prebuilt library
  elsewhere.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "liboracle_port.so")
REF_LIB = os.path.join(HERE, "_ref", "libcipher_ref.so")
# the reference's src/ directory: CIPHER_REF_SRC, else the location the
# build recipe (oracle/Makefile) assumes
REF_SRC = os.environ.get("CIPHER_REF_SRC") or "/root/reference/src"
# the reference's project root (its examples/ live there), when present
REF_ROOT = os.path.dirname(REF_SRC) if os.path.isdir(REF_SRC) else None

_port = None
_ref = None


def build(ref: bool = True) -> None:
    """Compile the port (and the reference build when its sources exist)."""
    targets = ["port"]
    if ref and os.path.isdir(REF_SRC):
        targets.append("ref")
    r = subprocess.run(["make", "-s", "-C", HERE, f"REF_SRC={REF_SRC}"] + targets, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_LIB):
            build(ref=False)
        lib = C.CDLL(PORT_LIB)
        lib.oracle_rhs.restype = C.c_int
        lib.oracle_rhs.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.oracle_poststep.restype = C.c_int
        lib.oracle_poststep.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]
        lib.oracle_initial_state.restype = C.c_int
        lib.oracle_initial_state.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]
        lib.oracle_output_fields.restype = C.c_int
        lib.oracle_output_fields.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32),
                                             C.POINTER(C.c_int32), C.c_int, C.POINTER(C.c_double)]
        lib.oracle_nucleation_step.restype = C.c_int
        lib.oracle_nucleation_step.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_int,
                                               C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                               C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_uint64),
                                               C.POINTER(C.c_int8), C.POINTER(C.c_double)]
        lib.oracle_nucleation_threshold.restype = C.c_double
        lib.oracle_nucleation_threshold.argtypes = [C.c_void_p, C.c_int] + [C.c_double] * 6 + [C.POINTER(C.c_int)]
        lib.oracle_ts_create.restype = C.c_void_p
        lib.oracle_ts_create.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.oracle_ts_destroy.restype = None
        lib.oracle_ts_destroy.argtypes = [C.c_void_p]
        lib.oracle_ts_step.restype = C.c_int
        lib.oracle_ts_step.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_double, C.POINTER(C.c_int)]
        lib.oracle_ts_solve.restype = C.c_int
        lib.oracle_ts_solve.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_double, C.c_double, C.c_void_p]
        lib.oracle_ts_get_stats.restype = None
        lib.oracle_ts_get_stats.argtypes = [C.c_void_p, C.c_void_p]
        lib.or_simplex_projection.restype = None
        lib.or_simplex_projection.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]
        _port = lib
    return _port


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError(f"{REF_LIB} not built (needs the reference sources)")
        lib = C.CDLL(REF_LIB)
        lib.ref_create.restype = C.c_int
        lib.ref_create.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_destroy.restype = None
        lib.ref_destroy.argtypes = []
        lib.ref_ndof.restype = C.c_int
        lib.ref_rhs.restype = C.c_int
        lib.ref_rhs.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.ref_poststep.restype = C.c_int
        lib.ref_poststep.argtypes = [C.POINTER(C.c_double), C.c_double, C.POINTER(C.c_double), C.c_int,
                                     C.POINTER(C.c_double)]
        lib.ref_set_nuclei.restype = C.c_int
        lib.ref_set_nuclei.argtypes = [C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int, C.c_void_p]
        lib.ref_nucleation_sites.restype = C.c_int
        lib.ref_nucleation_sites.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_int8),
                                             C.POINTER(C.c_double)]
        lib.ref_nucleation_event.restype = C.c_int
        lib.ref_nucleation_event.argtypes = [C.c_int] + [C.c_double] * 6 + [C.c_uint, C.POINTER(C.c_double)]
        lib.ref_output_fields.restype = C.c_int
        lib.ref_output_fields.argtypes = [C.POINTER(C.c_double), C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                          C.POINTER(C.c_double)]
        _ref = lib
    return _ref


def _addr(obj) -> C.c_void_p:
    """ctypes pointer of a cipher_b200 Problem/Mesh (or a raw pointer)."""
    p = getattr(obj, "ptr", obj)
    return C.cast(p, C.c_void_p)


# ---------------------------------------------------------------- port ----

def port_rhs(problem, mesh, X: np.ndarray, t: float = 0.0) -> np.ndarray:
    """F over owned cells; X holds owned then ghost cells (AoS doubles)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    F = np.zeros((mesh.nowned, X.shape[1]), dtype=np.float64)
    rc = port().oracle_rhs(_addr(problem), _addr(mesh), t, _dp(X), _dp(F))
    if rc:
        raise RuntimeError(f"oracle_rhs failed ({rc})")
    return F


def port_poststep(problem, mesh, X: np.ndarray) -> int:
    """Active-set update in place; returns 0, or 3 when a superset exceeds P."""
    assert X.flags.c_contiguous and X.dtype == np.float64
    return port().oracle_poststep(_addr(problem), _addr(mesh), _dp(X))


def port_initial_state(problem, mesh) -> np.ndarray:
    X = np.zeros((mesh.ncells, problem.ndof), dtype=np.float64)
    rc = port().oracle_initial_state(_addr(problem), _addr(mesh), _dp(X))
    if rc:
        raise RuntimeError(f"oracle_initial_state failed ({rc})")
    return X


def port_output_fields(problem, mesh, X: np.ndarray, kinds, idx) -> np.ndarray:
    """the output step's derived fields of the owned cells: [nfields, nowned]"""
    X = np.ascontiguousarray(X, dtype=np.float64)
    k = np.ascontiguousarray(kinds, dtype=np.int32)
    i = np.ascontiguousarray(idx, dtype=np.int32)
    out = np.zeros((len(k), mesh.nowned), dtype=np.float64)
    rc = port().oracle_output_fields(_addr(problem), _addr(mesh), _dp(X), k.ctypes.data_as(C.POINTER(C.c_int32)),
                                     i.ctypes.data_as(C.POINTER(C.c_int32)), len(k), _dp(out))
    if rc:
        raise RuntimeError(f"oracle_output_fields failed ({rc})")
    return out


def port_nucleation_threshold(nucleus, dim, t, dt, T, volume, gv, diffusivity):
    """(draws, threshold) of the event rule of a nucleus (a cipher_nucleus
    structure): the event fires when a draw happens and the number drawn is
    below the threshold"""
    draw = C.c_int(0)
    thr = port().oracle_nucleation_threshold(C.addressof(nucleus), dim, t, dt, T, volume, gv, diffusivity,
                                              C.byref(draw))
    return bool(draw.value), thr


class PortNucleation:
    """CPU restatement of nucleation with the library's event stream."""

    def __init__(self, problem, mesh, voxelsite, sitephase, sitenucleus, nuclei, seed: int = 1):
        self.problem, self.mesh = problem, mesh
        self.voxelsite = np.ascontiguousarray(voxelsite, dtype=np.int32)
        self.sitephase = np.ascontiguousarray(sitephase, dtype=np.int32)
        self.sitenucleus = np.ascontiguousarray(sitenucleus, dtype=np.int32)
        self.nuclei = nuclei
        self.nsites = len(self.sitephase)
        self.rng = C.c_uint64(int(seed))
        self.active = np.ones(self.nsites, dtype=np.int8)
        self.last = np.full((self.nsites, 4), np.nan)

    def step(self, X: np.ndarray, t: float, dt: float) -> int:
        assert X.flags.c_contiguous and X.dtype == np.float64
        out = np.full((self.nsites, 4), np.nan)
        i32 = C.POINTER(C.c_int32)
        nf = port().oracle_nucleation_step(_addr(self.problem), _addr(self.mesh), _dp(X), self.nsites,
                                           self.voxelsite.ctypes.data_as(i32), self.sitephase.ctypes.data_as(i32),
                                           self.sitenucleus.ctypes.data_as(i32), C.cast(self.nuclei, C.c_void_p),
                                           t, dt, C.byref(self.rng), self.active.ctypes.data_as(C.POINTER(C.c_int8)),
                                           _dp(out))
        if nf < 0:
            raise RuntimeError("oracle_nucleation_step failed")
        ev = ~np.isnan(out[:, 0])
        self.last[ev] = out[ev]
        return nf


def simplex_projection(v: np.ndarray) -> np.ndarray:
    v = np.ascontiguousarray(v, dtype=np.float64)
    out = np.zeros_like(v)
    port().or_simplex_projection(_dp(out), _dp(v), len(v))
    return out


class PortTS:
    """The CPU restatement of the library's RK stepper over the oracle RHS.
    `opts` and the returned stats are cipher_b200._lib.TSOpts / TSStats."""

    def __init__(self, problem, mesh, opts):
        self.lib = port()
        self.ptr = self.lib.oracle_ts_create(_addr(problem), _addr(mesh), C.cast(C.pointer(opts), C.c_void_p))
        if not self.ptr:
            raise RuntimeError("oracle_ts_create failed")
        self.problem, self.mesh = problem, mesh

    def step(self, X: np.ndarray, t_end: float) -> bool:
        assert X.flags.c_contiguous and X.dtype == np.float64
        acc = C.c_int(0)
        rc = self.lib.oracle_ts_step(self.ptr, _dp(X), t_end, C.byref(acc))
        if rc:
            raise RuntimeError(f"oracle_ts_step failed ({rc})")
        return bool(acc.value)

    def solve(self, X: np.ndarray, t0: float, t_end: float, stats):
        assert X.flags.c_contiguous and X.dtype == np.float64
        rc = self.lib.oracle_ts_solve(self.ptr, _dp(X), t0, t_end, C.cast(C.pointer(stats), C.c_void_p))
        if rc:
            raise RuntimeError(f"oracle_ts_solve failed ({rc})")
        return stats

    def stats(self, stats):
        self.lib.oracle_ts_get_stats(self.ptr, C.cast(C.pointer(stats), C.c_void_p))
        return stats

    def close(self):
        if self.ptr:
            self.lib.oracle_ts_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------- ref ----

class RefOracle:
    """The reference's RHSFunction/PostStep on one problem (one at a time)."""

    def __init__(self, problem, mesh, nucleation=None):
        """nucleation = (sitephase, sitenucleus, nuclei) makes the reference's
        nucleation helpers usable (nucleation_sites / nucleation_event)"""
        self.lib = ref()
        self.nsites = 0
        if nucleation is not None:
            sp, sn, nz = nucleation
            self._sp = np.ascontiguousarray(sp, dtype=np.int32)
            self._sn = np.ascontiguousarray(sn, dtype=np.int32)
            self.nsites = len(self._sp)
            i32 = C.POINTER(C.c_int32)
            rc = self.lib.ref_set_nuclei(self.nsites, self._sp.ctypes.data_as(i32), self._sn.ctypes.data_as(i32),
                                         len(nz), C.cast(nz, C.c_void_p))
            if rc:
                raise RuntimeError(f"ref_set_nuclei failed ({rc})")
        rc = self.lib.ref_create(_addr(problem), _addr(mesh))
        if rc:
            raise RuntimeError(f"ref_create failed ({rc})")
        self.problem, self.mesh = problem, mesh
        self.ndof = self.lib.ref_ndof()

    def rhs(self, X: np.ndarray, t: float = 0.0, with_time: bool = False):
        """X: owned then ghost cells (AoS); returns F over owned cells."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        nown = self.mesh.nowned
        own = np.ascontiguousarray(X[:nown])
        ghost = np.ascontiguousarray(X[nown:]) if X.shape[0] > nown else np.zeros((1, self.ndof))
        F = np.zeros_like(own)
        sec = C.c_double(0.0)
        rc = self.lib.ref_rhs(t, _dp(own), _dp(ghost), _dp(F), C.byref(sec))
        if rc:
            raise RuntimeError(f"reference RHSFunction failed ({rc})")
        return (F, sec.value) if with_time else F

    def poststep(self, X: np.ndarray, t: float = 0.0, dt: float = 0.0, step: int = 1) -> int:
        assert X.flags.c_contiguous and X.dtype == np.float64
        d = C.c_double(dt)
        return self.lib.ref_poststep(_dp(X), t, C.byref(d), step, None)

    def setup_problem(self, cellphase) -> np.ndarray:
        """the reference's SetUpProblem (src/init.c:1721-1830): the initial
        state of the owned cells from the phase of each cell"""
        cp = np.ascontiguousarray(cellphase, dtype=np.int32)
        X = np.zeros((self.mesh.nowned, self.ndof))
        self.lib.ref_setup_problem.restype = C.c_int
        self.lib.ref_setup_problem.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_int32)]
        rc = self.lib.ref_setup_problem(_dp(X), cp.ctypes.data_as(C.POINTER(C.c_int32)))
        if rc:
            raise RuntimeError(f"reference SetUpProblem failed ({rc})")
        return X

    def nucleation_sites(self, X: np.ndarray, cellsite, active=None):
        """the reference's per-site (barrier, diffusivity, temperature,
        volume) of state X, NaN rows for sites not evaluated; returns (out,
        active) with retired sites cleared"""
        X = np.ascontiguousarray(X, dtype=np.float64)
        cs = np.ascontiguousarray(cellsite, dtype=np.int32)
        act = np.ones(self.nsites, dtype=np.int8) if active is None else np.array(active, dtype=np.int8)
        out = np.full((max(self.nsites, 1), 4), np.nan)
        rc = self.lib.ref_nucleation_sites(_dp(X), cs.ctypes.data_as(C.POINTER(C.c_int32)),
                                           act.ctypes.data_as(C.POINTER(C.c_int8)), _dp(out))
        if rc:
            raise RuntimeError(f"ref_nucleation_sites failed ({rc})")
        return out[:self.nsites], act

    def nucleation_event(self, site, t, dt, T, volume, gv, diffusivity, seed):
        """(fired, first number the reference's generator gives for seed)"""
        draw = C.c_double(0.0)
        e = self.lib.ref_nucleation_event(site, t, dt, T, volume, gv, diffusivity, seed, C.byref(draw))
        if e < 0:
            raise RuntimeError("ref_nucleation_event failed")
        return bool(e), draw.value

    def output_fields(self, X: np.ndarray, names, components, t: float = 0.0, step: int = 0) -> np.ndarray:
        """the reference's PostStep with its output step on X (in place):
        the fields it writes, [len(names), nowned]"""
        assert X.flags.c_contiguous and X.dtype == np.float64
        nb = [n.encode() for n in names]
        cb_ = [c.encode() for c in components]
        na = (C.c_char_p * len(nb))(*nb)
        ca = (C.c_char_p * max(len(cb_), 1))(*cb_)
        out = np.zeros((self.mesh.nowned, len(nb)))
        rc = self.lib.ref_output_fields(_dp(X), t, step, len(nb), C.cast(na, C.c_void_p), C.cast(ca, C.c_void_p),
                                        _dp(out))
        if rc:
            raise RuntimeError(f"ref_output_fields failed ({rc})")
        return np.ascontiguousarray(out.T)

    def close(self):
        if self.lib is not None:
            self.lib.ref_destroy()
            self.lib = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
