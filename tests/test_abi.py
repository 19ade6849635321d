"""The C ABI library loads, exports every symbol include/*.h declares, and its
structs match the Python mirrors (CPU only; no compute calls on a device)."""
import ctypes as C
import os
import re

import cipher_b200._lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in ("cipher_b200.h", "cipher_problem.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(cipher_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_loads_and_exports_declared_symbols():
    lib = L.load()
    declared = _declared()
    assert len(declared) >= 20
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    # every declared symbol is bound with a signature in the Python mirror
    unbound = sorted(declared - set(L.EXPORTED))
    assert not unbound, unbound


def test_struct_sizes_match_mirrors():
    lib = L.load()
    out = (C.c_int64 * 12)()
    assert lib.cipher_abi_sizes(out, 12) == 12
    mirrors = [L.TSeries, L.RK, L.Mobility, L.Source, L.Material, L.Interface, L.BC, L.ProblemStruct,
               L.MeshStruct, L.Nucleus, L.OutputField, L.ConfigStruct]
    for size, m in zip(out, mirrors):
        assert size == C.sizeof(m), (m.__name__, size, C.sizeof(m))


def test_error_strings():
    lib = L.load()
    for code in range(0, 9):
        assert lib.cipher_strerror(code)
    assert b"cap" in lib.cipher_strerror(L.E_CAP)


def test_ctx_create_rejects_bad_input_without_device():
    """Argument checks run before any CUDA call."""
    lib = L.load()
    out = C.c_void_p()
    assert lib.cipher_ctx_create(None, None, 0, 0, C.byref(out)) == L.E_ARG
