"""The reference's own SetUpConfig (src/init.c:104-1716) on a configuration
file, its result written as arrays (test infrastructure: the checker of the
library's configuration loader).

libyaml is not installed, so the file's YAML events come from PyYAML (whose
event model is libyaml's) and are replayed to the reference's GetProperty
through oracle/shim/include/yaml.h.  The reference asserts on a file it
cannot use, which aborts the process, so this runs as its own process:

    python -m oracle.config_dump CONFIG.yaml OUT.npz

and the exit status tells whether the reference accepted the file.
"""
import ctypes as C
import sys

import numpy as np
import yaml

EVENT_CODES = {yaml.StreamStartEvent: 1, yaml.StreamEndEvent: 2, yaml.DocumentStartEvent: 3,
               yaml.DocumentEndEvent: 4, yaml.AliasEvent: 5, yaml.ScalarEvent: 6, yaml.SequenceStartEvent: 7,
               yaml.SequenceEndEvent: 8, yaml.MappingStartEvent: 9, yaml.MappingEndEvent: 10}


def events_of(text: str):
    types, values = [], []
    for ev in yaml.parse(text):
        types.append(EVENT_CODES[type(ev)])
        values.append(ev.value if isinstance(ev, yaml.ScalarEvent) else None)
    return types, values


def dump(path: str, out: str) -> None:
    import oracle
    from cipher_b200 import _lib as L
    lib = oracle.ref()
    lib.ref_config_events.restype = C.c_int
    lib.ref_config_events.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_char_p)]
    lib.ref_config_load.restype = C.c_int
    lib.ref_config_load.argtypes = [C.c_char_p]
    lib.ref_config_export.restype = C.c_int
    lib.ref_config_export.argtypes = [C.POINTER(L.ProblemStruct), C.POINTER(C.c_int64)]
    lib.ref_config_sites.restype = C.c_int
    lib.ref_config_sites.argtypes = [C.POINTER(C.c_int32)] * 3 + [C.c_void_p]
    lib.ref_config_string.restype = C.c_int
    lib.ref_config_string.argtypes = [C.c_int, C.c_int, C.c_char_p, C.c_int]

    text = open(path, encoding="utf-8", errors="surrogateescape").read()
    types, values = events_of(text)
    t = (C.c_int * len(types))(*types)
    v = (C.c_char_p * len(values))(*[None if x is None else x.encode() for x in values])
    assert lib.ref_config_events(len(types), t, v) == 0
    rc = lib.ref_config_load(path.encode())
    if rc:
        raise SystemExit(3)
    P = L.ProblemStruct()
    info = (C.c_int64 * 14)()
    assert lib.ref_config_export(C.byref(P), info) == 0
    nsites, nnuclei, noutputs, ncp = info[0], info[1], info[2], info[3]
    total = int(np.prod([P.resolution[d] for d in range(3)]))
    vs = np.full(total if nsites else 1, -1, dtype=np.int32)
    sp = np.zeros(max(nsites, 1), dtype=np.int32)
    sn = np.zeros(max(nsites, 1), dtype=np.int32)
    nz = (L.Nucleus * max(nnuclei, 1))()
    i32 = C.POINTER(C.c_int32)
    assert lib.ref_config_sites(vs.ctypes.data_as(i32), sp.ctypes.data_as(i32), sn.ctypes.data_as(i32),
                                C.cast(nz, C.c_void_p)) == 0
    buf = C.create_string_buffer(8192)

    def string(kind, i):
        assert lib.ref_config_string(kind, i, buf, 8192) == 0
        return buf.value.decode()

    scalars = {f: getattr(P, f) for f in ("dim", "npf", "ncp", "ndp", "nmat", "nf", "nbcs", "pf_size", "maxsites",
                                          "interpolation", "gradient_calculation", "junctionpenalty", "nloadcases",
                                          "has_temperature_rate", "timestep0", "mintimestep", "maxtimestep",
                                          "reltol", "abstol")}
    np.savez_compressed(
        out,
        scalars=np.array([scalars[k] for k in sorted(scalars)], dtype=np.float64),
        scalar_names=np.array(sorted(scalars)),
        resolution=np.array(list(P.resolution)), size=np.array(list(P.size)),
        time=np.array(list(P.time)), temperature_rate=np.array(list(P.temperature_rate)),
        material=np.frombuffer(C.string_at(P.material, P.nmat * C.sizeof(L.Material)), dtype=np.uint8),
        interface=np.frombuffer(C.string_at(P.interface, P.nf * C.sizeof(L.Interface)), dtype=np.uint8),
        bcs=np.frombuffer(C.string_at(C.addressof(P.bcs), P.nbcs * C.sizeof(L.BC)), dtype=np.uint8),
        interfacelist=np.ctypeslib.as_array(P.interfacelist, shape=(P.npf * P.npf,)).copy(),
        phasematerialmapping=np.ctypeslib.as_array(P.phasematerialmapping, shape=(P.npf,)).copy(),
        voxelphase=np.ctypeslib.as_array(P.voxelphase, shape=(total,)).copy(),
        info=np.array(list(info)), voxelsite=vs, sitephase=sp, sitenucleus=sn,
        nuclei=np.frombuffer(C.string_at(nz, nnuclei * C.sizeof(L.Nucleus)), dtype=np.uint8),
        components=np.array([string(0, i) for i in range(ncp)]),
        outputs=np.array([string(1, i) for i in range(noutputs)] or [""]),
        outfile=np.array(string(2, 0)), petscoptions=np.array(string(3, 0)))


if __name__ == "__main__":
    dump(sys.argv[1], sys.argv[2])
