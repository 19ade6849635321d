"""Compare a configuration read by the library (cipher_b200.Config) with
the reference's own SetUpConfig result as dumped by oracle.config_dump."""
import ctypes as C

import numpy as np

from cipher_b200 import _lib as L


def _bytes(ptr, n, T):
    return np.frombuffer(C.string_at(ptr, n * C.sizeof(T)), dtype=np.uint8) if n else np.zeros(0, np.uint8)


def _defined_materials(raw, nmat):
    """the reference's material tables with the one field it leaves
    unset: the T*ln(T) coefficient of the calphad2sl Redlich-Kister series
    (src/init.c:715-790 never assigns it; malloc'd memory), which the library
    sets to 0"""
    m = (L.Material * nmat).from_buffer_copy(raw.tobytes())
    for k in range(nmat):
        if m[k].model != L.CHEM_CALPHAD2SL:
            continue
        for tab in (m[k].binary, m[k].binaryq, m[k].ternary, m[k].ternaryq):
            for r in tab:
                for j in range(r.n):
                    r.h[j].logcoeff = 0.0
    return np.frombuffer(bytes(m), dtype=np.uint8)


def compare(cfg, g):
    """list of differences between Config `cfg` and dump `g` (empty: equal)"""
    P = cfg.problem.s
    diffs = []
    names = [str(n) for n in g["scalar_names"]]
    for name, v in zip(names, g["scalars"]):
        if float(getattr(P, name)) != float(v):
            diffs.append(f"{name}: {getattr(P, name)} != {v}")
    if list(P.resolution) != list(g["resolution"]):
        diffs.append(f"resolution {list(P.resolution)} != {list(g['resolution'])}")
    if list(P.size) != list(g["size"]):
        diffs.append(f"size {list(P.size)} != {list(g['size'])}")
    nl = P.nloadcases
    if list(P.time)[:nl] != list(g["time"])[:nl]:
        diffs.append("time")
    if P.has_temperature_rate and list(P.temperature_rate)[:nl] != list(g["temperature_rate"])[:nl]:
        diffs.append("temperature_rate")
    ref_tables = {"material": _defined_materials(g["material"], P.nmat), "interface": g["interface"], "bcs": g["bcs"]}
    for what, ptr, n, T in (("material", P.material, P.nmat, L.Material), ("interface", P.interface, P.nf, L.Interface),
                            ("bcs", C.addressof(P.bcs), P.nbcs, L.BC)):
        mine = _bytes(ptr, n, T)
        ref = ref_tables[what]
        if not np.array_equal(mine, ref):
            k = int(np.flatnonzero(mine != ref)[0]) if mine.size == ref.size else -1
            diffs.append(f"{what} tables differ (first byte {k} of {mine.size} / {ref.size})")
    npf = P.npf
    il = np.ctypeslib.as_array(P.interfacelist, shape=(npf * npf,)).reshape(npf, npf)
    ir = g["interfacelist"].reshape(npf, npf)
    up = np.triu(np.ones((npf, npf), bool), 1)
    if not np.array_equal(il[up], ir[up]):
        diffs.append("interface_mapping")
    if not np.array_equal(np.ctypeslib.as_array(P.phasematerialmapping, shape=(npf,)), g["phasematerialmapping"]):
        diffs.append("phase_material_mapping")
    if not np.array_equal(cfg.problem.voxelphase(), g["voxelphase"]):
        diffs.append("voxel_phase_mapping")
    info = [int(x) for x in g["info"]]
    s = cfg.s
    mine_info = [s.nsites, s.nnuclei, s.noutputs, s.ncomponents, s.outputfreq, s.random_seed if s.has_random_seed else
                 info[5], s.initrefine, s.initcoarsen, s.maxnrefine, s.minnrefine, s.amrinterval] + list(s.initblocksize)
    if mine_info != info:
        diffs.append(f"counts / amr parameters {mine_info} != {info}")
    if cfg.components != [str(c) for c in g["components"]]:
        diffs.append("components")
    outs = [str(o) for o in g["outputs"] if str(o)]
    if [o[0] for o in cfg.output_spec()] != outs:
        diffs.append("outputs")
    if s.outfile.decode() != str(g["outfile"]):
        diffs.append("outfile")
    # the reference appends its p4est brick options to petscoptions
    if not str(g["petscoptions"]).startswith(s.petscoptions.decode()):
        diffs.append("petscoptions")
    t = cfg.nucleation_tables()
    if s.nsites:
        vs, sp, sn, nz = t
        if not np.array_equal(vs, g["voxelsite"]):
            diffs.append("voxel_site_mapping")
        if not np.array_equal(sp, g["sitephase"][:s.nsites]) or not np.array_equal(sn, g["sitenucleus"][:s.nsites]):
            diffs.append("site mappings")
    if s.nnuclei:
        ref = (L.Nucleus * s.nnuclei).from_buffer_copy(g["nuclei"].tobytes())
        for k in range(s.nnuclei):
            r = ref[k]
            # the loader keeps each matrix list sorted (the site check intersects sorted lists)
            m = sorted(r.matrix[:r.nmatrix])
            for i, v in enumerate(m):
                r.matrix[i] = v
            if bytes(r) != C.string_at(C.addressof(s.nuclei[k]), C.sizeof(L.Nucleus)):
                diffs.append(f"nucleus {k}")
    return diffs
