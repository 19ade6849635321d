"""ctypes bindings of the C ABI in include/cipher_b200.h and include/cipher_problem.h.

The shared library is built in-tree (``cipher_b200/libcipher_b200.so``); this
module never falls back to anything else: if the library is missing the import
of the device API raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# CIPHER_B200_LIB selects another build of the same library (for example a
# build with different launch parameters); default: the in-tree build
LIB_PATH = os.environ.get("CIPHER_B200_LIB") or os.path.join(HERE, "libcipher_b200.so")

MAXCP = 5
MAXAP = 15
MAXTSER = 10
MAXRK = 4
MAXRKTAB = 50
MAXBIN = 10
MAXSRC = 2
MAXDIR = 8
MAXLC = 64
MAXBC = 6

CHEM_QUADRATIC, CHEM_CALPHADDIS, CHEM_CALPHAD2SL, CHEM_NONE = 0, 1, 2, 3
INTERP_LINEAR, INTERP_QUADRATIC, INTERP_CUBIC = 0, 1, 2
BC_NEUMANN, BC_DIRICHLET, BC_NONE = 0, 1, 2
SOURCE_SINK, SOURCE_RANDOM = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
ALLOY_SEGREGATION, ALLOY_ITF_MOBILITY, ALLOY_ACTIVATION, ALLOY_THERMAL = 0x01, 0x02, 0x04, 0x08
ALLOY_SOURCES, ALLOY_WALLS, ALLOY_TEMP_RATE, ALLOY_MIXED_MODELS = 0x10, 0x20, 0x40, 0x80
ALLOY_ALL = 0x7F
GG_ACTIVATION, GG_WIDTHS = 0x01, 0x02
RHS_REFERENCE_ORDER, RHS_CLOSED_FORM = 0, 1

OK = 0
E_ARG, E_NOMEM, E_CAP, E_NONFINITE, E_CUDA, E_TIMEOUT, E_UNSUPPORTED, E_STEP = range(1, 9)


class TSeries(C.Structure):
    _fields_ = [("n", C.c_int32), ("exp", C.c_int32 * MAXTSER), ("coeff", C.c_double * MAXTSER),
                ("logcoeff", C.c_double)]


class RK(C.Structure):
    _fields_ = [("n", C.c_int32), ("i", C.c_int32 * MAXRK), ("h", TSeries * MAXRK)]


class Mobility(C.Structure):
    _fields_ = [("m0", C.c_double), ("unary", TSeries * MAXCP), ("binary", RK * MAXBIN)]


class Source(C.Structure):
    _fields_ = [("model", C.c_int32), ("rate", C.c_double * MAXCP), ("ceq", C.c_double * MAXCP),
                ("amplitude", C.c_double * MAXCP)]


class Material(C.Structure):
    _fields_ = [("model", C.c_int32), ("nsites", C.c_int32), ("molarvolume", C.c_double),
                ("chempot_ex_kineticcoeff", C.c_double), ("c0", C.c_double * (2 * MAXCP)),
                ("stoichiometry", C.c_double * 2), ("p", C.c_double), ("q", C.c_double),
                ("ref", TSeries), ("unary", TSeries * (MAXCP * MAXCP)), ("quad_ceq", TSeries * MAXCP),
                ("quad_binary", TSeries * MAXCP), ("binary", RK * MAXRKTAB), ("ternary", RK * MAXRKTAB),
                ("binaryq", RK * MAXRKTAB), ("ternaryq", RK * MAXRKTAB), ("mobilityc", Mobility * MAXCP),
                ("temperature0", C.c_double), ("specific_heat", TSeries), ("latent_heat", TSeries),
                ("tconductivity", TSeries), ("nsources", C.c_int32), ("sources", Source * MAXSRC)]


class Interface(C.Structure):
    _fields_ = [("width", C.c_double), ("energy_m0", C.c_double), ("energy_activation", TSeries),
                ("energy_naniso", C.c_int32), ("energy_aniso_dir", C.c_double * (MAXDIR * 3)),
                ("energy_aniso_val", C.c_double * MAXDIR), ("mobility_m0", C.c_double),
                ("mobility_activation", TSeries), ("mobility_naniso", C.c_int32),
                ("mobility_aniso_dir", C.c_double * (MAXDIR * 3)), ("mobility_aniso_val", C.c_double * MAXDIR),
                ("has_potential", C.c_int32), ("potential", C.c_double * MAXCP), ("has_mobilityc", C.c_int32),
                ("mobilityc", C.c_double * MAXCP), ("nsources", C.c_int32), ("sources", Source * MAXSRC)]


class BC(C.Structure):
    _fields_ = [("boundaryid", C.c_int32), ("chem_bctype", C.c_int32), ("thermal_bctype", C.c_int32),
                ("chem_bcval", C.c_double * MAXCP), ("thermal_bcval", C.c_double),
                ("chem_bcbool", C.c_int8 * MAXCP)]


class ProblemStruct(C.Structure):
    _fields_ = [("dim", C.c_int32), ("npf", C.c_int32), ("ncp", C.c_int32), ("ndp", C.c_int32),
                ("nmat", C.c_int32), ("nf", C.c_int32), ("nbcs", C.c_int32), ("pf_size", C.c_int32),
                ("maxsites", C.c_int32), ("interpolation", C.c_int32), ("gradient_calculation", C.c_int32),
                ("junctionpenalty", C.c_double), ("nloadcases", C.c_int32), ("currentloadcase", C.c_int32),
                ("has_temperature_rate", C.c_int32), ("time", C.c_double * MAXLC),
                ("temperature_rate", C.c_double * MAXLC), ("timestep0", C.c_double), ("mintimestep", C.c_double),
                ("maxtimestep", C.c_double), ("reltol", C.c_double), ("abstol", C.c_double),
                ("resolution", C.c_int32 * 3), ("size", C.c_double * 3), ("periodic", C.c_int32 * 3),
                ("material", C.POINTER(Material)), ("interface", C.POINTER(Interface)),
                ("interfacelist", C.POINTER(C.c_int32)), ("phasematerialmapping", C.POINTER(C.c_int32)),
                ("voxelphase", C.POINTER(C.c_int32)), ("bcs", BC * MAXBC), ("centres", C.POINTER(C.c_double))]


class MeshStruct(C.Structure):
    _fields_ = [("dim", C.c_int32), ("ncells", C.c_int32), ("nowned", C.c_int32), ("nfaces", C.c_int32),
                ("face_cells", C.POINTER(C.c_int32)), ("nbfaces", C.c_int32), ("bface_cell", C.POINTER(C.c_int32)),
                ("bface_label", C.POINTER(C.c_int32)), ("cellgeom", C.POINTER(C.c_double)),
                ("cell_global", C.POINTER(C.c_int32)), ("uniform", C.c_int32), ("res", C.c_int32 * 3),
                ("periodic", C.c_int32 * 3), ("slab_lo", C.c_int32), ("slab_hi", C.c_int32)]


class AosLayout(C.Structure):
    _fields_ = [("as_offset", C.c_int32), ("pf_offset", C.c_int32), ("dp_offset", C.c_int32),
                ("ex_offset", C.c_int32), ("tm_offset", C.c_int32), ("ndof", C.c_int32),
                ("as_size", C.c_int32), ("pf_size", C.c_int32), ("dp_size", C.c_int32),
                ("ex_size", C.c_int32), ("sp_size", C.c_int32), ("sf_size", C.c_int32)]


class StateLayout(C.Structure):
    _fields_ = [("ncells", C.c_int64), ("stride", C.c_int64), ("pf_size", C.c_int32), ("dp_size", C.c_int32),
                ("ex_size", C.c_int32), ("precision", C.c_int32), ("as_offset", C.c_int64),
                ("pf_offset", C.c_int64), ("dp_offset", C.c_int64), ("ex_offset", C.c_int64),
                ("tm_offset", C.c_int64), ("bytes", C.c_int64), ("map_offset", C.c_int64),
                ("map_planes", C.c_int32)]


class GridDesc(C.Structure):
    _fields_ = [("dim", C.c_int32), ("res", C.c_int32 * 3), ("periodic", C.c_int32 * 3),
                ("ex_per_phase", C.c_int32), ("layout", StateLayout), ("npf", C.c_int32), ("ncp", C.c_int32),
                ("nmat", C.c_int32), ("materials", C.c_void_p), ("phasematerialmapping", C.c_void_p)]


class TSOpts(C.Structure):
    _fields_ = [("scheme", C.c_int32), ("poststep", C.c_int32), ("dt0", C.c_double), ("dtmin", C.c_double),
                ("dtmax", C.c_double), ("reltol", C.c_double), ("abstol", C.c_double), ("max_steps", C.c_int64)]


class AMROpts(C.Structure):
    _fields_ = [("nblocks", C.c_int32 * 3), ("lmin", C.c_int32), ("lmax", C.c_int32), ("initcoarsen", C.c_int32),
                ("interval", C.c_int32), ("precision", C.c_int32), ("device", C.c_int32), ("ts", TSOpts)]


class TSStats(C.Structure):
    _fields_ = [("steps", C.c_int64), ("rejected", C.c_int64), ("rhs_calls", C.c_int64), ("t", C.c_double),
                ("dt", C.c_double), ("last_norm", C.c_double)]


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("precision", C.c_int32), ("max_active", C.c_int32),
                ("hbm_budget", C.c_int64), ("ts", TSOpts)]


class ServerResult(C.Structure):
    _fields_ = [("state", C.c_int32), ("status", C.c_int32), ("error", C.c_int32), ("stats", TSStats),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_finish", C.c_double),
                ("ncells", C.c_int64), ("ndof", C.c_int32), ("footprint", C.c_int64)]


class ServerCounters(C.Structure):
    _fields_ = [("polls", C.c_int64), ("steps", C.c_int64), ("domain_steps", C.c_int64), ("rebuilds", C.c_int64),
                ("graph_steps", C.c_int64), ("direct_steps", C.c_int64), ("t_admit", C.c_double),
                ("t_step", C.c_double), ("t_retire", C.c_double)]


class Nucleus(C.Structure):
    _fields_ = [("model", C.c_int32), ("nmatrix", C.c_int32), ("matrix", C.c_int32 * 16),
                ("active_solutes", C.c_int8 * MAXCP), ("gamma", C.c_double), ("shapefactor", C.c_double),
                ("minsize", C.c_double), ("atomicvolume", C.c_double), ("lengthscale", C.c_double),
                ("incubationtimemin", C.c_double), ("liquidus", C.c_double), ("nucleation_rate", C.c_double),
                ("solvus_temperature_0", C.c_double), ("enthalpy_fusion_0", C.c_double),
                ("has_solvus_c", C.c_int32), ("has_enthalpy_c", C.c_int32),
                ("solvus_temperature_c", C.c_double * MAXCP), ("enthalpy_fusion_c", C.c_double * MAXCP)]


NUC_CNT, NUC_CONSTANT, NUC_THERMAL, NUC_NONE = 0, 1, 2, 3


class OutputField(C.Structure):
    _fields_ = [("kind", C.c_int32), ("index", C.c_int32), ("name", C.c_char * 48)]


OUT_PHASEID, OUT_MATID, OUT_INTERFACEID, OUT_CHEMPOT, OUT_COMP, OUT_PHI, OUT_TEMPERATURE = range(7)


class ConfigStruct(C.Structure):
    _fields_ = [("problem", C.POINTER(ProblemStruct)), ("ncomponents", C.c_int32),
                ("componentname", (C.c_char * 64) * MAXCP), ("nsites", C.c_int32), ("nnuclei", C.c_int32),
                ("voxelsite", C.POINTER(C.c_int32)), ("sitephase", C.POINTER(C.c_int32)),
                ("sitenucleus", C.POINTER(C.c_int32)), ("nuclei", C.POINTER(Nucleus)), ("noutputs", C.c_int32),
                ("outputs", C.POINTER(OutputField)), ("outputfreq", C.c_int32), ("outfile", C.c_char * 256),
                ("petscoptions", C.c_char * 1024), ("rk_type", C.c_char * 16), ("has_random_seed", C.c_int32),
                ("random_seed", C.c_int64), ("initblocksize", C.c_int32 * 3), ("initrefine", C.c_int32),
                ("initcoarsen", C.c_int32), ("maxnrefine", C.c_int32), ("minnrefine", C.c_int32),
                ("amrinterval", C.c_int32), ("max_phase_neighbours", C.c_int32)]
INIT_SHARP, INIT_DIFFUSE = 0, 1
TS_RK1FE, TS_RK2A, TS_RK3BS = 0, 1, 2
BATCH_RUNNING, BATCH_FINISHED, BATCH_FAILED = 0, 1, 2

PP = C.POINTER(ProblemStruct)
MP = C.POINTER(MeshStruct)

# (name, restype, argtypes)
_SIGNATURES = [
    ("cipher_strerror", C.c_char_p, [C.c_int]),
    ("cipher_last_error", C.c_char_p, []),
    ("cipher_abi_sizes", C.c_int, [C.POINTER(C.c_int64), C.c_int]),
    ("cipher_pool_trim", C.c_int, [C.c_int]),
    ("cipher_ctx_set_rhs_form", C.c_int, [C.c_void_p, C.c_int]),
    ("cipher_amr_create", C.c_int, [PP, C.POINTER(AMROpts), C.POINTER(C.c_void_p)]),
    ("cipher_amr_destroy", None, [C.c_void_p]),
    ("cipher_amr_solve", C.c_int, [C.c_void_p, C.c_double, C.c_int64, C.c_void_p]),
    ("cipher_amr_state", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(MP),
                                   C.POINTER(C.c_int64)]),
    ("cipher_forest_create", C.c_int, [C.c_int, C.POINTER(C.c_int32), C.c_int, C.c_int, C.c_int,
                                       C.POINTER(C.c_int32), C.POINTER(C.c_double), C.POINTER(C.c_void_p)]),
    ("cipher_forest_destroy", None, [C.c_void_p]),
    ("cipher_forest_nleaves", C.c_int64, [C.c_void_p]),
    ("cipher_forest_leaves", C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("cipher_forest_resolution", C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    ("cipher_forest_mark_active", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_int8)]),
    ("cipher_forest_adapt", C.c_int, [C.c_void_p, C.POINTER(C.c_int8), C.POINTER(C.c_double), C.c_int, C.c_int]),
    ("cipher_forest_transfer_plan", C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    ("cipher_forest_transfer_aos", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double)]),
    ("cipher_forest_mesh", C.c_int, [C.c_void_p, C.POINTER(MP)]),
    ("cipher_state_transfer", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int64),
                                        C.POINTER(C.c_int32), C.c_void_p]),
    ("cipher_problem_new", PP, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    ("cipher_problem_free", None, [PP]),
    ("cipher_problem_finalize", C.c_int, [PP]),
    ("cipher_problem_set_cap", C.c_int, [PP, C.c_int]),
    ("cipher_problem_aos_layout", AosLayout, [PP]),
    ("cipher_problem_grain_growth", C.c_int,
     [C.c_int, C.POINTER(C.c_int32), C.c_int, C.c_int, C.c_uint64, C.c_double, C.c_double, C.c_double,
      C.c_double, C.c_double, C.POINTER(PP)]),
    ("cipher_problem_grain_growth_multi", C.c_int,
     [C.c_int, C.POINTER(C.c_int32), C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_uint, C.POINTER(PP)]),
    ("cipher_voronoi", C.c_int, [C.c_int, C.POINTER(C.c_int32), C.c_int, C.c_uint64, C.POINTER(C.c_int32),
                                 C.POINTER(C.c_double)]),
    ("cipher_rand_uniform", C.c_double, [C.POINTER(C.c_uint64)]),
    ("cipher_problem_alloy", C.c_int,
     [C.c_int, C.POINTER(C.c_int32), C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_uint, C.POINTER(PP)]),
    ("cipher_mesh_uniform", C.c_int, [PP, C.c_int, C.c_int, C.POINTER(MP)]),
    ("cipher_mesh_grid", C.c_int, [PP, C.POINTER(MP)]),
    ("cipher_mesh_free", None, [MP]),
    ("cipher_initial_state_aos", C.c_int, [PP, MP, C.POINTER(C.c_double)]),
    ("cipher_initial_state_diffuse_aos", C.c_int, [PP, MP, C.c_double, C.POINTER(C.c_double)]),
    ("cipher_waxpy", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]),
    ("cipher_ctx_create", C.c_int, [PP, MP, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    ("cipher_ctx_destroy", None, [C.c_void_p]),
    ("cipher_ctx_layout", C.c_int, [C.c_void_p, C.POINTER(StateLayout)]),
    ("cipher_rhs", C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("cipher_poststep", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("cipher_ctx_check", C.c_int, [C.c_void_p, C.c_void_p]),
    ("cipher_chem_init", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("cipher_state_refresh", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("cipher_state_init_sharp", C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.c_void_p, C.c_void_p]),
    ("cipher_poststep_noalloc", C.c_int, [C.POINTER(GridDesc), C.c_void_p, C.c_void_p]),
    ("cipher_ts_default_opts", C.c_int, [PP, C.POINTER(TSOpts)]),
    ("cipher_ts_create", C.c_int, [C.c_void_p, C.POINTER(TSOpts), C.POINTER(C.c_void_p)]),
    ("cipher_ts_destroy", None, [C.c_void_p]),
    ("cipher_ts_step", C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.POINTER(C.c_int), C.c_void_p]),
    ("cipher_ts_solve", C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.POINTER(TSStats), C.c_void_p]),
    ("cipher_ts_get_stats", C.c_int, [C.c_void_p, C.POINTER(TSStats)]),
    ("cipher_ts_set_dt", C.c_int, [C.c_void_p, C.c_double]),
    ("cipher_batch_create", C.c_int, [C.c_int, C.c_int, C.POINTER(TSOpts), C.POINTER(C.c_void_p)]),
    ("cipher_batch_destroy", None, [C.c_void_p]),
    ("cipher_batch_footprint", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]),
    ("cipher_batch_attach", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                      C.POINTER(C.c_int)]),
    ("cipher_batch_detach", C.c_int, [C.c_void_p, C.c_int]),
    ("cipher_batch_step", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("cipher_batch_flush", C.c_int, [C.c_void_p]),
    ("cipher_batch_slot_stats", C.c_int, [C.c_void_p, C.c_int, C.POINTER(TSStats), C.POINTER(C.c_int),
                                          C.POINTER(C.c_int)]),
    ("cipher_batch_set_graphs", C.c_int, [C.c_void_p, C.c_int]),
    ("cipher_server_create", C.c_int, [C.POINTER(ServerOpts), C.POINTER(C.c_void_p)]),
    ("cipher_server_destroy", None, [C.c_void_p]),
    ("cipher_server_submit", C.c_int, [C.c_void_p, PP, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_int64)]),
    ("cipher_server_poll", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("cipher_server_result", C.c_int, [C.c_void_p, C.c_int64, C.POINTER(ServerResult), C.POINTER(C.c_double)]),
    ("cipher_server_release", C.c_int, [C.c_void_p, C.c_int64]),
    ("cipher_server_usage", C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("cipher_server_get_counters", C.c_int, [C.c_void_p, C.POINTER(ServerCounters)]),
    ("cipher_batch_get_counters", C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                            C.POINTER(C.c_int64)]),
    ("cipher_output_fields", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("cipher_write_vtu", C.c_int, [C.c_char_p, PP, C.c_void_p, C.c_int, C.POINTER(C.c_double)]),
    ("cipher_nucleation_create", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                           C.POINTER(C.c_int32), C.c_int, C.c_void_p, C.c_uint64,
                                           C.POINTER(C.c_void_p)]),
    ("cipher_nucleation_destroy", None, [C.c_void_p]),
    ("cipher_nucleation_step", C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_int),
                                         C.c_void_p]),
    ("cipher_nucleation_sites", C.c_int, [C.c_void_p, C.POINTER(C.c_int8), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("cipher_ts_set_nucleation", C.c_int, [C.c_void_p, C.c_void_p]),
    ("cipher_state_from_aos", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("cipher_state_to_aos", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("cipher_rhs_aos_host", C.c_int,
     [C.c_void_p, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p]),
    ("cipher_config_parse", C.c_int, [C.c_char_p, C.c_size_t, C.c_char_p, C.POINTER(C.POINTER(ConfigStruct))]),
    ("cipher_config_load", C.c_int, [C.c_char_p, C.POINTER(C.POINTER(ConfigStruct))]),
    ("cipher_config_free", None, [C.POINTER(ConfigStruct)]),
    ("cipher_output_field_parse", C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_char_p), C.POINTER(OutputField)]),
    ("cipher_yaml_to_json", C.c_int, [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
]

EXPORTED = [s[0] for s in _SIGNATURES]

_lib = None


class CipherError(RuntimeError):
    def __init__(self, code: int, where: str):
        lib = _lib
        msg = ""
        if lib is not None:
            msg = lib.cipher_last_error().decode(errors="replace")
            name = lib.cipher_strerror(code).decode()
        else:
            name = str(code)
        super().__init__(f"{where}: {name} ({code}) {msg}")
        self.code = code


def load() -> C.CDLL:
    """Load libcipher_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m cipher_b200.build` (needs nvcc)")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in _SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(rc: int, where: str) -> None:
    if rc != OK:
        raise CipherError(rc, where)
