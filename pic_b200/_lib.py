"""ctypes binding of libpicb200.so (the C ABI declared in include/picb200.h).

The library is built in-tree (``python -m pic_b200.build``) and loaded from
this package directory.  There is no fallback: if the library is missing or a
call fails, a ``PicError`` is raised with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpicb200.so")

PIC_MAX_SPECIES = 4
PIC_MAX_PROCESSES = 4

PIC_OK = 0
PIC_ERR_BAD_ARG = 1
PIC_ERR_CUDA = 2
PIC_ERR_NOT_CONVERGED = 3
PIC_ERR_TIMEOUT = 4
PIC_ERR_OUT_OF_CAPACITY = 5
PIC_ERR_NUMERIC = 6

STATUS_NAMES = {
    PIC_OK: "PIC_OK",
    PIC_ERR_BAD_ARG: "PIC_ERR_BAD_ARG",
    PIC_ERR_CUDA: "PIC_ERR_CUDA",
    PIC_ERR_NOT_CONVERGED: "PIC_ERR_NOT_CONVERGED",
    PIC_ERR_TIMEOUT: "PIC_ERR_TIMEOUT",
    PIC_ERR_OUT_OF_CAPACITY: "PIC_ERR_OUT_OF_CAPACITY",
    PIC_ERR_NUMERIC: "PIC_ERR_NUMERIC",
}

PIC_MG_MIXED = 0
PIC_MG_FP64 = 1

PIC_MG_PERSISTENT = 0
PIC_MG_HOST_LOOP = 1
PIC_MG_GRAPH_LOOP = 2
PIC_MG_CLUSTER = 3
PIC_MG_DST = 4
PIC_MG_HYBRID = 5
MG_LAUNCH_MODES = {"persistent": PIC_MG_PERSISTENT, "host": PIC_MG_HOST_LOOP, "graph": PIC_MG_GRAPH_LOOP,
                   "cluster": PIC_MG_CLUSTER, "dst": PIC_MG_DST, "hybrid": PIC_MG_HYBRID}

PIC_ELASTIC = 0
PIC_EXCITATION = 1
PIC_IONIZATION = 2
PIC_CHARGE_EXCHANGE = 3


class PicError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class MgOptions(C.Structure):
    _fields_ = [("precision", C.c_int), ("pre_sweeps", C.c_int), ("post_sweeps", C.c_int), ("omega", C.c_double),
                ("coarsest_max", C.c_int), ("launch_mode", C.c_int), ("geometry", C.c_int), ("coarse_fp32", C.c_int)]


GEOMETRIES = {"cartesian": 0, "rz": 1}


class MgInfo(C.Structure):
    _fields_ = [("cycles", C.c_int), ("rel_res", C.c_double), ("rhs_norm", C.c_double), ("converged", C.c_int)]


class MccSpeciesDesc(C.Structure):
    _fields_ = [("nproc", C.c_int), ("type", C.c_int * PIC_MAX_PROCESSES), ("threshold", C.c_double * PIC_MAX_PROCESSES),
                ("h_sigma", C.c_void_p * PIC_MAX_PROCESSES), ("born_electron_species", C.c_int),
                ("born_ion_species", C.c_int)]


class MccDesc(C.Structure):
    _fields_ = [("ne", C.c_int), ("h_energy", C.c_void_p), ("gas_density", C.c_double),
                ("gas_temperature", C.c_double), ("gas_mass", C.c_double),
                ("species", MccSpeciesDesc * PIC_MAX_SPECIES)]


class BirthBuffer(C.Structure):
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("vx", C.c_void_p), ("vy", C.c_void_p), ("vz", C.c_void_p),
                ("species", C.c_void_p), ("count", C.c_void_p), ("capacity", C.c_int)]


class SpeciesDesc(C.Structure):
    _fields_ = [("capacity", C.c_int), ("charge", C.c_double), ("mass", C.c_double), ("np2c", C.c_double)]


class SimDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double), ("dt", C.c_double),
                ("eps0", C.c_double), ("nspecies", C.c_int), ("species", SpeciesDesc * PIC_MAX_SPECIES),
                ("h_dirichlet", C.c_void_p), ("h_phi_bc", C.c_void_p), ("tol", C.c_double), ("max_cycles", C.c_int),
                ("mg", MgOptions), ("sort_interval", C.c_int), ("tile", C.c_int), ("mcc", C.c_void_p),
                ("seed", C.c_ulonglong), ("use_graph", C.c_int), ("min_cycles", C.c_int), ("push_kernel", C.c_int)]


PIC_MG_GEOMETRY_VALUES = 18

PUSH_KERNELS = {"ring": 0, "warp": 1, "warp_agg": 2, "pipe": 3}


PIC_ADJ_MAX_SEGMENTS = 16


class AdjSpecies(C.Structure):
    _fields_ = [("n", C.c_int), ("charge", C.c_double), ("mass", C.c_double), ("np2c", C.c_double)]


class AdjDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double), ("dt", C.c_double),
                ("eps0", C.c_double), ("nspecies", C.c_int), ("species", AdjSpecies * PIC_MAX_SPECIES),
                ("h_dirichlet", C.c_void_p), ("h_segment", C.c_void_p), ("h_phi_fixed", C.c_void_p),
                ("nseg", C.c_int), ("steps", C.c_int), ("checkpoint_every", C.c_int), ("loss_species", C.c_int),
                ("tol", C.c_double), ("max_cycles", C.c_int)]


class SimDiag(C.Structure):
    _fields_ = [("live", C.c_longlong * PIC_MAX_SPECIES), ("kinetic", C.c_double * PIC_MAX_SPECIES),
                ("momentum", (C.c_double * 3) * PIC_MAX_SPECIES), ("field_energy", C.c_double),
                ("gauss_flux", C.c_double), ("gauss_charge", C.c_double), ("div_error_l2", C.c_double)]


class SimCounters(C.Structure):
    _fields_ = [("absorbed", C.c_ulonglong * PIC_MAX_SPECIES),
                ("collisions", (C.c_ulonglong * PIC_MAX_PROCESSES) * PIC_MAX_SPECIES),
                ("null_candidates", C.c_ulonglong * PIC_MAX_SPECIES), ("born", C.c_ulonglong * PIC_MAX_SPECIES),
                ("dropped_births", C.c_ulonglong), ("nu_overflow", C.c_ulonglong), ("count", C.c_int * PIC_MAX_SPECIES),
                ("last_cycles", C.c_int), ("last_rel_res", C.c_double), ("steps", C.c_longlong), ("electrode_absorbed", C.c_ulonglong * PIC_MAX_SPECIES),
                ("candidate_overflow", C.c_ulonglong)]


_vp = C.c_void_p
_i = C.c_int
_f = C.c_float
_d = C.c_double

# name -> argtypes (restype is int unless listed in _RESTYPE)
SIGNATURES = {
    "pic_abi_version": [],
    "pic_last_error": [],
    "pic_update_R": [_vp, _vp, _vp, _vp, _i, _f, _f, _vp, _vp, _vp],
    "pic_absorb": [_vp, _vp, _i, _i, _i, _vp, _vp],
    "pic_update_V": [_vp, _vp, _vp, _vp, _i, _vp, _vp, _i, _i, _f, _vp],
    "pic_deposit": [_vp, _vp, _i, _f, _vp, _i, _i, _vp],
    "pic_update_E": [_vp, _vp, _vp, _i, _i, _d, _d, _vp],
    "pic_form_rhs": [_vp, _vp, _d, _vp, _i, _i, _vp],
    "pic_update_E_rz": [_vp, _vp, _vp, _i, _i, _d, _d, _vp],
    "pic_sim_solver_mode": [_vp, C.POINTER(_i)],
    "pic_cg_create": [_i, _i, _d, _d, _vp, _vp, C.POINTER(_vp)],
    "pic_cg_solve": [_vp, _vp, _vp, _d, _i, C.POINTER(MgInfo), _vp],
    "pic_cg_destroy": [_vp],
    "pic_sim_particle_buffer": [_vp, _vp, _i, _d, _d, _d, _d, C.POINTER(_i), _vp],
    "pic_rz_density": [_vp, _i, _i, _d, _vp],
    "pic_update_R_rz": [_vp, _vp, _vp, _vp, _vp, _i, _f, _f, _vp],
    "pic_mg_create": [_i, _i, _d, _d, _vp, C.POINTER(MgOptions), C.POINTER(_vp)],
    "pic_mg_destroy": [_vp],
    "pic_mg_solve": [_vp, _vp, _vp, _d, _i, C.POINTER(MgInfo), _vp],
    "pic_mg_solve_async": [_vp, _vp, _vp, _d, _i, _vp],
    "pic_mg_read_info": [_vp, _d, C.POINTER(MgInfo)],
    "pic_mg_effective_launch_mode": [_vp, C.POINTER(_i)],
    "pic_mg_set_wait_limit": [_vp, C.c_longlong],
    "pic_mg_tile_geometry": [_i, _vp],
    "pic_sorter_create": [_i, _i, _i, _i, C.POINTER(_vp)],
    "pic_sorter_destroy": [_vp],
    "pic_sort": [_vp, _vp, _vp, _vp, _vp, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "pic_sort_static": [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "pic_mcc_create": [C.POINTER(MccDesc), _i, C.POINTER(_d), _d, C.POINTER(_vp)],
    "pic_mcc_destroy": [_vp],
    "pic_mcc_query": [_vp, _i, C.POINTER(_d), C.POINTER(_d), C.POINTER(_d)],
    "pic_mcc_apply": [_vp, _i, _vp, _vp, _vp, _vp, _vp, _i, C.c_ulonglong, C.c_uint, C.POINTER(BirthBuffer), _vp, _vp],
    "pic_sim_create": [C.POINTER(SimDesc), _vp, C.POINTER(_vp)],
    "pic_sim_destroy": [_vp],
    "pic_sim_load_species": [_vp, _i, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp],
    "pic_sim_init": [_vp, _vp],
    "pic_sim_step": [_vp, _i, _vp],
    "pic_sim_sync": [_vp, _vp],
    "pic_sim_species_arrays": [_vp, _i, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)],
    "pic_sim_fields": [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)],
    "pic_sim_read_particles": [_vp, _i, _vp, C.c_longlong, C.POINTER(_i), _vp],
    "pic_sim_sort": [_vp, _vp],
    "pic_sim_read_counters": [_vp, C.POINTER(SimCounters), _vp],
    "pic_sim_diagnostics": [_vp, C.c_void_p, _vp],
    "pic_sim_kernel_launches": [_vp],
    "pic_sim_set_profiling": [_vp, _i],
    "pic_sim_set_wait_limit": [_vp, C.c_longlong],
    "pic_sim_read_profile": [_vp, C.c_void_p],
    "pic_ens_create": [C.POINTER(_vp), _i, C.POINTER(_vp)],
    "pic_ens_destroy": [_vp],
    "pic_ens_step": [_vp, _i, _vp],
    "pic_ens_fused_pass": [_vp, C.POINTER(_i)],
    "pic_ens_set_fused_pass": [_vp, _i],
    "pic_adj_create": [_vp, C.POINTER(_vp)],
    "pic_adj_destroy": [_vp],
    "pic_adj_set_particles": [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "pic_adj_set_target": [_vp, _vp, _vp],
    "pic_adj_forward": [_vp, _vp, C.c_double, C.POINTER(C.c_double), _vp],
    "pic_adj_backward": [_vp, _vp, C.POINTER(C.c_double), _vp],
    "pic_adj_freeze_absorption": [_vp, _i],
    "pic_adj_state": [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp),
                      C.POINTER(_vp)],
}
_RESTYPE = {"pic_last_error": C.c_char_p, "pic_sim_kernel_launches": C.c_longlong}

PHASES = ["build", "push", "merge", "rhs", "solve", "efield", "sort"]


class SimProfile(C.Structure):
    _fields_ = [("ms", C.c_double * len(PHASES)), ("count", C.c_longlong * len(PHASES)), ("mg_cycles", C.c_longlong)]

_lib = None


def load() -> C.CDLL:
    """Load libpicb200.so once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PicError(PIC_ERR_CUDA, f"{LIB_PATH} is missing; build it with `python -m pic_b200.build`")
        lib = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, C.c_int)
        _lib = lib
    return _lib


def last_error() -> str:
    return load().pic_last_error().decode()


def check(rc: int, what: str = "") -> int:
    if rc != PIC_OK:
        raise PicError(rc, f"{what}: {last_error()}" if what else last_error())
    return rc


def call(name: str, *args) -> int:
    """Call an ABI function and raise PicError on a non-zero status."""
    return check(getattr(load(), name)(*args), name)


def stream_ptr(stream=None):
    """cudaStream_t of a torch stream (None = torch's current stream)."""
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def ptr(t) -> C.c_void_p:
    """Device pointer of a torch tensor (None -> NULL)."""
    if t is None:
        return C.c_void_p(None)
    return C.c_void_p(t.data_ptr())
