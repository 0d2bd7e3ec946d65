"""ctypes binding of libisinggpu.so (the C-ABI declared in include/ising_gpu.h).

The shared object is built in-tree by ``ising_b200/build.py``.  There is no fallback: if
the library is missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libisinggpu.so")
HEADER = os.path.join(HERE, "..", "include", "ising_gpu.h")

ISING_OK = 0
STATUS = {1: "ISING_ERR_ARG", 2: "ISING_ERR_NAN", 3: "ISING_ERR_BOUNDS", 4: "ISING_ERR_TIMEOUT",
          5: "ISING_ERR_UNSUPPORTED", 6: "ISING_ERR_CUDA", 7: "ISING_ERR_ALLOC", 8: "ISING_ERR_LATTICE",
          9: "ISING_ERR_CAPACITY"}

CELL_SC, CELL_BCC, CELL_HYPER_KAGOME = 0, 1, 2
DMI_INTERFACIAL, DMI_BULK = 0, 1
MOVE_UNIFORM, MOVE_BALL = 0, 1
PT_EVEN_ODD, PT_RANDOM_PAIRS = 0, 1


class IsingError(RuntimeError):
    """Raised for a non-zero status; .status holds the code (the reference would error stop)."""

    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS.get(status, status)}: {msg}")
        self.status = status


class MeshInfo(C.Structure):
    _fields_ = [("num_atoms", C.c_int64), ("num_cells", C.c_int64), ("nx", C.c_int), ("ny", C.c_int),
                ("nz", C.c_int), ("n_sub", C.c_int), ("n_shells", C.c_int), ("n_replicas", C.c_int),
                ("shell_size", C.c_int * 2), ("checkerboard", C.c_int), ("a_vec", C.c_double * 3),
                ("b_vec", C.c_double * 3), ("c_vec", C.c_double * 3)]


class Params(C.Structure):
    _fields_ = [("J", C.c_double), ("J_prime", C.c_double), ("Dz", C.c_double), ("Dz_prime", C.c_double),
                ("B", C.c_double), ("K", C.c_double), ("K_axis", C.c_double * 3),
                ("zeeman_factor", C.c_double), ("include_Jp", C.c_int), ("dmi_mode", C.c_int),
                ("dmi_axis", C.c_double * 3), ("legacy_neighbours", C.c_int), ("demag", C.c_int)]


class PTOptions(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("ensemble", C.c_uint32), ("move", C.c_int), ("r", C.c_double),
                ("scheme", C.c_int), ("resync_every", C.c_int), ("record", C.c_int),
                ("record_capacity", C.c_int), ("l2_group", C.c_int), ("sweep_kernel", C.c_int)]


class EnsembleDesc(C.Structure):
    _fields_ = [("mesh", C.c_void_p), ("n_temps", C.c_int), ("betas", C.POINTER(C.c_double)),
                ("params", Params), ("ensemble", C.c_uint32)]


class EnsemblesOptions(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("move", C.c_int), ("r", C.c_double), ("scheme", C.c_int),
                ("resync_every", C.c_int), ("wait_timeout_ms", C.c_int)]


class EnsSchedule(C.Structure):
    _fields_ = [("block_threads", C.c_int), ("chunk_pairs", C.c_int), ("order", C.c_int),
                ("group_bytes", C.c_int64), ("ms_per_round", C.c_double), ("loader", C.c_int)]


ENS_ORDER_PHASE, ENS_ORDER_GROUPS, ENS_ORDER_WAVE = 0, 1, 2
ENS_LOADER_REGISTERS, ENS_LOADER_STAGED, ENS_LOADER_FUSED = 0, 1, 2

_P = C.POINTER
_d, _i, _i64, _u32, _u64, _vp = C.c_double, C.c_int, C.c_int64, C.c_uint32, C.c_uint64, C.c_void_p

_SIGS = {
    "ising_status_string": (C.c_char_p, [_i]),
    "ising_last_error": (C.c_char_p, []),
    "ising_version": (C.c_char_p, []),
    "ising_unit_cell": (_i, [_i, _P(_d), _P(_d), _P(_d), _P(_d), _P(_d), _P(_d), _P(C.c_float), _P(_i)]),
    "ising_mesh_create": (_i, [_P(C.c_float), _i, _i, _i, _i, _d, _d, _d, _d, _d, _d, _d, _i, _i, _i, _P(_vp)]),
    "ising_mesh_destroy": (_i, [_vp]),
    "ising_mesh_get_info": (_i, [_vp, _P(MeshInfo)]),
    "ising_mesh_set_stream": (_i, [_vp, _vp]),
    "ising_mesh_positions": (_i, [_vp, _P(C.c_float)]),
    "ising_mesh_neighbours": (_i, [_vp, _i64, _i, _P(_i64), _i, _P(_i)]),
    "ising_mesh_derivative_list": (_i, [_vp, _P(_i64)]),
    "ising_mesh_colouring": (_i, [_vp, _P(Params), _P(_i), _P(_i)]),
    "ising_spins_set": (_i, [_vp, _i, _P(_d)]),
    "ising_spins_get": (_i, [_vp, _i, _P(_d)]),
    "ising_spins_set_async": (_i, [_vp, _i, _P(_d)]),
    "ising_spins_get_async": (_i, [_vp, _i, _P(_d)]),
    "ising_spins_wait": (_i, [_vp]),
    "ising_spins_init_uniform": (_i, [_vp, _u64, _u32]),
    "ising_params_reference": (_i, [_i, _d, _d, _d, _d, _d, _P(Params)]),
    "ising_local_energy": (_i, [_vp, _i, _i, _P(Params), _P(_d), _P(_d), _P(_d)]),
    "ising_local_energy_batch": (_i, [_vp, _i, _i, _P(_i64), _P(_d), _P(Params), _P(_d), _P(_d)]),
    "ising_total_energy": (_i, [_vp, _i, _P(Params), _P(_d)]),
    "ising_total_energy_noalloc": (_i, [_vp, _i, _P(Params), _P(_d)]),
    "ising_observables": (_i, [_vp, _P(Params), _P(_d), _P(_d)]),
    "ising_metropolis_mcs": (_i, [_vp, _i, _d, _i, _P(Params), _d, _u64]),
    "ising_winding_number": (_i, [_vp, _i, _i, _P(_d)]),
    "ising_winding_all_slices": (_i, [_vp, _i, _P(_d)]),
    "ising_statistics": (_i, [_vp, _i, _P(_d), _P(_d), _P(_d)]),
    "ising_winding_density": (_i, [_vp, _i, _i, _P(_d)]),
    "ising_winding_density_all": (_i, [_vp, _i, _P(_d)]),
    "ising_mesh_set_interpolation_scale": (_i, [_vp, _i, _i]),
    "ising_mesh_interpolation_scale": (_i, [_vp, _P(_i), _P(_i)]),
    "ising_winding_density_interpolated": (_i, [_vp, _i, _i, _P(_d)]),
    "ising_skyrmion_number": (_i, [_vp, _i, _i, _d, _i, _d, _P(_i)]),
    "ising_skyrmion_distribution": (_i, [_vp, _i, _i, _d, _d, _i, _i, _P(_i)]),
    "ising_chain_mesh_statistics": (_i, [_vp, _i, _P(_i), _P(_d), _P(_d), _P(_d)]),
    "ising_gaussian_filter_2d": (_i, [_P(_d), _i, _i, _d]),
    "ising_skyrmion_number_density": (_i, [_P(_d), _i, _i, _i, _i, _d, _i, _d, _P(_i)]),
    "ising_pt_create": (_i, [_vp, _i, _P(_d), _P(Params), _P(PTOptions), _P(_vp)]),
    "ising_pt_destroy": (_i, [_vp]),
    "ising_pt_run": (_i, [_vp, _i, _i]),
    "ising_pt_relax": (_i, [_vp, _i]),
    "ising_pt_schedule": (_i, [_vp, _i, _P(_i), _P(_i), _P(_i)]),
    "ising_pt_permutation": (_i, [_vp, _P(_i)]),
    "ising_pt_energies": (_i, [_vp, _P(_d), _P(_d)]),
    "ising_pt_resync": (_i, [_vp]),
    "ising_pt_inject_stall": (_i, [_vp, _i]),
    "ising_pt_swap_stats": (_i, [_vp, _P(_u64), _P(_u64)]),
    "ising_pt_series": (_i, [_vp, _P(_d), _P(_i)]),
    "ising_ensembles_create": (_i, [_i, _P(EnsembleDesc), _P(EnsemblesOptions), _P(_vp)]),
    "ising_ensembles_destroy": (_i, [_vp]),
    "ising_ensembles_set_stream": (_i, [_vp, _vp]),
    "ising_ensembles_run": (_i, [_vp, _i, _i]),
    "ising_ensembles_set_schedule": (_i, [_vp, _P(EnsSchedule)]),
    "ising_ensembles_get_schedule": (_i, [_vp, _P(EnsSchedule), _P(_i), _P(_i64)]),
    "ising_ensembles_autotune": (_i, [_vp, _i, _i, _P(EnsSchedule), _i, _P(_i)]),
    "ising_ensembles_permutation": (_i, [_vp, _i, _P(_i)]),
    "ising_ensembles_energies": (_i, [_vp, _i, _P(_d), _P(_d)]),
    "ising_ensembles_swap_stats": (_i, [_vp, _i, _P(_u64), _P(_u64)]),
    "ising_ensembles_resync": (_i, [_vp]),
    "ising_ensembles_inject_stall": (_i, [_vp, _i]),
    "ising_ensembles_set_resync": (_i, [_vp, _i]),
    "ising_demag_field": (_i, [_vp, _i, _P(_d)]),
    "ising_write_demag_csv": (_i, [_vp, _i, C.c_char_p]),
    "ising_conv3_bf16": (_i, [_vp, _i, _i, _i, _i, _i, _vp, _i, _i, _vp, _vp, _i, _vp, _i, _i, _i, _vp]),
    "ising_bf16_gemm": (_i, [_vp, _i, _vp, _i, _i, _i, _i, _P(C.c_float), _P(C.c_float), _i, _vp, _i, _i, _vp]),
    "ising_net_create": (_i, [_i, _i, _u64, _P(_vp)]),
    "ising_net_destroy": (_i, [_vp]),
    "ising_net_param_count": (_i, []),
    "ising_net_set_params": (_i, [_vp, _P(C.c_float)]),
    "ising_net_get_params": (_i, [_vp, _P(C.c_float)]),
    "ising_net_forward": (_i, [_vp, _P(C.c_float), _i, _P(C.c_float)]),
    "ising_net_loss_grad": (_i, [_vp, _P(C.c_float), _P(C.c_float), _i, _P(_d), _P(C.c_float)]),
    "ising_net_train_step": (_i, [_vp, _P(C.c_float), _P(C.c_float), _i, _d, _P(_d)]),
    "ising_pt_patch_step": (_i, [_vp, _vp, _i, _i, _i, _i, _i]),
    "ising_pt_patch_count": (_i, [_vp, _i, _P(_i64)]),
    "ising_pt_patch_set_scale": (_i, [_vp, _P(C.c_float), C.c_float]),
    "ising_pt_patch_samples": (_i, [_vp, _i, _i, _i, _i, _i, _i, _P(C.c_float), _P(C.c_float)]),
    "ising_pt_patch_stats": (_i, [_vp, _P(_u64), _P(_u64)]),
    "ising_pt_patch_jump": (_i, [_vp, _P(_d)]),
    "ising_pt_patch_last": (_i, [_vp, _i, _P(C.c_float), _P(C.c_float), _P(_d), _P(_d), _P(_i)]),
    "ising_write_spins_csv": (_i, [_vp, _i, C.c_char_p, _i, _i, _i]),
    "ising_write_pt_data_csv": (_i, [C.c_char_p, _d, _d, _d, _d, _d, _i, _d, _P(_d)]),
    "ising_pt_file_tag": (_i, [C.c_char_p, C.c_size_t, _d, _d, _d, _d]),
    "ising_write_winding_density_csv": (_i, [_vp, _i, C.c_char_p]),
    "ising_frame_filename": (_i, [C.c_char_p, C.c_size_t, C.c_char_p, _i]),
    "ising_write_winding_density_interpolated_csv": (_i, [_vp, _i, C.c_char_p]),
    "ising_write_frame_info": (_i, [C.c_char_p, _i, _i, C.c_float]),
}

_lib = None


def header_symbols(path: str = HEADER):
    """Function names declared in include/*.h (every one must be exported)."""
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ising_[a-z0-9_]+)\s*\(", txt)))


def load():
    """Load libisinggpu.so; raises if it is absent (there is no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python ising_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str):
    if status != ISING_OK:
        msg = load().ising_last_error().decode(errors="replace")
        raise IsingError(status, where, msg)


def call(name: str, *args):
    st = getattr(load(), name)(*args)
    check(st, name)
    return st
