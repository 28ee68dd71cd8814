"""Loader and ctypes declarations for the C ABI in include/hpcrack.h.

The shared library is built in-tree (``make -C hpcrack_b200`` or :func:`build`) as
``hpcrack_b200/libhpcrack_b200.so``.  There is no CPU path: if the library is
missing or no CUDA device is usable, calls fail with an exception.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
# HPCRACK_LIB selects another build of the same library (e.g. two builds timed against each other).
LIB_PATH = os.environ.get("HPCRACK_LIB") or os.path.join(HERE, "libhpcrack_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "hpcrack.h")

HPC_OK = 0
STATUS = {0: "HPC_OK", 1: "HPC_ERR_ARG", 2: "HPC_ERR_CUDA", 3: "HPC_ERR_NOMEM", 4: "HPC_ERR_DIVZERO",
          5: "HPC_ERR_INPUT", 6: "HPC_ERR_NODEVICE", 7: "HPC_ERR_IO"}


class HpcError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, fn: str, status: int, message: str):
        super().__init__(f"{fn} -> {STATUS.get(status, status)}: {message}")
        self.status = status


class hpc_geometry(C.Structure):
    _fields_ = [("maxlevel", C.c_int), ("element_nb", C.c_int * 3), ("x_start", C.c_double * 3),
                ("roi_start", C.c_int * 3)]


class hpc_mg(C.Structure):
    _fields_ = [("nu0", C.c_int), ("nu1", C.c_int), ("nu2", C.c_int), ("gamma", C.c_int), ("ncy", C.c_int)]


class hpc_step_params(C.Structure):
    _fields_ = [("t", C.c_int), ("mg_u", hpc_mg), ("mg_d", hpc_mg), ("small_k", C.c_double), ("lc", C.c_double),
                ("voxel_size", C.c_double), ("ut0", C.c_double), ("du", C.c_double), ("du_factor", C.c_double),
                ("mech_tol", C.c_double), ("pf_tol", C.c_double), ("mech_solver", C.c_int)]


_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_i = C.c_int
_d = C.c_double
_ctx = C.c_void_p

# name -> argtypes (every function returns int status unless listed in _RESTYPE)
SIGNATURES = {
    "hpc_create": [C.POINTER(C.c_void_p), C.POINTER(hpc_geometry), _i],
    "hpc_destroy": [_ctx],
    "hpc_footprint": [C.POINTER(hpc_geometry), C.POINTER(C.c_size_t)],
    "hpc_level_dims": [_ctx, _i, _ip, _dp],
    "hpc_sync": [_ctx],
    "hpc_last_error": [],
    "hpc_set_choice_quirk": [_ctx, _i],
    "hpc_set_autotune": [_ctx, _i],
    "hpc_set_fused_coarsest": [_ctx, _i],
    "hpc_set_tensor_apply": [_ctx, _i],
    "hpc_set_tma_staging": [_ctx, _i],
    "hpc_tuned_shapes": [_ip, _i, _ip],
    "hpc_launch_count": [_ctx, C.POINTER(C.c_longlong), _i],
    "hpc_binary_version": [_ip],
    "hpc_batch_create": [C.POINTER(C.c_void_p)],
    "hpc_batch_destroy": [_vp],
    "hpc_batch_step": [_vp, C.POINTER(C.c_void_p), _i, C.POINTER(hpc_step_params), _dp],
    "hpc_batch_timing": [_vp, _i, _dp],
    "hpc_stream": [_ctx],
    "hpc_kernel_timing": [_ctx, _i],
    "hpc_kernel_time": [_ctx, C.POINTER(C.c_longlong), _dp],
    "hpc_upload": [_ctx, _i, _i, _i, _dp],
    "hpc_download": [_ctx, _i, _i, _i, _dp],
    "hpc_upload_choice": [_ctx, _i, C.POINTER(C.c_int16)],
    "hpc_download_choice": [_ctx, _i, C.POINTER(C.c_int16)],
    "hpc_get_state": [_ctx, _dp],
    "hpc_set_state": [_ctx, _dp],
    "hpc_checkpoint_begin": [_ctx, _i],
    "hpc_vtk_write": [_ctx, C.c_char_p, _i, _i, _d, C.c_char_p, C.c_char_p, _i],
    "hpc_vtk_wait": [_ctx],
    "hpc_checkpoint_wait": [_ctx, _ip, C.POINTER(_dp), _dp],
    "hpc_checkpoint_restore": [_ctx, _dp, _dp, _dp, _dp, _dp, _dp, _dp],
    "hpc_internal_force": [_ctx, _i, _i, _i, _d],
    "hpc_prem_u": [_ctx, _i, _i, _d],
    "hpc_fld": [_ctx, _i, _i, _i, _d],
    "hpc_precondition_m": [_ctx, _i, _i, _d],
    "hpc_initial_residual_u": [_ctx, _i, _d, _dp],
    "hpc_pcg_u": [_ctx, _i, _d, _d, _i, _i, _dp],
    "hpc_initial_residual_d": [_ctx, _i, _d, _dp],
    "hpc_pcg_d": [_ctx, _i, _d, _i, _i, _dp],
    "hpc_cycle_u": [_ctx, _i, C.POINTER(hpc_mg), _d, _d, _i, _dp],
    "hpc_cycle_d": [_ctx, _i, C.POINTER(hpc_mg), _d, _i, _dp],
    "hpc_u_entire": [_ctx, C.POINTER(hpc_mg), _d, _d, _i, _dp, _d, _ip, _ip],
    "hpc_phase_field": [_ctx, C.POINTER(hpc_mg), _d, _i, _dp, _d, _ip, _ip],
    "hpc_step": [_ctx, C.POINTER(hpc_step_params), _dp],
    "hpc_u_entire_fcg": [_ctx, C.POINTER(hpc_mg), _d, _d, _i, _dp, _d, _i, _ip, _ip],
    "hpc_mp_choice": [_ctx],
    "hpc_mp_all_element": [_ctx, _d],
    "hpc_vr_all_level": [_ctx, _i],
    "hpc_voigt_all_level": [_ctx, _i],
    "hpc_coarse_vr": [_ctx, _i],
    "hpc_strain_history": [_ctx, _d, _d],
    "hpc_fd_h": [_ctx, _i],
    "hpc_delta_d_max": [_ctx, _dp],
    "hpc_d_max": [_ctx, _dp],
    "hpc_U_e": [_ctx, _d, _dp],
    "hpc_externe_force_nodal": [_ctx, _d, _d],
    "hpc_externe_force_sum": [_ctx, _dp],
    "hpc_initial_crack": [_ctx, _d, _i],
    "hpc_dirichlet_bd": [_ctx, _i, _i, _d],
    "hpc_dirichlet_force": [_ctx, _i, _i, _i],
    "hpc_dirichlet_residual": [_ctx, _i, _i],
    "hpc_solution_injection": [_ctx, _i, _i, _i],
    "hpc_coarsen_f_standard": [_ctx, _i, _i, _i, _i, _i],
    "hpc_refine_standard": [_ctx, _i, _i, _i, _i, _i],
    "hpc_image_material": [_ctx, C.POINTER(C.c_uint8), _ip, _i, _ip, _dp, _dp, _dp, _d],
    "hpc_dmax_noalloc": [C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p],
    "hpc_slab_level": [C.POINTER(hpc_geometry), _i, _i, _i, _ip],
    "hpc_create_slab": [C.POINTER(C.c_void_p), C.POINTER(hpc_geometry), _i, _i, _i],
    "hpc_footprint_slab": [C.POINTER(hpc_geometry), _i, _i, C.POINTER(C.c_size_t)],
    "hpc_slab_group_create": [C.POINTER(C.c_void_p), _i],
    "hpc_slab_group_join": [_vp, _ctx],
    "hpc_slab_group_abort": [_vp],
    "hpc_slab_group_destroy": [_vp],
    "hpc_nccl_unique_id": [C.POINTER(C.c_ubyte)],
    "hpc_slab_join_nccl": [_ctx, C.POINTER(C.c_ubyte)],
}
_RESTYPE = {"hpc_last_error": C.c_char_p, "hpc_stream": C.c_void_p}

_lib = None


def build(verbose: bool = False) -> str:
    """Compile the CUDA library for sm_100a in-tree (nvcc cross-compiles without a GPU)."""
    out = subprocess.run(["make", "-C", HERE, "all"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("hpcrack_b200 build failed:\n" + out.stdout + out.stderr)
    if verbose:
        print(out.stdout)
    return LIB_PATH


def load() -> C.CDLL:
    """Load the in-tree library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} not built: run `make -C hpcrack_b200`")
    lib = C.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            if os.environ.get("HPCRACK_LIB"):  # an older build: calls to what it lacks fail when made
                continue
            raise AttributeError(f"{LIB_PATH} lacks {name}")
        fn.argtypes = args
        fn.restype = _RESTYPE.get(name, C.c_int)
    _lib = lib
    return lib


def check(fn_name: str, status: int) -> None:
    if status != HPC_OK:
        msg = load().hpc_last_error()
        raise HpcError(fn_name, status, msg.decode(errors="replace") if msg else "")


def declared_symbols(header: str = HEADER) -> list[str]:
    """Function names declared in include/hpcrack.h (for the export check)."""
    import re
    text = open(header).read()
    return sorted(set(re.findall(r"\b(hpc_[a-zA-Z_0-9]+)\s*\(", text)))
