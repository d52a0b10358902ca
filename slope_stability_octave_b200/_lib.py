"""ctypes binding of libslopegpu.so, the C ABI declared in include/slopegpu.h.

The library is loaded from this package directory (built in-tree by
``python -m slope_stability_octave_b200.build``).  There is no fallback: if the shared
library is missing or a call fails, a ``SlopeGPUError`` is raised.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libslopegpu.so")

vp = C.c_void_p
i32, i64, f64, ch = C.c_int32, C.c_int64, C.c_double, C.c_char
cint = C.c_int

# name -> argtypes (restype int unless listed in _RESTYPES)
SIGNATURES = {
    "sg_abi_version": [],
    "sg_last_error": [],
    "sg_device_count": [],
    "sg_constitutive3d": [vp] * 6 + [i64, vp, vp, vp],
    "sg_constitutive3d_dev": [vp] * 6 + [i64, vp, vp, vp, vp],
    "sg_constitutive2d": [vp] * 6 + [i64, vp, vp, vp],
    "sg_constitutive2d_dev": [vp] * 6 + [i64, vp, vp, vp, vp],
    "sg_constitutive3d_noalloc": [vp] * 6 + [i64, vp, vp, vp],
    "sg_reduction_dev": [vp, vp, vp, f64, ch, i64, vp, vp, vp],
    "sg_potential_dev": [cint] + [vp] * 7 + [i64, vp, vp],
    "sg_assemble_ktangent3d": [vp] * 6 + [i32, i64, i64, i32, i64, vp],
    "sg_assemble_ktangent2d": [vp] * 5 + [i32, i64, i64, i32, i64, vp],
    "sg_assemble_ktangent_dev": [cint] + [vp] * 6 + [i32, i64, i32, i64, vp, vp],
    # mesh and element operators
    "sg_mesh_create": [cint, i32, i32, i64, i64, vp, vp, vp, vp, vp, vp, vp],
    "sg_mesh_destroy": [vp],
    "sg_mesh_sizes": [vp, vp],
    "sg_mesh_bsr": [vp, vp],
    "sg_mesh_pattern": [vp, vp, vp, vp],
    "sg_mesh_scatter_map": [vp, vp],
    "sg_mesh_free_dofs": [vp, vp],
    "sg_strain_dev": [vp, vp, vp, vp],
    "sg_force_dev": [vp, vp, i32, vp, vp],
    "sg_residual_dev": [vp] * 9,
    "sg_assemble_bsr_dev": [vp, vp, vp, vp],
    "sg_elastic_ds_dev": [vp, vp, vp, vp, vp],
    "sg_symmetrize_bsr_dev": [vp, vp, vp, vp],
    "sg_kr_blend_dev": [vp, f64, vp, vp, vp, vp],
    "sg_assemble_kr_dev": [vp, vp, f64, vp, vp, vp, vp],
    "sg_bsr_to_ref_dev": [vp, vp, vp, vp],
    # seepage (pore pressure) systems on the mesh
    "sg_mesh_bsr_scalar": [vp, vp],
    "sg_seepage_system_dev": [vp, vp, vp, vp, vp, vp, f64, i32, vp, vp, vp, vp],
    "sg_point_gradient_dev": [vp, vp, vp, vp],
    "sg_seepage_saturation_dev": [vp, vp, vp, vp, vp, vp, vp],
    # sparse and vector operations
    "sg_bsr_info": [vp, vp],
    "sg_bsr_spmv_dev": [vp, vp, vp, vp, vp],
    "sg_dot_dev": [i64, vp, vp, vp, vp],
    "sg_masked_diff_norm2_dev": [i64, vp, vp, vp, vp, vp],
    "sg_axpby_dev": [i64, f64, vp, f64, vp, vp],
    # AMG
    "sg_amg_create": [vp, vp, vp, i32, vp, vp, i32, vp, vp],
    "sg_amg_destroy": [vp],
    "sg_amg_update": [vp, vp, vp],
    "sg_amg_clone": [vp, vp],
    "sg_krylov_set_graph": [vp, i32],
    "sg_krylov_set_aorth": [vp, i32],
    "sg_amg_setup_ijv": [C.c_char_p, vp, vp, vp, i64, i64, vp, i32, vp, i32, vp, i32, i32, vp],
    "sg_amg_update_values": [C.c_char_p, vp, i64, vp],
    "sg_amg_apply_host": [C.c_char_p, vp, vp, i64],
    "sg_amg_clear": [C.c_char_p],
    "sg_amg_ijv_info": [C.c_char_p, vp, i32],
    "sg_amg_apply": [vp, vp, vp, vp],
    "sg_amg_info": [vp, vp, i32],
    "sg_amg_export": [vp, i32, vp, vp, vp, vp, vp, vp],
    "sg_amg_set_correction": [vp, vp, vp],
    # learned node-wise correction of the V-cycle
    "sg_mlp_forward_dev": [vp, vp, i64, vp, vp, vp],
    "sg_mlp_part_size": [i64],
    "sg_mlp_backward_dev": [vp, vp, vp, i64, vp, vp, vp, vp],
    "sg_learned_create": [vp, vp, i32, C.c_uint64, vp],
    "sg_learned_destroy": [vp],
    "sg_learned_params": [vp, vp, i32],
    "sg_learned_features": [vp, vp, vp, vp, vp, vp],
    "sg_learned_correction": [vp, vp, vp, vp],
    "sg_learned_collect": [vp, vp, vp, vp, vp, i32, i32, i32, vp],
    "sg_learned_set_loss": [vp, i32],
    "sg_learned_loss": [vp, vp, vp, i32, vp, vp],
    "sg_learned_gradient": [vp, vp, vp, i32, vp, vp, vp],
    "sg_learned_train": [vp, vp, vp, i32, f64, vp, vp],
    "sg_learned_export": [vp, i32, i32, vp],
    "sg_learned_info": [vp, vp],
    # Krylov
    "sg_krylov_create": [i64, i32, vp],
    "sg_krylov_destroy": [vp],
    "sg_dfgmres_solve": [vp, vp, vp, vp, vp, vp, i32, vp, vp, f64, i32, vp, vp, vp, vp],
    "sg_a_orthogonalize": [vp, vp, vp, vp, vp, i32, f64, vp, vp],
    # live kernel timing
    "sg_instr_enable": [cint, cint],
    "sg_instr_read": [vp, vp, vp, i32],
    "sg_launch_count": [cint],
    "sg_instr_units": [vp, i32],
    "sg_device_alloc_count": [cint],
    "sg_device_status": [C.c_int32, vp],
}
_RESTYPES = {"sg_last_error": C.c_char_p, "sg_launch_count": C.c_int64, "sg_device_alloc_count": C.c_int64, "sg_mlp_part_size": C.c_int64}


class SlopeGPUError(RuntimeError):
    pass


_lib = None


def lib() -> C.CDLL:
    """Load (once) and return the native library; raise if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SlopeGPUError(
                f"{LIB_PATH} not found: build it with `python -m slope_stability_octave_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            # a symbol missing from an out-of-date build fails when it is called (AttributeError)
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, cint)
        _lib = L
    return _lib


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        msg = lib().sg_last_error().decode(errors="replace")
        raise SlopeGPUError(f"{what or 'slopegpu'} failed ({rc}): {msg}")


def call(name: str, *args) -> None:
    """Call a status-returning C-ABI function and raise on failure."""
    check(getattr(lib(), name)(*args), name)
