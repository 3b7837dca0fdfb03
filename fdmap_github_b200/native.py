"""ctypes binding of libfdmap_gpu.so (include/fdmap_host.h, include/fdmap_gpu.h).

The library is loaded from the package directory; there is no fallback: if
it is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfdmap_gpu.so"

FDMAP_ERRORS = {
    0: "ok",
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "non-finite value detected",
    -4: "friction Newton solver did not converge",
    -5: "device wait timed out",
    -6: "unsupported configuration",
    -7: "I/O error",
    -8: "out of memory",
}

# FDMAP_FAULT_* (include/fdmap_desc.h), checkpoint order of friction.f90:528-546
FAULT_FIELDS = ["D", "Psi", "DPsi", "trup", "V", "O", "S", "N", "S0", "N0",
                "Ds", "Dn", "DDs", "DDn", "W", "DW", "Nreg", "DNreg"]
FAULT_INDEX = {n: i for i, n in enumerate(FAULT_FIELDS)}

# FDMAP_INIT_BODY_ON_DEVICE (include/fdmap_host.h)
INIT_BODY_ON_DEVICE = 1

# FDMAP_METRIC_* (include/fdmap_gpu.h)
METRIC_INDEX = {"xq": 0, "xr": 1, "yq": 2, "yr": 3, "Ji": 4, "J": 5}

# every exported entry point with (restype, argtypes)
_DP = C.POINTER(C.c_double)
_VP = C.c_void_p
SIGNATURES = {
    # fdmap_host.h
    "fdmap_host_init": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(_VP)]),
    "fdmap_host_init_ex": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(_VP)]),
    "fdmap_host_set_spacing": (C.c_int, [_VP, C.c_double, C.c_double]),
    "fdmap_host_desc": (_VP, [_VP]),
    "fdmap_host_desc_mut": (_VP, [_VP]),
    "fdmap_host_free": (None, [_VP]),
    "fdmap_host_info": (C.c_int, [_VP, C.POINTER(C.c_int), _DP]),
    "fdmap_host_iface_n": (C.c_int, [_VP, C.c_int]),
    "fdmap_host_body_flags": (C.c_int, [_VP, C.POINTER(C.c_int)]),
    "fdmap_host_block_limits": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_int)]),
    "fdmap_host_block_pml": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_int), _DP]),
    "fdmap_host_block_cdiss": (C.c_double, [_VP, C.c_int]),
    "fdmap_host_iface_info": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_int)]),
    "fdmap_host_iface_xy": (_DP, [_VP, C.c_int, C.c_int]),
    "fdmap_host_iface_blocks": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_int)]),
    "fdmap_host_side_array": (_DP, [_VP, C.c_int, C.c_int, C.c_char_p, C.POINTER(C.c_longlong)]),
    "fdmap_host_array": (_DP, [_VP, C.c_char_p, C.POINTER(C.c_longlong)]),
    "fdmap_host_last_error": (C.c_char_p, []),
    # fdmap_gpu.h
    "fdmap_gpu_create": (C.c_int, [_VP, C.c_int, C.c_int, C.POINTER(_VP)]),
    "fdmap_gpu_init_edges": (C.c_int, [_VP, C.c_double]),
    "fdmap_gpu_time_step": (C.c_int, [_VP, C.c_double, C.c_double, C.c_int]),
    "fdmap_gpu_run": (C.c_int, [_VP, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]),
    "fdmap_gpu_synchronize": (C.c_int, [_VP]),
    "fdmap_gpu_set_stream": (C.c_int, [_VP, _VP]),
    "fdmap_gpu_profile": (C.c_int, [_VP, C.c_int]),
    "fdmap_gpu_profile_read": (C.c_int, [_VP, _DP, C.POINTER(C.c_longlong)]),
    "fdmap_gpu_profile_read_kinds": (C.c_int, [_VP, C.c_int, _DP, C.POINTER(C.c_longlong)]),
    "fdmap_gpu_set_pairs": (C.c_int, [_VP, C.c_int]),
    "fdmap_gpu_get_pairs": (C.c_int, [_VP]),
    "fdmap_gpu_get_fields": (C.c_int, [_VP, _DP, _DP]),
    "fdmap_gpu_set_fields": (C.c_int, [_VP, _DP, _DP]),
    "fdmap_gpu_get_fault": (C.c_int, [_VP, C.c_int, C.c_int, _DP]),
    "fdmap_gpu_set_fault": (C.c_int, [_VP, C.c_int, C.c_int, _DP]),
    "fdmap_gpu_get_fhat": (C.c_int, [_VP, C.c_int, C.c_int, _DP]),
    "fdmap_gpu_status": (C.c_int, [_VP, C.POINTER(C.c_longlong)]),
    "fdmap_gpu_check_finite": (C.c_int, [_VP, C.POINTER(C.c_longlong)]),
    "fdmap_gpu_newton_counts": (C.c_int, [_VP, C.POINTER(C.c_longlong)]),
    "fdmap_gpu_clear_status": (C.c_int, [_VP]),
    "fdmap_gpu_set_newton_limit": (C.c_int, [_VP, C.c_int]),
    "fdmap_gpu_set_tile": (C.c_int, [_VP, C.c_int]),
    "fdmap_gpu_get_tile": (C.c_int, [_VP, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "fdmap_gpu_tune": (C.c_int, [_VP, C.c_double, C.c_int, C.POINTER(C.c_int), _DP]),
    "fdmap_gpu_test_wait_timeout": (C.c_int, [_VP, C.c_double]),
    "fdmap_gpu_time_params": (C.c_int, [_VP, _DP, C.POINTER(C.c_int)]),
    "fdmap_gpu_get_metric": (C.c_int, [_VP, C.c_int, _DP]),
    "fdmap_gpu_get_side_impedance": (C.c_int, [_VP, C.c_int, C.c_int, _DP]),
    "fdmap_gpu_get_pml": (C.c_int, [_VP, C.c_int, _DP]),
    "fdmap_gpu_get_side_displacement": (C.c_int, [_VP, C.c_int, C.c_int, _DP, _DP]),
    "fdmap_gpu_get_energy": (C.c_int, [_VP, _DP]),
    "fdmap_gpu_get_displacement": (C.c_int, [_VP, _DP, _DP]),
    "fdmap_gpu_set_displacement": (C.c_int, [_VP, _DP, _DP]),
    "fdmap_gpu_get_peak": (C.c_int, [_VP, _DP, _DP]),
    "fdmap_gpu_set_peak": (C.c_int, [_VP, _DP, _DP]),
    "fdmap_gpu_set_side_displacement": (C.c_int, [_VP, C.c_int, C.c_int, _DP, _DP]),
    "fdmap_gpu_set_pml": (C.c_int, [_VP, C.c_int, _DP]),
    "fdmap_gpu_fault_max_noalloc": (C.c_int, [_VP, C.c_int, C.c_int, _DP]),
    "fdmap_gpu_output_add": (C.c_int, [_VP, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_int, C.c_int, C.c_int, C.c_longlong, C.c_longlong, C.c_int]),
    "fdmap_gpu_output_open": (C.c_int, [_VP, C.c_char_p, C.c_int]),
    "fdmap_gpu_output_flush": (C.c_int, [_VP]),
    "fdmap_gpu_output_close": (C.c_int, [_VP]),
    "fdmap_gpu_create_part": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_int), C.POINTER(_VP)]),
    "fdmap_gpu_part_interfaces": (C.c_int, [_VP, C.POINTER(C.c_int), C.c_int]),
    "fdmap_gpu_part_buffers": (C.c_int, [_VP, C.c_int, C.c_longlong, C.POINTER(_DP), C.POINTER(_DP),
                                         C.POINTER(C.c_longlong)]),
    "fdmap_gpu_set_exchange": (C.c_int, [_VP, _VP, _VP]),
    "fdmap_gpu_group_init_edges": (C.c_int, [C.POINTER(_VP), C.c_int, C.c_double]),
    "fdmap_gpu_group_time_step": (C.c_int, [C.POINTER(_VP), C.c_int, C.c_double, C.c_double, C.c_int]),
    "fdmap_gpu_group_run": (C.c_int, [C.POINTER(_VP), C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                      C.c_int]),
    "fdmap_gpu_trace": (C.c_int, [_VP, C.c_int]),
    "fdmap_gpu_trace_read": (C.c_int, [_VP, C.POINTER(C.c_ulonglong), C.c_int]),
    "fdmap_gpu_launch_count": (C.c_longlong, [_VP]),
    "fdmap_gpu_device_bytes": (C.c_longlong, [_VP]),
    "fdmap_gpu_destroy": (None, [_VP]),
    "fdmap_gpu_strerror": (C.c_char_p, [C.c_int]),
    "fdmap_gpu_last_error": (C.c_char_p, []),
    # fdmap_gpu.h: batched ensemble
    "fdmap_gpu_ensemble_create": (C.c_int, [C.POINTER(_VP), C.c_int, C.c_int, C.c_int, C.POINTER(_VP)]),
    "fdmap_gpu_ensemble_size": (C.c_int, [_VP]),
    "fdmap_gpu_ensemble_instance": (C.c_int, [_VP, C.c_int, C.POINTER(_VP)]),
    "fdmap_gpu_ensemble_time_step": (C.c_int, [_VP, C.c_double, C.c_double, C.c_int]),
    "fdmap_gpu_ensemble_run": (C.c_int, [_VP, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]),
    "fdmap_gpu_ensemble_synchronize": (C.c_int, [_VP]),
    "fdmap_gpu_ensemble_set_shape": (C.c_int, [_VP, C.POINTER(C.c_int)]),
    "fdmap_gpu_ensemble_get_shape": (C.c_int, [_VP, C.POINTER(C.c_int)]),
    "fdmap_gpu_ensemble_tune": (C.c_int, [_VP, C.c_double, C.c_int, C.POINTER(C.c_int), _DP]),
    "fdmap_gpu_ensemble_set_tile": (C.c_int, [_VP, C.c_int]),
    "fdmap_gpu_ensemble_set_pairs": (C.c_int, [_VP, C.c_int]),
    "fdmap_gpu_ensemble_get_pairs": (C.c_int, [_VP]),
    "fdmap_gpu_ensemble_get_tile": (C.c_int, [_VP, C.POINTER(C.c_int)]),
    "fdmap_gpu_ensemble_launch_count": (C.c_longlong, [_VP]),
    "fdmap_gpu_ensemble_destroy": (None, [_VP]),
    # fdmap_gpu.h: forward/backward pair
    "fdmap_gpu_adjoint_create": (C.c_int, [_VP, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int,
                                           C.POINTER(_VP)]),
    "fdmap_gpu_adjoint_set_material": (C.c_int, [_VP, _DP, _DP]),
    "fdmap_gpu_adjoint_forward": (C.c_int, [_VP, C.c_double, C.c_double, C.c_int, _DP, _DP, _DP]),
    "fdmap_gpu_adjoint_backward": (C.c_int, [_VP, _DP, _DP]),
    "fdmap_gpu_adjoint_fields": (C.c_int, [_VP, _DP]),
    "fdmap_gpu_adjoint_fault_size": (C.c_int, [_VP]),
    "fdmap_gpu_adjoint_time_params": (C.c_int, [_VP, _DP, C.POINTER(C.c_int)]),
    "fdmap_gpu_adjoint_set_prestress": (C.c_int, [_VP, _DP]),
    "fdmap_gpu_adjoint_get_prestress": (C.c_int, [_VP, _DP]),
    "fdmap_gpu_adjoint_prestress_gradient": (C.c_int, [_VP, _DP]),
    "fdmap_gpu_adjoint_set_store_budget": (C.c_int, [_VP, C.c_longlong]),
    "fdmap_gpu_adjoint_segment_bytes": (C.c_longlong, [_VP]),
    "fdmap_gpu_adjoint_resident_segments": (C.c_int, [_VP]),
    "fdmap_gpu_adjoint_destroy": (None, [_VP]),
}

_lib = None


class FdmapError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str = ""):
        self.code = code
        msg = f"{where}: {FDMAP_ERRORS.get(code, 'error')} ({code})"
        if detail:
            msg += f": {detail}"
        super().__init__(msg)


def lib() -> C.CDLL:
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `python -m fdmap_github_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def dptr(a) -> C.POINTER(C.c_double):
    """Pointer to a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    assert a.dtype.name == "float64" and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_DP)


def check_host(rc: int, where: str, L=None) -> None:
    if rc != 0:
        raise FdmapError(rc, where, (L if L is not None else lib()).fdmap_host_last_error().decode())


def check_gpu(rc: int, where: str) -> None:
    if rc != 0:
        raise FdmapError(rc, where, lib().fdmap_gpu_last_error().decode())
