"""ctypes binding of libgpulsm.so (the C ABI declared in include/gpulsm.h).

The library is the only compute path: there is no CPU fallback.  Loading
fails loudly when libgpulsm.so has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpulsm.so")
HEADER_PATH = os.path.join(HERE, "..", "include", "gpulsm.h")

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CAPACITY = 2
ERR_PUBLICATION = 3
ERR_TIMEOUT = 4
ERR_CUDA = 5
ERR_OUT_OF_MEMORY = 6
ERR_LENGTH = 7

STATUS_OUTPUT_OVERFLOW = 1 << 3
STATUS_WAIT_TIMEOUT = 1 << 8
STATUS_BAD_INPUT = 1 << 9

SEARCH_DIRECTORY = 0
SEARCH_LEARNED = 1
SEARCH_BINARY = 2


class GpuLsmError(RuntimeError):
    """Base class of errors reported through the C ABI; `.status` is the gpulsm_status."""

    status = -1

    def __init__(self, message: str, status: int):
        super().__init__(message)
        self.status = status


class InvalidArgument(GpuLsmError, ValueError):
    """std::invalid_argument in the reference (null pointers, bad configuration)."""


class CapacityError(GpuLsmError):
    """runtime_error '... capacity exhausted ...' in the reference (GPULSMOpt.cuh:6819-6837)."""


class PublicationError(GpuLsmError):
    """runtime_error 'publication failed' in the reference."""


class DeviceTimeout(GpuLsmError):
    """A bounded device wait gave up (status bit 8); the context stays usable."""


class CudaError(GpuLsmError):
    """A CUDA runtime error (CUDA_CHECK in the reference)."""


class OutOfDeviceMemory(GpuLsmError, MemoryError):
    """std::bad_alloc in the reference."""


class LengthError(GpuLsmError, ValueError):
    """std::length_error in the reference."""


_ERRORS = {
    ERR_INVALID_ARGUMENT: InvalidArgument,
    ERR_CAPACITY: CapacityError,
    ERR_PUBLICATION: PublicationError,
    ERR_TIMEOUT: DeviceTimeout,
    ERR_CUDA: CudaError,
    ERR_OUT_OF_MEMORY: OutOfDeviceMemory,
    ERR_LENGTH: LengthError,
}


class DictConfig(C.Structure):
    _fields_ = [
        ("max_elements", C.c_uint64),
        ("batch_capacity", C.c_uint64),
        ("level_zero_capacity", C.c_uint64),
        ("fan_in", C.c_uint32),
        ("rows_per_bucket_log2", C.c_uint32),
        ("search_mode", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class FlixConfig(C.Structure):
    _fields_ = [
        ("key_bits", C.c_uint32),
        ("node_size", C.c_uint32),
        ("fill_percent", C.c_uint32),
        ("search_mode", C.c_uint32),
        ("max_elements", C.c_uint64),
    ]


class ServeStats(C.Structure):
    _fields_ = [
        ("completed", C.c_uint64),
        ("rejected", C.c_uint64),
        ("rounds", C.c_uint64),
        ("keys", C.c_uint64),
        ("p50_us", C.c_double),
        ("p99_us", C.c_double),
        ("max_us", C.c_double),
        ("mean_us", C.c_double),
        ("mean_round_keys", C.c_double),
        ("wall_s", C.c_double),
        ("gpu_busy_s", C.c_double),
        ("host_launch_s", C.c_double),
        ("graph_rounds", C.c_uint64),
        ("kind_gpu_s", C.c_double * 4),
        ("host_copy_s", C.c_double),
        ("host_scatter_s", C.c_double),
        ("graph_updates", C.c_uint64),
        ("stage_flushes", C.c_uint64),
        ("max_round_gpu_us", C.c_double),
        ("max_launch_us", C.c_double),
    ]


def stats_dict(s: ServeStats) -> dict:
    """A ServeStats as a dict (array fields as lists)."""
    out = {}
    for k, _ in ServeStats._fields_:
        v = getattr(s, k)
        out[k] = list(v) if isinstance(v, C.Array) else v
    return out


class LoadSpec(C.Structure):
    _fields_ = [
        ("rate_per_s", C.c_double),
        ("seconds", C.c_double),
        ("mix", C.c_double * 4),
        ("zipf_s", C.c_double),
        ("max_outstanding", C.c_uint32),
        ("min_keys", C.c_uint32),
        ("max_keys", C.c_uint32),
        ("range_width_max", C.c_uint32),
        ("seed", C.c_uint64),
        ("universe", C.c_void_p),
        ("universe_n", C.c_uint64),
    ]


_lib = None


def header_functions() -> list[str]:
    """Names of every function declared in include/gpulsm.h."""
    with open(HEADER_PATH) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gpulsm_[a-z0-9_]+)\s*\(", text)))


def load() -> C.CDLL:
    """Load libgpulsm.so and declare every entry point; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python gpu-lsm-tree_b200/build.py` "
            "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    vp, u64, u32, i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int
    pvp = C.POINTER(C.c_void_p)
    sig = {
        "gpulsm_last_error": (C.c_char_p, []),
        "gpulsm_version": (C.c_char_p, []),
        "gpulsm_launch_count": (C.c_uint64, []),
        "gpulsm_dict_create": (i32, [C.POINTER(DictConfig), pvp]),
        "gpulsm_dict_destroy": (i32, [vp]),
        "gpulsm_dict_clear": (i32, [vp, vp]),
        "gpulsm_dict_join": (i32, [vp, vp]),
        "gpulsm_dict_bulk_build": (i32, [vp, vp, vp, u64, vp]),
        "gpulsm_dict_insert": (i32, [vp, vp, vp, u64, vp]),
        "gpulsm_dict_erase": (i32, [vp, vp, u64, vp]),
        "gpulsm_dict_update": (i32, [vp, vp, vp, vp, u64, vp]),
        "gpulsm_dict_lookup": (i32, [vp, vp, u64, vp, vp, vp]),
        "gpulsm_dict_range_sum": (i32, [vp, vp, vp, u64, vp, vp]),
        "gpulsm_dict_range_count": (i32, [vp, vp, vp, u64, vp, vp]),
        "gpulsm_dict_range_offsets": (i32, [vp, vp, vp, u64, vp, vp]),
        "gpulsm_dict_range_pairs": (i32, [vp, vp, vp, u64, vp, vp, vp, vp]),
        "gpulsm_dict_successor": (i32, [vp, vp, u64, vp, vp]),
        "gpulsm_dict_status": (i32, [vp, C.POINTER(u32)]),
        "gpulsm_dict_resident_bytes": (i32, [vp, C.POINTER(u64)]),
        "gpulsm_dict_kernel_timing": (i32, [vp, i32]),
        "gpulsm_dict_kernel_timing_read": (i32, [vp, C.POINTER(u64), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "gpulsm_dict_size": (i32, [vp, C.POINTER(u64), C.POINTER(u32)]),
        "gpulsm_dict_cleanup": (i32, [vp, vp, C.POINTER(u64)]),
        "gpulsm_flix_create": (i32, [C.POINTER(FlixConfig), pvp]),
        "gpulsm_flix_destroy": (i32, [vp]),
        "gpulsm_flix_build": (i32, [vp, vp, vp, u64, u64, vp]),
        "gpulsm_flix_insert": (i32, [vp, vp, vp, u64, vp]),
        "gpulsm_flix_remove": (i32, [vp, vp, u64, vp]),
        "gpulsm_flix_lookups_ordered": (i32, [vp, vp, u64, vp, vp]),
        "gpulsm_flix_lookups_successor": (i32, [vp, vp, u64, vp, vp]),
        "gpulsm_flix_lookup": (i32, [vp, vp, u64, vp, vp]),
        "gpulsm_flix_successor": (i32, [vp, vp, u64, vp, vp]),
        "gpulsm_flix_rebuild": (i32, [vp, vp]),
        "gpulsm_flix_resident_bytes": (i32, [vp, C.POINTER(u64)]),
        "gpulsm_flix_size": (i32, [vp, C.POINTER(u64)]),
        "gpulsm_flix_status": (i32, [vp, C.POINTER(u32)]),
        "gpulsm_flix_allocation_state": (i32, [vp, C.POINTER(u64), C.POINTER(u64), C.POINTER(u64),
                                               C.POINTER(u32)]),
        "gpulsm_sort_pairs": (i32, [vp, vp, vp, vp, u64, u32, u32, u32, vp]),
        "gpulsm_sort_pairs_noalloc": (i32, [vp, vp, vp, vp, u64, u32, u32, u32, vp]),
        "gpulsm_sort_noalloc_scratch_bytes": (u64, []),
        "gpulsm_tenants_create": (i32, [u32, vp, u64, u32, u32, u32, pvp]),
        "gpulsm_tenants_destroy": (i32, [vp]),
        "gpulsm_tenants_set_tuning": (i32, [vp, u32, u32, u32]),
        "gpulsm_tenants_insert_round": (i32, [vp, vp, vp, vp, vp]),
        "gpulsm_tenants_round_graph": (i32, [vp, vp, vp, vp, vp]),
        "gpulsm_tenants_lookup": (i32, [vp, vp, vp, u64, vp, vp, vp]),
        "gpulsm_tenants_sizes": (i32, [vp, vp]),
        "gpulsm_tenants_status": (i32, [vp, C.POINTER(u32)]),
        "gpulsm_tenants_resident_bytes": (i32, [vp, C.POINTER(u64)]),
        "gpulsm_server_create": (i32, [C.POINTER(DictConfig), u64, u32, u32, pvp]),
        "gpulsm_server_destroy": (i32, [vp]),
        "gpulsm_server_bulk_build": (i32, [vp, vp, vp, u64, vp]),
        "gpulsm_server_submit": (i32, [vp, u32, vp, vp, u64, vp, vp, C.POINTER(u64)]),
        "gpulsm_server_poll": (i32, [vp, u64, C.POINTER(C.c_int32)]),
        "gpulsm_server_wait": (i32, [vp, u64, C.POINTER(C.c_int32)]),
        "gpulsm_server_wait_round": (i32, [vp, u64, C.POINTER(C.c_int32), C.POINTER(u64)]),
        "gpulsm_server_drain": (i32, [vp]),
        "gpulsm_server_stats": (i32, [vp, C.POINTER(ServeStats)]),
        "gpulsm_server_reset_stats": (i32, [vp]),
        "gpulsm_server_set_staged_updates": (i32, [vp, C.c_int]),
        "gpulsm_server_run_load": (i32, [vp, C.POINTER(LoadSpec), C.POINTER(ServeStats)]),
        "gpulsm_server_resident_bytes": (i32, [vp, C.POINTER(u64)]),
        "gpulsm_model_bytes": (u64, [u32]),
        "gpulsm_model_fit": (i32, [vp, u64, u32, u32, u32, vp, vp, vp]),
        "gpulsm_model_gradients": (i32, [vp, u64, u32, u32, vp, vp, vp, vp]),
        "gpulsm_model_lower_bound": (i32, [vp, u64, u32, u32, vp, vp, u64, vp, vp]),
        "gpulsm_binary_lower_bound": (i32, [vp, u64, u32, vp, u64, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(code: int) -> None:
    """Raise the mapped exception for a non-zero gpulsm_status."""
    if code == OK:
        return
    msg = load().gpulsm_last_error()
    msg = msg.decode() if msg else f"gpulsm status {code}"
    raise _ERRORS.get(code, GpuLsmError)(msg, code)
