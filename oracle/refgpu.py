"""ctypes wrappers of the reference's own GPU engines, compiled from the
reference headers in place by oracle/Makefile:
  oracle/_ref/libref_gpulsmopt.so  GPULSMOpt (ref_gpulsmopt_shim.cu)
  oracle/_ref/libref_flix.so       FliX's bucket layer (ref_flix_shim.cu)
TEST INFRASTRUCTURE ONLY: used by tests to pin the oracle and to compare our
engine with the reference kernels on the same GPU."""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "libref_gpulsmopt.so")
FLIX_LIB = os.path.join(_HERE, "_ref", "libref_flix.so")
_lib = None
_flib = None


def available() -> bool:
    return os.path.exists(LIB)


def flix_available() -> bool:
    return os.path.exists(FLIX_LIB)


def _load():
    global _lib
    if _lib is None:
        lib = C.CDLL(LIB)
        vp, u64, i32 = C.c_void_p, C.c_uint64, C.c_int
        sig = {
            "ref_last_error": (C.c_char_p, []),
            "ref_create": (i32, [u64, u64, u64, C.POINTER(C.c_void_p)]),
            "ref_destroy": (i32, [vp]),
            "ref_clear": (i32, [vp, vp]),
            "ref_bulk_build": (i32, [vp, vp, vp, u64, vp]),
            "ref_insert": (i32, [vp, vp, vp, u64, vp]),
            "ref_erase": (i32, [vp, vp, u64, vp]),
            "ref_lookup": (i32, [vp, vp, u64, vp, vp, i32, vp]),
            "ref_range": (i32, [vp, vp, vp, u64, vp, vp]),
            "ref_successor": (i32, [vp, vp, u64, vp, vp]),
            "ref_status": (i32, [vp, C.POINTER(C.c_uint32)]),
            "ref_resident_bytes": (i32, [vp, C.POINTER(C.c_uint64)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class RefError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _chk(code: int):
    if code:
        raise RefError(code, _load().ref_last_error().decode())


def _stream(s):
    import torch

    return (s or torch.cuda.current_stream()).cuda_stream or None


class RefGPULSMOpt:
    """Reference GPULSMOpt over torch CUDA tensors (32-bit bit patterns)."""

    def __init__(self, max_elements: int, batch_capacity: int = 0, level_zero_capacity: int = 0):
        self._lib = _load()
        h = C.c_void_p()
        _chk(self._lib.ref_create(max_elements, batch_capacity, level_zero_capacity, C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ref_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clear(self, stream=None):
        _chk(self._lib.ref_clear(self._h, _stream(stream)))

    def bulk_build(self, keys, values, stream=None):
        _chk(self._lib.ref_bulk_build(self._h, keys.data_ptr(), values.data_ptr(), keys.numel(), _stream(stream)))

    def insert(self, keys, values, stream=None):
        _chk(self._lib.ref_insert(self._h, keys.data_ptr(), values.data_ptr(), keys.numel(), _stream(stream)))

    def erase(self, keys, stream=None):
        _chk(self._lib.ref_erase(self._h, keys.data_ptr(), keys.numel(), _stream(stream)))

    def lookup(self, queries, out_values, out_found=None, grouped=False, stream=None):
        _chk(self._lib.ref_lookup(self._h, queries.data_ptr(), queries.numel(), out_values.data_ptr(),
                                  out_found.data_ptr() if out_found is not None else None, int(grouped),
                                  _stream(stream)))

    def range(self, lo, hi, out_sums, stream=None):
        _chk(self._lib.ref_range(self._h, lo.data_ptr(), hi.data_ptr(), lo.numel(), out_sums.data_ptr(),
                                 _stream(stream)))

    def successor(self, queries, out_keys, stream=None):
        _chk(self._lib.ref_successor(self._h, queries.data_ptr(), queries.numel(), out_keys.data_ptr(),
                                     _stream(stream)))

    def status(self) -> int:
        v = C.c_uint32()
        _chk(self._lib.ref_status(self._h, C.byref(v)))
        return int(v.value)


def _load_flix():
    global _flib
    if _flib is None:
        lib = C.CDLL(FLIX_LIB)
        vp, u64, i32 = C.c_void_p, C.c_uint64, C.c_int
        p64 = C.POINTER(C.c_uint64)
        sig = {
            "reff_last_error": (C.c_char_p, []),
            "reff_create": (i32, [i32, C.POINTER(C.c_void_p)]),
            "reff_destroy": (i32, [vp]),
            "reff_build": (i32, [vp, vp, u64, u64]),
            "reff_rebuild": (i32, [vp]),
            "reff_insert": (i32, [vp, vp, vp, u64, vp]),
            "reff_remove": (i32, [vp, vp, u64, vp]),
            "reff_lookups_ordered": (i32, [vp, vp, vp, u64, vp]),
            "reff_lookups_successor": (i32, [vp, vp, vp, u64, vp]),
            "reff_total_keys": (i32, [vp, vp, p64]),
            "reff_resident_bytes": (i32, [vp, p64]),
            "reff_allocation_state": (i32, [vp, p64, p64, p64]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _flib = lib
    return _flib


def _fchk(code: int):
    if code:
        raise RefError(code, _load_flix().reff_last_error().decode())


class RefFlix:
    """The reference's FliX bucket layer (class cg_rtx_index_updates with 32-key
    nodes, FliX/impl_cg_rtx_index_updates.cuh:1422) over torch CUDA tensors.

    Its interface contract holds here too: build keys are unique, insert and
    remove batches are sorted and unique, probes of lookups_ordered and
    lookups_successor are sorted (FliX/benchmarks_updates.cuh:252-360)."""

    def __init__(self, key_bits: int = 64):
        self._lib = _load_flix()
        self.key_bits = key_bits
        h = C.c_void_p()
        _fchk(self._lib.reff_create(key_bits, C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.reff_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build_bucket_layer_only(self, keys, max_size: int):
        _fchk(self._lib.reff_build(self._h, keys.data_ptr(), keys.numel(), max_size))

    def rebuild_bucket_layer_only(self):
        _fchk(self._lib.reff_rebuild(self._h))

    def insert(self, keys, values, stream=None):
        _fchk(self._lib.reff_insert(self._h, keys.data_ptr(), values.data_ptr(), keys.numel(), _stream(stream)))

    def remove(self, keys, stream=None):
        _fchk(self._lib.reff_remove(self._h, keys.data_ptr(), keys.numel(), _stream(stream)))

    def lookups_ordered(self, keys, out, stream=None):
        _fchk(self._lib.reff_lookups_ordered(self._h, keys.data_ptr(), out.data_ptr(), keys.numel(), _stream(stream)))

    def lookups_successor(self, keys, out, stream=None):
        _fchk(self._lib.reff_lookups_successor(self._h, keys.data_ptr(), out.data_ptr(), keys.numel(),
                                               _stream(stream)))

    def total_keys(self, stream=None) -> int:
        v = C.c_uint64()
        _fchk(self._lib.reff_total_keys(self._h, _stream(stream), C.byref(v)))
        return int(v.value)

    def allocation_state(self) -> tuple[int, int, int]:
        """(next free allocation-region node, allocation-region nodes, buckets incl. overflow)."""
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _fchk(self._lib.reff_allocation_state(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return int(a.value), int(b.value), int(c.value)
