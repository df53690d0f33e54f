"""ctypes wrapper of oracle/_ref/libref_gpulsmopt.so: the reference's own
GPULSMOpt engine (compiled from its header, see ref_gpulsmopt_shim.cu).
TEST INFRASTRUCTURE ONLY: used by tests to pin the oracle and to compare our
engine with the reference kernels on the same GPU."""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "libref_gpulsmopt.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


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
