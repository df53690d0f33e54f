"""ctypes front end of the CPU oracle (liboracle.so).  TEST INFRASTRUCTURE ONLY.

The C sources (lsm_oracle.c, flix_oracle.c) restate the reference semantics and
cite the reference file:line of each rule.  This module only marshals numpy
arrays; it contains no dictionary logic of its own.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def build_oracle(reference: str | None = None) -> None:
    """Compile liboracle.so and, when `reference` names a reference checkout,
    the reference engines under oracle/_ref (read in place, never copied)."""
    if reference:
        subprocess.run(["make", "-s", "-C", _HERE, "all", f"REFERENCE={reference}"], check=True)
    else:
        subprocess.run(["make", "-s", "-C", _HERE, os.path.join(_HERE, "liboracle.so"),
                        os.path.join(_HERE, "libcpubaselines.so")], check=True)


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build_oracle()
    lib = C.CDLL(_LIB_PATH)
    vp = C.c_void_p
    u64 = C.c_uint64
    sig = {
        "orc_set_threads": (C.c_int, [C.c_int]),
        "orc_get_threads": (C.c_int, []),
        "orc_lsm_create": (vp, []),
        "orc_lsm_destroy": (None, [vp]),
        "orc_lsm_clear": (None, [vp]),
        "orc_lsm_size": (u64, [vp]),
        "orc_lsm_dump": (u64, [vp, _u32p, _u32p]),
        "orc_lsm_bulk_build": (None, [vp, _u32p, _u32p, u64]),
        "orc_lsm_insert": (None, [vp, _u32p, _u32p, u64]),
        "orc_lsm_erase": (None, [vp, _u32p, u64]),
        "orc_lsm_lookup": (None, [vp, _u32p, u64, _u32p, vp]),
        "orc_lsm_range_sum": (None, [vp, _u32p, _u32p, u64, _u32p]),
        "orc_lsm_range_count": (None, [vp, _u32p, _u32p, u64, _u32p]),
        "orc_lsm_range_offsets": (u64, [vp, _u32p, _u32p, u64, _u64p]),
        "orc_lsm_range_pairs": (None, [vp, _u32p, _u32p, u64, _u64p, _u32p, _u32p]),
        "orc_lsm_successor": (None, [vp, _u32p, u64, _u32p]),
        "orc_flix_create": (vp, [C.c_int]),
        "orc_flix_destroy": (None, [vp]),
        "orc_flix_size": (u64, [vp]),
        "orc_flix_dump": (u64, [vp, _u64p, _u32p]),
        "orc_flix_build": (None, [vp, _u64p, vp, u64]),
        "orc_flix_insert": (None, [vp, _u64p, vp, u64]),
        "orc_flix_remove": (None, [vp, _u64p, u64]),
        "orc_flix_lookup": (None, [vp, _u64p, u64, _u32p]),
        "orc_flix_successor": (None, [vp, _u64p, u64, _u64p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def oracle_threads(threads: int = 0) -> int:
    """Set the oracle's OpenMP thread count (0 = every host core); returns it."""
    return _load().orc_set_threads(int(threads))


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def _u64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64))


class OracleLSM:
    """GPULSMOpt semantics (upsert, tombstones) on the CPU: the std::map oracle."""

    def __init__(self):
        self._lib = _load()
        self._h = self._lib.orc_lsm_create()

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.orc_lsm_destroy(self._h)
            self._h = None

    def clear(self):
        self._lib.orc_lsm_clear(self._h)

    def __len__(self):
        return int(self._lib.orc_lsm_size(self._h))

    def dump(self):
        n = len(self)
        k = np.empty(n, np.uint32)
        v = np.empty(n, np.uint32)
        self._lib.orc_lsm_dump(self._h, k, v)
        return k, v

    def bulk_build(self, keys, values):
        k, v = _u32(keys), _u32(values)
        self._lib.orc_lsm_bulk_build(self._h, k, v, k.size)

    def insert(self, keys, values):
        k, v = _u32(keys), _u32(values)
        assert k.size == v.size
        self._lib.orc_lsm_insert(self._h, k, v, k.size)

    def erase(self, keys):
        k = _u32(keys)
        self._lib.orc_lsm_erase(self._h, k, k.size)

    def update(self, keys, values, erase):
        """Rows applied one at a time in input order: row i erases keys[i]
        when erase[i] is nonzero, else inserts (keys[i], values[i]).  Only the
        last row of each key matters, so those rows are applied as one erase
        and one insert (their key sets are disjoint)."""
        k, v, e = _u32(keys), _u32(values), np.asarray(erase, np.uint8)
        assert k.size == v.size == e.size
        _, first_from_end = np.unique(k[::-1], return_index=True)
        last = k.size - 1 - first_from_end
        er = e[last] != 0
        self.erase(k[last[er]])
        self.insert(k[last[~er]], v[last[~er]])

    def lookup(self, queries, with_found: bool = False):
        q = _u32(queries)
        out = np.empty(q.size, np.uint32)
        if with_found:
            found = np.empty(q.size, np.uint8)
            self._lib.orc_lsm_lookup(self._h, q, q.size, out, found.ctypes.data_as(C.c_void_p))
            return out, found
        self._lib.orc_lsm_lookup(self._h, q, q.size, out, None)
        return out

    def range_sum(self, lo, hi):
        lo, hi = _u32(lo), _u32(hi)
        out = np.empty(lo.size, np.uint32)
        self._lib.orc_lsm_range_sum(self._h, lo, hi, lo.size, out)
        return out

    def range_count(self, lo, hi):
        lo, hi = _u32(lo), _u32(hi)
        out = np.empty(lo.size, np.uint32)
        self._lib.orc_lsm_range_count(self._h, lo, hi, lo.size, out)
        return out

    def range_pairs(self, lo, hi):
        """Returns (offsets[n+1] u64, keys, values) with each query's live pairs in key order."""
        lo, hi = _u32(lo), _u32(hi)
        offsets = np.empty(lo.size + 1, np.uint64)
        total = int(self._lib.orc_lsm_range_offsets(self._h, lo, hi, lo.size, offsets))
        keys = np.empty(total, np.uint32)
        vals = np.empty(total, np.uint32)
        self._lib.orc_lsm_range_pairs(self._h, lo, hi, lo.size, offsets, keys, vals)
        return offsets, keys, vals

    def successor(self, queries):
        q = _u32(queries)
        out = np.empty(q.size, np.uint32)
        self._lib.orc_lsm_successor(self._h, q, q.size, out)
        return out


class OracleFlix:
    """FliX bucket-layer semantics (insert-if-absent, physical delete) on the CPU."""

    def __init__(self, key_bits: int = 64):
        assert key_bits in (32, 64)
        self.key_bits = key_bits
        self._lib = _load()
        self._h = self._lib.orc_flix_create(key_bits)

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.orc_flix_destroy(self._h)
            self._h = None

    def __len__(self):
        return int(self._lib.orc_flix_size(self._h))

    def dump(self):
        n = len(self)
        k = np.empty(n, np.uint64)
        v = np.empty(n, np.uint32)
        self._lib.orc_flix_dump(self._h, k, v)
        return k, v

    def build(self, keys, values=None):
        k = _u64(keys)
        v = None if values is None else _u32(values)
        self._lib.orc_flix_build(self._h, k, None if v is None else v.ctypes.data_as(C.c_void_p), k.size)

    def insert(self, keys, values):
        k, v = _u64(keys), _u32(values)
        assert k.size == v.size
        self._lib.orc_flix_insert(self._h, k, v.ctypes.data_as(C.c_void_p), k.size)

    def remove(self, keys):
        k = _u64(keys)
        self._lib.orc_flix_remove(self._h, k, k.size)

    def lookup(self, probes):
        p = _u64(probes)
        out = np.empty(p.size, np.uint32)
        self._lib.orc_flix_lookup(self._h, p, p.size, out)
        return out

    def successor(self, probes):
        p = _u64(probes)
        out = np.empty(p.size, np.uint64)
        self._lib.orc_flix_successor(self._h, p, p.size, out)
        return out


def model_gradients(keys, kmin: int, shift: int, nseg: int, a, b):
    """float64 gradients of the learned model's mean squared error (model_oracle.c)."""
    lib = _load()
    fn = lib.orc_model_gradients
    fn.restype = None
    fn.argtypes = [_u64p, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32,
                   np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"),
                   np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"),
                   np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"),
                   np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"), C.POINTER(C.c_double)]
    k = _u64(keys)
    ga = np.zeros(nseg, np.float64)
    gb = np.zeros(nseg, np.float64)
    loss = C.c_double()
    fn(k, k.size, kmin, shift, nseg, np.ascontiguousarray(a, np.float32), np.ascontiguousarray(b, np.float32),
       ga, gb, C.byref(loss))
    return ga, gb, loss.value


# ----------------------------------------------------------------------------
# CPU baselines (libcpubaselines.so, cpu_baselines.cpp): engines with the same
# semantics as OracleLSM, timed beside the GPU.  Test infrastructure only.
_CPU_LIB_PATH = os.path.join(_HERE, "libcpubaselines.so")
_cpu = None


def _load_cpu():
    global _cpu
    if _cpu is not None:
        return _cpu
    if not os.path.exists(_CPU_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE, _CPU_LIB_PATH], check=True)
    lib = C.CDLL(_CPU_LIB_PATH)
    vp, u64 = C.c_void_p, C.c_uint64
    sig = {}
    for pre in ("cpumap", "cpulsm"):
        sig.update({
            f"{pre}_destroy": (None, [vp]),
            f"{pre}_insert": (None, [vp, _u32p, _u32p, u64]),
            f"{pre}_erase": (None, [vp, _u32p, u64]),
            f"{pre}_lookup": (None, [vp, _u32p, u64, _u32p, vp]),
            f"{pre}_range_offsets": (u64, [vp, _u32p, _u32p, u64, _u64p]),
            f"{pre}_range_pairs": (None, [vp, _u32p, _u32p, u64, _u64p, _u32p, _u32p]),
        })
    sig["cpumap_create"] = (vp, [])
    sig["cpulsm_create"] = (vp, [u64, C.c_uint32])
    sig["cpulsm_levels"] = (C.c_uint32, [vp])
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _cpu = lib
    return lib


class _CpuBaseline:
    _pre = ""

    def __del__(self):
        if getattr(self, "_h", None):
            getattr(self._lib, f"{self._pre}_destroy")(self._h)
            self._h = None

    def insert(self, keys, values):
        k, v = _u32(keys), _u32(values)
        getattr(self._lib, f"{self._pre}_insert")(self._h, k, v, k.size)

    def erase(self, keys):
        k = _u32(keys)
        getattr(self._lib, f"{self._pre}_erase")(self._h, k, k.size)

    def lookup(self, queries, with_found: bool = False):
        q = _u32(queries)
        out = np.empty(q.size, np.uint32)
        found = np.empty(q.size, np.uint8) if with_found else None
        getattr(self._lib, f"{self._pre}_lookup")(self._h, q, q.size, out,
                                                  found.ctypes.data_as(C.c_void_p) if with_found else None)
        return (out, found) if with_found else out

    def range_pairs(self, lo, hi):
        lo, hi = _u32(lo), _u32(hi)
        offsets = np.empty(lo.size + 1, np.uint64)
        total = int(getattr(self._lib, f"{self._pre}_range_offsets")(self._h, lo, hi, lo.size, offsets))
        keys = np.empty(total, np.uint32)
        vals = np.empty(total, np.uint32)
        getattr(self._lib, f"{self._pre}_range_pairs")(self._h, lo, hi, lo.size, offsets, keys, vals)
        return offsets, keys, vals


class CpuMap(_CpuBaseline):
    """Single-thread std::map with GPULSMOpt's semantics."""
    _pre = "cpumap"

    def __init__(self):
        self._lib = _load_cpu()
        self._h = self._lib.cpumap_create()


class CpuLsm(_CpuBaseline):
    """Multi-threaded leveled LSM on every host core (OpenMP), GPULSMOpt's semantics."""
    _pre = "cpulsm"

    def __init__(self, cap0: int = 1 << 22, fan_in: int = 4):
        self._lib = _load_cpu()
        self._h = self._lib.cpulsm_create(cap0, fan_in)

    def levels(self) -> int:
        return int(self._lib.cpulsm_levels(self._h))
