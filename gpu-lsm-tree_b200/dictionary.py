"""Python mirror of the reference's GPU dictionary interfaces over the C ABI.

`GPULSMOpt` mirrors class GPULSMOpt (GPULSMOpt.cuh:5599-5881): the same method
names, argument meaning and error classes (ValueError for invalid_argument,
CapacityError for the "capacity" runtime_error, MemoryError for bad_alloc).
`GpuLsmOptIndex` mirrors FliX's index-concept adapter around it
(FliX/impl_gpulsmopt.cuh:137-311).  Device buffers are torch CUDA tensors of
32-bit integers (int32 or uint32 bit patterns); torch only supplies memory and
streams - every operation runs in libgpulsm.so.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _native as N


def _stream(stream) -> int | None:
    import torch

    if stream is None:
        return torch.cuda.current_stream().cuda_stream or None
    if isinstance(stream, int):
        return stream or None
    return stream.cuda_stream or None


def _ptr(t, name: str, elem_bytes: int = 4, count: int | None = None) -> int | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise N.InvalidArgument(f"{name} must be a CUDA tensor", N.ERR_INVALID_ARGUMENT)
    if not t.is_contiguous():
        raise N.InvalidArgument(f"{name} must be contiguous", N.ERR_INVALID_ARGUMENT)
    if t.element_size() != elem_bytes:
        raise N.InvalidArgument(f"{name} must hold {elem_bytes}-byte elements", N.ERR_INVALID_ARGUMENT)
    if count is not None and t.numel() < count:
        raise N.InvalidArgument(f"{name} holds {t.numel()} < {count} elements", N.ERR_INVALID_ARGUMENT)
    return t.data_ptr()


@dataclass
class DictionaryConfig:
    """gpu_dictionary_adapter.cuh:16-23 plus the B200 tunables."""

    max_elements: int = 0
    batch_capacity: int = 0
    level_zero_capacity: int = 0
    fan_in: int = 0
    rows_per_bucket_log2: int = 0
    search_mode: int = N.SEARCH_DIRECTORY


class GPULSMOpt:
    """GPU LSM dictionary with GPULSMOpt semantics (upsert, tombstones, u32 keys/values)."""

    def __init__(self, config: DictionaryConfig | None = None, **kw):
        cfg = config or DictionaryConfig(**kw)
        self._lib = N.load()
        c = N.DictConfig(cfg.max_elements, cfg.batch_capacity, cfg.level_zero_capacity, cfg.fan_in,
                         cfg.rows_per_bucket_log2, cfg.search_mode, 0)
        h = C.c_void_p()
        N.check(self._lib.gpulsm_dict_create(C.byref(c), C.byref(h)))
        self._h = h
        self.config = cfg

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gpulsm_dict_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- updates -----------------------------------------------------------
    def clear(self, stream=None):
        N.check(self._lib.gpulsm_dict_clear(self._h, _stream(stream)))

    def join(self, stream=None):
        """Make `stream` wait until every update enqueued so far has been merged
        (updates return once admitted; reads join by themselves)."""
        N.check(self._lib.gpulsm_dict_join(self._h, _stream(stream)))

    def bulk_build(self, keys, values, count: int | None = None, stream=None):
        n = keys.numel() if count is None else count
        N.check(self._lib.gpulsm_dict_bulk_build(self._h, _ptr(keys, "keys", count=n),
                                                 _ptr(values, "values", count=n), n, _stream(stream)))

    def insert(self, keys, values, count: int | None = None, stream=None):
        n = keys.numel() if count is None else count
        N.check(self._lib.gpulsm_dict_insert(self._h, _ptr(keys, "keys", count=n),
                                             _ptr(values, "values", count=n), n, _stream(stream)))

    def erase(self, keys, count: int | None = None, stream=None):
        n = keys.numel() if count is None else count
        N.check(self._lib.gpulsm_dict_erase(self._h, _ptr(keys, "keys", count=n), n, _stream(stream)))

    def update(self, keys, values, erase, count: int | None = None, stream=None):
        """One batch of inserts and erases (no GPULSMOpt counterpart): row i
        erases keys[i] when erase[i] (uint8) is nonzero, else inserts
        (keys[i], values[i]); the last row of a key wins."""
        n = keys.numel() if count is None else count
        N.check(self._lib.gpulsm_dict_update(self._h, _ptr(keys, "keys", count=n), _ptr(values, "values", count=n),
                                             _ptr(erase, "erase", 1, n), n, _stream(stream)))

    # --- queries -----------------------------------------------------------
    def lookup(self, queries, out_values, out_found=None, count: int | None = None, stream=None):
        n = queries.numel() if count is None else count
        N.check(self._lib.gpulsm_dict_lookup(
            self._h, _ptr(queries, "queries", count=n), n, _ptr(out_values, "out_values", count=n),
            _ptr(out_found, "out_found", 1, n), _stream(stream)))

    def range(self, lo, hi, out_sums, count: int | None = None, stream=None):
        """GPULSMOpt::range: u32 sum of live values in [lo, hi] (wraps at 2^32)."""
        n = lo.numel() if count is None else count
        N.check(self._lib.gpulsm_dict_range_sum(self._h, _ptr(lo, "lo", count=n), _ptr(hi, "hi", count=n),
                                                n, _ptr(out_sums, "out_sums", count=n), _stream(stream)))

    def range_count(self, lo, hi, out_counts, count: int | None = None, stream=None):
        n = lo.numel() if count is None else count
        N.check(self._lib.gpulsm_dict_range_count(self._h, _ptr(lo, "lo", count=n), _ptr(hi, "hi", count=n),
                                                  n, _ptr(out_counts, "out_counts", count=n), _stream(stream)))

    def range_offsets(self, lo, hi, offsets, count: int | None = None, stream=None):
        n = lo.numel() if count is None else count
        N.check(self._lib.gpulsm_dict_range_offsets(self._h, _ptr(lo, "lo", count=n), _ptr(hi, "hi", count=n),
                                                    n, _ptr(offsets, "offsets", 8, n + 1), _stream(stream)))

    def range_pairs(self, lo, hi, offsets, out_keys, out_values, count: int | None = None, stream=None):
        n = lo.numel() if count is None else count
        N.check(self._lib.gpulsm_dict_range_pairs(
            self._h, _ptr(lo, "lo", count=n), _ptr(hi, "hi", count=n), n,
            _ptr(offsets, "offsets", 8, n + 1), _ptr(out_keys, "out_keys"), _ptr(out_values, "out_values"),
            _stream(stream)))

    def range_query(self, lo, hi, stream=None):
        """Convenience: offsets, then allocate and fill (keys, values) pairs.  Synchronises."""
        import torch

        n = lo.numel()
        offsets = torch.empty(n + 1, dtype=torch.int64, device=lo.device)
        self.range_offsets(lo, hi, offsets, stream=stream)
        total = int(offsets[n].item())
        keys = torch.empty(max(total, 1), dtype=torch.int32, device=lo.device)
        vals = torch.empty(max(total, 1), dtype=torch.int32, device=lo.device)
        self.range_pairs(lo, hi, offsets, keys, vals, stream=stream)
        return offsets, keys[:total], vals[:total]

    def successor(self, queries, out_keys, count: int | None = None, stream=None):
        n = queries.numel() if count is None else count
        N.check(self._lib.gpulsm_dict_successor(self._h, _ptr(queries, "queries", count=n), n,
                                                _ptr(out_keys, "out_keys", count=n), _stream(stream)))

    # --- introspection ------------------------------------------------------
    def canonical_carry_status(self) -> int:
        v = C.c_uint32()
        N.check(self._lib.gpulsm_dict_status(self._h, C.byref(v)))
        return int(v.value)

    def gpu_resident_bytes(self) -> int:
        v = C.c_uint64()
        N.check(self._lib.gpulsm_dict_resident_bytes(self._h, C.byref(v)))
        return int(v.value)

    def kernel_timing(self, enable: bool) -> None:
        """Bracket every merge kernel launch with CUDA events (measurement hook)."""
        N.check(self._lib.gpulsm_dict_kernel_timing(self._h, 1 if enable else 0))

    def kernel_timing_read(self) -> dict:
        """Merges timed since the last read: launches, summed device ms, algorithmic bytes."""
        n, ms, b = C.c_uint64(), C.c_double(), C.c_double()
        N.check(self._lib.gpulsm_dict_kernel_timing_read(self._h, C.byref(n), C.byref(ms), C.byref(b)))
        return {"launches": int(n.value), "ms": float(ms.value), "bytes": float(b.value)}

    def cleanup(self, stream=None) -> int:
        """LSMu's explicit cleanup (FliX/impl_lsm_tree.cuh:1256-1400): one level of
        the newest live versions; returns the live key count."""
        v = C.c_uint64()
        N.check(self._lib.gpulsm_dict_cleanup(self._h, _stream(stream), C.byref(v)))
        return int(v.value)

    def size(self) -> tuple[int, int]:
        rows, levels = C.c_uint64(), C.c_uint32()
        N.check(self._lib.gpulsm_dict_size(self._h, C.byref(rows), C.byref(levels)))
        return int(rows.value), int(levels.value)


class GpuLsmOptIndex:
    """FliX index-concept adapter (FliX/impl_gpulsmopt.cuh:137-311) over GPULSMOpt.

    build() assigns values 0..n-1 (:223-229); lookup() passes no out_found, so a
    miss reads 0xffffffff (:247-259).
    """

    def __init__(self, batch_capacity: int = 1 << 20, level_zero_capacity: int = 0):
        self.batch_capacity = batch_capacity
        self.level_zero_capacity = level_zero_capacity
        self.dictionary: GPULSMOpt | None = None

    def build(self, keys, size: int, max_size: int | None = None, stream=None):
        import torch

        configured = max(max_size or size, size)
        if configured > (0xFFFFFFFF // 2):
            raise RuntimeError("GPULSMOpt supports at most 2^31-1 records")
        self.dictionary = GPULSMOpt(DictionaryConfig(
            max_elements=configured,
            batch_capacity=max(1, min(configured or size, self.batch_capacity)),
            level_zero_capacity=self.level_zero_capacity))
        values = torch.arange(size, dtype=torch.int32, device=keys.device)
        self.dictionary.bulk_build(keys, values, size, stream)

    def _d(self) -> GPULSMOpt:
        if self.dictionary is None:
            raise RuntimeError("GPULSMOpt index used before build")
        return self.dictionary

    def lookup(self, keys, result, size: int, stream=None):
        if size:
            self._d().lookup(keys, result, None, size, stream)

    def range_lookup_sum(self, lower, upper, result, size: int, stream=None):
        if size:
            self._d().range(lower, upper, result, size, stream)

    def insert(self, update_list, offsets, size: int, stream=None):
        self._d().insert(update_list, offsets, size, stream)

    def remove(self, update_list, size: int, stream=None):
        self._d().erase(update_list, size, stream)

    def lookups_successor(self, keys, result, size: int, stream=None):
        if size:
            self._d().successor(keys, result, size, stream)

    def gpu_resident_bytes(self) -> int:
        return self.dictionary.gpu_resident_bytes() if self.dictionary else 0


def sort_pairs(keys_in, values_in, keys_out, values_out, begin_bit: int = 0, end_bit: int | None = None,
               stream=None):
    """Stable onesweep radix sort of (key, u32 value) pairs (gpulsm_sort_pairs)."""
    lib = N.load()
    kb = keys_in.element_size() * 8
    end = kb if end_bit is None else end_bit
    n = keys_in.numel()
    N.check(lib.gpulsm_sort_pairs(_ptr(keys_in, "keys_in", kb // 8), _ptr(values_in, "values_in"),
                                  _ptr(keys_out, "keys_out", kb // 8, n), _ptr(values_out, "values_out"),
                                  n, kb, begin_bit, end, _stream(stream)))
