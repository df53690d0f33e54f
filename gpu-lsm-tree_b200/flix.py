"""Python mirror of FliX's bucket-layer index surface over the C ABI.

`FlixIndex` follows class cg_rtx_index_updates in its bucket-layer
configuration (FliX/impl_cg_rtx_index_updates.cuh:1711-2677): the same method
names and argument meaning - build_bucket_layer_only, insert, remove,
lookups_ordered, lookups_successor, rebuild_bucket_layer_only,
gpu_resident_bytes - with 32- or 64-bit keys and u32 values ("offsets").
Semantics: insert if absent, physical delete, misses read 0xffffffff, a
successor miss reads 0xffffffff widened to the key type.  Unlike the
reference, insert/remove accept unsorted batches with duplicates (they are
sorted inside; the first occurrence of a key applies) and lookup()/successor()
accept unsorted probes.
"""
from __future__ import annotations

import ctypes as C

from . import _native as N
from .dictionary import _ptr, _stream


class FlixIndex:
    def __init__(self, key_bits: int = 64, node_size: int = 32, fill_percent: int = 50,
                 search_mode: int = N.SEARCH_DIRECTORY, max_elements: int = 0):
        self._lib = N.load()
        self.key_bits = key_bits
        self._kb = key_bits // 8
        c = N.FlixConfig(key_bits, node_size, fill_percent, search_mode, max_elements)
        h = C.c_void_p()
        N.check(self._lib.gpulsm_flix_create(C.byref(c), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gpulsm_flix_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _k(self, t, name, n=None):
        return _ptr(t, name, self._kb, n)

    # --- construction -------------------------------------------------------
    def build_bucket_layer_only(self, keys, size: int | None = None, max_size: int | None = None,
                                values=None, stream=None):
        """Values default to the input index of each key (the reference's offsets)."""
        n = keys.numel() if size is None else size
        N.check(self._lib.gpulsm_flix_build(self._h, self._k(keys, "keys", n), _ptr(values, "values", 4, n),
                                            n, max_size or n, _stream(stream)))

    build = build_bucket_layer_only

    def rebuild_bucket_layer_only(self, stream=None):
        N.check(self._lib.gpulsm_flix_rebuild(self._h, _stream(stream)))

    rebuild = rebuild_bucket_layer_only

    # --- updates -------------------------------------------------------------
    def insert(self, update_list, offsets, size: int | None = None, stream=None):
        n = update_list.numel() if size is None else size
        N.check(self._lib.gpulsm_flix_insert(self._h, self._k(update_list, "update_list", n),
                                             _ptr(offsets, "offsets", 4, n), n, _stream(stream)))

    def remove(self, update_list, size: int | None = None, stream=None):
        n = update_list.numel() if size is None else size
        N.check(self._lib.gpulsm_flix_remove(self._h, self._k(update_list, "update_list", n), n,
                                             _stream(stream)))

    # --- queries ---------------------------------------------------------------
    def lookups_ordered(self, sorted_keys, result, size: int | None = None, stream=None):
        n = sorted_keys.numel() if size is None else size
        N.check(self._lib.gpulsm_flix_lookups_ordered(self._h, self._k(sorted_keys, "keys", n),
                                                      n, _ptr(result, "result", 4, n), _stream(stream)))

    def lookups_successor(self, sorted_keys, result, size: int | None = None, stream=None):
        n = sorted_keys.numel() if size is None else size
        N.check(self._lib.gpulsm_flix_lookups_successor(self._h, self._k(sorted_keys, "keys", n), n,
                                                        self._k(result, "result", n), _stream(stream)))

    def lookup(self, keys, result, size: int | None = None, stream=None):
        n = keys.numel() if size is None else size
        N.check(self._lib.gpulsm_flix_lookup(self._h, self._k(keys, "keys", n), n,
                                             _ptr(result, "result", 4, n), _stream(stream)))

    def successor(self, keys, result, size: int | None = None, stream=None):
        n = keys.numel() if size is None else size
        N.check(self._lib.gpulsm_flix_successor(self._h, self._k(keys, "keys", n), n,
                                                self._k(result, "result", n), _stream(stream)))

    # --- introspection -------------------------------------------------------------
    def gpu_resident_bytes(self) -> int:
        v = C.c_uint64()
        N.check(self._lib.gpulsm_flix_resident_bytes(self._h, C.byref(v)))
        return int(v.value)

    def size(self) -> int:
        v = C.c_uint64()
        N.check(self._lib.gpulsm_flix_size(self._h, C.byref(v)))
        return int(v.value)

    def status(self) -> int:
        v = C.c_uint32()
        N.check(self._lib.gpulsm_flix_status(self._h, C.byref(v)))
        return int(v.value)

    def allocation_state(self) -> dict:
        """Allocation region: nodes taken by splits, nodes it holds, head
        buckets, and how often it was grown (allocation_buffer_next_free /
        allocation_buffer_total_nodes in the reference)."""
        used, total, buckets, grows = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint32()
        N.check(self._lib.gpulsm_flix_allocation_state(self._h, C.byref(used), C.byref(total), C.byref(buckets),
                                                       C.byref(grows)))
        return {"used_nodes": int(used.value), "region_nodes": int(total.value), "buckets": int(buckets.value),
                "grows": int(grows.value)}
