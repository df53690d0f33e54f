"""Multi-tenant batched dictionary over the C ABI (gpulsm_tenants_*).

Many independent u32 dictionaries with GPULSMOpt upsert semantics, updated in
rounds: one round carries one batch per tenant as a CSR batch (concatenated
keys/values plus int64 offsets[tenants + 1], all CUDA tensors) and costs a
handful of launches for all tenants together.  The reference has no
multi-tenant facility; per-tenant answers equal a GPULSMOpt per tenant.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .dictionary import _ptr, _stream


class TenantPool:
    def __init__(self, capacities, max_round_keys: int, tile: int = 0, fan_in: int = 0, fanout: int = 0):
        self._lib = N.load()
        caps = np.ascontiguousarray(np.asarray(capacities, dtype=np.uint64))
        self.tenants = int(caps.size)
        h = C.c_void_p()
        N.check(self._lib.gpulsm_tenants_create(self.tenants, caps.ctypes.data_as(C.c_void_p), int(max_round_keys),
                                                tile, fan_in, fanout, C.byref(h)))
        self._h = h
        self.capacities = caps

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gpulsm_tenants_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tuning(self, tile: int, fan_in: int, fanout: int):
        N.check(self._lib.gpulsm_tenants_set_tuning(self._h, tile, fan_in, fanout))

    def insert_round(self, keys, values, offsets, stream=None, graph: bool = False):
        """offsets: int64 CUDA tensor [tenants + 1]; keys/values: 32-bit CUDA tensors.
        graph=True replays a CUDA graph captured for these exact buffers."""
        fn = self._lib.gpulsm_tenants_round_graph if graph else self._lib.gpulsm_tenants_insert_round
        N.check(fn(self._h, _ptr(keys, "keys"), _ptr(values, "values"), _ptr(offsets, "offsets", 8, self.tenants + 1),
                   _stream(stream)))

    def lookup(self, tenant_ids, keys, out_values, out_found=None, stream=None):
        n = keys.numel()
        N.check(self._lib.gpulsm_tenants_lookup(self._h, _ptr(tenant_ids, "tenant_ids", count=n),
                                                _ptr(keys, "keys", count=n), n, _ptr(out_values, "out_values", count=n),
                                                _ptr(out_found, "out_found", 1, n), _stream(stream)))

    def sizes(self) -> np.ndarray:
        out = np.zeros(self.tenants, np.uint64)
        N.check(self._lib.gpulsm_tenants_sizes(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def status(self) -> int:
        v = C.c_uint32()
        N.check(self._lib.gpulsm_tenants_status(self._h, C.byref(v)))
        return int(v.value)

    def gpu_resident_bytes(self) -> int:
        v = C.c_uint64()
        N.check(self._lib.gpulsm_tenants_resident_bytes(self._h, C.byref(v)))
        return int(v.value)
