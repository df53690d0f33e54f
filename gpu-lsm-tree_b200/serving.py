"""Serving loop over one LSM dictionary (gpulsm_server_* in include/gpulsm.h).

Continuous batching of mixed lookup / insert / erase / range-sum requests
with host buffers: a native worker thread takes the queue, in arrival order,
into rounds of at most three dictionary calls (the round's inserts and erases
as one update batch, its lookups, its range sums), admits updates by a
device-memory budget, and pipelines rounds through staging slots.  Results
equal applying the rounds in order, each round's updates one at a time in
submission order before its reads (every request of a round is in flight
while it runs, so this is a linearization); `Ticket.round` tells the round.  The reference has no counterpart: GPULSMOpt serialises
every call behind a mutex and an operation event (GPULSMOpt.cuh:6852-6858).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .dictionary import DictionaryConfig

LOOKUP, INSERT, ERASE, RANGE_SUM = 0, 1, 2, 3


class Ticket:
    """A submitted request; keeps its host buffers alive until collected."""

    __slots__ = ("id", "kind", "bufs", "out", "found", "state", "round")

    def __init__(self, tid, kind, bufs, out, found):
        self.id, self.kind, self.bufs, self.out, self.found, self.state = tid, kind, bufs, out, found, 0
        self.round = None  # set by wait(): the round that ran the request (0: none)


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a).astype(np.uint32, copy=False))


class Server:
    """GPU dictionary server; see the module docstring."""

    def __init__(self, config: DictionaryConfig | None = None, budget_bytes: int = 16 << 30,
                 max_round_keys: int = 1 << 20, depth: int = 3, **kw):
        cfg = config or DictionaryConfig(**kw)
        self._lib = N.load()
        c = N.DictConfig(cfg.max_elements, cfg.batch_capacity, cfg.level_zero_capacity, cfg.fan_in,
                         cfg.rows_per_bucket_log2, cfg.search_mode, 0)
        h = C.c_void_p()
        N.check(self._lib.gpulsm_server_create(C.byref(c), budget_bytes, max_round_keys, depth, C.byref(h)))
        self._h = h
        self.max_round_keys = max_round_keys

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gpulsm_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_staged_updates(self, staged: bool) -> None:
        """Staged (graph-replayed admission, merges deferred) or direct update runs."""
        N.check(self._lib.gpulsm_server_set_staged_updates(self._h, int(bool(staged))))

    def bulk_build(self, keys, values, stream=None):
        """Preload from device tensors (torch), as GPULSMOpt.bulk_build."""
        from .dictionary import _ptr, _stream

        n = keys.numel()
        N.check(self._lib.gpulsm_server_bulk_build(self._h, _ptr(keys, "keys", count=n),
                                                   _ptr(values, "values", count=n), n, _stream(stream)))

    def _submit(self, kind, keys, aux=None, out=False, found=False) -> Ticket:
        keys = _u32(keys)
        n = keys.size
        aux = _u32(aux) if aux is not None else None
        if aux is not None and aux.size != n:
            raise ValueError("keys and values / upper bounds differ in length")
        o = np.empty(n, np.uint32) if out else None
        f = np.empty(n, np.uint8) if found else None
        t = C.c_uint64()
        ptr = lambda a: a.ctypes.data if a is not None and a.size else None
        N.check(self._lib.gpulsm_server_submit(self._h, kind, ptr(keys), ptr(aux), n, ptr(o), ptr(f), C.byref(t)))
        return Ticket(t.value, kind, (keys, aux), o, f)

    def submit_lookup(self, keys, with_found: bool = False) -> Ticket:
        return self._submit(LOOKUP, keys, out=True, found=with_found)

    def submit_insert(self, keys, values) -> Ticket:
        return self._submit(INSERT, keys, values)

    def submit_erase(self, keys) -> Ticket:
        return self._submit(ERASE, keys)

    def submit_range_sum(self, lo, hi) -> Ticket:
        return self._submit(RANGE_SUM, lo, hi, out=True)

    def _finish(self, t: Ticket, state: int):
        t.state = state
        if state < 0:
            raise N._ERRORS.get(-state, N.GpuLsmError)(f"request {t.id} failed with status {-state}", -state)
        if t.kind == LOOKUP:
            return (t.out, t.found) if t.found is not None else t.out
        return t.out

    def wait(self, t: Ticket):
        """Block until the request is done; returns its output (lookup values,
        (values, found), range sums, or None for updates)."""
        st, rd = C.c_int32(), C.c_uint64()
        N.check(self._lib.gpulsm_server_wait_round(self._h, t.id, C.byref(st), C.byref(rd)))
        t.round = rd.value
        return self._finish(t, st.value)

    def poll(self, t: Ticket) -> bool:
        """True once done (the result is then read with `result`)."""
        if t.state:
            return True
        st = C.c_int32()
        N.check(self._lib.gpulsm_server_poll(self._h, t.id, C.byref(st)))
        t.state = st.value
        return st.value != 0

    def result(self, t: Ticket):
        if not t.state:
            return self.wait(t)
        return self._finish(t, t.state)

    def drain(self):
        N.check(self._lib.gpulsm_server_drain(self._h))

    def stats(self) -> dict:
        s = N.ServeStats()
        N.check(self._lib.gpulsm_server_stats(self._h, C.byref(s)))
        return N.stats_dict(s)

    def reset_stats(self):
        N.check(self._lib.gpulsm_server_reset_stats(self._h))

    def resident_bytes(self) -> int:
        v = C.c_uint64()
        N.check(self._lib.gpulsm_server_resident_bytes(self._h, C.byref(v)))
        return v.value

    def run_load(self, universe, rate_per_s: float = 0.0, seconds: float = 1.0, mix=(0.6, 0.2, 0.1, 0.1),
                 min_keys: int = 1, max_keys: int = 1 << 16, zipf_s: float = 1.1, range_width_max: int = 1 << 16,
                 max_outstanding: int = 64, seed: int = 1) -> dict:
        """Native load generator: Poisson arrivals at rate_per_s (0 = closed
        loop with max_outstanding in flight); returns the latency statistics."""
        u = _u32(universe)
        spec = N.LoadSpec(rate_per_s, seconds, (C.c_double * 4)(*mix), zipf_s, max_outstanding, min_keys,
                          max_keys, range_width_max, seed, u.ctypes.data, u.size)
        s = N.ServeStats()
        N.check(self._lib.gpulsm_server_run_load(self._h, C.byref(spec), C.byref(s)))
        return N.stats_dict(s)
