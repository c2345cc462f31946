"""Python handle on the native serving loop (tp_server_* in include/toothpaste_gpu.h)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat


def _check(st: int) -> None:
    if st != nat.TP_OK:
        raise nat.TpError(st, nat.lib().tp_server_last_error().decode())


class BootstrapServer:
    """Continuous batching of single blind rotations over resident parameter sets."""

    def __init__(self, device: int = 0, max_queue: int = 0):
        self._h = ctypes.c_void_p()
        _check(nat.lib().tp_server_create(device, max_queue, ctypes.byref(self._h)))
        self.sets: list = []
        self._keep: list = []

    def add_set(self, rotator, max_batch: int, buffers: int = 2, out_coef: bool = False) -> int:
        sid = ctypes.c_uint32()
        _check(nat.lib().tp_server_add_set(self._h, rotator.handle, rotator.ctx.N, rotator.ctx.n, max_batch, buffers,
                                           int(out_coef), ctypes.byref(sid)))
        self.sets.append(rotator)
        return sid.value

    def set_memory_budget(self, nbytes: int) -> None:
        """Device bytes admitted requests may reserve (default: free device memory at start)."""
        _check(nat.lib().tp_server_set_memory_budget(self._h, nbytes))

    def memory(self) -> dict:
        b, u, r = nat.U64(), nat.U64(), nat.U64()
        _check(nat.lib().tp_server_memory(self._h, ctypes.byref(b), ctypes.byref(u), ctypes.byref(r)))
        return {"budget_bytes": b.value, "in_use_bytes": u.value, "rejected_for_memory": r.value}

    def start(self) -> None:
        _check(nat.lib().tp_server_start(self._h))

    def submit(self, set_id: int, lwe: np.ndarray, acc: np.ndarray, result: np.ndarray) -> int:
        """Queues one rotation; the three arrays must stay alive until wait() returns."""
        t = nat.U64()
        self._keep.append((lwe, acc, result))
        _check(nat.lib().tp_server_submit(self._h, set_id, nat.ptr(lwe), nat.ptr(acc), nat.ptr(result),
                                          ctypes.byref(t)))
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 120000) -> None:
        _check(nat.lib().tp_server_wait(self._h, ticket, timeout_ms))

    def drain(self, timeout_ms: int = 300000) -> None:
        _check(nat.lib().tp_server_drain(self._h, timeout_ms))
        self._keep.clear()

    def stats(self) -> dict:
        s = (ctypes.c_double * 8)()
        _check(nat.lib().tp_server_stats(self._h, s))
        return {"completed": int(s[0]), "rejected": int(s[1]), "launches": int(s[2]), "seconds": s[3],
                "p50_ms": s[4], "p99_ms": s[5], "p999_ms": s[6], "max_ms": s[7]}

    def reset_stats(self) -> None:
        _check(nat.lib().tp_server_reset_stats(self._h))

    def run_poisson(self, rate: float, seconds: float, mix, pools, seed: int = 5) -> dict:
        """pools: one (lwes, accs) pair of 2-D uint64 arrays per set, in set order."""
        k = len(pools)
        mixv = (ctypes.c_double * k)(*mix)
        lw = (nat.U64P * k)(*[nat.ptr(np.ascontiguousarray(p[0])) for p in pools])
        ac = (nat.U64P * k)(*[nat.ptr(np.ascontiguousarray(p[1])) for p in pools])
        cnt = np.array([p[0].shape[0] for p in pools], dtype=np.uint64)
        self.reset_stats()
        _check(nat.lib().tp_server_run_poisson(self._h, rate, seconds, mixv, k, lw, ac, nat.ptr(cnt), seed))
        st = self.stats()
        st["offered_per_s"] = rate
        st["achieved_per_s"] = st["completed"] / st["seconds"] if st["seconds"] else 0.0
        return st

    def close(self) -> None:
        if getattr(self, "_h", None):
            nat.lib().tp_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
