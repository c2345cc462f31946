"""SAP digit decomposition over the C ABI.

GpuSAPDecomposer mirrors SAPDecomposer::Decompose
(lib/src/operators/sap_decomposer.cpp:353-464) of a
SAPDecompositionContext(rotation, trace, LWE conversion N -> n, radix)
(lines 15-186) on the Goldilocks modulus, for a batch of LWEs per call: per
digit a blind rotation of each LWE's running accumulator, the digit's
SampleExtract, the optional ResetAccumulator and HomTrunc (partial trace and the
truncation tree of automorphism key switches).

Keys come in the reference layouts: the rotator's m_brk, the trace evaluators'
m_ksk for indices 3, 5, 9, .., N+1 concatenated, and the LWE converter's m_ksk.
`hamming_weight` is the reference's m_beta (nonzero words of the LWE key) and
`restart_period` its GetRestartIteration() (UINT64_MAX: never reset).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat

NEVER = 2**64 - 1


class GpuSAPDecomposer:
    """`rotation` = (variant, N, n, basis, digits); `trace`, `ks` = (basis, digits)."""

    def __init__(self, rotation: tuple[int, int, int, int, int], trace: tuple[int, int], ks: tuple[int, int],
                 brk: np.ndarray, trace_keys: np.ndarray, lwe_ksk: np.ndarray, hamming_weight: int,
                 restart_period: int = NEVER, device: int = 0):
        variant, N, n, basis, digits = rotation
        p = nat.BrParams(variant, nat.GOLDILOCKS, N, n, basis, digits)
        h = ctypes.c_void_p()
        nat.check(nat.lib().tp_sap_create(ctypes.byref(p), trace[0], trace[1], ks[0], ks[1], device,
                                          ctypes.byref(h)))
        self._h = h
        self.N, self.n = N, n
        self.beta, self.restart = int(hamming_weight), int(restart_period)
        keys = [np.ascontiguousarray(k, dtype=np.uint64) for k in (brk, trace_keys, lwe_ksk)]
        nat.check(nat.lib().tp_sap_upload_keys(self._h, nat.ptr(keys[0]), keys[0].size, nat.ptr(keys[1]),
                                               keys[1].size, nat.ptr(keys[2]), keys[2].size))

    def close(self) -> None:
        if getattr(self, "_h", None):
            nat.lib().tp_sap_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def key_words(self, which: int) -> int:
        """Words of key `which` (0 rotation, 1 trace, 2 LWE key switch)."""
        return int(nat.lib().tp_sap_key_words(self._h, which))

    def decompose_batch(self, batch: int, out_ptr: int, out_digits: int, lwes_ptr: int, radix: int,
                        stream=None) -> np.ndarray:
        """Device buffers: lwes batch x (n+1), out batch x out_digits x (N+1). Returns the digit counts."""
        digits = np.zeros(batch, np.uint32)
        nat.check(nat.lib().tp_sap_decompose_batch(self._h, batch, out_ptr, out_digits, lwes_ptr, radix, self.beta,
                                                   self.restart,
                                                   digits.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), stream))
        return digits

    def homtrunc_batch(self, batch: int, out_ptr: int, in_ptr: int, radix: int, stream=None) -> None:
        """HomTrunc of `batch` NTT-domain RLWEs (device, 2N words each) into out (NTT domain)."""
        nat.check(nat.lib().tp_sap_homtrunc_batch(self._h, batch, out_ptr, in_ptr, radix, stream))

    def reset_batch(self, batch: int, acc_ptr: int, radix: int = 0, stream=None) -> None:
        """ResetAccumulator of `batch` NTT-domain accumulators in place (radix 0 as Decompose passes it)."""
        nat.check(nat.lib().tp_sap_reset_batch(self._h, batch, acc_ptr, radix, stream))

    def HomTrunc(self, rlwes: np.ndarray, radix: int) -> np.ndarray:
        import torch
        x = np.ascontiguousarray(rlwes, dtype=np.uint64).reshape(-1, 2 * self.N)
        d_in = torch.from_numpy(x.view(np.int64)).cuda()
        d_out = torch.empty_like(d_in)
        self.homtrunc_batch(x.shape[0], d_out.data_ptr(), d_in.data_ptr(), radix)
        return d_out.cpu().numpy().view(np.uint64)

    def ResetAccumulator(self, accs: np.ndarray, radix: int = 0) -> np.ndarray:
        import torch
        x = np.ascontiguousarray(accs, dtype=np.uint64).reshape(-1, 2 * self.N)
        d = torch.from_numpy(x.copy().view(np.int64)).cuda()
        self.reset_batch(x.shape[0], d.data_ptr(), radix)
        return d.cpu().numpy().view(np.uint64)

    def Decompose(self, lwes: np.ndarray, radix: int, out_digits: int) -> tuple[np.ndarray, np.ndarray]:
        """Decomposes rows of n+1 words; returns (digit counts, batch x out_digits x (N+1) words, zero-initialised)."""
        import torch
        lw = np.ascontiguousarray(lwes, dtype=np.uint64).reshape(-1, self.n + 1)
        d_in = torch.from_numpy(lw.view(np.int64)).cuda()
        d_out = torch.zeros((lw.shape[0], out_digits, self.N + 1), dtype=torch.int64, device="cuda")
        digits = self.decompose_batch(lw.shape[0], d_out.data_ptr(), out_digits, d_in.data_ptr(), radix)
        return digits, d_out.cpu().numpy().view(np.uint64)
