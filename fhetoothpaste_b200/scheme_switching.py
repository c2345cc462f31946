"""LWE -> RGSW scheme switching over the C ABI.

GpuLWEtoRGSWConverter mirrors LWEtoRGSWConverter::Convert
(lib/src/operators/lwe_to_rgsw_conversion.cpp:168-225) for a
SchemeSwitchingContext(rotation, trace, squaring, out_digits, out_basis)
(lines 10-110) on the Goldilocks modulus: one blind rotation of the converter's
test polynomial, the Lev rows, a trace per row and an RLWE key switch from s^2
to s, for a whole batch of LWE ciphertexts per call.

Keys come in the reference layouts: the rotator's m_brk, the trace's
automorphism keys for indices 3, 5, 9, .., N+1 concatenated (the m_ksk of each
evaluator in m_trace_evaluators order), and the squaring converter's m_ksk.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat


class GpuLWEtoRGSWConverter:
    """Batched LWE -> RGSW conversion. `rotation` = (variant, N, n, basis, digits)."""

    def __init__(self, rotation: tuple[int, int, int, int, int], trace: tuple[int, int], square: tuple[int, int],
                 out_digits: int, out_basis: int, brk: np.ndarray, trace_keys: np.ndarray, square_key: np.ndarray,
                 device: int = 0):
        variant, N, n, basis, digits = rotation
        p = nat.BrParams(variant, nat.GOLDILOCKS, N, n, basis, digits)
        h = ctypes.c_void_p()
        nat.check(nat.lib().tp_ss_create(ctypes.byref(p), trace[0], trace[1], square[0], square[1], out_digits,
                                         out_basis, device, ctypes.byref(h)))
        self._h = h
        self.N, self.n, self.out_digits = N, n, out_digits
        keys = [np.ascontiguousarray(k, dtype=np.uint64) for k in (brk, trace_keys, square_key)]
        nat.check(nat.lib().tp_ss_upload_keys(self._h, nat.ptr(keys[0]), keys[0].size, nat.ptr(keys[1]),
                                              keys[1].size, nat.ptr(keys[2]), keys[2].size))

    def close(self) -> None:
        if getattr(self, "_h", None):
            nat.lib().tp_ss_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def key_words(self, which: int) -> int:
        """Words of key `which` (0 rotation, 1 trace, 2 squaring)."""
        return int(nat.lib().tp_ss_key_words(self._h, which))

    def accumulator(self) -> np.ndarray:
        """The converter's test polynomial buffer m_acc = [0 | -tp | tp] (3N words)."""
        out = np.zeros(3 * self.N, np.uint64)
        nat.check(nat.lib().tp_ss_accumulator(self._h, nat.ptr(out)))
        return out

    @property
    def output_words(self) -> int:
        """Words of one RGSW output: [lev_left rows | lev_right rows], 4 N out_digits."""
        return 4 * self.N * self.out_digits

    def convert_batch(self, batch: int, out_ptr: int, lwes_ptr: int, stream=None) -> None:
        """Device buffers: lwes batch x (n+1) words, out batch x 4 N out_digits. Asynchronous."""
        nat.check(nat.lib().tp_lwe_to_rgsw_batch(self._h, batch, out_ptr, lwes_ptr, stream))

    def Convert(self, lwes: np.ndarray) -> np.ndarray:
        """Converts rows of n+1 words; returns one RGSW (4 N out_digits words, NTT domain) per row."""
        import torch
        lw = np.ascontiguousarray(lwes, dtype=np.uint64).reshape(-1, self.n + 1)
        d_in = torch.from_numpy(lw.view(np.int64)).cuda()
        d_out = torch.empty((lw.shape[0], self.output_words), dtype=torch.int64, device="cuda")
        self.convert_batch(lw.shape[0], d_out.data_ptr(), d_in.data_ptr())
        return d_out.cpu().numpy().view(np.uint64)
