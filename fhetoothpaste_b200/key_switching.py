"""Python mirrors of the reference's key-switching operators over the C ABI.

  GpuRLWEtoRLWEConverter  RLWEtoRLWEConverter::Convert  (lib/src/operators/rlwe_conversion.cpp:224-249)
  GpuAutomorphismEvaluator AutomorphismEvaluator::Eval  (lib/src/operators/automorphism_evaluation.cpp:150-159)
  GpuLWEtoRLWEPacker      LWEtoRLWEPacker::Pack          (lib/src/operators/lwe_to_rlwe_packing.cpp:129-236)
  GpuLWEtoLWEConverter    LWEtoLWEConverter::Convert     (lib/src/operators/lwe_conversion.cpp:205-239)
  GpuTraceEvaluator       TraceEvaluator::Eval / EvalAuto (lib/src/operators/trace_evaluation.cpp:135-179)

Each takes its key in the reference layout (the operator's m_ksk; for the
packer the automorphism keys for indices 2^j + 1, j = 1..log2 N, concatenated).
The batch methods take device pointers and run asynchronously on `stream`;
the numpy methods copy in and out and wait.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat


def _dev(torch, a: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64)).cuda()


class _KsBase:
    def __init__(self, handle: ctypes.c_void_p, key: np.ndarray):
        self._h = handle
        key = np.ascontiguousarray(key, dtype=np.uint64)
        nat.check(nat.lib().tp_ks_upload_key(self._h, nat.ptr(key), key.size))

    def set_tile(self, coef_per_thread: int) -> None:
        """4 or 8 coefficients per thread for this context's kernels (same results)."""
        nat.check(nat.lib().tp_ks_set_tile(self._h, coef_per_thread))

    @property
    def tile(self) -> int:
        return int(nat.lib().tp_ks_get_tile(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            nat.lib().tp_ks_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuRLWEtoRLWEConverter(_KsBase):
    def __init__(self, ring_dim: int, basis: int, digits: int, ksk: np.ndarray, device: int = 0):
        h = ctypes.c_void_p()
        nat.check(nat.lib().tp_rlwe_ks_create(ring_dim, basis, digits, device, ctypes.byref(h)))
        self.N = ring_dim
        super().__init__(h, ksk)

    def convert_batch(self, batch: int, out_ptr: int, in_ptr: int, stream=None) -> None:
        nat.check(nat.lib().tp_rlwe_ks_batch(self._h, batch, out_ptr, in_ptr, stream))

    def Convert(self, out: np.ndarray, inp: np.ndarray) -> None:
        """out -= KS(inp.A); out.B += inp.B, rows of 2N words (numpy, in place)."""
        import torch
        d_in, d_out = _dev(torch, inp), _dev(torch, out)
        self.convert_batch(d_in.numel() // (2 * self.N), d_out.data_ptr(), d_in.data_ptr())
        out[...] = d_out.cpu().numpy().view(np.uint64).reshape(out.shape)


class GpuAutomorphismEvaluator(_KsBase):
    def __init__(self, ring_dim: int, basis: int, digits: int, index: int, ksk: np.ndarray, device: int = 0):
        h = ctypes.c_void_p()
        nat.check(nat.lib().tp_auto_create(ring_dim, basis, digits, index, device, ctypes.byref(h)))
        self.N = ring_dim
        super().__init__(h, ksk)

    def eval_batch(self, batch: int, out_ptr: int, in_ptr: int, stream=None) -> None:
        nat.check(nat.lib().tp_auto_eval_batch(self._h, batch, out_ptr, in_ptr, stream))

    def Eval(self, out: np.ndarray, inp: np.ndarray) -> None:
        import torch
        d_in, d_out = _dev(torch, inp), _dev(torch, out)
        self.eval_batch(d_in.numel() // (2 * self.N), d_out.data_ptr(), d_in.data_ptr())
        out[...] = d_out.cpu().numpy().view(np.uint64).reshape(out.shape)


class GpuLWEtoRLWEPacker(_KsBase):
    def __init__(self, ring_dim: int, basis: int, digits: int, keys: np.ndarray, device: int = 0):
        h = ctypes.c_void_p()
        nat.check(nat.lib().tp_pack_create(ring_dim, basis, digits, device, ctypes.byref(h)))
        self.N = ring_dim
        super().__init__(h, keys)

    def pack_batch(self, packs: int, length: int, out_ptr: int, in_ptr: int, stream=None) -> None:
        nat.check(nat.lib().tp_pack_batch(self._h, packs, length, out_ptr, in_ptr, stream))

    def pack_consecutive_batch(self, packs: int, length: int, out_ptr: int, in_ptr: int, stream=None) -> None:
        nat.check(nat.lib().tp_pack_consecutive_batch(self._h, packs, length, out_ptr, in_ptr, stream))

    def pack_subtree_batch(self, packs: int, length: int, out_ptr: int, in_ptr: int, stream=None) -> None:
        """Subtrees of `length` inputs: L0 set-up and merges, roots in the coefficient domain
        (one shard of a packing split over devices; see sharded_pack)."""
        nat.check(nat.lib().tp_pack_subtree_batch(self._h, packs, length, out_ptr, in_ptr, stream))

    def pack_merge_batch(self, packs: int, count: int, level0: int, finish: bool, out_ptr: int, nodes_ptr: int,
                         stream=None) -> None:
        """The tree above `count` roots of level `level0` per pack; with `finish` the
        trailing traces too, giving what pack_batch gives for the whole tree."""
        nat.check(nat.lib().tp_pack_merge_batch(self._h, packs, count, level0, int(bool(finish)), out_ptr,
                                                nodes_ptr, stream))

    def PackConsecutively(self, lwes: np.ndarray, length: int) -> np.ndarray:
        """PackConsecutively of `lwes` (packs*length rows of N+1 words); packs x 2N coefficients."""
        import torch
        d_in = _dev(torch, lwes)
        packs = d_in.numel() // (length * (self.N + 1))
        d_out = torch.empty((packs, 2 * self.N), dtype=torch.int64, device="cuda")
        self.pack_consecutive_batch(packs, length, d_out.data_ptr(), d_in.data_ptr())
        return d_out.cpu().numpy().view(np.uint64)

    def Pack(self, lwes: np.ndarray, length: int) -> np.ndarray:
        """Packs `lwes` (packs*length rows of N+1 words); returns packs x 2N coefficients."""
        import torch
        d_in = _dev(torch, lwes)
        packs = d_in.numel() // (length * (self.N + 1))
        d_out = torch.empty((packs, 2 * self.N), dtype=torch.int64, device="cuda")
        self.pack_batch(packs, length, d_out.data_ptr(), d_in.data_ptr())
        return d_out.cpu().numpy().view(np.uint64)


class GpuTraceEvaluator(_KsBase):
    """TraceEvaluator (lib/src/operators/trace_evaluation.cpp:135-186) with its automorphism keys
    for indices 2^j + 1, j = 1..log2 N, concatenated (the packer's key layout)."""

    def __init__(self, ring_dim: int, basis: int, digits: int, keys: np.ndarray, device: int = 0):
        h = ctypes.c_void_p()
        nat.check(nat.lib().tp_pack_create(ring_dim, basis, digits, device, ctypes.byref(h)))
        self.N = ring_dim
        super().__init__(h, keys)

    def eval_batch(self, batch: int, out_ptr: int, in_ptr: int, stream=None) -> None:
        nat.check(nat.lib().tp_trace_eval_batch(self._h, batch, out_ptr, in_ptr, stream))

    def eval_auto_batch(self, batch: int, out_ptr: int, in_ptr: int, auto_index: int, stream=None) -> None:
        nat.check(nat.lib().tp_trace_eval_auto_batch(self._h, batch, out_ptr, in_ptr, auto_index, stream))

    def Eval(self, inp: np.ndarray) -> np.ndarray:
        """Rows of 2N coefficient words -> the trace, NTT domain."""
        import torch
        d = _dev(torch, inp)
        out = torch.empty_like(d)
        self.eval_batch(d.numel() // (2 * self.N), out.data_ptr(), d.data_ptr())
        return out.cpu().numpy().view(np.uint64)

    def EvalAuto(self, inp: np.ndarray, auto_index: int) -> np.ndarray:
        """AutomorphismEvaluator::Eval with the trace's key for auto_index = 2^j + 1 (fresh output)."""
        import torch
        d = _dev(torch, inp)
        out = torch.zeros_like(d)
        self.eval_auto_batch(d.numel() // (2 * self.N), out.data_ptr(), d.data_ptr(), auto_index)
        return out.cpu().numpy().view(np.uint64)


class GpuLWEtoLWEConverter:
    def __init__(self, n_in: int, n_out: int, basis: int, digits: int, ksk: np.ndarray | None, device: int = 0,
                 modulus: int = nat.GOLDILOCKS, key_file=None):
        h = ctypes.c_void_p()
        nat.check(nat.lib().tp_lwe_ks_create(modulus, n_in, n_out, basis, digits, device, ctypes.byref(h)))
        self._h = h
        self.n_in, self.n_out = n_in, n_out
        if key_file is not None:
            nat.check(nat.lib().tp_lwe_ks_upload_key_file(self._h, str(key_file).encode()))
        else:
            ksk = np.ascontiguousarray(ksk, dtype=np.uint64)
            nat.check(nat.lib().tp_lwe_ks_upload_key(self._h, nat.ptr(ksk), ksk.size))

    def close(self) -> None:
        if getattr(self, "_h", None):
            nat.lib().tp_lwe_ks_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def convert_batch(self, batch: int, out_ptr: int, in_ptr: int, stream=None) -> None:
        nat.check(nat.lib().tp_lwe_ks_batch(self._h, batch, out_ptr, in_ptr, stream))

    def pbs_epilogue_batch(self, batch: int, out_ptr: int, rlwe_ptr: int, target_modulus: int, stream=None) -> None:
        """SampleExtract(0) of each RLWE (coefficients, N = n_in) -> this key switch -> FLOOR switch to target."""
        nat.check(nat.lib().tp_pbs_epilogue_batch(self._h, batch, out_ptr, rlwe_ptr, target_modulus, stream))

    def Convert(self, out: np.ndarray, inp: np.ndarray) -> None:
        import torch
        d_in, d_out = _dev(torch, inp), _dev(torch, out)
        self.convert_batch(d_in.numel() // (self.n_in + 1), d_out.data_ptr(), d_in.data_ptr())
        out[...] = d_out.cpu().numpy().view(np.uint64).reshape(out.shape)


def modulus_switch_batch(count: int, vec_ptr: int, target_modulus: int, stream=None, kind: str = "floor") -> None:
    """In-place modulus switch of `count` device words from p to a power of two; kind 'round' | 'floor' |
    'ceil', each word as the reference's long-double ModulusSwitch gives it."""
    code = {"round": nat.TP_MS_ROUND, "floor": nat.TP_MS_FLOOR, "ceil": nat.TP_MS_CEIL}[kind]
    nat.check(nat.lib().tp_modulus_switch_batch(count, vec_ptr, nat.GOLDILOCKS, target_modulus, code, stream))
