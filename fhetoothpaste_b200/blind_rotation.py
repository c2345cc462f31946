"""Python mirror of the reference's blind-rotation operator API over the C ABI.

Mirrors CGGIBlindRotationContext / BMMPBlindRotationContext and
BlindRotator::BlindRotate (lib/include/interfaces/blindrotation_operator.h:20-49
of the reference) for tests, the benchmark and the serving loop. Key
generation stays with the caller (the C++ adapters in fhetoothpaste_b200/host/
run it on the host); this class takes the generated key words.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat

BINARY, TERNARY = "binary", "ternary"


class BlindRotationContext:
    """Parameters of one blind-rotation operator (CGGI binary/ternary or BMMP)."""

    def __init__(self, variant: int, ring_dim: int, lwe_dim: int, basis: int, digits: int,
                 modulus: int = nat.GOLDILOCKS, std: float = 0.0):
        self.variant = int(variant)
        self.modulus = int(modulus)
        self.N = int(ring_dim)
        self.n = int(lwe_dim)
        self.basis = int(basis)
        self.basis_log2 = self.basis.bit_length() - 1
        self.digits = int(digits)
        self.std = float(std)

    def params(self) -> nat.BrParams:
        return nat.BrParams(self.variant, self.modulus, self.N, self.n, self.basis, self.digits)

    def key_words(self) -> int:
        g = {nat.TP_BR_CGGI_BINARY: 1, nat.TP_BR_CGGI_TERNARY: 2, nat.TP_BR_BMMP_BINARY: 3}[self.variant]
        groups = self.n // 2 if self.variant == nat.TP_BR_BMMP_BINARY else self.n
        return groups * g * 4 * self.N * self.digits


class GpuBlindRotator:
    """A blind-rotation key resident on one GPU plus its launch context."""

    def __init__(self, ctx: BlindRotationContext, brk: np.ndarray | None, device: int = 0, key_file=None):
        """`brk` in the reference's m_brk layout, or `key_file` (a key file of kind blind_rotation)."""
        L = nat.lib()
        self.ctx = ctx
        self.device = device
        h = ctypes.c_void_p()
        prm = ctx.params()
        nat.check(L.tp_br_create(ctypes.byref(prm), device, ctypes.byref(h)))
        self._h = h
        if key_file is not None:
            nat.check(L.tp_br_upload_key_file(self._h, str(key_file).encode()))
        else:
            brk = np.ascontiguousarray(brk, dtype=np.uint64)
            nat.check(L.tp_br_upload_key(self._h, nat.ptr(brk), brk.size))

    @classmethod
    def from_key_file(cls, path, device: int = 0) -> "GpuBlindRotator":
        """Context and key from a key file (parameters read from its header)."""
        from .keyfile import key_file_info
        i = key_file_info(path)
        ctx = BlindRotationContext(i["variant"], i["ring_dim"], i["lwe_dim"], i["basis"], i["digits"], i["modulus"])
        return cls(ctx, None, device=device, key_file=path)

    def close(self) -> None:
        if getattr(self, "_h", None):
            nat.lib().tp_br_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    # BlindRotator::BlindRotate(result, lwe, accumulator, output_as_coefficients)
    def BlindRotate(self, result: np.ndarray, lwe: np.ndarray, acc: np.ndarray,
                    output_as_coefficients: bool = False) -> None:
        for a, w in ((result, 2 * self.ctx.N), (lwe, self.ctx.n + 1), (acc, 2 * self.ctx.N)):
            if a.dtype != np.uint64 or not a.flags.c_contiguous or a.size < w:
                raise ValueError("buffers must be contiguous uint64 arrays of the operator's sizes")
        nat.check(nat.lib().tp_br_blind_rotate(self._h, nat.ptr(result), nat.ptr(lwe), nat.ptr(acc),
                                               int(bool(output_as_coefficients))))

    def blind_rotate_batch_host(self, lwes: np.ndarray, accs: np.ndarray, out_coef: bool = False,
                                stream: int | None = None) -> np.ndarray:
        """Rotates every row of `lwes` (batch x (n+1)); `accs` is batch x 2N or one 2N row."""
        lwes = np.ascontiguousarray(lwes, dtype=np.uint64)
        accs = np.ascontiguousarray(accs, dtype=np.uint64)
        batch = lwes.shape[0]
        shared = accs.ndim == 1
        out = np.empty((batch, 2 * self.ctx.N), dtype=np.uint64)
        nat.check(nat.lib().tp_br_blind_rotate_batch_host(
            self._h, batch, nat.ptr(out), nat.ptr(lwes), lwes.shape[1], nat.ptr(accs),
            0 if shared else accs.shape[1], int(bool(out_coef)), stream))
        nat.check(nat.lib().tp_br_check(self._h, stream))
        return out

    def blind_rotate_batch(self, results_ptr: int, lwes_ptr: int, lwe_stride: int, accs_ptr: int,
                           acc_stride: int, batch: int, out_coef: bool = False, stream: int | None = None) -> None:
        """Device-pointer batch launch (asynchronous on `stream`)."""
        nat.check(nat.lib().tp_br_blind_rotate_batch(self._h, batch, results_ptr, lwes_ptr, lwe_stride, accs_ptr,
                                                     acc_stride, int(bool(out_coef)), stream))

    def check(self, stream: int | None = None) -> None:
        nat.check(nat.lib().tp_br_check(self._h, stream))

    @property
    def tile(self) -> int:
        """Coefficients per thread of the rotation kernel (8 or 4)."""
        return int(nat.lib().tp_br_get_tile(self._h))

    def set_tile(self, coef_per_thread: int) -> None:
        nat.check(nat.lib().tp_br_set_tile(self._h, coef_per_thread))

    @property
    def split(self) -> int:
        """Thread blocks per rotation (1, or 2 / 4 for the cluster kernels)."""
        return int(nat.lib().tp_br_get_split(self._h))

    def set_split(self, blocks_per_rotation: int) -> None:
        nat.check(nat.lib().tp_br_set_split(self._h, blocks_per_rotation))

    @property
    def mac_form(self) -> int:
        """Multiply-accumulate form of the one-block kernel at tile 4 (0 row by row, 1 digit-staged)."""
        return int(nat.lib().tp_br_get_mac_form(self._h))

    def set_mac_form(self, form: int) -> None:
        nat.check(nat.lib().tp_br_set_mac_form(self._h, form))

    @property
    def radix(self) -> int:
        """NTT radix of the one-block kernel at tile 4 (2, or 4 for the fused radix-4 passes)."""
        return int(nat.lib().tp_br_get_radix(self._h))

    def set_radix(self, radix: int) -> None:
        nat.check(nat.lib().tp_br_set_radix(self._h, radix))

    def autotune(self, batch: int) -> tuple[int, float]:
        """Times every tile (and the two- and four-block splits) on `batch` synthetic rotations and keeps
        the fastest."""
        coef, rate = ctypes.c_uint32(), ctypes.c_double()
        nat.check(nat.lib().tp_br_autotune(self._h, batch, ctypes.byref(coef), ctypes.byref(rate)))
        return int(coef.value), float(rate.value)

    def capture_batch(self, results_ptr: int, lwes_ptr: int, lwe_stride: int, accs_ptr: int, acc_stride: int,
                      batch: int, out_coef: bool = False, extract_ptr: int | None = None) -> "BatchGraph":
        """Records one batch launch (plus SampleExtract into extract_ptr) as a CUDA graph."""
        g = ctypes.c_void_p()
        nat.check(nat.lib().tp_br_batch_graph_create(self._h, batch, results_ptr, lwes_ptr, lwe_stride, accs_ptr,
                                                     acc_stride, int(bool(out_coef)), extract_ptr, ctypes.byref(g)))
        return BatchGraph(g, self)

    def capture_bootstrap(self, key_switch, batch: int, rlwe_scratch_ptr: int, lwes_ptr: int, accs_ptr: int,
                          acc_stride: int, out_lwe_ptr: int) -> "BatchGraph":
        """Records rotation (coefficient output) + SampleExtract + LWE key switch + FLOOR switch to 2N."""
        g = ctypes.c_void_p()
        nat.check(nat.lib().tp_pbs_graph_create(self._h, key_switch._h, batch, rlwe_scratch_ptr, lwes_ptr, accs_ptr,
                                                acc_stride, out_lwe_ptr, ctypes.byref(g)))
        return BatchGraph(g, (self, key_switch))


class NegacyclicFunctionEvaluator:
    """NegacyclicFunctionEvaluator (lib/src/operators/negacyclic_function_evaluator.cpp:72-101):
    BlindRotate with coefficient output, then SampleExtract at index 0 into the caller's buffer
    (words stay untouched where the rotated A coefficient is 0, as in the reference)."""

    def __init__(self, rotator: GpuBlindRotator):
        self.rot = rotator
        self.N = rotator.ctx.N

    @staticmethod
    def _extract(out: np.ndarray, rl: np.ndarray) -> None:
        N = rl.size // 2
        out[0] = rl[0]
        a = rl[N - np.arange(1, N)]
        nz = a != 0
        idx = np.arange(1, N)[nz]
        out[idx] = np.uint64(nat.GOLDILOCKS) - a[nz]
        out[N] = rl[N]

    def EvalFunc(self, result: np.ndarray, input_lwe: np.ndarray, lut) -> None:
        """lut: an RLWE [A | B] (2N words), or a function f: the test RLWE is then built as the
        reference builds it (f(0) at A[0], -f(N - i) at B[i], lines 82-84)."""
        N = self.N
        if callable(lut):
            rl = np.zeros(2 * N, np.uint64)
            rl[0] = int(lut(0)) % nat.GOLDILOCKS
            for i in range(1, N):
                rl[i + N] = (nat.GOLDILOCKS - int(lut(N - i)) % nat.GOLDILOCKS) % nat.GOLDILOCKS
            lut = rl
        acc = np.empty(2 * N, np.uint64)
        self.rot.BlindRotate(acc, np.ascontiguousarray(input_lwe, np.uint64), np.ascontiguousarray(lut, np.uint64),
                             True)
        self._extract(result, acc)

    def eval_func_batch(self, lwes: np.ndarray, luts: np.ndarray, results: np.ndarray | None = None) -> np.ndarray:
        """Many at once: lwes batch x (n+1), luts batch x 2N or one 2N row; returns batch x (N+1)."""
        rl = self.rot.blind_rotate_batch_host(lwes, luts, out_coef=True)
        out = np.zeros((rl.shape[0], self.N + 1), np.uint64) if results is None else results
        for b in range(rl.shape[0]):
            self._extract(out[b], rl[b])
        return out


class BatchGraph:
    """A recorded batch launch; replays read the device buffers' current contents."""

    def __init__(self, handle: ctypes.c_void_p, owner: GpuBlindRotator):
        self._g = handle
        self._owner = owner  # keeps the key alive while the graph exists

    def launch(self, stream: int | None = None) -> None:
        nat.check(nat.lib().tp_graph_launch(self._g, stream))

    def close(self) -> None:
        if getattr(self, "_g", None):
            nat.lib().tp_graph_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ntt_forward(ring_dim: int, count: int, out_ptr: int, in_ptr: int, stream: int | None = None) -> None:
    nat.check(nat.lib().tp_ntt_forward(ring_dim, count, out_ptr, in_ptr, stream))


def ntt_backward(ring_dim: int, count: int, out_ptr: int, in_ptr: int, stream: int | None = None) -> None:
    nat.check(nat.lib().tp_ntt_backward(ring_dim, count, out_ptr, in_ptr, stream))


def sample_extract_batch(ring_dim: int, batch: int, out_ptr: int, rlwe_ptr: int, stream: int | None = None) -> None:
    nat.check(nat.lib().tp_sample_extract_batch(ring_dim, batch, out_ptr, rlwe_ptr, stream))
