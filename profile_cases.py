"""Runs each GPU kernel of the library on one small case, for profiler captures.

    python profile_cases.py CASE [CASE ...]   (or: all)

Every case launches its kernel(s) twice: one warm-up launch, then the launch to
capture (so `ncu -s <launches per warm-up> -c <launches>` selects the second).
Inputs are seeded uniform residues; keys are uniform words (the kernels' timing
does not depend on their values). Sizes keep device memory to a few GB while the
streamed operands stay larger than L2 where the kernel streams them.
"""
from __future__ import annotations

import argparse
import sys

import numpy as np

P = 0xFFFFFFFF00000001


def _u64(seed: int, shape, bound: int = P) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.integers(0, 2**63, shape, dtype=np.uint64) % np.uint64(bound)


def _dev(torch, a: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint64).view(np.int64)).cuda()


def _rotation(torch, variant: int, N: int, n: int, beta: int, digits: int, batch: int, tile: int = 0):
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    ctx = BlindRotationContext(variant, N, n, 1 << beta, digits)
    rot = GpuBlindRotator(ctx, _u64(1, ctx.key_words()))  # key_relayout_kernel
    if tile:
        rot.set_tile(tile)                                 # key_retile_kernel
    lw = _dev(torch, _u64(2, (batch, n + 1), 2 * N))
    ac = _dev(torch, _u64(3, (batch, 2 * N)))
    out = torch.empty((batch, 2 * N), dtype=torch.int64, device="cuda")
    for _ in range(2):
        rot.blind_rotate_batch(out.data_ptr(), lw.data_ptr(), n + 1, ac.data_ptr(), 2 * N, batch)
    rot.check()
    rot.close()


def case_br_ternary_n2048(torch):
    """br_kernel, CGGI ternary N=2048 base 2^12 l=3, n reduced to 64, one wave (148)."""
    _rotation(torch, 1, 2048, 64, 12, 3, 148)


def case_br_binary_n1024(torch):
    """br_kernel, CGGI binary N=1024 base 2^16 l=4, n reduced to 64, one wave (296)."""
    _rotation(torch, 0, 1024, 64, 16, 4, 296)


def case_br_bmmp_n2048(torch):
    """br_kernel, BMMP N=2048 base 2^16 l=4, n reduced to 64 (32 pairs), one wave (148)."""
    _rotation(torch, 2, 2048, 64, 16, 4, 148)


def case_br_ternary_n4096(torch):
    """br_kernel, CGGI ternary N=4096 base 2^12 l=3, n reduced to 32, one wave (148)."""
    _rotation(torch, 1, 4096, 32, 12, 3, 148)


def case_br_ternary_n8192(torch):
    """br_kernel on two-CTA clusters, CGGI ternary N=8192 base 2^12 l=3, n reduced to 32, one wave (74)."""
    _rotation(torch, 1, 8192, 32, 12, 3, 74)


def case_br_pair_ternary_n2048(torch):
    """br_pair_kernel (two blocks per rotation), CGGI ternary N=2048 l=3, n reduced to 64, batch 37."""
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    N, n, batch = 2048, 64, 37
    ctx = BlindRotationContext(1, N, n, 1 << 12, 3)
    rot = GpuBlindRotator(ctx, _u64(1, ctx.key_words()))
    rot.set_split(2)
    lw = _dev(torch, _u64(2, (batch, n + 1), 2 * N))
    ac = _dev(torch, _u64(3, (batch, 2 * N)))
    out = torch.empty((batch, 2 * N), dtype=torch.int64, device="cuda")
    for _ in range(2):
        rot.blind_rotate_batch(out.data_ptr(), lw.data_ptr(), n + 1, ac.data_ptr(), 2 * N, batch)
    rot.check()
    rot.close()


def case_br_quad_ternary_n2048(torch):
    """br_quad_kernel (four blocks per rotation), CGGI ternary N=2048 l=3, n reduced to 64, batch 16."""
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    N, n, batch = 2048, 64, 16
    ctx = BlindRotationContext(1, N, n, 1 << 12, 3)
    rot = GpuBlindRotator(ctx, _u64(1, ctx.key_words()))
    rot.set_tile(4)
    rot.set_split(4)
    lw = _dev(torch, _u64(2, (batch, n + 1), 2 * N))
    ac = _dev(torch, _u64(3, (batch, 2 * N)))
    out = torch.empty((batch, 2 * N), dtype=torch.int64, device="cuda")
    for _ in range(2):
        rot.blind_rotate_batch(out.data_ptr(), lw.data_ptr(), n + 1, ac.data_ptr(), 2 * N, batch)
    rot.check()
    rot.close()


def case_pbs_epilogue_n1024(torch):
    """lwe_ks_kernel as the bootstrap epilogue: 4096 RLWEs N=1024 -> extract -> KS to n=500
    (base 2^16, l=4, 16 MB key) -> FLOOR switch to 2N."""
    from fhetoothpaste_b200 import GpuLWEtoLWEConverter
    N, n, l, batch = 1024, 500, 4, 4096
    conv = GpuLWEtoLWEConverter(N, n, 1 << 16, l, _u64(15, N * l * (n + 1)))
    x = _dev(torch, _u64(16, (batch, 2 * N)))
    y = torch.empty((batch, n + 1), dtype=torch.int64, device="cuda")
    for _ in range(2):
        conv.pbs_epilogue_batch(batch, y.data_ptr(), x.data_ptr(), 2 * N)
    torch.cuda.synchronize()
    conv.close()


def case_ntt_n2048(torch):
    """ntt_batch_kernel forward then backward, 8192 polynomials of N=2048 (134 MB)."""
    from fhetoothpaste_b200 import ntt_backward, ntt_forward
    N, count = 2048, 8192
    x = _dev(torch, _u64(4, (count, N)))
    for _ in range(2):
        ntt_forward(N, count, x.data_ptr(), x.data_ptr())
        ntt_backward(N, count, x.data_ptr(), x.data_ptr())
    torch.cuda.synchronize()


def case_rlwe_ks_n2048(torch):
    """ks_kernel (RLWE->RLWE), 4096 ciphertexts of N=2048, base 2^16 l=4."""
    from fhetoothpaste_b200 import GpuRLWEtoRLWEConverter
    N, l, batch = 2048, 4, 4096
    conv = GpuRLWEtoRLWEConverter(N, 1 << 16, l, _u64(5, 2 * N * l))
    x = _dev(torch, _u64(6, (batch, 2 * N)))
    y = torch.zeros((batch, 2 * N), dtype=torch.int64, device="cuda")
    for _ in range(2):
        conv.convert_batch(batch, y.data_ptr(), x.data_ptr())
    torch.cuda.synchronize()
    conv.close()


def case_auto_n2048(torch):
    """ks_kernel (automorphism X -> X^5 + key switch), 4096 ciphertexts of N=2048, l=4."""
    from fhetoothpaste_b200 import GpuAutomorphismEvaluator
    N, l, batch = 2048, 4, 4096
    ev = GpuAutomorphismEvaluator(N, 1 << 16, l, 5, _u64(7, 2 * N * l))
    x = _dev(torch, _u64(8, (batch, 2 * N)))
    y = torch.zeros((batch, 2 * N), dtype=torch.int64, device="cuda")
    for _ in range(2):
        ev.eval_batch(batch, y.data_ptr(), x.data_ptr())
    torch.cuda.synchronize()
    ev.close()


def case_pack_n2048(torch):
    """pack_l0_kernel + ks_kernel merge levels: 8 packs of 2048 LWEs (n=N=2048), l=4."""
    from fhetoothpaste_b200 import GpuLWEtoRLWEPacker
    N, L, packs, l = 2048, 2048, 8, 4
    packer = GpuLWEtoRLWEPacker(N, 1 << 16, l, _u64(9, 11 * 2 * N * l))
    x = _dev(torch, _u64(10, (packs * L, N + 1)))
    y = torch.empty((packs, 2 * N), dtype=torch.int64, device="cuda")
    for _ in range(2):
        packer.pack_batch(packs, L, y.data_ptr(), x.data_ptr())
    torch.cuda.synchronize()
    packer.close()


def case_lwe_ks_2048_630(torch):
    """lwe_ks_kernel: 4096 LWE ciphertexts n=2048 -> n=630, base 2^16 l=4 (41 MB key)."""
    from fhetoothpaste_b200 import GpuLWEtoLWEConverter
    n_in, n_out, l, batch = 2048, 630, 4, 4096
    conv = GpuLWEtoLWEConverter(n_in, n_out, 1 << 16, l, _u64(11, n_in * l * (n_out + 1)))
    x = _dev(torch, _u64(12, (batch, n_in + 1)))
    y = torch.zeros((batch, n_out + 1), dtype=torch.int64, device="cuda")
    for _ in range(2):
        conv.convert_batch(batch, y.data_ptr(), x.data_ptr())
    torch.cuda.synchronize()
    conv.close()


def case_sample_extract_n2048(torch):
    """sample_extract0_kernel, 16384 ciphertexts of N=2048 (537 MB in)."""
    from fhetoothpaste_b200 import sample_extract_batch
    N, batch = 2048, 16384
    x = _dev(torch, _u64(13, (batch, 2 * N)))
    y = torch.empty((batch, N + 1), dtype=torch.int64, device="cuda")
    for _ in range(2):
        sample_extract_batch(N, batch, y.data_ptr(), x.data_ptr())
    torch.cuda.synchronize()


def case_key_retile_n2048(torch):
    """key_relayout_kernel (upload) and key_retile_kernel (tile 4 -> 8 -> 4), ternary N=2048 n=630 key."""
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    ctx = BlindRotationContext(1, 2048, 630, 1 << 12, 3)
    rot = GpuBlindRotator(ctx, _u64(14, ctx.key_words()))
    rot.set_tile(8)
    rot.set_tile(4)
    rot.close()


def case_lwe_to_rgsw_n2048(torch):
    """LWE -> RGSW scheme switching, 256 LWEs (CGGI binary n=100, N=2048, gadgets 2^14 l=4, out 4
    digits): br_kernel, ss_rows_kernel, 11 trace ks_kernel launches, ntt_batch_kernel x2,
    ks_kernel (s^2 -> s), ss_assemble_kernel per conversion call."""
    from fhetoothpaste_b200 import BlindRotationContext, GpuLWEtoRGSWConverter
    N, n, beta, l, D, batch = 2048, 100, 14, 4, 4, 256
    words = BlindRotationContext(0, N, n, 1 << beta, l).key_words()
    conv = GpuLWEtoRGSWConverter((0, N, n, 1 << beta, l), (1 << beta, l), (1 << beta, l), D, 1 << beta,
                                 _u64(61, words), _u64(62, 11 * 2 * N * l), _u64(63, 2 * N * l))
    lw = _dev(torch, _u64(64, (batch, n + 1), 2 * N))
    out = torch.empty((batch, 4 * N * D), dtype=torch.int64, device="cuda")
    for _ in range(2):
        conv.convert_batch(batch, out.data_ptr(), lw.data_ptr())
    torch.cuda.synchronize()
    conv.close()


def case_sap_n4096(torch):
    """SAP digit decomposition, 16 LWEs (CGGI binary n=10, N=4096, gadgets 2^16 l=4, radix 32,
    inputs mod 2^40: 8 digits): br_kernel, ks_kernel (trace and split modes), ntt_batch_kernel,
    lwe_ks_kernel and the element-wise SAP kernels, per decomposition call."""
    from fhetoothpaste_b200 import BlindRotationContext, GpuSAPDecomposer
    N, n, l, batch = 4096, 10, 4, 16
    words = BlindRotationContext(0, N, n, 1 << 16, l).key_words()
    dec = GpuSAPDecomposer((0, N, n, 1 << 16, l), (1 << 16, l), (1 << 16, l), _u64(71, words),
                           _u64(72, 12 * 2 * N * l), _u64(73, N * l * (n + 1)), hamming_weight=5)
    lw = _dev(torch, _u64(74, (batch, n + 1), 1 << 40))
    out = torch.zeros((batch, 9, N + 1), dtype=torch.int64, device="cuda")
    for _ in range(2):
        dec.decompose_batch(batch, out.data_ptr(), 9, lw.data_ptr(), 32)
    torch.cuda.synchronize()
    dec.close()


def case_sap_reset_n4096(torch):
    """The SAP case above with an accumulator reset every 2 digits (restart period 2), so the
    reset path (epilogue, fresh rotation, sap_select_kernel) runs too."""
    from fhetoothpaste_b200 import BlindRotationContext, GpuSAPDecomposer
    N, n, l, batch = 4096, 10, 4, 16
    words = BlindRotationContext(0, N, n, 1 << 16, l).key_words()
    dec = GpuSAPDecomposer((0, N, n, 1 << 16, l), (1 << 16, l), (1 << 16, l), _u64(71, words),
                           _u64(72, 12 * 2 * N * l), _u64(73, N * l * (n + 1)), hamming_weight=5,
                           restart_period=2)
    lw = _dev(torch, _u64(74, (batch, n + 1), 1 << 40))
    out = torch.zeros((batch, 9, N + 1), dtype=torch.int64, device="cuda")
    for _ in range(2):
        dec.decompose_batch(batch, out.data_ptr(), 9, lw.data_ptr(), 32)
    torch.cuda.synchronize()
    dec.close()


def case_lwe_to_rgsw_n2048_b1024(torch):
    """As lwe_to_rgsw_n2048 with 1024 LWEs, so the element-wise kernels' rows (134 MB) exceed L2."""
    from fhetoothpaste_b200 import BlindRotationContext, GpuLWEtoRGSWConverter
    N, n, beta, l, D, batch = 2048, 100, 14, 4, 4, 1024
    words = BlindRotationContext(0, N, n, 1 << beta, l).key_words()
    conv = GpuLWEtoRGSWConverter((0, N, n, 1 << beta, l), (1 << beta, l), (1 << beta, l), D, 1 << beta,
                                 _u64(61, words), _u64(62, 11 * 2 * N * l), _u64(63, 2 * N * l))
    lw = _dev(torch, _u64(64, (batch, n + 1), 2 * N))
    out = torch.empty((batch, 4 * N * D), dtype=torch.int64, device="cuda")
    for _ in range(2):
        conv.convert_batch(batch, out.data_ptr(), lw.data_ptr())
    torch.cuda.synchronize()
    conv.close()


def case_modswitch_round(torch):
    """ms_pow2_kernel: ROUND switch of 64 M words (512 MB) from p to 2^12, twice."""
    from fhetoothpaste_b200 import modulus_switch_batch
    x = _dev(torch, _u64(81, 1 << 26))
    for _ in range(2):
        modulus_switch_batch(x.numel(), x.data_ptr(), 1 << 12, kind="round")
    torch.cuda.synchronize()


def case_pack_consecutive_n2048(torch):
    """pack_l0_idx_kernel + compacted merges: 64 consecutive packings of 64 LWEs (n = N = 2048)."""
    from fhetoothpaste_b200 import GpuLWEtoRLWEPacker
    N, L, packs, l = 2048, 64, 64, 4
    pk = GpuLWEtoRLWEPacker(N, 1 << 16, l, _u64(82, 11 * 2 * N * l))
    lw = _dev(torch, _u64(83, (packs * L, N + 1)))
    out = torch.empty((packs, 2 * N), dtype=torch.int64, device="cuda")
    for _ in range(2):
        pk.pack_consecutive_batch(packs, L, out.data_ptr(), lw.data_ptr())
    torch.cuda.synchronize()
    pk.close()


def case_trace_n2048(torch):
    """scale_kernel + trace steps + NTT: TraceEvaluator::Eval of 4096 RLWEs (N = 2048, l = 4)."""
    from fhetoothpaste_b200 import GpuTraceEvaluator
    N, l, batch = 2048, 4, 4096
    tr = GpuTraceEvaluator(N, 1 << 16, l, _u64(84, 11 * 2 * N * l))
    x = _dev(torch, _u64(85, (batch, 2 * N)))
    y = torch.empty_like(x)
    for _ in range(2):
        tr.eval_batch(batch, y.data_ptr(), x.data_ptr())
    torch.cuda.synchronize()
    tr.close()


CASES = {name[5:]: fn for name, fn in globals().items() if name.startswith("case_")}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("cases", nargs="+", help="case names or 'all': " + ", ".join(sorted(CASES)))
    args = ap.parse_args(argv)
    names = sorted(CASES) if args.cases == ["all"] else args.cases
    unknown = [c for c in names if c not in CASES]
    if unknown:
        ap.error(f"unknown case(s): {unknown}")
    import torch
    if not torch.cuda.is_available():
        print("profile_cases needs a CUDA device", file=sys.stderr)
        return 2
    for name in names:
        CASES[name](torch)
        print(f"{name}: ok", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
