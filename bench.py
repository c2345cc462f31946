"""Benchmark of the batched blind rotation on B200 (one JSON line on rank 0).

Workload (default): batched CGGI blind rotation with a ternary LWE secret,
n = 630, N = 2048, Goldilocks, signed gadget base 2^12 with l = 3; 4096
independent LWE ciphertexts per step, each with its own seeded 16-entry LUT
test polynomial (trivial RLWE, coefficient domain), NTT-domain output. One
step = one persistent launch over the whole batch.

  value  blind rotations/s with inputs resident in HBM (kernel time, CUDA events)
  e2e    the same through the host-buffer C-ABI call (tp_br_blind_rotate_batch_host):
         host->device copy of the step's LWEs and test polynomials, the launch,
         device->host copy of the results, all inside the timed region
  plain  the one-rotation-per-launch form (batch 1) for the batched/plain ratio, also
         with the rotation split over two and four SMs (cluster kernels)

`--impl reference` times the reference library's own CPU blind rotation (built
from its sources into oracle/_ref/, one rotator per host thread) on a bounded
sample of the same workload. Multi-GPU runs (torchrun) shard the batch: every
rank rotates its own 4096 ciphertexts, no collective on the data path
(weak scaling); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

P = 0xFFFFFFFF00000001

WORKLOADS = {
    # name: variant, N, n, basis_log2, digits, batch
    "cggi_ternary_n2048": (1, 2048, 630, 12, 3, 4096),
    "cggi_binary_n1024": (0, 1024, 500, 16, 4, 4096),
    "bmmp_binary_n2048": (2, 2048, 768, 16, 4, 2048),
    "cggi_ternary_n4096": (1, 4096, 900, 12, 3, 1024),
}
DESCR = {
    "cggi_ternary_n2048": "batched CGGI blind rotation, ternary n=630, N=2048, Goldilocks, base 2^12 l=3",
    "cggi_binary_n1024": "CGGI blind rotation, binary n=500, N=1024, Goldilocks, base 2^16 l=4",
    "bmmp_binary_n2048": "BMMP blind rotation, binary n=768 (384 pairs), N=2048, base 2^16 l=4",
    "cggi_ternary_n4096": "CGGI blind rotation, ternary n=900, N=4096, base 2^12 l=3",
}


def ntt_mm(N: int) -> int:
    return N // 2 * (N.bit_length() - 1)


def modmul_per_iteration(variant: int, N: int, l: int) -> int:
    """Algorithmic modmul count of one CMux iteration (NTT counted as N/2 log2 N)."""
    if variant == 0:
        return 2 * N + (2 + 2 * l) * ntt_mm(N) + 4 * l * N
    if variant == 1:
        return (2 + 2 * l) * ntt_mm(N) + 8 * l * N + 4 * N
    return (2 + 2 * l) * ntt_mm(N) + 12 * l * N + 6 * N


def workload_modmuls(variant: int, N: int, n: int, l: int, lwes: np.ndarray) -> int:
    """Modmuls of one launch over `lwes` (CGGI skips a_i = 0, BMMP does not)."""
    if variant == 2:
        iters = lwes.shape[0] * (n // 2)
    else:
        iters = int(np.count_nonzero(lwes[:, :n]))
    edge = lwes.shape[0] * (2 * ntt_mm(N) + 2 * N)  # prologue NTTs and X^b
    return iters * modmul_per_iteration(variant, N, l) + edge


def lut_polys(N: int, count: int, seed: int) -> np.ndarray:
    """count x 2N trivial RLWEs (A = 0) of random 16-entry negacyclic LUT test polynomials."""
    from oracle.oracle import sm64
    delta = P // 16
    tables = (sm64(seed, count * 16) % np.uint64(16)).reshape(count, 16)
    vals = np.array([(int(v) * delta) % P for v in range(16)], dtype=np.uint64)
    B = np.repeat(vals[tables.astype(np.int64)], N // 16, axis=1)
    return np.concatenate([np.zeros((count, N), np.uint64), B], axis=1)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def traffic_from_profiles(workload: str):
    """DRAM bytes per launch from the committed ncu summary of this workload, if any."""
    f = ROOT / "profiles" / "traffic.json"
    if not f.exists():
        return None, None
    d = json.loads(f.read_text()).get(workload)
    if not d:
        return None, None
    return d.get("dram_bytes_per_launch"), d.get("source")


def bench_config(wl: str, batch: int, n: int) -> dict:
    """The `config` object of the JSON line, the same keys in both arms."""
    variant, N, _, bl, l, _ = WORKLOADS[wl]
    key_bytes = BlindRotationKeyWords(variant, N, n, l) * 8
    return {"workload": DESCR[wl], "batch_per_gpu": batch, "ring_dim": N, "lwe_dim": n, "gadget": f"2^{bl} l={l}",
            "output": "NTT domain",
            "inputs": "seeded synthetic LWEs + per-ciphertext 16-entry LUT test polynomials",
            "l2": f"inputs larger than L2: {key_bytes / 2**20:.0f} MiB key streamed per launch"}


def BlindRotationKeyWords(variant: int, N: int, n: int, l: int) -> int:
    """Words of the reference's m_brk: per iteration group 2l rows of G RGSWs x [A|B]."""
    groups = n // 2 if variant == 2 else n
    g = 1 if variant == 0 else (2 if variant == 1 else 3)
    return groups * g * 4 * N * l


def cpu_reference_sample(variant, N, n, bl, l, lwes, accs, seconds_target=15.0):
    """Times the reference library's CPU blind rotation on a bounded sample,
    one rotator per host thread. Returns (BR/s, threads, rotations, seconds)."""
    import ctypes

    from oracle.oracle import Reference, lwe_secret, ptr, rlwe_secret
    ref = Reference()
    L = ref.L
    cores = os.cpu_count() or 1
    key_bytes = (n if variant < 2 else n // 2) * (1 if variant == 0 else (2 if variant == 1 else 3)) * 4 * N * l * 8
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError):
        avail = 16 << 30
    threads = max(1, min(cores, int(avail * 0.5 // max(key_bytes, 1))))
    lk = lwe_secret(variant, n, N, 1)
    rk = rlwe_secret(N, 2)
    L.ref_seed(3)
    h = L.ref_br_create(variant, N, n, bl, l, 0.0, ptr(lk), ptr(rk))
    # one warm rotation to size the sample
    one = np.empty(2 * N, np.uint64)
    t0 = time.perf_counter()
    L.ref_br_rotate(h, ptr(one), ptr(np.ascontiguousarray(lwes[0])), ptr(np.ascontiguousarray(accs[0])), 0)
    t1 = time.perf_counter() - t0
    per_thread = max(1, int(seconds_target / max(t1, 1e-3) / 4))
    count = min(threads * per_thread, lwes.shape[0])
    res = np.empty((count, 2 * N), np.uint64)
    secs = L.ref_br_rotate_many(h, ptr(res), ptr(np.ascontiguousarray(lwes[:count])),
                                ptr(np.ascontiguousarray(accs[:count])), count, 0, threads)
    key = np.empty(L.ref_br_key_words(h), np.uint64)
    L.ref_br_key_copy(h, ptr(key))
    L.ref_br_destroy(h)
    return count / secs, threads, count, secs, key, res


def gpu_matches_reference(variant, N, n, bl, l, key, lwes, accs, ref_out, device) -> bool:
    """Rotates the CPU sample on the GPU with the reference's own key and compares every word."""
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    rot = GpuBlindRotator(BlindRotationContext(variant, N, n, 1 << bl, l), key, device=device)
    got = rot.blind_rotate_batch_host(np.ascontiguousarray(lwes), np.ascontiguousarray(accs), out_coef=False)
    rot.close()
    return bool(np.array_equal(got, ref_out))


def run_reference(args, wl):
    variant, N, n, bl, l, batch = WORKLOADS[wl]
    from oracle.oracle import lwe_inputs
    lwes = lwe_inputs(N, n, batch, 7)
    accs = lut_polys(N, batch, 8)
    vals = []
    for s in range(args.warmup + args.steps):
        v, threads, count, secs = cpu_reference_sample(variant, N, n, bl, l, lwes, accs,
                                                       seconds_target=args.ref_seconds)[:4]
        if s >= args.warmup:
            vals.append((v, threads, count, secs))
    v = statistics.median([x[0] for x in vals])
    threads, count = vals[-1][1], vals[-1][2]
    cfg = bench_config(wl, batch, n)
    line = {"impl": "reference", "metric": "blind rotations/sec", "value": round(v, 3), "unit": "BR/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(statistics.median([x[3] for x in vals]) * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (mod p)",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": round(v, 3), "unit": "BR/s", "cores": threads, "kind": "reference",
                             "sample": f"{count} rotations per step on {threads} threads (one rotator each), "
                                       "reference library built from its own sources (oracle/_ref)"},
            "e2e": {"value": round(v, 3), "unit": "BR/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _timed(torch, fn, warmup: int, reps: int, stream) -> float:
    """Mean ms of fn() over reps launches on `stream` (CUDA events), after warmup."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _uniform_key(words: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.integers(0, 2**63, words, dtype=np.uint64)  # residues below p


BMMP_BATCHES = (1, 37, 512, 2048, 8192)


def bmmp_batch_sweep(device: int) -> dict:
    """BMMP (binary n=768 as 384 pairs, N=2048, base 2^16 l=4) at uneven batch sizes,
    identity test polynomials; per batch size the autotuner picks the tile and the
    blocks per rotation, then one graph-recorded launch per step is timed."""
    import torch
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    from oracle.oracle import lwe_inputs
    N, n = 2048, 768
    ctx = BlindRotationContext(2, N, n, 1 << 16, 4)
    rot = GpuBlindRotator(ctx, _uniform_key(ctx.key_words(), 31), device=device)
    stream = torch.cuda.current_stream().cuda_stream
    ident = np.zeros(2 * N, np.uint64)
    ident[N:] = np.arange(N, dtype=np.uint64)
    out = {"workload": "BMMP n=768 (384 pairs), N=2048, base 2^16 l=4, identity LUT", "unit": "BR/s"}
    lw_all = torch.from_numpy(lwe_inputs(N, n, max(BMMP_BATCHES), 33).view(np.int64)).cuda()
    ac = torch.from_numpy(ident.view(np.int64)).cuda()
    res = torch.empty((max(BMMP_BATCHES), 2 * N), dtype=torch.int64, device="cuda")
    key = _uniform_key(ctx.key_words(), 31)
    lw_host = lwe_inputs(N, n, max(BMMP_BATCHES), 33)
    for b in BMMP_BATCHES:
        coef, _ = rot.autotune(b)
        g = rot.capture_batch(res.data_ptr(), lw_all.data_ptr(), n + 1, ac.data_ptr(), 0, b)
        reps = 3 if b >= 512 else 5
        ms = _timed(torch, lambda: g.launch(stream), 2, reps, stream)
        g.close()
        out[str(b)] = {"BR_per_s": round(b / (ms * 1e-3), 1), "ms_per_launch": round(ms, 3),
                       "tile": {"coef_per_thread": coef, "blocks_per_rotation": rot.split,
                                "mac_form": rot.mac_form}}
        if b >= 2048:
            # sampled parity of the timed launch's results: the oracle with the same key words
            from oracle.oracle import Oracle
            idx = sorted({0, 147, 148, b // 2, b - 1})
            got = res[idx].cpu().numpy().view(np.uint64)
            want = Oracle().blind_rotate_many(2, N, n, 16, 4, key, lw_host[idx],
                                              np.repeat(ident[None, :], len(idx), axis=0), False, 8)
            out[str(b)]["sampled_parity"] = {"ciphertexts": idx, "equal_to_oracle": bool(np.array_equal(got, want))}
    rot.check(stream)
    rot.close()
    return out


LARGE_RINGS = ((8192, 2), (16384, 4), (32768, 8), (65536, 16))  # (N, CTAs per rotation)


def large_ring_run(device: int) -> dict:
    """CGGI ternary rotations (base 2^12, l = 3, n = 64) at the ring sizes that run one rotation
    per cluster of CTAs, two waves of the resident clusters each (uniform key words; the
    parity of these sizes is in tests/test_gpu_largen.py)."""
    import torch
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    from oracle.oracle import lwe_inputs
    n = 64
    out = {"workload": "CGGI ternary, base 2^12 l=3, n=64, one rotation per cluster", "unit": "BR/s"}
    stream = torch.cuda.current_stream().cuda_stream
    for N, ctas in LARGE_RINGS:
        ctx = BlindRotationContext(1, N, n, 1 << 12, 3)
        rot = GpuBlindRotator(ctx, _uniform_key(ctx.key_words(), 41), device=device)
        batch = 2 * (torch.cuda.get_device_properties(device).multi_processor_count // ctas)
        lw = torch.from_numpy(lwe_inputs(N, n, batch, 43).view(np.int64)).cuda()
        ac = torch.from_numpy(lut_polys(N, batch, 44).view(np.int64)).cuda()
        res = torch.empty((batch, 2 * N), dtype=torch.int64, device="cuda")
        ms = _timed(torch, lambda: rot.blind_rotate_batch(res.data_ptr(), lw.data_ptr(), n + 1, ac.data_ptr(),
                                                          2 * N, batch, stream=stream), 1, 3, stream)
        rot.check(stream)
        out[str(N)] = {"BR_per_s": round(batch / (ms * 1e-3), 1), "batch": batch, "ms_per_launch": round(ms, 3),
                       "ctas_per_rotation": ctas}
        rot.close()
        del lw, ac, res
    return out


def packing_run(device: int) -> dict:
    """Config-4 key switching: 2048 LWEs (n = N = 2048) packed into one RLWE with the
    11 automorphism keys (base 2^16, l = 4), 64 packings per launch; then RLWE->RLWE
    key switching of 1024 ciphertexts in one launch."""
    import torch
    from fhetoothpaste_b200 import GpuLWEtoRLWEPacker, GpuRLWEtoRLWEConverter
    N, L, packs, beta, l = 2048, 2048, 64, 16, 4
    stream = torch.cuda.current_stream().cuda_stream
    packer = GpuLWEtoRLWEPacker(N, 1 << beta, l, _uniform_key(11 * 2 * N * l, 41), device=device)
    rng = np.random.default_rng(42)
    lw = torch.from_numpy(rng.integers(0, 2**63, (packs * L, N + 1), dtype=np.uint64).view(np.int64)).cuda()
    po = torch.empty((packs, 2 * N), dtype=torch.int64, device="cuda")
    pack_ms = _timed(torch, lambda: packer.pack_batch(packs, L, po.data_ptr(), lw.data_ptr(), stream), 1, 2, stream)
    del lw
    packer.close()
    conv = GpuRLWEtoRLWEConverter(N, 1 << beta, l, _uniform_key(2 * N * l, 43), device=device)
    cts = 1024
    ci = torch.from_numpy(rng.integers(0, 2**63, (cts, 2 * N), dtype=np.uint64).view(np.int64)).cuda()
    co = torch.zeros((cts, 2 * N), dtype=torch.int64, device="cuda")
    ks_ms = _timed(torch, lambda: conv.convert_batch(cts, co.data_ptr(), ci.data_ptr(), stream), 2, 5, stream)
    conv.close()
    return {"workload": "pack 2048 LWE (n=2048) -> RLWE N=2048, base 2^16 l=4; RLWE KS x1024",
            "packs_per_launch": packs, "ms_per_pack_launch": round(pack_ms, 3),
            "packs_per_s": round(packs / (pack_ms * 1e-3), 2),
            "lwe_packed_per_s": round(packs * L / (pack_ms * 1e-3), 1),
            "rlwe_ks_per_s": round(cts / (ks_ms * 1e-3), 1), "ms_per_ks_launch": round(ks_ms, 3)}


def bootstrap_run(device: int) -> dict:
    """Whole bootstraps (config-1 shape: CGGI binary n=500, N=1024, base 2^16 l=4): blind rotation
    with coefficient output, SampleExtract, LWE key switch N=1024 -> n=500 (base 2^16, l=4) and the
    FLOOR switch to 2N, recorded as one graph over a batch of 4096; the output LWEs are valid inputs
    of the next rotation."""
    import torch
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator, GpuLWEtoLWEConverter
    from oracle.oracle import lwe_inputs
    N, n, beta, l, batch = 1024, 500, 16, 4, 4096
    stream = torch.cuda.current_stream().cuda_stream
    ctx = BlindRotationContext(0, N, n, 1 << beta, l)
    rot = GpuBlindRotator(ctx, _uniform_key(ctx.key_words(), 51), device=device)
    conv = GpuLWEtoLWEConverter(N, n, 1 << beta, l, _uniform_key(N * l * (n + 1), 52), device=device)
    lw = torch.from_numpy(lwe_inputs(N, n, batch, 53).view(np.int64)).cuda()
    ac = torch.from_numpy(lut_polys(N, batch, 54).view(np.int64)).cuda()
    rl = torch.empty((batch, 2 * N), dtype=torch.int64, device="cuda")
    out = torch.empty((batch, n + 1), dtype=torch.int64, device="cuda")
    g = rot.capture_bootstrap(conv, batch, rl.data_ptr(), lw.data_ptr(), ac.data_ptr(), 2 * N, out.data_ptr())
    ms = _timed(torch, lambda: g.launch(stream), 2, 3, stream)
    g.close()
    rot.check(stream)
    # the epilogue alone, for its share of the bootstrap
    ep = _timed(torch, lambda: conv.pbs_epilogue_batch(batch, out.data_ptr(), rl.data_ptr(), 2 * N, stream), 1, 3,
                stream)
    rot.close()
    conv.close()
    return {"workload": "bootstrap: CGGI binary n=500 N=1024 2^16 l=4 + extract + LWE KS 1024->500 + switch to 2N",
            "batch": batch, "bootstraps_per_s": round(batch / (ms * 1e-3), 1), "ms_per_batch": round(ms, 3),
            "epilogue_ms": round(ep, 3)}


def scheme_switch_run(device: int) -> dict:
    """LWE -> RGSW scheme switching at the shape of the reference's scheme-switch tests (CGGI
    binary n=100, N=2048; rotation, trace and squaring gadgets base 2^14 l=4; output 4 digits of
    base 2^14), 1024 conversions per call: rotation of the test polynomial, Lev rows, the trace
    (11 automorphism key switches per row) and the s^2 -> s key switch."""
    import torch
    from fhetoothpaste_b200 import BlindRotationContext, GpuLWEtoRGSWConverter
    from oracle.oracle import lwe_inputs
    N, n, beta, l, D, batch = 2048, 100, 14, 4, 4, 1024
    stream = torch.cuda.current_stream().cuda_stream
    brk_words = BlindRotationContext(0, N, n, 1 << beta, l).key_words()
    conv = GpuLWEtoRGSWConverter((0, N, n, 1 << beta, l), (1 << beta, l), (1 << beta, l), D, 1 << beta,
                                 _uniform_key(brk_words, 61), _uniform_key(11 * 2 * N * l, 62),
                                 _uniform_key(2 * N * l, 63), device=device)
    lw = torch.from_numpy(lwe_inputs(N, n, batch, 64).view(np.int64)).cuda()
    out = torch.empty((batch, 4 * N * D), dtype=torch.int64, device="cuda")
    ms = _timed(torch, lambda: conv.convert_batch(batch, out.data_ptr(), lw.data_ptr(), stream), 1, 3, stream)
    conv.close()
    return {"workload": "LWE->RGSW: CGGI binary n=100 N=2048, gadgets 2^14 l=4, out 4 digits 2^14",
            "batch": batch, "conversions_per_s": round(batch / (ms * 1e-3), 1), "ms_per_batch": round(ms, 3)}


def sap_run(device: int) -> dict:
    """SAP digit decomposition at the shape of the reference's SAP tests (CGGI binary n=10,
    N=4096, rotation / trace / LWE key-switch gadgets base 2^16 l=4, radix 32, inputs mod 2^40:
    8 digits, each a rotation, an extraction and a truncation of 5 trace steps and a 127-node
    key-switch tree), 64 LWEs per call."""
    import torch
    from fhetoothpaste_b200 import BlindRotationContext, GpuSAPDecomposer
    N, n, beta, l, radix, batch = 4096, 10, 16, 4, 32, 64
    stream = torch.cuda.current_stream().cuda_stream
    brk_words = BlindRotationContext(0, N, n, 1 << beta, l).key_words()
    dec = GpuSAPDecomposer((0, N, n, 1 << beta, l), (1 << beta, l), (1 << beta, l), _uniform_key(brk_words, 71),
                           _uniform_key(12 * 2 * N * l, 72), _uniform_key(N * l * (n + 1), 73), hamming_weight=5,
                           device=device)
    rng = np.random.default_rng(74)
    lw = torch.from_numpy(rng.integers(0, 1 << 40, (batch, n + 1), dtype=np.uint64).view(np.int64)).cuda()
    out = torch.zeros((batch, 9, N + 1), dtype=torch.int64, device="cuda")
    ms = _timed(torch, lambda: dec.decompose_batch(batch, out.data_ptr(), 9, lw.data_ptr(), radix, stream), 1, 3,
                stream)
    dec.close()
    return {"workload": "SAP: CGGI binary n=10 N=4096, gadgets 2^16 l=4, radix 32, inputs mod 2^40 (8 digits)",
            "batch": batch, "decompositions_per_s": round(batch / (ms * 1e-3), 1), "ms_per_batch": round(ms, 3)}


SERVING_SETS = [(1024, 500), (2048, 630), (4096, 900)]  # ternary, base 2^12, l = 3
SERVING_MIX = [0.5, 0.35, 0.15]


SERVING_LIGHT_RATE = 300.0  # requests/s of the light-load point (launches of a few requests)


def serving_run(device: int, rate: float, seconds: float) -> dict:
    """Config-5 serving loop: Poisson single-bootstrap requests over three resident
    ternary parameter sets, continuous batching in the native scheduler. Three load
    points: the offered rate (overload), 80% of what that achieved (sustainable), and
    a light load whose latency is one small launch."""
    from fhetoothpaste_b200 import BlindRotationContext, BootstrapServer, GpuBlindRotator
    from oracle.oracle import lwe_inputs
    rots, pools = [], []
    for i, (N, n) in enumerate(SERVING_SETS):
        ctx = BlindRotationContext(1, N, n, 1 << 12, 3)
        kw = ctx.key_words()
        rng = np.random.default_rng(77 + i)
        brk = rng.integers(0, 2**63, kw, dtype=np.uint64)  # below p; timing does not depend on key values
        rots.append(GpuBlindRotator(ctx, brk, device=device))
        del brk
        pools.append((lwe_inputs(N, n, 256, 900 + i), lut_polys(N, 256, 950 + i)))
    out = {"sets": [f"N={N} n={n}" for N, n in SERVING_SETS], "mix": SERVING_MIX,
           "key_bytes_resident": sum(r.ctx.key_words() * 8 for r in rots), "duration_s": seconds}
    for label, r in (("offered", rate), ("sustainable", None), ("light", SERVING_LIGHT_RATE)):
        srv = BootstrapServer(device=device, max_queue=2500)
        for rot, mb in zip(rots, (296, 148, 148)):
            srv.add_set(rot, max_batch=mb, buffers=2)
        srv.start()
        if r is None:
            # 80% of the throughput the overloaded run achieved
            r = 0.8 * out["offered"]["achieved_per_s"]
        st = srv.run_poisson(rate=r, seconds=seconds, mix=SERVING_MIX, pools=pools, seed=5)
        srv.close()
        out[label] = {k: (round(v, 3) if isinstance(v, float) else v) for k, v in st.items()}
    for rot in rots:
        rot.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cggi_ternary_n2048", choices=sorted(WORKLOADS))
    ap.add_argument("--batch", type=int, default=0, help="override the per-GPU batch")
    ap.add_argument("--ref-seconds", type=float, default=15.0, help="CPU work per reference sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="full", choices=["full", "kernel"],
                    help="kernel: only warm-up + timed batch launches (for profiler captures)")
    ap.add_argument("--lwe-dim", type=int, default=0, help="override n (smaller profiler captures)")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=10.0)
    ap.add_argument("--serve-rate", type=float, default=50000.0)
    ap.add_argument("--no-extras", action="store_true", help="skip the BMMP batch sweep and the packing run")
    args = ap.parse_args()

    from fhetoothpaste_b200.dist_util import aggregate_rate, env_ranks, init, max_over_ranks, weak_seed
    rank, world, local = env_ranks()
    wl = args.workload

    if args.impl == "reference":
        if rank == 0:
            run_reference(args, wl)
        return

    import torch
    torch.cuda.set_device(local)
    dist = init("nccl", timeout_s=120.0)  # None on one GPU

    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator, _native
    from oracle.oracle import lwe_inputs

    variant, N, n, bl, l, batch = WORKLOADS[wl]
    if args.batch:
        batch = args.batch
    if args.lwe_dim:
        n = args.lwe_dim
    ctx = BlindRotationContext(variant, N, n, 1 << bl, l)
    # Key words are uniform residues: timing does not depend on their values
    # (parity with real keys is covered by the test suite).
    kw = ctx.key_words()
    rng = np.random.default_rng(weak_seed(1234, rank))
    brk = rng.integers(0, 2**63, kw, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, kw, dtype=np.uint64)
    brk = np.where(brk >= np.uint64(P), brk - np.uint64(P), brk)
    rot = GpuBlindRotator(ctx, brk, device=local)
    del brk

    lwes_h = lwe_inputs(N, n, batch, weak_seed(7, rank))   # each rank rotates its own batch
    accs_h = lut_polys(N, batch, weak_seed(8, rank))
    lw = torch.from_numpy(lwes_h.view(np.int64)).cuda()
    ac = torch.from_numpy(accs_h.view(np.int64)).cuda()
    out = torch.empty((batch, 2 * N), dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    # one step = one replay of the recorded batch launch (CUDA graph)
    graph = rot.capture_batch(out.data_ptr(), lw.data_ptr(), n + 1, ac.data_ptr(), 2 * N, batch)

    def step():
        graph.launch(stream)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    for _ in range(args.warmup):
        step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lib = _native.lib()
    with ClockSampler(local) as clk:
        c0 = lib.tp_kernel_launches()
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        c1 = lib.tp_kernel_launches()
        barrier()
    rot.check(stream)
    ms = e0.elapsed_time(e1) / args.steps
    graph.close()
    if args.mode == "kernel":
        if rank == 0:
            print(json.dumps({"mode": "kernel", "workload": wl, "batch": batch, "lwe_dim": n,
                              "ms_per_launch": round(ms, 3), "rotations_per_s": round(batch / (ms * 1e-3), 1)}))
        rot.close()
        if dist:
            dist.destroy_process_group()
        return
    ms = max_over_ranks(ms, dist, "cuda")
    value = aggregate_rate(batch, world, ms * 1e-3)
    timed_launches = c1 - c0

    # end-to-end through the host-buffer call: pinned host inputs, copies inside
    lw_p = torch.from_numpy(lwes_h.view(np.int64)).pin_memory()
    ac_p = torch.from_numpy(accs_h.view(np.int64)).pin_memory()
    res_p = torch.empty((batch, 2 * N), dtype=torch.int64).pin_memory()
    L = _native.lib()

    def e2e_step():
        _native.check(L.tp_br_blind_rotate_batch_host(
            rot.handle, batch, _native.ctypes.cast(res_p.data_ptr(), _native.U64P),
            _native.ctypes.cast(lw_p.data_ptr(), _native.U64P), n + 1,
            _native.ctypes.cast(ac_p.data_ptr(), _native.U64P), 2 * N, 0, stream))

    e2e_steps = args.steps
    for _ in range(1):
        e2e_step()
    barrier()
    # CUDA events on the launching stream: the call's host->device copies, the
    # launch and the device->host copy of the results are all on this stream
    c2 = L.tp_kernel_launches()
    e0.record()
    for _ in range(e2e_steps):
        e2e_step()
    e1.record()
    e2e_launches = L.tp_kernel_launches() - c2
    barrier()
    e2e_s = max_over_ranks(e0.elapsed_time(e1) * 1e-3 / e2e_steps, dist, "cuda")
    e2e_val = aggregate_rate(batch, world, e2e_s)
    h2d = lwes_h.nbytes + accs_h.nbytes
    d2h = batch * 2 * N * 8

    # plain form: one rotation per launch (one thread block, as the batched kernel
    # runs it), and the same with the rotation split over two and four SMs
    one_out = torch.empty((1, 2 * N), dtype=torch.int64, device="cuda")
    plain_reps = 3

    def plain_time() -> float:
        rot.blind_rotate_batch(one_out.data_ptr(), lw.data_ptr(), n + 1, ac.data_ptr(), 2 * N, 1, stream=stream)
        torch.cuda.synchronize()
        e0.record()
        for i in range(plain_reps):
            rot.blind_rotate_batch(one_out.data_ptr(), lw[i:].data_ptr(), n + 1, ac[i:].data_ptr(), 2 * N, 1,
                                   stream=stream)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / plain_reps

    plain_ms = plain_time()
    rot.set_split(2)
    plain2_ms = plain_time()
    plain4_ms = None
    try:
        rot.set_split(4)
        plain4_ms = plain_time()
    except _native.TpError:  # the four-block kernel does not fit this parameter set
        pass
    rot.set_split(1)

    # roofline: algorithmic modmuls per launch over the kernel's launch time,
    # against the measured 64x64->128 product rate of this GPU
    import ctypes
    prod, imad = ctypes.c_double(), ctypes.c_double()
    _native.check(L.tp_measure_int_peak(local, ctypes.byref(prod), ctypes.byref(imad)))
    mm = workload_modmuls(variant, N, n, l, lwes_h)
    achieved = mm / (ms * 1e-3)
    traffic, tsrc = traffic_from_profiles(wl)
    key_bytes = kw * 8

    plain = {"value": round(1e3 / plain_ms, 3), "unit": "BR/s", "ms_per_rotation": round(plain_ms, 3),
             "batched_over_plain": round(value / world / (1e3 / plain_ms), 1),
             "two_blocks": {"value": round(1e3 / plain2_ms, 3), "ms_per_rotation": round(plain2_ms, 3),
                            "batched_over_plain": round(value / world / (1e3 / plain2_ms), 1)},
             "four_blocks": None if plain4_ms is None else {
                 "value": round(1e3 / plain4_ms, 3), "ms_per_rotation": round(plain4_ms, 3),
                 "batched_over_plain": round(value / world / (1e3 / plain4_ms), 1)}}
    imad8 = imad.value / 8  # 8 IMAD issues per 64x64 modmul at the measured IMAD rate
    line = {
        "metric": "blind rotations/sec", "value": round(value, 2), "unit": "BR/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 (mod p)", "data": "synthetic",
        "gpu_launches": int(timed_launches),
        "config": bench_config(wl, batch, n),
        "roofline": {"bound": "int32", "achieved": round(achieved / 1e9, 1), "peak": round(prod.value / 1e9, 1),
                     "unit": "Gmodmul/s", "frac": round(achieved / prod.value, 4), "traffic": traffic,
                     "traffic_source": tsrc,
                     "peak_source": "measured 64x64->128 IMAD-chain product rate of this GPU (tp_measure_int_peak)",
                     "frac_imad8": round(achieved / imad8, 4),
                     "peak_imad8": round(imad8 / 1e9, 1),
                     "imad8_source": "measured mad.lo.u32 rate / 8 IMAD per modmul (the scope table's formula)",
                     "imad_per_s": round(imad.value / 1e12, 2),
                     "algorithmic_modmul_per_launch": mm,
                     "key_hbm": {"bytes_per_launch": key_bytes,
                                 "achieved_gbs": round(key_bytes / (ms * 1e-3) / 1e9, 1)}},
        "e2e": {"value": round(e2e_val, 2), "unit": "BR/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": e2e_steps},
        "clocks": clk.summary(),
        "launch": {"form": "CUDA graph, one kernel per step", "coef_per_thread": rot.tile,
                   "blocks_per_rotation": rot.split, "mac_form": rot.mac_form, "radix": rot.radix,
                   "key": "uniform random key words (timing does not depend on key values)"},
    }
    if rank == 0 and world == 1 and not args.no_serving:
        line["serving"] = serving_run(local, args.serve_rate, args.serve_seconds)
    if rank == 0 and world == 1 and not args.no_extras:
        line["bmmp_batches"] = bmmp_batch_sweep(local)
        line["packing"] = packing_run(local)
        line["bootstrap"] = bootstrap_run(local)
        line["scheme_switch"] = scheme_switch_run(local)
        line["sap"] = sap_run(local)
        line["large_rings"] = large_ring_run(local)
    line["gpu_launches_detail"] = {"timed_region": int(timed_launches), "e2e_timed_region": int(e2e_launches),
                                   "counted_by": "tp_kernel_launches() deltas (graph replays count their kernels)"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, threads, count, secs, ref_key, ref_out = cpu_reference_sample(variant, N, n, bl, l, lwes_h, accs_h,
                                                                             seconds_target=args.ref_seconds)
            line["cpu_baseline"] = {"value": round(v, 3), "unit": "BR/s", "cores": threads, "kind": "reference",
                                    "ms_per_rotation_per_core": round(1e3 * threads / v, 1),
                                    "sample": f"{count} rotations on {threads} threads in {secs:.1f}s "
                                              "(reference library, one rotator per thread)",
                                    "gpu_outputs_match": gpu_matches_reference(variant, N, n, bl, l, ref_key,
                                                                               lwes_h[:count], accs_h[:count],
                                                                               ref_out, local)}
        except Exception as exc:  # the baseline is reported, not required
            line["cpu_baseline"] = {"value": None, "unit": "BR/s", "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {exc}"}
    rot.close()
    line["gpu_launches_detail"]["whole_run"] = int(_native.lib().tp_kernel_launches())
    # last, so that a reader keeping the end of the line sees the batched/plain ratio
    line["plain"] = plain
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
