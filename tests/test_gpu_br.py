"""Blind-rotation parity on the GPU through the C ABI.

Bit-exact against the golden vectors recorded from the reference library and
against the C oracle on fresh seeded inputs.
"""
import numpy as np
import pytest

from brcases import case_inputs, case_key
from oracle.oracle import lwe_inputs, random_acc

pytestmark = pytest.mark.gpu

ALL_CASES = ["small_binary_n256", "small_ternary_n128", "small_bmmp_n512", "cfg1_binary_n1024",
             "cfg5a_ternary_n1024", "cfg2_ternary_n2048", "cfg3_bmmp_n2048", "cfg5c_ternary_n4096"]
SMALL = ["small_binary_n256", "small_ternary_n128", "small_bmmp_n512"]


def rotator(oracle, golden, name):
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    manifest, _ = golden
    case = manifest["br"][name]
    _, _, brk = case_key(oracle, name, case)
    ctx = BlindRotationContext(case["variant"], case["N"], case["n"], 1 << case["basis_log2"], case["digits"])
    return case, GpuBlindRotator(ctx, brk)


@pytest.mark.parametrize("name", ALL_CASES)
def test_plain_blind_rotate_matches_reference(native, oracle, golden, name):
    case, rot = rotator(oracle, golden, name)
    lwes, accs, coefs = case_inputs(name, case)
    expect = golden[1][f"br_{name}"]
    for i, oc in enumerate(coefs):
        res = np.zeros(2 * case["N"], np.uint64)
        rot.BlindRotate(res, np.ascontiguousarray(lwes[i]), np.ascontiguousarray(accs[i]), bool(oc))
        np.testing.assert_array_equal(res, expect[i])


@pytest.mark.parametrize("name", ALL_CASES)
def test_batched_blind_rotate_matches_reference(native, oracle, golden, name):
    case, rot = rotator(oracle, golden, name)
    lwes, accs, coefs = case_inputs(name, case)
    expect = golden[1][f"br_{name}"]
    for oc in (0, 1):
        idx = [i for i, c in enumerate(coefs) if c == oc]
        got = rot.blind_rotate_batch_host(lwes[idx], accs[idx], out_coef=bool(oc))
        np.testing.assert_array_equal(got, expect[idx])


@pytest.mark.parametrize("name", SMALL)
def test_batch_against_oracle_fresh_inputs(native, oracle, golden, name):
    """A batch larger than the resident grid, so blocks loop over ciphertexts."""
    case, rot = rotator(oracle, golden, name)
    N, n = case["N"], case["n"]
    _, _, brk = case_key(oracle, name, case)
    batch = 2 * 148 * 8 + 5
    lwes = lwe_inputs(N, n, batch, 777)
    accs = random_acc(N, batch, 778)
    for oc in (0, 1):
        got = rot.blind_rotate_batch_host(lwes, accs, out_coef=bool(oc))
        for b in (0, 1, 148, batch // 2, batch - 1):
            exp = oracle.blind_rotate(case["variant"], N, n, case["basis_log2"], case["digits"], brk, lwes[b],
                                      accs[b], oc)
            np.testing.assert_array_equal(got[b], exp, err_msg=f"ciphertext {b}")


@pytest.mark.parametrize("name", SMALL)
def test_shared_accumulator_and_edge_words(native, oracle, golden, name):
    """acc_stride 0 (one test polynomial for the whole batch); a_i in {0, N, 2N-1}, b >= N."""
    case, rot = rotator(oracle, golden, name)
    N, n = case["N"], case["n"]
    _, _, brk = case_key(oracle, name, case)
    lwes = lwe_inputs(N, n, 6, 91)
    lwes[0, :] = 0                      # every a_i = 0 and b = 0: the accumulator only goes through the NTTs
    lwes[1, :] = N                      # X^N = -1 everywhere
    lwes[2, :] = 2 * N - 1
    lwes[3, n] = N + 1
    acc = random_acc(N, 1, 92)[0]
    got = rot.blind_rotate_batch_host(lwes, acc, out_coef=True)
    for b in range(6):
        exp = oracle.blind_rotate(case["variant"], N, n, case["basis_log2"], case["digits"], brk, lwes[b], acc, 1)
        np.testing.assert_array_equal(got[b], exp, err_msg=f"ciphertext {b}")


def test_out_of_range_lwe_is_reported(native, oracle, golden):
    from fhetoothpaste_b200 import TpError
    case, rot = rotator(oracle, golden, "small_ternary_n128")
    N, n = case["N"], case["n"]
    lwes = lwe_inputs(N, n, 2, 5)
    lwes[1, 3] = 2 * N + 3
    acc = random_acc(N, 1, 6)[0]
    with pytest.raises(TpError) as ei:
        rot.blind_rotate_batch_host(lwes, acc)
    assert ei.value.status == 1
    # the flag is cleared once reported
    rot.blind_rotate_batch_host(lwes[:1], acc)


def test_result_may_alias_accumulator(native, oracle, golden, cuda):
    """SAP passes result == accumulator (sap_decomposer.cpp:369); the batch kernel reads every
    accumulator word of a ciphertext before writing its result."""
    torch = cuda
    case, rot = rotator(oracle, golden, "small_binary_n256")
    N, n = case["N"], case["n"]
    _, _, brk = case_key(oracle, "small_binary_n256", case)
    lwes = lwe_inputs(N, n, 3, 21)
    accs = random_acc(N, 3, 22)
    d_lwe = torch.from_numpy(lwes.view(np.int64)).cuda()
    d_acc = torch.from_numpy(accs.view(np.int64)).cuda()
    rot.blind_rotate_batch(d_acc.data_ptr(), d_lwe.data_ptr(), n + 1, d_acc.data_ptr(), 2 * N, 3, out_coef=True)
    rot.check()
    got = d_acc.cpu().numpy().view(np.uint64)
    for b in range(3):
        exp = oracle.blind_rotate(case["variant"], N, n, case["basis_log2"], case["digits"], brk, lwes[b], accs[b], 1)
        np.testing.assert_array_equal(got[b], exp)


@pytest.mark.parametrize("name", SMALL)
def test_graph_replays_read_fresh_inputs(native, oracle, golden, cuda, name):
    """One recorded graph (rotation + SampleExtract), replayed over two different input sets."""
    torch = cuda
    case, rot = rotator(oracle, golden, name)
    N, n = case["N"], case["n"]
    _, _, brk = case_key(oracle, name, case)
    batch = 150
    d_lwe = torch.empty((batch, n + 1), dtype=torch.int64, device="cuda")
    d_acc = torch.empty((batch, 2 * N), dtype=torch.int64, device="cuda")
    d_res = torch.empty((batch, 2 * N), dtype=torch.int64, device="cuda")
    d_ext = torch.empty((batch, N + 1), dtype=torch.int64, device="cuda")
    graph = rot.capture_batch(d_res.data_ptr(), d_lwe.data_ptr(), n + 1, d_acc.data_ptr(), 2 * N, batch,
                              out_coef=True, extract_ptr=d_ext.data_ptr())
    for seed in (31, 41):
        lwes = lwe_inputs(N, n, batch, seed)
        accs = random_acc(N, batch, seed + 1)
        d_lwe.copy_(torch.from_numpy(lwes.view(np.int64)))
        d_acc.copy_(torch.from_numpy(accs.view(np.int64)))
        graph.launch()
        rot.check()
        res = d_res.cpu().numpy().view(np.uint64)
        ext = d_ext.cpu().numpy().view(np.uint64)
        for b in (0, 77, batch - 1):
            exp = oracle.blind_rotate(case["variant"], N, n, case["basis_log2"], case["digits"], brk, lwes[b],
                                      accs[b], 1)
            np.testing.assert_array_equal(res[b], exp)
            lwe = np.zeros(N + 1, np.uint64)
            oracle.L.tpo_sample_extract(oracle_ptr(lwe), oracle_ptr(exp), 0, N)
            np.testing.assert_array_equal(ext[b], lwe)
    graph.close()


def test_launch_counter(native, oracle, golden, cuda):
    """tp_kernel_launches: a batch launch counts one kernel; recording a graph counts nothing;
    each replay counts the graph's kernels (rotation + SampleExtract = 2)."""
    torch = cuda
    case, rot = rotator(oracle, golden, "small_binary_n256")
    N, n = case["N"], case["n"]
    batch = 8
    d_lwe = torch.zeros((batch, n + 1), dtype=torch.int64, device="cuda")
    d_acc = torch.zeros((batch, 2 * N), dtype=torch.int64, device="cuda")
    d_res = torch.empty((batch, 2 * N), dtype=torch.int64, device="cuda")
    d_ext = torch.empty((batch, N + 1), dtype=torch.int64, device="cuda")
    count = native.tp_kernel_launches
    c0 = count()
    rot.blind_rotate_batch(d_res.data_ptr(), d_lwe.data_ptr(), n + 1, d_acc.data_ptr(), 2 * N, batch)
    assert count() - c0 == 1
    c1 = count()
    graph = rot.capture_batch(d_res.data_ptr(), d_lwe.data_ptr(), n + 1, d_acc.data_ptr(), 2 * N, batch,
                              out_coef=True, extract_ptr=d_ext.data_ptr())
    assert count() == c1
    graph.launch()
    graph.launch()
    torch.cuda.synchronize()
    assert count() - c1 == 4
    graph.close()


def test_short_names_rotate_like_the_oracle(native, oracle, golden, cuda):
    """tp_ctx_create / tp_brk_upload / tp_blind_rotate(_batch): the same calls under the short names."""
    import ctypes
    from fhetoothpaste_b200 import _native as nat
    torch = cuda
    name = "small_binary_n256"
    case = golden[0]["br"][name]
    _, _, brk = case_key(oracle, name, case)
    N, n = case["N"], case["n"]
    p = nat.BrParams(case["variant"], nat.GOLDILOCKS, N, n, 1 << case["basis_log2"], case["digits"])
    h = ctypes.c_void_p()
    assert native.tp_ctx_create(ctypes.byref(p), ctypes.byref(h)) == nat.TP_OK
    assert native.tp_brk_upload(h, nat.ptr(brk), brk.size, 1) == nat.TP_ERR_LAYOUT
    assert native.tp_brk_upload(h, nat.ptr(brk), brk.size, 0) == nat.TP_OK
    lwes = lwe_inputs(N, n, 5, 91)
    accs = random_acc(N, 5, 92)
    d_l = torch.from_numpy(lwes.view(np.int64)).cuda()
    d_a = torch.from_numpy(accs.view(np.int64)).cuda()
    d_r = torch.empty((5, 2 * N), dtype=torch.int64, device="cuda")
    assert native.tp_blind_rotate_batch(h, 5, d_r.data_ptr(), d_l.data_ptr(), d_a.data_ptr(), 2 * N, 1,
                                        None) == nat.TP_OK
    got = d_r.cpu().numpy().view(np.uint64)
    one = np.empty(2 * N, np.uint64)
    assert native.tp_blind_rotate(h, nat.ptr(one), nat.ptr(np.ascontiguousarray(lwes[2])),
                                  nat.ptr(np.ascontiguousarray(accs[2])), 1) == nat.TP_OK
    for b in range(5):
        want = oracle.blind_rotate(case["variant"], N, n, case["basis_log2"], case["digits"], brk, lwes[b], accs[b], 1)
        np.testing.assert_array_equal(got[b], want)
    np.testing.assert_array_equal(one, got[2])
    assert native.tp_ctx_destroy(h) == nat.TP_OK


def test_graph_refuses_extract_without_coefficients(native, oracle, golden, cuda):
    from fhetoothpaste_b200 import TpError
    torch = cuda
    case, rot = rotator(oracle, golden, "small_binary_n256")
    N, n = case["N"], case["n"]
    buf = torch.zeros(4 * (2 * N + n + 1), dtype=torch.int64, device="cuda")
    with pytest.raises(TpError):
        rot.capture_batch(buf.data_ptr(), buf.data_ptr(), n + 1, buf.data_ptr(), 2 * N, 1, out_coef=False,
                          extract_ptr=buf.data_ptr())


def oracle_ptr(a):
    from oracle.oracle import ptr
    return ptr(a)


@pytest.mark.parametrize("name", ALL_CASES)
def test_tile_of_four_matches_reference(native, oracle, golden, name):
    """4 coefficients per thread (radix-4 passes), key re-tiled on the device after upload."""
    case, rot = rotator(oracle, golden, name)
    lwes, accs, coefs = case_inputs(name, case)
    expect = golden[1][f"br_{name}"]
    for tile in (4, 8):
        rot.set_tile(tile)
        assert rot.tile == tile
        for oc in (0, 1):
            idx = [i for i, c in enumerate(coefs) if c == oc]
            got = rot.blind_rotate_batch_host(lwes[idx], accs[idx], out_coef=bool(oc))
            np.testing.assert_array_equal(got, expect[idx], err_msg=f"tile {tile}")


@pytest.mark.parametrize("name", ALL_CASES)
def test_both_accumulation_forms_match_reference(native, oracle, golden, name):
    """Tile 4 with the row-by-row multiply-accumulate and, where it is built (3 or 4 digits,
    N <= 2048), the digit-staged form that sums every output word over all rows before one
    reduction."""
    from fhetoothpaste_b200 import _native
    case, rot = rotator(oracle, golden, name)
    lwes, accs, coefs = case_inputs(name, case)
    expect = golden[1][f"br_{name}"]
    rot.set_tile(4)
    staged = case["digits"] in (3, 4) and case["N"] <= 2048
    assert rot.mac_form == (1 if staged else 0)  # the staged form is the default where it is built
    for form in (0, 1):
        if form == 1 and not staged:
            with pytest.raises(_native.TpError):
                rot.set_mac_form(1)
            continue
        rot.set_mac_form(form)
        for oc in (0, 1):
            idx = [i for i, c in enumerate(coefs) if c == oc]
            got = rot.blind_rotate_batch_host(lwes[idx], accs[idx], out_coef=bool(oc))
            np.testing.assert_array_equal(got, expect[idx], err_msg=f"form {form}")


@pytest.mark.parametrize("name", ALL_CASES)
def test_radix4_passes_match_reference(native, oracle, golden, name):
    """The fused radix-4 passes (N = 1024 .. 4096) give the radix-2 words, with either
    multiply-accumulate form that fits."""
    from fhetoothpaste_b200 import _native
    case, rot = rotator(oracle, golden, name)
    rot.set_tile(4)
    if not 1024 <= case["N"] <= 4096:
        with pytest.raises(_native.TpError):
            rot.set_radix(4)
        return
    rot.set_radix(4)
    assert rot.radix == 4
    lwes, accs, coefs = case_inputs(name, case)
    expect = golden[1][f"br_{name}"]
    for form in (0, 1):
        try:
            rot.set_mac_form(form)
        except _native.TpError:
            continue
        for oc in (0, 1):
            idx = [i for i, c in enumerate(coefs) if c == oc]
            got = rot.blind_rotate_batch_host(lwes[idx], accs[idx], out_coef=bool(oc))
            np.testing.assert_array_equal(got, expect[idx], err_msg=f"radix 4, form {form}")


def test_autotune_picks_a_tile_and_keeps_results(native, oracle, golden):
    name = "small_bmmp_n512"
    case, rot = rotator(oracle, golden, name)
    coef, rate = rot.autotune(300)
    assert coef in (4, 8) and rot.tile == coef and rate > 0
    lwes, accs, coefs = case_inputs(name, case)
    idx = [i for i, c in enumerate(coefs) if c == 0]
    np.testing.assert_array_equal(rot.blind_rotate_batch_host(lwes[idx], accs[idx]), golden[1][f"br_{name}"][idx])


@pytest.mark.parametrize("name", ALL_CASES)
def test_two_block_rotation_matches_reference(native, oracle, golden, name):
    """Two thread blocks per ciphertext (cluster kernel): same words as the reference."""
    case, rot = rotator(oracle, golden, name)
    rot.set_tile(4)
    rot.set_split(2)
    assert rot.split == 2
    lwes, accs, coefs = case_inputs(name, case)
    expect = golden[1][f"br_{name}"]
    for oc in (0, 1):
        idx = [i for i, c in enumerate(coefs) if c == oc]
        got = rot.blind_rotate_batch_host(lwes[idx], accs[idx], out_coef=bool(oc))
        np.testing.assert_array_equal(got, expect[idx], err_msg="two blocks per rotation")
    # one ciphertext through the reference-signature call, result aliasing the accumulator
    res = np.ascontiguousarray(accs[0])
    rot.BlindRotate(res, np.ascontiguousarray(lwes[0]), res, bool(coefs[0]))
    np.testing.assert_array_equal(res, expect[0])


@pytest.mark.parametrize("name", SMALL)
def test_two_block_batches_of_any_size(native, oracle, golden, name):
    """Batch 1, 37 and more pairs than fit on the device (pairs loop over ciphertexts)."""
    case, rot = rotator(oracle, golden, name)
    N, n = case["N"], case["n"]
    _, _, brk = case_key(oracle, name, case)
    rot.set_split(2)
    for batch in (1, 37, 2 * 148 + 3):
        lwes = lwe_inputs(N, n, batch, 500 + batch)
        accs = random_acc(N, batch, 600 + batch)
        got = rot.blind_rotate_batch_host(lwes, accs, out_coef=False)
        for b in sorted({0, batch // 2, batch - 1}):
            exp = oracle.blind_rotate(case["variant"], N, n, case["basis_log2"], case["digits"], brk, lwes[b],
                                      accs[b], 0)
            np.testing.assert_array_equal(got[b], exp, err_msg=f"batch {batch}, ciphertext {b}")


@pytest.mark.parametrize("split", [2, 4])
def test_split_needs_tile_of_four(native, oracle, golden, split):
    from fhetoothpaste_b200 import TpError
    case, rot = rotator(oracle, golden, "small_binary_n256")
    rot.set_tile(8)
    with pytest.raises(TpError):
        rot.set_split(split)
    rot.set_tile(4)
    rot.set_split(split)
    with pytest.raises(TpError):
        rot.set_tile(8)
    with pytest.raises(TpError):
        rot.set_split(3)
    rot.set_split(1)
    rot.set_tile(8)


@pytest.mark.parametrize("name", ALL_CASES)
def test_four_block_rotation_matches_reference(native, oracle, golden, name):
    """Four thread blocks per ciphertext (two per accumulator half, the half's gadget
    digits split between them): same words as the reference. A parameter set whose
    shared-memory plan does not fit one SM refuses the split."""
    from fhetoothpaste_b200 import TpError
    case, rot = rotator(oracle, golden, name)
    rot.set_tile(4)
    try:
        rot.set_split(4)
    except TpError:
        assert case["N"] == 4096 and case["variant"] == 2, "only N = 4096 BMMP sets may refuse"
        pytest.skip("the four-block kernel does not fit this parameter set")
    assert rot.split == 4
    lwes, accs, coefs = case_inputs(name, case)
    expect = golden[1][f"br_{name}"]
    for oc in (0, 1):
        idx = [i for i, c in enumerate(coefs) if c == oc]
        got = rot.blind_rotate_batch_host(lwes[idx], accs[idx], out_coef=bool(oc))
        np.testing.assert_array_equal(got, expect[idx], err_msg="four blocks per rotation")
    res = np.ascontiguousarray(accs[0])
    rot.BlindRotate(res, np.ascontiguousarray(lwes[0]), res, bool(coefs[0]))
    np.testing.assert_array_equal(res, expect[0])


@pytest.mark.parametrize("name", SMALL)
def test_four_block_batches_of_any_size(native, oracle, golden, name):
    """Batch 1, 37 and more clusters than fit on the device (clusters loop over ciphertexts)."""
    case, rot = rotator(oracle, golden, name)
    N, n = case["N"], case["n"]
    _, _, brk = case_key(oracle, name, case)
    rot.set_split(4)
    for batch in (1, 37, 4 * 148 + 3):
        lwes = lwe_inputs(N, n, batch, 700 + batch)
        accs = random_acc(N, batch, 800 + batch)
        got = rot.blind_rotate_batch_host(lwes, accs, out_coef=False)
        for b in sorted({0, batch // 2, batch - 1}):
            exp = oracle.blind_rotate(case["variant"], N, n, case["basis_log2"], case["digits"], brk, lwes[b],
                                      accs[b], 0)
            np.testing.assert_array_equal(got[b], exp, err_msg=f"batch {batch}, ciphertext {b}")


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("digits", [1, 2])
def test_four_block_uneven_digit_split(native, oracle, variant, digits):
    """One or two gadget digits: the second digit subset's CTAs hold one digit or none and
    only relay partial sums. Words equal the oracle's and the one-block kernel's."""
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    from oracle.oracle import lwe_secret, rlwe_secret
    N, n, beta = 256, 8, 16
    lk = lwe_secret(variant, n, N, seed=71)
    rk = rlwe_secret(N, seed=72)
    brk = oracle.br_keygen(variant, N, n, beta, digits, 3.2, lk, rk, seed=73)
    rot = GpuBlindRotator(BlindRotationContext(variant, N, n, 1 << beta, digits), brk)
    rot.set_tile(4)
    lwes = lwe_inputs(N, n, 5, 74)
    accs = random_acc(N, 5, 75)
    one = rot.blind_rotate_batch_host(lwes, accs)
    rot.set_split(4)
    four = rot.blind_rotate_batch_host(lwes, accs)
    np.testing.assert_array_equal(four, one)
    for b in range(5):
        exp = oracle.blind_rotate(variant, N, n, beta, digits, brk, lwes[b], accs[b], 0)
        np.testing.assert_array_equal(four[b], exp, err_msg=f"ciphertext {b}")


def test_function_evaluator_like_oracle(native, oracle, golden):
    from fhetoothpaste_b200 import NegacyclicFunctionEvaluator
    from oracle.oracle import ptr
    name = "small_binary_n256"
    case, rot = rotator(oracle, golden, name)
    N, n = case["N"], case["n"]
    _, _, brk = case_key(oracle, name, case)
    ev = NegacyclicFunctionEvaluator(rot)
    lwes = lwe_inputs(N, n, 3, 81)
    f = lambda x: (5 * x + 2) % 11  # noqa: E731
    res = np.full(N + 1, 9, np.uint64)
    ev.EvalFunc(res, lwes[0], f)
    acc = np.zeros(2 * N, np.uint64)
    acc[0] = 2
    for i in range(1, N):
        acc[i + N] = (0xFFFFFFFF00000001 - (5 * (N - i) + 2) % 11) % 0xFFFFFFFF00000001
    rl = oracle.blind_rotate(case["variant"], N, n, case["basis_log2"], case["digits"], brk, lwes[0], acc, 1)
    want = np.full(N + 1, 9, np.uint64)
    oracle.L.tpo_sample_extract(ptr(want), ptr(rl), 0, N)
    np.testing.assert_array_equal(res, want)
    luts = random_acc(N, 3, 82)
    batch = ev.eval_func_batch(lwes, luts)
    for b in range(3):
        rl = oracle.blind_rotate(case["variant"], N, n, case["basis_log2"], case["digits"], brk, lwes[b], luts[b], 1)
        np.testing.assert_array_equal(batch[b], oracle.sample_extract(rl))


def test_four_block_binary_n4096(native, oracle):
    """Binary N = 4096 fits the four-block plan with two exchange buffers (one RGSW per
    iteration); BMMP (three RGSWs per pair) refuses the split there."""
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator, TpError
    from oracle.oracle import lwe_secret, rlwe_secret
    N, n, beta, digits = 4096, 6, 16, 4
    lk = lwe_secret(0, n, N, seed=81)
    rk = rlwe_secret(N, seed=82)
    brk = oracle.br_keygen(0, N, n, beta, digits, 3.2, lk, rk, seed=83)
    rot = GpuBlindRotator(BlindRotationContext(0, N, n, 1 << beta, digits), brk)
    rot.set_tile(4)
    lwes = lwe_inputs(N, n, 3, 84)
    accs = random_acc(N, 3, 85)
    rot.set_split(4)
    for oc in (False, True):
        got = rot.blind_rotate_batch_host(lwes, accs, out_coef=oc)
        for b in range(3):
            exp = oracle.blind_rotate(0, N, n, beta, digits, brk, lwes[b], accs[b], int(oc))
            np.testing.assert_array_equal(got[b], exp, err_msg=f"ciphertext {b}, out_coef {oc}")
    bctx = BlindRotationContext(2, N, n, 1 << 16, 4)
    brot = GpuBlindRotator(bctx, np.zeros(bctx.key_words(), np.uint64))
    brot.set_tile(4)
    with pytest.raises(TpError):
        brot.set_split(4)
