"""The carry-form Goldilocks reduction, adds, power-of-two multiplies and the wide product
accumulator of csrc/gl_arith.cuh, step by step in exact 32-bit word arithmetic (each line one
instruction of the device sequence, carries and borrows explicit), against Python integers: all
combinations of edge words and seeded random values. The device functions themselves are tested
on the GPU (tests/test_gpu_arith.py) and inside every transform the parity tests run."""
import random

P = 2**64 - 2**32 + 1
M32 = 2**32 - 1
EDGE32 = [0, 1, 2, M32, M32 - 1, 2**31, 2**31 - 1]


def _sub(a, b, borrow_in=0):
    d = a - b - borrow_in
    return d & M32, 1 if d < 0 else 0


def _add(a, b, carry_in=0):
    s = a + b + carry_in
    return s & M32, s >> 32


def reduce96(w0, w1, w2):
    """(w1:w0) + w2 2^64: S + eps = (w1:w0) + (w2, ~w2); the carry out selects the
    correction 0xFFFFFFFF + carry (0 or eps) to take off."""
    n = ~w2 & M32
    s0, cf = _add(w0, n)
    s1, cf = _add(w1, w2, cf)
    m, _ = _add(M32, 0, cf)
    s0, bw = _sub(s0, m)
    s1, _ = _sub(s1, 0, bw)
    return (s1 << 32) | s0


def reduce_sub64(r0, r1, r2, r3, r4=0):
    """t = (r1:r0) - (r4:r3) (a borrow takes eps off), then reduce96(t, r2)."""
    t0, bw = _sub(r0, r3)
    t1, bw = _sub(r1, r4, bw)
    b = (0 - bw) & M32
    t0, bw = _sub(t0, b)
    t1, _ = _sub(t1, 0, bw)
    return reduce96(t0, t1, r2)


def reduce128(r0, r1, r2, r3):
    """t = (r1:r0) - r3 (a borrow takes eps off); S + eps = t + (r2, ~r2); the carry out
    selects the correction 0xFFFFFFFF + carry (0 or eps) to take off."""
    return reduce_sub64(r0, r1, r2, r3, 0)


def shl(x, k):
    """gl_shl<k>, k in [0, 64): the three words of x 2^(k mod 32), one word higher for k >= 32."""
    x0, x1 = x & M32, x >> 32
    r = k & 31
    w = (x0, x1, 0) if r == 0 else ((x0 << r) & M32, ((x1 << r) | (x0 >> (32 - r))) & M32, x1 >> (32 - r))
    if k == 0:
        return x - P if x >= P else x
    if k < 32:
        return reduce96(*w)
    return reduce128(0, *w)


def shr(x, k):
    """gl_shr<k>, k in [1, 32]: x 2^-k = (h + y) - y 2^32, h = x >> k, y = x0 << (32 - k)."""
    x0, x1 = x & M32, x >> 32
    if k < 32:
        h0, h1, y = ((x0 >> k) | (x1 << (32 - k))) & M32, x1 >> k, (x0 << (32 - k)) & M32
    else:
        h0, h1, y = x1, 0, x0
    a0, cf = _add(h0, y)
    a1, _ = _add(h1, 0, cf)
    d1, bw = _sub(a1, y)
    m, _ = _sub(0, 0, bw)
    r0, bw = _sub(a0, m)
    r1, _ = _sub(d1, 0, bw)
    return (r1 << 32) | r0


def pow2(e):
    """Pow2<e>: (sign, shift) with 2^e = sign * 2^shift, shift in (-32, 64)."""
    e %= 192
    if e < 64:
        return False, e
    return (True, e - 96) if e < 160 else (False, e - 192)


def wide_mad(acc, x, k):
    """wide_mad: D (five words) += x0 k0 + x1 k1 2^64, M (three words) += x0 k1 + x1 k0."""
    d, m = list(acc[0]), list(acc[1])
    x0, x1, k0, k1 = x & M32, x >> 32, k & M32, k >> 32
    d[0], cf = _add(d[0], (x0 * k0) & M32)
    d[1], cf = _add(d[1], (x0 * k0) >> 32, cf)
    d[2], cf = _add(d[2], (x1 * k1) & M32, cf)
    d[3], cf = _add(d[3], (x1 * k1) >> 32, cf)
    d[4], _ = _add(d[4], 0, cf)
    for a, b in ((x0, k1), (x1, k0)):
        m[0], cf = _add(m[0], (a * b) & M32)
        m[1], cf = _add(m[1], (a * b) >> 32, cf)
        m[2], _ = _add(m[2], 0, cf)
    return d, m


def wide_reduce(acc):
    """wide_reduce: s = D + M 2^32 (four adds), then the reduction with subtrahend (s4:s3)."""
    d, m = acc
    s1, cf = _add(d[1], m[0])
    s2, cf = _add(d[2], m[1], cf)
    s3, cf = _add(d[3], m[2], cf)
    s4, _ = _add(d[4], 0, cf)
    return reduce_sub64(d[0], s1, s2, s3, s4)


def add(a, b):
    """a + (b + eps); without a carry out the eps is taken back (0xFFFFFFFF + carry)."""
    bl, cf = _add(b & M32, M32)
    bh, _ = _add(b >> 32, 0, cf)
    s0, cf = _add(a & M32, bl)
    s1, cf = _add(a >> 32, bh, cf)
    m, _ = _add(M32, 0, cf)
    s0, bw = _sub(s0, m)
    s1, _ = _sub(s1, 0, bw)
    return (s1 << 32) | s0


def add_lazy(a, b):
    """a + b; a carry out is folded back as eps (read with addc, negated with sub)."""
    s0, cf = _add(a & M32, b & M32)
    s1, cf = _add(a >> 32, b >> 32, cf)
    c, _ = _add(0, 0, cf)
    m = (0 - c) & M32
    s0, cf = _add(s0, m)
    s1, _ = _add(s1, 0, cf)
    return (s1 << 32) | s0


def test_reduction_is_canonical_for_any_128_bit_value():
    rng = random.Random(1)
    cases = [(a, b, c, d) for a in EDGE32 for b in EDGE32 for c in EDGE32 for d in EDGE32]
    cases += [tuple(rng.getrandbits(32) for _ in range(4)) for _ in range(20000)]
    for c in cases:
        x = c[0] + (c[1] << 32) + (c[2] << 64) + (c[3] << 96)
        assert reduce128(*c) == x % P, c


def test_adds_canonical_and_lazy():
    rng = random.Random(2)
    e64 = [0, 1, 2, P - 1, P - 2, P - 2**32, 2**63, 2**32, 2**32 - 1, 2**64 - 2**33]
    e64 = [v % P for v in e64]
    pairs = [(a, b) for a in e64 for b in e64] + [(rng.randrange(P), rng.randrange(P)) for _ in range(20000)]
    for a, b in pairs:
        assert add(a, b) == (a + b) % P, (a, b)
    # left operand any 64-bit value, right canonical: congruent and below 2^64
    anyl = [0, 1, P - 1, P, P + 1, 2**64 - 2**32, 2**64 - 2, 2**64 - 1]
    pairs = [(a, b) for a in anyl for b in e64] + [(rng.getrandbits(64), rng.randrange(P)) for _ in range(20000)]
    for a, b in pairs:
        for f in (add, add_lazy):
            r = f(a, b)
            assert 0 <= r < 2**64 and r % P == (a + b) % P, (f.__name__, a, b)


def test_power_of_two_multiplies_for_every_exponent():
    rng = random.Random(3)
    xs = [0, 1, 2, P - 1, P, P + 1, 2**64 - 1, 2**64 - 2**32, 2**63, M32, 2**32, M32 << 32]
    xs += [rng.getrandbits(64) for _ in range(3000)]
    for e in range(192):
        neg, k = pow2(e)
        for x in xs:  # any 64-bit x, canonical result
            t = shl(x, k) if k >= 0 else shr(x, -k)
            assert 0 <= t < P, (e, x)
            assert ((P - t) % P if neg else t) == x * pow(2, e, P) % P, (e, x)


def test_power_of_two_twiddle_exponents():
    """pow2_twiddle_exp (csrc/ntt_block.cuh): psi^(+-brv(2^l + i)) = 2^e for the levels l < 5,
    the same exponents for every ring size."""
    def brv(x, bits):
        return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0
    g = [48, 120, 156, 78, 39]
    for N in (128, 256, 1024, 4096, 65536):
        logn = N.bit_length() - 1
        psi = pow(7, (P - 1) // (2 * N), P)
        for lvl in range(min(5, logn)):
            for i in range(1 << lvl):
                e = g[lvl] * (2 * brv(i, lvl) + 1) % 192
                w = pow(psi, brv((1 << lvl) + i, logn), P)
                assert w == pow(2, e, P), (N, lvl, i)
                assert pow(w, P - 2, P) == pow(2, (192 - e) % 192, P)


def test_wide_accumulator_sums_exactly():
    rng = random.Random(4)
    edge = [0, 1, P - 1, 2**64 - 1, 2**63, M32, M32 << 32]
    for terms in (1, 2, 3, 6, 8, 12, 16):
        for trial in range(400):
            pick = (lambda: rng.choice(edge)) if trial < 100 else (lambda: rng.getrandbits(64))
            pairs = [(pick(), pick()) for _ in range(terms)]
            acc = ([0] * 5, [0] * 3)
            for x, k in pairs:
                acc = wide_mad(acc, x, k)
            got = wide_reduce(acc)
            assert got == sum(x * k for x, k in pairs) % P, (terms, pairs)


def test_integer_pass0_for_small_digits():
    """ntt_pass0_small (csrc/ntt_block.cuh): levels 0 and 1 of the forward transform on small
    signed digits as exact 64-bit integer sums, against the butterflies with the reference's
    twiddles psi^brv(1), psi^brv(2), psi^brv(3), at the largest digits allowed (|d| <= 2^14)."""
    rng = random.Random(6)
    D = 1 << 14
    for N in (1024, 2048, 4096):
        logn = N.bit_length() - 1
        psi = pow(7, (P - 1) // (2 * N), P)
        w1, w2, w3 = (pow(psi, int(format(k, f"0{logn}b")[::-1], 2), P) for k in (1, 2, 3))
        cases = [[D, D, D, D], [-D, -D, -D, -D], [D, -D, D, -D], [-D, D, -D, D], [0, 0, 0, 0]]
        cases += [[rng.randint(-D, D) for _ in range(4)] for _ in range(3000)]
        for d in cases:
            x = [v % P for v in d]
            a0, a2 = (x[0] + w1 * x[2]) % P, (x[0] - w1 * x[2]) % P
            a1, a3 = (x[1] + w1 * x[3]) % P, (x[1] - w1 * x[3]) % P
            want = [(a0 + w2 * a1) % P, (a0 - w2 * a1) % P, (a2 + w3 * a3) % P, (a2 - w3 * a3) % P]
            a, b = d[0] + (d[2] << 48), d[0] - (d[2] << 48)
            pp = (d[1] << 24) + (d[3] << 40) - (d[3] << 8)
            qq = (d[1] << 40) - (d[1] << 8) + (d[3] << 24)
            v = [a - pp, a + pp, b - qq, b + qq]
            for j in range(4):
                assert -2**63 <= v[j] < 2**63
                u = v[j] & (2**64 - 1)           # the 64-bit pattern
                got = u - (M32 if v[j] < 0 else 0)  # eps off for negative values
                assert got == want[j] and 0 <= got < P, (N, d, j)
