"""The carry-form Goldilocks reduction and adds of csrc/gl_arith.cuh, step by step in exact
32-bit word arithmetic (each line one instruction of the device sequence, carries and borrows
explicit), against Python integers: all combinations of edge words and seeded random values.
The device functions themselves are tested on the GPU (tests/test_gpu_arith.py)."""
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


def reduce128(r0, r1, r2, r3):
    """t = (r1:r0) - r3 (a borrow takes eps off); S + eps = t + (r2, ~r2); the carry out
    selects the correction 0xFFFFFFFF + carry (0 or eps) to take off."""
    t0, bw = _sub(r0, r3)
    t1, bw = _sub(r1, 0, bw)
    b = (0 - bw) & M32
    t0, bw = _sub(t0, b)
    t1, _ = _sub(t1, 0, bw)
    n = ~r2 & M32
    s0, cf = _add(t0, n)
    s1, cf = _add(t1, r2, cf)
    m, _ = _add(M32, 0, cf)
    s0, bw = _sub(s0, m)
    s1, _ = _sub(s1, 0, bw)
    return (s1 << 32) | s0


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
