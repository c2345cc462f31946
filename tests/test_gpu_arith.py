"""Device Goldilocks primitives against exact integer arithmetic, on random
values and on the edges of their input ranges (0, 1, p-1, p..2^64-1, 2^32 +- 1)."""
import numpy as np
import pytest

from oracle.oracle import P, sm64

pytestmark = pytest.mark.gpu

EDGE = [0, 1, 2, 2**32 - 1, 2**32, 2**32 + 1, 2**63, P - 2, P - 1]
EDGE_ANY = EDGE + [P, P + 1, 2**64 - 2**32, 2**64 - 2, 2**64 - 1]


def run(native, cuda, op, a, b, c=None):
    from fhetoothpaste_b200 import _native
    torch = cuda
    a = np.asarray(a, dtype=np.uint64)
    b = np.asarray(b, dtype=np.uint64)
    c = np.zeros_like(a) if c is None else np.asarray(c, dtype=np.uint64)
    da, db, dc = (torch.from_numpy(x.view(np.int64)).cuda() for x in (a, b, c))
    out = torch.empty_like(da)
    _native.check(native.tp_debug_arith(op, a.size, out.data_ptr(), da.data_ptr(), db.data_ptr(), dc.data_ptr(),
                                        None))
    return out.cpu().numpy().view(np.uint64)


def grid(vals):
    a, b = np.meshgrid(np.array(vals, dtype=np.uint64), np.array(vals, dtype=np.uint64))
    return a.ravel(), b.ravel()


def canon_rand(seed, n):
    x = sm64(seed, n)
    return np.where(x >= np.uint64(P), x - np.uint64(P), x)


@pytest.mark.parametrize("op,fn", [(0, lambda a, b: (a + b) % P), (1, lambda a, b: (a - b) % P),
                                   (2, lambda a, b: a * b % P)])
def test_canonical_ops(native, cuda, op, fn):
    a, b = grid(EDGE)
    a = np.concatenate([a, canon_rand(1, 20000)])
    b = np.concatenate([b, canon_rand(2, 20000)])
    got = run(native, cuda, op, a, b)
    exp = np.array([fn(int(x), int(y)) for x, y in zip(a, b)], dtype=np.uint64)
    np.testing.assert_array_equal(got, exp)


def test_fused_multiply_add_any_inputs(native, cuda):
    a, b = grid(EDGE_ANY)
    c = np.resize(np.array(EDGE_ANY[::-1], dtype=np.uint64), a.size)
    a = np.concatenate([a, sm64(3, 20000)])
    b = np.concatenate([b, sm64(4, 20000)])
    c = np.concatenate([c, sm64(5, 20000)])
    got = run(native, cuda, 3, a, b, c)
    exp = np.array([(int(z) + int(x) * int(y)) % P for x, y, z in zip(a, b, c)], dtype=np.uint64)
    np.testing.assert_array_equal(got, exp)


def test_reduce128_any_value(native, cuda):
    lo, hi = grid(EDGE_ANY)
    lo = np.concatenate([lo, sm64(6, 20000)])
    hi = np.concatenate([hi, sm64(7, 20000)])
    got = run(native, cuda, 4, lo, hi)
    exp = np.array([(int(x) + (int(y) << 64)) % P for x, y in zip(lo, hi)], dtype=np.uint64)
    np.testing.assert_array_equal(got, exp)


def test_canonical_reduction_any_value(native, cuda):
    # the canonical reduction's own output must already be below p
    lo, hi = grid(EDGE_ANY)
    lo = np.concatenate([lo, sm64(8, 20000), np.zeros(4, np.uint64)])
    hi = np.concatenate([hi, sm64(9, 20000), np.array([1 << 32, 2**32 - 1, 2**64 - 2**32, 2**64 - 1], np.uint64)])
    got = run(native, cuda, 6, lo, hi)
    exp = np.array([(int(x) + (int(y) << 64)) % P for x, y in zip(lo, hi)], dtype=np.uint64)
    np.testing.assert_array_equal(got, exp)


@pytest.mark.parametrize("op,fn", [(7, lambda a, b: (a + b) % P), (8, lambda a, b: (a + b) % P),
                                   (9, lambda a, b: (a - b) % P)])
def test_add_sub_any_left_operand(native, cuda, op, fn):
    # left operand any 64-bit value (a lazily reduced butterfly input), right canonical
    a, b = np.meshgrid(np.array(EDGE_ANY, dtype=np.uint64), np.array(EDGE, dtype=np.uint64))
    a = np.concatenate([a.ravel(), sm64(10, 20000)])
    b = np.concatenate([b.ravel(), canon_rand(11, 20000)])
    got = run(native, cuda, op, a, b)
    exp = np.array([fn(int(x), int(y)) for x, y in zip(a, b)], dtype=np.uint64)
    np.testing.assert_array_equal(got, exp)
