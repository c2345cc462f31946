"""Serving loop: mixed parameter sets under continuous batching give, for every
request, exactly the words the same request gives alone (integer results: the
tolerance is zero), and admission control rejects beyond the queue bound and beyond the
device-memory budget, admitting again as launches complete."""
import threading

import numpy as np
import pytest

from oracle.oracle import lwe_inputs, lwe_secret, random_acc, rlwe_secret

pytestmark = pytest.mark.gpu

SETS = [  # variant, N, n, basis_log2, digits
    (1, 256, 16, 12, 3),
    (0, 512, 20, 16, 4),
    (2, 1024, 12, 16, 3),
]


@pytest.fixture(scope="module")
def rotators(native, oracle):
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    rots, keys = [], []
    for i, (v, N, n, bl, dg) in enumerate(SETS):
        brk = oracle.br_keygen(v, N, n, bl, dg, 3.2, lwe_secret(v, n, N, 40 + i), rlwe_secret(N, 50 + i), 60 + i)
        rots.append(GpuBlindRotator(BlindRotationContext(v, N, n, 1 << bl, dg), brk))
        keys.append(brk)
    return rots, keys


def test_results_same_alone_and_in_mix(rotators, oracle):
    from fhetoothpaste_b200 import BootstrapServer
    rots, keys = rotators
    srv = BootstrapServer(max_queue=10000)
    sids = [srv.add_set(r, max_batch=16, buffers=2, out_coef=True) for r in rots]
    srv.start()
    rng = np.random.default_rng(3)
    reqs = []
    for k in range(240):
        s = int(rng.integers(0, len(SETS)))
        v, N, n, bl, dg = SETS[s]
        reqs.append((s, lwe_inputs(N, n, 1, 1000 + k)[0], random_acc(N, 1, 2000 + k)[0], np.zeros(2 * N, np.uint64)))
    # in the mix: three client threads submitting concurrently
    tickets = [None] * len(reqs)

    def client(idx):
        for i in idx:
            s, lwe, acc, res = reqs[i]
            tickets[i] = srv.submit(sids[s], lwe, acc, res)

    th = [threading.Thread(target=client, args=(range(j, len(reqs), 3),)) for j in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for t in tickets:
        srv.wait(t)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["rejected"] == 0
    assert st["launches"] < len(reqs)  # requests were batched together
    # alone: one request at a time through the same server
    for i in range(0, len(reqs), 7):
        s, lwe, acc, mixed = reqs[i]
        alone = np.zeros_like(mixed)
        srv.wait(srv.submit(sids[s], lwe, acc, alone))
        np.testing.assert_array_equal(alone, mixed, err_msg=f"request {i}")
    # and against the oracle for a few
    for i in (0, 1, 2, 100):
        s, lwe, acc, mixed = reqs[i]
        v, N, n, bl, dg = SETS[s]
        np.testing.assert_array_equal(mixed, oracle.blind_rotate(v, N, n, bl, dg, keys[s], lwe, acc, 1))
    srv.drain()
    srv.close()


def test_admission_control_bounds_the_queue(rotators):
    from fhetoothpaste_b200 import BootstrapServer, TpError
    rots, _ = rotators
    srv = BootstrapServer(max_queue=4)
    sid = srv.add_set(rots[2], max_batch=2, buffers=1)
    # not started yet: nothing drains the queue, so the fifth request is refused
    v, N, n, bl, dg = SETS[2]
    bufs = [(lwe_inputs(N, n, 1, k)[0], random_acc(N, 1, k)[0], np.zeros(2 * N, np.uint64)) for k in range(5)]
    tickets = [srv.submit(sid, *bufs[k]) for k in range(4)]
    with pytest.raises(TpError):
        srv.submit(sid, *bufs[4])
    srv.start()
    for t in tickets:
        srv.wait(t)
    assert srv.stats()["rejected"] == 1
    srv.close()


def test_memory_budget_refuses_then_readmits(rotators, oracle):
    from fhetoothpaste_b200 import BootstrapServer, TpError, _native
    rots, keys = rotators
    v, N, n, bl, dg = SETS[1]
    req_bytes = ((n + 1) + 4 * N) * 8  # LWE, test polynomial and result of one request
    srv = BootstrapServer(max_queue=1000)
    sid = srv.add_set(rots[1], max_batch=4, buffers=1, out_coef=True)
    srv.set_memory_budget(3 * req_bytes)
    bufs = [(lwe_inputs(N, n, 1, 300 + k)[0], random_acc(N, 1, 400 + k)[0], np.zeros(2 * N, np.uint64))
            for k in range(6)]
    # not started: the first three fill the budget, the next two are refused for memory
    tickets = [srv.submit(sid, *bufs[k]) for k in range(3)]
    assert srv.memory()["in_use_bytes"] == 3 * req_bytes
    for k in (3, 4):
        with pytest.raises(TpError) as e:
            srv.submit(sid, *bufs[k])
        assert e.value.status == _native.TP_ERR_OOM
    srv.start()
    for t in tickets:
        srv.wait(t)
    srv.drain()
    m = srv.memory()
    assert m["in_use_bytes"] == 0 and m["rejected_for_memory"] == 2 and m["budget_bytes"] == 3 * req_bytes
    # the completed launches returned their bytes: refused requests are admitted now
    for k in (3, 4, 5):
        srv.wait(srv.submit(sid, *bufs[k]))
    for k in (0, 3, 5):
        lwe, acc, res = bufs[k]
        np.testing.assert_array_equal(res, oracle.blind_rotate(v, N, n, bl, dg, keys[1], lwe, acc, 1))
    assert srv.stats()["rejected"] == 2
    srv.close()


def test_default_memory_budget_is_free_device_memory(rotators):
    from fhetoothpaste_b200 import BootstrapServer
    import torch
    rots, _ = rotators
    srv = BootstrapServer(max_queue=16)
    srv.add_set(rots[0], max_batch=8, buffers=2)
    srv.start()
    free, _ = torch.cuda.mem_get_info()
    budget = srv.memory()["budget_bytes"]
    assert 0.5 * free < budget < 1.5 * free + (1 << 30)
    srv.close()


def test_poisson_load_generator_reports_latency(rotators):
    from fhetoothpaste_b200 import BootstrapServer
    rots, _ = rotators
    srv = BootstrapServer(max_queue=100000)
    for r in rots:
        srv.add_set(r, max_batch=64, buffers=2)
    srv.start()
    pools = [(lwe_inputs(N, n, 32, 7 + i), random_acc(N, 32, 8 + i)) for i, (v, N, n, bl, dg) in enumerate(SETS)]
    st = srv.run_poisson(rate=2000.0, seconds=1.0, mix=[0.5, 0.35, 0.15], pools=pools)
    assert st["completed"] > 1000
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["p999_ms"] <= st["max_ms"]
    srv.close()


def test_cluster_ring_set_in_the_mix(native, oracle):
    """A set of ring size 8192 (one rotation per cluster of four CTAs) served beside a small set:
    every request equals the oracle."""
    from fhetoothpaste_b200 import BlindRotationContext, BootstrapServer, GpuBlindRotator
    sets = [(1, 8192, 4, 12, 3), (0, 512, 20, 16, 4)]
    rots, keys = [], []
    for i, (v, N, n, bl, dg) in enumerate(sets):
        brk = oracle.br_keygen(v, N, n, bl, dg, 3.2, lwe_secret(v, n, N, 70 + i), rlwe_secret(N, 80 + i), 90 + i)
        rots.append(GpuBlindRotator(BlindRotationContext(v, N, n, 1 << bl, dg), brk))
        keys.append(brk)
    srv = BootstrapServer(max_queue=1000)
    sids = [srv.add_set(r, max_batch=8, buffers=2, out_coef=True) for r in rots]
    srv.start()
    reqs = []
    for k in range(24):
        s = k % 2
        v, N, n, bl, dg = sets[s]
        req = (s, lwe_inputs(N, n, 1, 3000 + k)[0], random_acc(N, 1, 4000 + k)[0], np.zeros(2 * N, np.uint64))
        reqs.append((req, srv.submit(sids[s], req[1], req[2], req[3])))
    for _, t in reqs:
        srv.wait(t)
    for (s, lwe, acc, res), _ in reqs[:6]:
        v, N, n, bl, dg = sets[s]
        np.testing.assert_array_equal(res, oracle.blind_rotate(v, N, n, bl, dg, keys[s], lwe, acc, 1))
    srv.drain()
    srv.close()
    for r in rots:
        r.close()
