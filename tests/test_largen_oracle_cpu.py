"""Ring sizes above 4096 on the CPU: the C oracle (oracle/tp_oracle.c) regenerates the keys of
tests/golden/largen.json (made by the reference library, tests/golden/make_largen_golden.py)
word for word and reproduces the reference's rotations (SHA-256 of every output), so the GPU
tests at those sizes can compare against the oracle directly."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import lwe_secret, rlwe_secret, sha256

GOLDEN = Path(__file__).resolve().parent / "golden" / "largen.json"
CASES = json.loads(GOLDEN.read_text())["br"]


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_at_large_ring_sizes(oracle, name):
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    from make_golden import br_inputs
    c = CASES[name]
    N, n, v = c["N"], c["n"], c["variant"]
    lk, rk = lwe_secret(v, n, N, c["seed"] + 10), rlwe_secret(N, c["seed"] + 11)
    brk = oracle.br_keygen(v, N, n, c["basis_log2"], c["digits"], c["std"], lk, rk, c["key_seed"])
    assert sha256(brk) == c["key_sha256"]
    lwes, accs, coefs = br_inputs(name, N, n, c["seed"])
    assert sha256(lwes) == c["lwe_sha256"] and sha256(accs) == c["acc_sha256"]
    for i, oc in enumerate(coefs):
        out = oracle.blind_rotate(v, N, n, c["basis_log2"], c["digits"], brk, lwes[i], accs[i], oc)
        assert sha256(np.ascontiguousarray(out)) == c["out_sha256"][i], (name, i)


KS_CASES = json.loads(GOLDEN.read_text())["ks"]


@pytest.mark.parametrize("name", sorted(KS_CASES))
def test_oracle_key_switching_matches_reference_at_large_ring_sizes(oracle, name):
    """RLWE key switches, automorphisms and packings at N = 8192 .. 32768: the oracle's keys
    and results hash to the reference's."""
    from kscases import ks_inputs, ks_key
    c = KS_CASES[name]
    N, bl, dg = c["N"], c["basis_log2"], c["digits"]
    key = ks_key(oracle, name, c)
    x = ks_inputs(c)
    if c["kind"] == "rlwe_ks":
        got = [oracle.rlwe_ks(N, bl, dg, key, x[i]) for i in range(2)]
    elif c["kind"] == "auto":
        got = [oracle.auto_eval(N, bl, dg, c["index"], key, x[i]) for i in range(2)]
    else:
        got = [oracle.pack(N, bl, dg, key, x, c["len"])]
    assert [sha256(np.ascontiguousarray(g)) for g in got] == c["out_sha256"], name
