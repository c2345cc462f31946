"""Keys stored in key files and uploaded to GPU contexts rotate / switch exactly like keys uploaded
from memory; a file whose header does not match the context is refused."""
import numpy as np
import pytest

from brcases import case_inputs, case_key

pytestmark = pytest.mark.gpu


def test_rotation_key_from_file(native, oracle, golden, cuda, tmp_path):
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator, TpError
    from fhetoothpaste_b200 import _native as nat
    from fhetoothpaste_b200.keyfile import write_key_file
    name = "cfg1_binary_n1024"
    case = golden[0]["br"][name]
    _, _, brk = case_key(oracle, name, case)
    path = tmp_path / "cfg1.tpkey"
    write_key_file(path, "blind_rotation", brk, ring_dim=case["N"], lwe_dim=case["n"], digits=case["digits"],
                   basis=1 << case["basis_log2"], variant=case["variant"])
    rot = GpuBlindRotator.from_key_file(path)
    lwes, accs, coefs = case_inputs(name, case)
    idx = [i for i, c in enumerate(coefs) if c == 0]
    np.testing.assert_array_equal(rot.blind_rotate_batch_host(lwes[idx], accs[idx]), golden[1][f"br_{name}"][idx])
    # same key, context with another LWE dimension: refused before any upload
    with pytest.raises(TpError) as ei:
        GpuBlindRotator(BlindRotationContext(case["variant"], case["N"], case["n"] - 2, 1 << case["basis_log2"],
                                             case["digits"]), None, key_file=path)
    assert ei.value.status == nat.TP_ERR_LAYOUT


def test_lwe_switch_key_from_file(native, oracle, cuda, tmp_path):
    from fhetoothpaste_b200 import GpuLWEtoLWEConverter
    from fhetoothpaste_b200.keyfile import write_key_file
    from oracle.oracle import P, random_acc, rlwe_secret, lwe_secret
    N, n, beta, digits, batch = 512, 40, 16, 4, 9
    ksk = oracle.lwe_ks_keygen(P, N, n, beta, digits, 3.2, rlwe_secret(N, 1), lwe_secret(0, n, N, 2), 3)
    path = tmp_path / "ks.tpkey"
    write_key_file(path, "lwe_switch", ksk, ring_dim=N, lwe_dim=n, digits=digits, basis=1 << beta)
    mem = GpuLWEtoLWEConverter(N, n, 1 << beta, digits, ksk)
    fil = GpuLWEtoLWEConverter(N, n, 1 << beta, digits, None, key_file=path)
    rl = cuda.from_numpy(random_acc(N, batch, 4).view(np.int64)).cuda()
    outs = []
    for conv in (mem, fil):
        o = cuda.empty((batch, n + 1), dtype=cuda.int64, device="cuda")
        conv.pbs_epilogue_batch(batch, o.data_ptr(), rl.data_ptr(), 2 * N)
        outs.append(o.cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])
