"""Shared-memory plans of the rotation kernels (br_kernels.cuh, br_pair_kernel.cuh) on the
CPU: every plan the library builds fits one SM's 227 KB with a 1023-word LWE; the four-block
kernel is built for every set but BMMP at N = 4096, and only ternary N = 4096 needs the
single NTT exchange buffer. Host code only (nvcc builds it; no kernel runs)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIMIT_WORDS = 227 * 1024 // 8


@pytest.fixture(scope="module")
def driver_output():
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not on PATH")
    out_dir = ROOT / "tests" / "_build"  # git-ignored build folder
    out_dir.mkdir(exist_ok=True)
    exe = out_dir / "smem_plan_driver"
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O1",
                    f"-I{ROOT / 'include'}", f"-I{ROOT / 'fhetoothpaste_b200' / 'csrc'}",
                    str(ROOT / "tests" / "cpp" / "smem_plan_driver.cu"), "-o", str(exe)], check=True)
    return subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines()


@pytest.fixture(scope="module")
def plans(driver_output):
    rows = {}
    for line in driver_output:
        if line.startswith("C "):
            continue
        logn, v, one, pair, qfits, quad, qxb, ppf, qpf = map(int, line.split())
        rows[(logn, v)] = dict(one=one, pair=pair, quad_fits=qfits, quad=quad, quad_xbufs=qxb)
    assert len(rows) == 18
    return rows


@pytest.fixture(scope="module")
def cluster_plans(driver_output):
    rows = {}
    for line in driver_output:
        if line.startswith("C "):
            logn, v, logs, one, ks = map(int, line.split()[1:])
            rows[(logn, v)] = dict(logs=logs, one=one, ks=ks)
    assert len(rows) == 12
    return rows


def test_every_built_plan_fits_one_sm(plans):
    for (logn, v), r in plans.items():
        assert r["one"] <= LIMIT_WORDS, (logn, v)
        assert r["pair"] <= LIMIT_WORDS, (logn, v)
        if r["quad_fits"]:
            assert r["quad"] <= LIMIT_WORDS, (logn, v)


def test_four_block_kernel_sets(plans):
    refused = {k for k, r in plans.items() if not r["quad_fits"]}
    assert refused == {(12, 2)}
    single = {k for k, r in plans.items() if r["quad_fits"] and r["quad_xbufs"] == 1}
    assert single == {(12, 1)}


def test_cluster_plans(cluster_plans):
    """Rings above 4096: 2, 4, 8, 16 CTAs of 4096 coefficients for N = 8192 .. 65536, and every
    per-CTA plan (rotation with a 1023-word LWE, key switching) fits one SM."""
    for (logn, v), r in cluster_plans.items():
        assert r["logs"] == logn - 12, (logn, v)
        assert r["one"] <= LIMIT_WORDS, (logn, v)
        assert r["ks"] <= LIMIT_WORDS, (logn, v)
