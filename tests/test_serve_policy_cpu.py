"""The serving loop's choice of blocks per rotation (csrc/serve_policy.h), on the CPU:
four for small launches that fit on the SMs left free, two when the two-block kernel holds
the launch, else one; and the blocks a launch keeps busy."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def policy():
    out_dir = ROOT / "tests" / "_build"  # git-ignored build folder
    out_dir.mkdir(exist_ok=True)
    exe = out_dir / "serve_policy_driver"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'fhetoothpaste_b200' / 'csrc'}",
                    str(ROOT / "tests" / "cpp" / "serve_policy_driver.cpp"), "-o", str(exe)], check=True)

    def run(lines):
        res = subprocess.run([str(exe)], input="\n".join(lines) + "\n", capture_output=True, text=True, check=True)
        return [int(x) for x in res.stdout.split()]
    return run


# (take, busy blocks, SMs, four-block capacity, two-block capacity) -> blocks per rotation
SPLIT_CASES = [
    ((1, 0, 148, 32, 74), 4),      # light load: one request on an idle device
    ((8, 0, 148, 32, 74), 4),      # the largest four-block launch
    ((9, 0, 148, 32, 74), 2),      # above it: two blocks
    ((8, 116, 148, 32, 74), 4),    # 116 + 32 = 148 blocks: still fits
    ((8, 117, 148, 32, 74), 2),    # one block over: two blocks
    ((1, 148, 148, 32, 74), 2),    # busy device
    ((3, 0, 148, 0, 74), 2),       # the set's four-block kernel does not fit (capacity 0)
    ((5, 0, 148, 4, 74), 2),       # more requests than four-block clusters fit at once
    ((74, 0, 148, 32, 74), 2),     # a full two-block wave
    ((75, 0, 148, 32, 74), 1),     # beyond it: one block per rotation
    ((3, 0, 148, 32, 0), 4),       # no two-block kernel, four-block fits
    ((20, 0, 148, 32, 0), 1),      # neither holds it
]


def test_serving_split_policy(policy):
    got = policy([f"split {' '.join(map(str, args))}" for args, _ in SPLIT_CASES])
    assert got == [want for _, want in SPLIT_CASES]


def test_serving_blocks_in_flight(policy):
    cases = [((4, 3, 32), 12), ((2, 100, 74), 148), ((1, 4096, 148), 148), ((1, 5, 0), 1), ((4, 8, 32), 32)]
    got = policy([f"blocks {' '.join(map(str, args))}" for args, _ in cases])
    assert got == [want for _, want in cases]
