"""Host logic of the warp row-block layout (nirnaya_b200/csrc/row_blocks.hpp).

The iteration kernels index a per-warp shared slice of kWarpCapMax (256)
products by the block descriptors, so a malformed list is a memory-safety
bug, not just a wrong answer. These tests build the layout on the CPU
through a small harness: single LPs and block-diagonal batches of uneven
instances (empty rows, instances without rows, rows longer than the block
capacity) must satisfy the invariants, match a Python restatement of the
greedy packing, and a corrupted list must be rejected before upload.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "nirnaya_b200", "csrc")
CUDA_INC = os.environ.get("CUDA_HOME", "/usr/local/cuda") + "/include"

CAP_MAX, ROWS_MAX = 256, 32


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("rb") / "row_blocks_harness")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", CSRC, "-I", CUDA_INC,
                    os.path.join(ROOT, "tests", "native", "row_blocks_harness.cpp"), "-o", exe], check=True)
    return exe


def run(exe, rp, off, cap, corrupt=None):
    words = [cap, len(off) - 1, len(rp) - 1, *rp, *off]
    words += [0] if corrupt is None else [1, corrupt]
    out = subprocess.run([exe], input=" ".join(map(str, words)), capture_output=True, text=True, check=True).stdout
    lines = dict(line.split(" ", 1) if " " in line else (line, "") for line in out.strip().splitlines())
    if "error" in lines:
        return lines["error"]
    ints = {k: [int(v) for v in s.split()] for k, s in lines.items()}
    blk = np.array(ints["blocks"]).reshape(-1, 2)
    return blk, ints["owner"], ints["lo"]


def greedy(rp, cap):
    """Python restatement: consecutive rows while their nonzeros fit `cap`
    and at most 32 rows; a row longer than `cap` alone."""
    rows = len(rp) - 1
    out, s = [], 0
    while s < rows:
        r = s + 1
        if rp[s + 1] - rp[s] <= cap:
            while r < rows and rp[r + 1] - rp[s] <= cap and r - s < ROWS_MAX:
                r += 1
        out.append(s)
        s = r
    return out


def check_invariants(blk, owner, lo, rp, off, cap):
    rows = len(rp) - 1
    assert blk[0, 0] == 0 and blk[-1, 0] == rows and blk[-1, 1] == rp[rows]
    for k in range(len(owner)):
        r0, p0 = blk[k]
        r1, p1 = blk[k + 1]
        assert r0 < r1 and p0 == rp[r0] and p1 == rp[r1]
        assert r1 - r0 == 1 or (p1 - p0 <= cap and r1 - r0 <= ROWS_MAX)
        i = owner[k]
        assert off[i] <= r0 and r1 <= off[i + 1], "a block crosses an instance"
        assert lo[i] <= k < lo[i + 1]


def random_batch(rng, count, cap):
    lens, off = [], [0]
    for i in range(count):
        nr = 0 if i % 5 == 3 else int(rng.integers(1, 200))
        ln = rng.integers(0, 12, size=nr)
        if nr:
            ln[rng.integers(0, nr)] = int(rng.integers(cap + 1, 3 * cap + 2))  # one long row
            if nr > 2:
                ln[-1] = int(rng.integers(cap + 1, 2 * cap + 2))  # a long row last
        lens.extend(ln.tolist())
        off.append(off[-1] + nr)
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(int).tolist()
    return rp, off


@pytest.mark.parametrize("cap", [32, 64, 128, 256])
def test_batch_layout_invariants_and_restatement(harness, cap):
    rng = np.random.default_rng(cap)
    for trial in range(5):
        rp, off = random_batch(rng, 1 + 4 * trial, cap)
        blk, owner, lo = run(harness, rp, off, cap)
        check_invariants(blk, owner, lo, rp, off, cap)
        want = []
        for i in range(len(off) - 1):
            seg = rp[off[i]:off[i + 1] + 1]
            want += [off[i] + s for s in greedy(seg, cap)] if off[i + 1] > off[i] else []
        assert blk[:-1, 0].tolist() == want


def test_single_lp_and_empty_layouts(harness):
    rp = [0, 3, 3, 300, 301]
    blk, owner, lo = run(harness, rp, [0, 4], 64)
    check_invariants(blk, owner, lo, rp, [0, 4], 64)
    assert blk[:, 0].tolist() == [0, 2, 3, 4]
    # an orientation without rows: one empty block
    blk, owner, lo = run(harness, [0], [0, 0, 0], 64)
    assert blk.tolist() == [[0, 0], [0, 0]] and owner == [] and lo == [0, 0, 0]


def test_second_instance_starts_at_its_own_nonzero(harness):
    # the first block of every instance after the first starts at that
    # instance's first nonzero, not at zero
    rp = [0, 300, 305, 310, 600]
    off = [0, 1, 4]
    blk, owner, lo = run(harness, rp, off, 32)
    check_invariants(blk, owner, lo, rp, off, 32)
    assert blk[lo[1]].tolist() == [1, 300]


def test_corrupted_descriptor_is_rejected(harness):
    rp, off = random_batch(np.random.default_rng(1), 4, 32)
    for k in (1, 2):
        msg = run(harness, rp, off, 32, corrupt=k)
        assert isinstance(msg, str) and "internal" in msg
    assert "capacity" in run(harness, [0, 10, 20], [0, 2], 0)

