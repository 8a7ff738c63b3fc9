"""CPU checks of bench.py's measurement plumbing: the algorithmic-byte
formulas the roofline divides by, the lookups of the committed ncu traffic
and reference iteration counts, and the reference arm's JSON line (the
reference's own PdhgSolver::solve, compiled from source, on the host)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


class _Lp:
    nrow, ncol, nnz = 200000, 500000, 5005134


def test_algorithmic_bytes_of_the_fused_kernels():
    # unfused SpMV + update, as the profiles state them for C2
    assert bench.primal_bytes(_Lp, 8) == 95661612
    assert bench.dual_bytes(_Lp, 8) == 74461612
    assert bench.primal_bytes(_Lp, 4) == 58841076
    assert bench.dual_bytes(_Lp, 4) == 47641076
    # FP32 values with FP64 vectors: 8 bytes per nonzero streamed, vectors at 8
    assert bench.dual_bytes(_Lp, 8, 4) == bench.dual_bytes(_Lp, 8) - 4 * 5005134
    assert bench.primal_bytes(_Lp, 8, 4) == bench.primal_bytes(_Lp, 8) - 4 * 5005134
    # plain SpMV: (index + value) per nonzero, row pointers, x read, y written
    assert bench.spmv_bytes(_Lp, False, 4) == 8 * 5005134 + 4 * 200001 + 4 * 500000 + 4 * 200000
    assert bench.spmv_bytes_w(_Lp, False, 4, 8) == 8 * 5005134 + 4 * 200001 + 8 * 500000 + 8 * 200000


def test_committed_profile_lookups():
    # every fused iteration kernel the C2 line can name as dominant, in both layouts
    for fam in ("warp", "cta"):
        t = bench.committed_traffic(f"k_dual<double,double>[{fam}]:zipf_200000x500000_nnz5M")
        assert t is not None and 0.9 * 74461612 < t < 1.1 * 74461612
        t = bench.committed_traffic(f"k_primal<double,double>[{fam}]:zipf_200000x500000_nnz5M")
        assert t is not None and 0.8 * 95661612 < t < 1.1 * 95661612
    assert bench.committed_ref_iterations("random_eq_2000x5000_nnz40000") == (187424, False)
    n, lower = bench.committed_ref_iterations("zipf_200000x500000_nnz5M")
    assert n > 1_000_000 and lower
    assert bench.committed_traffic("no_such_kernel") is None


def test_workloads_name_the_configs():
    labels = {k: v["label"] for k, v in bench.WORKLOADS.items()}
    assert set(labels) == {"c1", "c2", "c3", "c4", "c5"}
    assert labels["c2"] == "zipf_200000x500000_nnz5M"


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_nirnaya.so")),
                    reason="oracle/_ref not built from the reference sources")
def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "c1",
                          "--steps", "1", "--warmup", "0", "--cpu-seconds", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "s" and line["higher_is_better"] is False
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["lower_bound"] in (True, False) and line["per_iteration_s"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and "PdhgSolver::solve" in cb["sample"]
    assert set(cb["iterations_per_s_by_threads"]) >= {"1"}


def _bench_line(tmp_path, *args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args, "--mps-dir", str(tmp_path)],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_mps_read_mode_line(tmp_path):
    line = _bench_line(tmp_path, "--mps-read", "--workload", "c1", "--steps", "2", "--warmup", "1")
    assert line["metric"] == "mps_read_throughput" and line["unit"] == "MB/s" and line["value"] > 0
    assert line["config"]["workload"] == "random_eq_2000x5000_nnz40000.mps" and line["config"]["nnz"] == 40000
    assert set(line["seconds_by_threads"]) >= {"1"}
    if line["reference"] is not None:
        assert line["reference"]["models_bit_identical"] is True


def test_host_path_mode_line(tmp_path):
    line = _bench_line(tmp_path, "--host-path", "--workload", "c1")
    assert line["metric"] == "host_path_seconds" and line["higher_is_better"] is False
    assert set(line["seconds"]) == {"read", "presolve", "scale", "verify", "write_sol"}
    if line["reference"] is not None:
        ref = line["reference"]
        assert ref["scaled_model_bit_identical"] and ref["verification_bit_identical"] and ref["sol_bytes_identical"]


def test_verify_batch_mode_is_wired_and_needs_a_gpu():
    """--verify-batch (the device check on the batch) is a bench.py mode;
    its device legs run on a GPU only."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0 and "--verify-batch" in out.stdout
    import bench

    assert callable(bench.verify_batch_bench)
