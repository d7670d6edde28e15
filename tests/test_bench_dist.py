"""The multi-GPU bench path's cross-rank logic on CPU (gloo, 2 ranks): every
rank sees the slowest rank's time, and the job's throughput is all ranks'
units over that time; the reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_ranks_time_by_the_slowest_and_sum_units():
    port = str(_free_port())
    procs = [subprocess.Popen([sys.executable, os.path.join(HERE, "_bench_rank.py"), str(r), "2",
                               port], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
             for r in range(2)]
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["slowest"] == 5.0            # rank 1 took 5 s, rank 0 took 3 s
        assert o["value"] == 2 * 1000 / 5.0   # 2 ranks x 1000 units in 5 s


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        workload, steps, warmup = "ntt64", 1, 3
    assert bench.run_reference(Args(), 1, 2) is None
    assert capsys.readouterr().out == ""


def test_reference_arm_line_keeps_the_contract(capsys):
    """Rank 0 of the reference arm prints one JSON line with the contract's keys."""
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        workload, steps, warmup = "ntt64", 1, 3
    bench.run_reference(Args(), 0, 1)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC
    assert line["unit"] == "polys/s" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["n_gpus"] == 1 and line["steps"] == 1 and line["warmup"] >= 3
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert cb["host"]["nproc"] >= 1 and cb["host"]["model"]
    assert line["e2e"] == {"value": line["value"], "unit": "polys/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_secondary_summary_is_short_and_names_the_metric_figures():
    """The JSON line's `secondary` holds the figures the metric names, flat,
    and stays short enough for a log tail (the full detail goes to a file)."""
    sys.path.insert(0, ROOT)
    import bench
    rate = {"p99_ms": 1.0, "commits_per_s": 10.0, "req_per_s": 20.0}
    detail = {
        "commit": {"commits_per_s": 4e6, "commits_per_s_graph": 8e6, "per_call_commits_per_s": 1e5,
                   "e2e_commits_per_s": 9e5,
                   "cpu_oracle_commits_per_s": {"threads_1": 7e3, "threads_all": 9e4}},
        "round": {"round_ms_p50": 0.7, "round_ms_p99": 0.8, "e2e_round_ms_p50": 1.5,
                  "cpu_oracle_round_ms": {"threads_1": 18000.0, "threads_all": 2000.0}},
        "batch": {"batched_commits_per_s": 1.5e6, "per_call_commits_per_s": 2e4,
                  "batched_ms_p50": 2.7},
        "ntt256": {"polys_per_s": 7.8e8, "frac": 0.36},
        "ntt64_transforms": {"forward": {"frac": 0.8}, "inverse": {"frac": 0.8}},
        "ring_round": {"round_ms_p50": 2.0},
        "serve": {"commits_per_s_ratio": 8.8, "saturated_req_per_s_ratio": 3.0,
                  "saturated": {"continuous": rate, "plain": rate},
                  "rates": {str(k): {"continuous": rate, "plain": rate}
                            for k in (1000, 5000, 50000)}},
    }
    out = bench.secondary_summary(detail)
    for key in ("round_ms_p50", "round_ms_p99", "served_commits_per_s_ratio",
                "served_req_per_s_ratio", "config0_commits_per_s", "config3_commits_per_s"):
        assert out[key] is not None, key
    assert len(json.dumps(out)) < 2000
