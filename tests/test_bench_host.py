"""bench.py's host-side pieces that need no GPU: the clock record taken
beside the timed region (median SM clock, the throttle reasons that reject a
run), the profiled DRAM traffic read from the committed ncu summary and
scaled by the state size, and the latency percentiles of the serving run."""
import os

import bench


class _Done:
    def terminate(self):
        pass

    def wait(self):
        pass


def clock_record(lines):
    c = bench.Clocks(0)
    c.f = open(c.path, "w")
    c.f.write("".join(line + "\n" for line in lines))
    c.f.flush()
    c.proc = _Done()
    rec = c.stop()
    assert not os.path.exists(c.path)  # the record is removed once read
    return rec


def test_clocks_median_and_power_cap():
    rec = clock_record([
        "0, 1882, 1965, 990.1, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1875, 1965, 995.0, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1890, 1965, 998.2, 0x0, Not Active, Not Active, Not Active, Not Active",
    ])
    assert rec["sm_mhz"] == 1882 and rec["sm_max_mhz"] == 1965 and rec["samples"] == 3
    assert rec["reasons"] == ["sw_power_cap"]


def test_clocks_report_the_reasons_that_reject_a_run():
    rec = clock_record([
        "0, 1200, 1965, 700.0, 0x48, Active, Not Active, Active, Not Active",
        "garbage line",
        "0, N/A, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ])
    assert rec["sm_mhz"] == 1200 and rec["samples"] == 1
    assert rec["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]


def test_clocks_without_nvidia_smi():
    c = bench.Clocks(0)
    c.proc = None
    assert c.stop()["reasons"] == ["nvidia-smi unavailable"]


def test_profiled_traffic_scales_with_the_state():
    t30 = bench.profiled_traffic(30)
    assert t30 is not None and t30 > 2 * (16 << 30) * 0.9
    assert abs(bench.profiled_traffic(28) * 4 - t30) <= 4


def test_percentile():
    assert bench.percentile([], 50) is None
    xs = [5, 1, 4, 2, 3]
    assert bench.percentile(xs, 0) == 1 and bench.percentile(xs, 50) == 3 and bench.percentile(xs, 100) == 5


def _run_reference(env_extra):
    import json
    import subprocess
    import sys
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, os.path.join(os.path.dirname(bench.__file__), "bench.py"), "--impl",
                        "reference", "--qubits", "16", "--steps", "1", "--warmup", "3", "--no-reference-gpu"],
                       capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    return lines


def test_reference_arm_line(ref):
    """The reference arm on the host cores (oracle/_ref): one JSON line with
    the contract's keys; its e2e moves no bytes."""
    (line,) = _run_reference({})
    assert line["impl"] == "reference" and line["unit"] == "circuits/s" and line["value"] > 0
    assert line["higher_is_better"] is True and line["n_gpus"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "circuits/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_do_no_work(ref):
    assert _run_reference({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []
