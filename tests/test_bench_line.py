"""bench.py's host-side logic, without a GPU (the measurements are
stand-ins):

- the JSON line assembled from the measurements: the contract's keys with
  their types and units, the whole-job value over N GPUs, the roofline against
  the given peak, and the claims (Dirac roofline, the FP64 arm, mixed over
  FP64) at the end of the line, where a log tail keeps them;
- the clock summary from the sampler's CSV: only the timed region's samples,
  and the throttle reasons seen there.
"""
import json
import sys
from pathlib import Path
from types import SimpleNamespace

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402

CONTRACT = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
            "vs_baseline", "dtype", "data", "config", "clocks", "gpu_launches", "e2e", "cpu_baseline", "roofline")


def _inputs(world):
    a = SimpleNamespace(steps=5, warmup=3, md_steps=10, eps=0.05, tol=1e-10)
    out = [{"inner_iterations": 13500, "reliable_updates": 210, "accepted": 1, "dH": 0.01, "cg_iterations": 13300}
           for _ in range(5)]
    clocks = {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": []}
    results = {"mixed": {"ms": 5 * 62.5, "out": out, "clocks": clocks, "launches": 87.0},
               "fp64": {"ms": 5 * 97.0, "out": out, "clocks": clocks, "launches": 60.0}}
    roof = {"gbs": 2800.0, "kernel": "cg_mixed_duo_kernel", "note": "310 inner iterations", "traffic": 6790400}
    peaks = {"hbm_gbs": 6424.4, "src": "measured"}
    cpu = {"value": 0.013, "unit": "traj/s", "cores": 1, "kind": "reference", "sample": "one trajectory"}
    detail = {"batched": {"value": 396.0, "solver_gbs": 4100.0},
              "serving_sharded": {"n_gpus": world, "offered_req_per_s": 100.0 * world,
                                  "throughput_req_per_s": 95.0 * world, "p50_ms": 110.0, "p99_ms": 800.0}}
    return a, world, 64, 64 ** 3, results, 5 * 63.0 / 1000.0, roof, {"gbs": 4850.0}, peaks, cpu, detail


def test_line_keys_units_and_order():
    args = _inputs(1)
    line = bench.bench_line(*args)
    for k in CONTRACT:
        assert k in line, k
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["higher_is_better"] is True and line["scaling"] == "weak" and line["vs_baseline"] is None
    assert abs(line["value"] - 5 / 0.3125) < 1e-12 and abs(line["ms_per_step"] - 62.5) < 1e-12
    assert line["gpu_launches"] == 435 and isinstance(line["gpu_launches"], int)
    e2e = line["e2e"]
    assert abs(e2e["value"] - 5 / 0.315) < 1e-12 and e2e["unit"] == bench.UNIT
    assert e2e["h2d_bytes_per_step"] == 3 * 64 ** 3 * 8 and e2e["d2h_bytes_per_step"] == 2 * 64 ** 3 * 8
    r = line["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["peak"] == 6424.4
    assert abs(r["frac"] - 2800.0 / 6424.4) < 1e-15 and r["traffic"] == 6790400
    assert "workload" in line["config"] and "L=64" in line["config"]["workload"]
    # the claims close the line
    assert list(line)[-3:] == ["dirac_roofline", "fp64", "mixed_over_fp64"]
    assert abs(line["mixed_over_fp64"] - round((5 / 0.3125) / (5 / 0.485), 3)) < 1e-12
    assert abs(line["dirac_roofline"]["frac"] - round(4850.0 / 6424.4, 3)) < 1e-12
    json.loads(json.dumps(line))  # plain JSON


def test_line_over_gpus():
    args = _inputs(4)
    line = bench.bench_line(*args)
    assert line["n_gpus"] == 4 and line["config"]["parallelism"] == "replicas x4"
    assert abs(line["value"] - 4 * 5 / 0.3125) < 1e-12  # the whole job's trajectories per second
    assert abs(line["e2e"]["value"] - 4 * 5 / 0.315) < 1e-12
    assert line["serving"]["n_gpus"] == 4 and line["serving"]["done_req_per_s"] == 380.0
    assert line["batched"]["fp64_traj_s"] is None  # the FP64 chains run on one GPU only


class _FakeSampler:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def test_clock_summary_counts_the_timed_region_only(tmp_path):
    """The clock sampler reports the median SM clock, the maximum and the
    throttle reasons seen after mark() (the timed region), not before."""
    c = bench.Clocks(0)
    c.path = str(tmp_path / "clocks.csv")
    c.fh = open(c.path, "w")
    c.proc = _FakeSampler()
    warm = "0, 1200, 1965, 300.0, 0x1, Active, Not Active, Not Active, Not Active\n"  # hw_slowdown before timing
    c.fh.write(warm * 3)
    c.mark()
    rows = ["0, 1965, 1965, 900.5, 0x4, Not Active, Not Active, Not Active, Active\n",
            "0, 1950, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active\n",
            "0, 1965, 1965, 950.0, 0x0, Not Active, Not Active, Not Active, Not Active\n",
            "garbled line\n"]
    c.fh.writelines(rows)
    got = c.stop()
    assert got == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3,
                   "power_w_max": 990.0}


def test_clock_summary_without_sampler():
    assert bench.Clocks(0).stop()["reasons"] == ["nvidia-smi unavailable"]
