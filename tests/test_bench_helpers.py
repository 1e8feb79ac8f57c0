"""bench.py's host-side helpers (no GPU): the roofline denominator comes from
the measured peaks file, the ncu traffic from the committed profile summary,
algorithmic bytes follow B = B_fmt + 8 n + 16 m, and the clock sampler's
parse keeps only the throttle reasons nvidia-smi reports Active."""
import json
import os

import bench


def test_peak_is_the_measured_copy_bandwidth():
    p = os.path.join(bench.ROOT, "MEASURED_PEAKS.json")
    if not os.path.exists(p):  # the file is written per machine; without it the stated fallback
        assert bench.hbm_peak() == (bench.FALLBACK_HBM_GBS, "fallback")
        return
    with open(p) as f:
        want = float(json.load(f)["hbm_gbs"])
    assert bench.hbm_peak() == (want, "measured")


def test_ncu_traffic_comes_from_the_committed_summary():
    t = bench.ncu_traffic_per_launch("reference", bench.DEFAULT_N)
    assert t is not None and t > 0
    assert bench.ncu_traffic_per_launch("reference", bench.DEFAULT_N // 2) is None  # other sizes: not captured


def test_algorithmic_bytes():
    assert bench.algorithmic_bytes({"format_bytes": 1000}, m=3, n=5) == 1000 + 8 * 5 + 16 * 3


class _FakeSmi:
    def __init__(self, text):
        self.text = text

    def terminate(self):
        pass

    def communicate(self, timeout=None):
        return self.text, ""


def test_clock_sampler_parse():
    rows = [
        "0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1800, 1965, 990.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1700, 1965, 999.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "garbage line",
    ]
    cs = object.__new__(bench.ClockSampler)
    cs.proc = _FakeSmi("\n".join(rows) + "\n")
    cs.idx = 0
    got = cs.stop()
    assert got == {"sm_mhz": 1800.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    cs.proc = None
    assert cs.stop() is None


def test_block_kernel_lines_parse():
    text = ("Bitmap SpMV type: \x1b[1;33mBITMAP TEMP\x1b[0m\n"
            "Block nonzeros = \x1b[0;36m   1\x1b[0m, MFLOP/s: min = \x1b[1;32m    425.55\x1b[0m, avg = \x1b[1;32m"
            "    430.74\x1b[0m, max = \x1b[1;32m    436.60\x1b[0m; y-vector sum: \x1b[0;31m4.697620400000000e+09\x1b[0m\n"
            "Block nonzeros =    2, MFLOP/s: min =     767.85, avg =     822.91, max =     861.93; "
            "y-vector sum: 7.381974950000000e+09\n")
    got = bench.block_kernel_lines(text)
    assert [g["bnnz"] for g in got] == [1, 2]
    assert got[0] == {"bnnz": 1, "mflops_min": 425.55, "mflops_avg": 430.74, "mflops_max": 436.6,
                      "y_sum": 4.6976204e9}
    assert bench.block_kernel_lines("") == []


def test_ingest_leg_keeps_stdout_to_the_json_line():
    """The ingest leg times abhsf_read_mtx and, where it is built, the
    reference's reader on the same sample file; they read the same elements,
    and the reference reader's log does not reach stdout (which carries only
    the bench's JSON line)."""
    import subprocess
    import sys
    code = ("import sys, json; sys.path.insert(0, %r)\n"
            "import bench\n"
            "from abhsf_b200 import workloads as W\n"
            "r = bench.ingest_run(W.tiled_mixture(n=65536), 20000)\n"
            "print(json.dumps(r))\n") % bench.ROOT
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = p.stdout.strip().splitlines()
    assert len(lines) == 1
    r = json.loads(lines[0])
    assert r["entries"] > 0 and r["abhsf_read_mtx"]["MB/s"] > 0
    ref = r["reference_reader"]
    assert "unavailable" in ref or ref["same_elements"] is True
