"""The benchmark's CPU-side pieces: the reference arm's JSON line (the oracle
port timed on the host cores), the roofline arithmetic and the per-sample
work model fed by the oracle's counters."""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402
import oracle as O  # noqa: E402
from zigtrace_b200 import scenes, workmodel  # noqa: E402


def _run_reference(extra_env=None):
    env = dict(os.environ, **(extra_env or {}))
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "cornell",
                           "--steps", "1", "--warmup", "0", "--cpu-seconds", "1"],
                          capture_output=True, text=True, timeout=600, env=env, cwd=str(ROOT))


def test_reference_arm_prints_one_contract_line():
    r = _run_reference()
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "Msamples/s" and d["unit"] == "Msamples/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 0
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "Msamples/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]


def test_reference_arm_never_loads_the_product_library():
    """The reference arm times the oracle only: the product's shared library
    must not even be mapped into its process."""
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'cornell', "
            "'--steps', '1', '--warmup', '0', '--cpu-seconds', '1']; "
            "runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('PRODUCT_LIB_MAPPED' if 'libzt_b200' in maps else 'PRODUCT_LIB_ABSENT'); "
            "print('ORACLE_MAPPED' if 'libzt_oracle' in maps else 'ORACLE_ABSENT')")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    assert "PRODUCT_LIB_ABSENT" in r.stdout and "ORACLE_MAPPED" in r.stdout


def test_reference_arm_other_ranks_print_nothing():
    r = _run_reference({"RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_roofline_entry_arithmetic():
    work = {"flop": 600.0, "bytes": 2000.0, "ext_rays": 2.0, "shadow_rays": 0.5, "box_tests": 40.0,
            "prim_tests": 3.0}
    r = bench.roofline_entry(work, samples=10_000_000, kernel_ms=5.0, sms=148, traffic=123,
                             traffic_note="n", execution={"issue_active_pct": 1.0})
    peak = 148 * bench.FP64_LANES_PER_SM * 2 * bench.NOMINAL_SM_MHZ * 1e6 / 1e12
    assert r["bound"] == "fp64" and r["unit"] == "TFLOP/s"
    assert r["achieved"] == pytest.approx(600.0 * 1e7 / 5e-3 / 1e12, rel=1e-3)
    assert r["peak"] == pytest.approx(peak, abs=0.05)
    assert r["frac"] == pytest.approx(r["achieved"] / peak, rel=1e-2)
    assert r["traffic"] == 123 and r["ncu_execution"] == {"issue_active_pct": 1.0}
    assert r["memory"]["achieved_gbs"] == pytest.approx(2000.0 * 1e7 / 5e-3 / 1e9, rel=1e-3)
    assert r["per_sample"] == {"ext_rays": 2.0, "shadow_rays": 0.5, "box_tests": 40.0, "prim_tests": 3.0}


def test_roofline_with_single_precision_box_tests():
    """Fast traversal: box-test FLOP against the FP32 peak, the rest against
    FP64; frac is the time both need at peak over the kernel time."""
    work = {"flop": 600.0, "flop_f32": 480.0, "bytes": 2000.0, "box_tests": 40.0}
    r = bench.roofline_entry(work, samples=10_000_000, kernel_ms=5.0, sms=148, traffic=None, traffic_note="n",
                             execution=None)
    p64 = 148 * 64 * 2 * bench.NOMINAL_SM_MHZ * 1e6
    p32 = 148 * 128 * 2 * bench.NOMINAL_SM_MHZ * 1e6
    want = (120.0 * 1e7 / p64 + 480.0 * 1e7 / p32) / 5e-3
    assert r["bound"] == "fp64+fp32" and r["frac"] == pytest.approx(want, abs=1e-4)  # frac has 4 decimals
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"], rel=1e-2)  # frac = achieved / peak
    assert r["split"]["fp32_tflops"] == pytest.approx(480.0 * 1e7 / 5e-3 / 1e12, rel=1e-3)
    assert "flop_f32" not in r["per_sample"]


def test_work_model_from_oracle_counters():
    scene = scenes.cornell().build()
    os_ = O.OracleScene.from_scene(scene)
    pix = np.arange(0, 64 * 64, 7, dtype=np.uint64)
    _, st = os_.render_pixels(64, 64, 4, 16, pix, threads=2, stats=True)
    assert st["samples"] == len(pix) * 4
    w = workmodel.per_sample(st, 4)
    assert w["ext_rays"] >= 1.0 and w["shadow_rays"] > 0 and w["box_tests"] > 0
    expect = (workmodel.FLOP_SLAB * st["slab_tests"] + workmodel.FLOP_SPHERE * st["sphere_tests"] +
              workmodel.FLOP_TRIANGLE * st["tri_tests"] + workmodel.FLOP_PLANE * st["plane_tests"] +
              workmodel.FLOP_SHADE * st["hits"] + workmodel.FLOP_NEE * st["nee_samples"]) / st["samples"]
    assert w["flop"] == pytest.approx(expect)
    assert w["bytes"] > workmodel.BYTES_PIXEL / 4
    f = workmodel.per_sample(st, 4, fast=True)
    assert f["flop"] == w["flop"] and f["flop_f32"] == pytest.approx(workmodel.FLOP_SLAB * st["slab_tests"] / st["samples"])
    assert w["flop_f32"] == 0 and f["bytes"] < w["bytes"]


def test_wavefront_queue_bytes():
    st = {"samples": 100, "ext_rays": 157, "hits": 61, "shadow_rays": 33}
    b = workmodel.wavefront_queue_bytes(st, 4)
    want = (workmodel.WF_BYTES_SAMPLE + (workmodel.WF_BYTES_RAY * 157 + workmodel.WF_BYTES_HIT * 61 +
                                         workmodel.WF_BYTES_SHADOW * 33) / 100 + workmodel.BYTES_PIXEL / 4)
    assert b == pytest.approx(want)
    assert 700 < b < 1000  # the 1M-triangle workload's counters give about 830 bytes per sample


def test_native_stdout_writes_do_not_mix_with_the_json_line():
    """Libraries that write to descriptor 1 themselves (NCCL's version banner
    on rank 0) land on standard error; standard output carries the JSON line
    alone, and descriptor 1 is restored when main() returns."""
    code = ("import os, sys; sys.path.insert(0, '.'); import bench; "
            "bench.reference_arm = lambda args: (os.write(1, b'NCCL version banner\\n'), bench.emit({'metric': 'm'})); "
            "sys.argv = ['bench.py', '--impl', 'reference']; bench.main(); print('AFTER_MAIN')")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.splitlines() == ['{"metric": "m"}', "AFTER_MAIN"]
    assert "NCCL version banner" in r.stderr
