"""Host helpers of bench.py on CPU: the defaults the benchmark contract asks
for, the lattice option, and the roofline denominators."""
import json
import os
import subprocess
import sys
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_defaults_are_one_gpu_and_three_warmup_steps():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True,
                         text=True, check=True).stdout
    assert "--gpus" in out and "--steps" in out and "--warmup" in out and "--impl" in out
    src = open(os.path.join(ROOT, "bench.py")).read()
    assert 'ap.add_argument("--gpus", type=int, default=1)' in src
    assert 'ap.add_argument("--warmup", type=int, default=3)' in src   # W >= 3


def test_lattice_option_overrides_the_workload_default():
    assert bench.lattice_of(types.SimpleNamespace(lattice=None), "32,32,32,64") == (32, 32, 32, 64)
    assert bench.lattice_of(types.SimpleNamespace(lattice="8,8,8,16"), "32,32,32,64") == (8, 8, 8, 16)


def test_peak_is_the_measured_copy_bandwidth_else_the_fallback(tmp_path, monkeypatch):
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6547.8}))
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.peaks() == (6547.8, "measured")
    monkeypatch.setattr(bench, "ROOT", str(tmp_path / "absent"))
    assert bench.peaks() == (6650.0, "fallback")
    assert bench.NOMINAL_HBM_GBS == 7700.0
