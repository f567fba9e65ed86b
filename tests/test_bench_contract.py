"""bench.py's reference arm runs on the host alone: its JSON line carries the keys the
benchmark contract asks for (the GPU arm is exercised on the GPU)."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1"], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


class _RecordingFixer:
    """Stands in for GaugeFixer: records the launch-shape calls an autotuner code turns into."""

    def __init__(self):
        self.calls = []

    def set_pass_shape(self, real, variant, warps):
        self.calls.append(("shape", real, variant, warps))

    def set_pass_order(self, real, alternate, capped=False):
        self.calls.append(("order", real, bool(alternate), bool(capped)))

    def set_pass_stages(self, real, stages):
        self.calls.append(("stages", real, stages))


def test_autotuner_codes_map_to_launch_shapes():
    """gf_autotune's output codes (variant code + 1000 alternating walk + 10000 capped + 100000 three
    cp.async stages) set the same shape again through the setters, and name the kernel they stand for."""
    sys.path.insert(0, str(ROOT))
    import bench

    cases = {
        0: [("shape", "fp32", 0, 4), ("order", "fp32", False, False)],
        11116: [("shape", "fp32", 7, 4), ("order", "fp32", True, True)],
        1004: [("shape", "fp64", 1, 4), ("order", "fp64", True, False)],
        101004: [("shape", "fp64", 1, 4), ("order", "fp64", True, False), ("stages", "fp64", 3)],
        1100: [("shape", "fp32", 3, 4), ("order", "fp32", True, False)],
        8: [("shape", "fp64", 1, 8), ("order", "fp64", False, False)],
    }
    for code, want in cases.items():
        real = want[0][1]
        gf = _RecordingFixer()
        bench.apply_pass_code(gf, real, code)
        assert gf.calls == want, code
    assert "pair_rp" in bench.pass_kernel_name(11116, "fp32", True)
    assert "registers capped" in bench.pass_kernel_name(11116, "fp32", True)
    assert "three cp.async stages" in bench.pass_kernel_name(101004, "fp64", False)
    assert "k_batched_pass_staged<double" in bench.pass_kernel_name(101004, "fp64", False)
