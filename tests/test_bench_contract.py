"""bench.py's output contract, on CPU: the reference arm (the PyTorch-CPU
FP64 port of the reference algorithm) prints one JSON line with the same
metric, unit and direction as the GPU arm, its own CPU baseline and a zero
host<->device byte count; and the workload description says whether the
inputs exceed L2."""
import contextlib
import io
import json
from types import SimpleNamespace

import bench


def test_reference_arm_json_line():
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        rc = bench.main(["--impl", "reference", "--steps", "1", "--warmup", "0", "--workload", "tgv32"])
    assert rc in (0, None)
    lines = [l for l in buf.getvalue().splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "Mcell-stages/s"
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"] and cb["cores"] >= 1
    assert cb["kind"] in ("port", "reference") and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("tgv32")


def test_l2_note_follows_the_workload_size():
    args = SimpleNamespace(n=128, precision="f32", seed=0, workload="tgv32")
    small = SimpleNamespace(name="tgv32", qs=[None], interior_cells=32 ** 3, padded_cells=36 ** 3,
                            cfg=SimpleNamespace(ghost=2))
    assert "not flushed" in bench.workload_desc(small, args)["l2"]
    args.workload = "wavy4"
    big = SimpleNamespace(name="wavy4", qs=[None] * 4, interior_cells=4 * 128 ** 3, padded_cells=4 * 132 ** 3,
                          cfg=SimpleNamespace(ghost=2))
    assert "larger than L2" in bench.workload_desc(big, args)["l2"]
