"""bench.py's mesh workload on CPU: the reference arm runs the reference's own
hmvm_omp_2 on the ppohBEM matrix of a mesh, and vs_baseline is looked up only
for the reference's published matrices at their own size and precision."""
import json
import os
import subprocess
import sys
from types import SimpleNamespace

import pytest

from helpers import ROOT, SAMPLE_PBF


@pytest.mark.skipif(not os.path.exists(SAMPLE_PBF), reason="the reference's sample mesh is not present")
def test_reference_arm_on_mesh():
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--mesh", SAMPLE_PBF,
                        "--steps", "3", "--warmup", "1"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "HMVM/s"
    cfg = line["config"]
    assert cfg["mesh"] == "input_sample.pbf" and cfg["n"] == 600 and cfg["nlf"] == 1426
    assert "input_sample.pbf" in line["data"] and "fits the 126 MB L2" in cfg["l2"]


def test_published_lookup():
    sys.path.insert(0, ROOT)
    import bench

    hm = SimpleNamespace(nd=600)
    a = SimpleNamespace(mesh="/any/where/input_sample.pbf", nrhs=1, precision="fp64")
    assert bench.published_hmvm_per_s(a, hm) == pytest.approx(1 / 1.920e-5)
    a.precision = "fp32"
    assert bench.published_hmvm_per_s(a, hm) == pytest.approx(1 / 1.674e-5)
    assert bench.published_hmvm_per_s(SimpleNamespace(mesh=a.mesh, nrhs=1, precision="mixed"), hm) is None
    assert bench.published_hmvm_per_s(SimpleNamespace(mesh=a.mesh, nrhs=8, precision="fp64"), hm) is None
    assert bench.published_hmvm_per_s(a, SimpleNamespace(nd=601)) is None  # not the published matrix
    big = SimpleNamespace(mesh="input_216h.pbf", nrhs=1, precision="fp64")
    assert bench.published_hmvm_per_s(big, SimpleNamespace(nd=21600)) == pytest.approx(1 / 1.002e-3)
    assert bench.published_hmvm_per_s(SimpleNamespace(mesh=None, nrhs=1, precision="fp64"), hm) is None


def test_traffic_ratios_from_committed_profiles():
    """The roofline's traffic field scales the DRAM-bytes ratios that the
    committed ncu summaries carry; both single-vector kernels have them."""
    sys.path.insert(0, ROOT)
    import bench

    for prec in ("fp64", "mixed"):
        for stage in (1, 2):
            r = bench.traffic_ratio(stage, prec)
            assert r is not None and 1.0 <= r < 1.2, (prec, stage, r)
    assert bench.traffic_ratio(2, "fp32") is None
