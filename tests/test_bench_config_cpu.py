"""bench.py's two arms print the same workload ``config``, which the reference
line is compared on. The tests below check the reference arm's line on a small
Cartesian block through the CPU oracle against the config the GPU arm builds
for the same arguments. They also check the one-block-per-GPU layout that the
curvilinear two-block workload takes at even process counts. No GPU is
needed."""
import json
import os
import subprocess
import sys
from types import SimpleNamespace

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_gpu_arm_config():
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = "2"
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "cartesian", "--n", "25",
                        "--steps", "1", "--warmup", "0"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["steps"] >= 1
    import bench
    args = SimpleNamespace(workload="cartesian", n=25, dist_backend="nccl")
    p, name = bench.make_problem(args, 3)
    expect = bench.workload_config(args, name, sum(b.npoints for b in p.blocks), len(p.blocks), 1)
    assert line["config"] == expect
    assert line["cpu_baseline"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0


def test_config_names_the_process_layout():
    import bench
    args = SimpleNamespace(workload="hill", n=None, dist_backend="nccl")
    one = bench.workload_config(args, "w", 100, 2, 1)
    assert one["parallelism"] == "replicas1" and one["points"] == 100 and one["blocks"] == 2
    four = bench.workload_config(args, "w", 100, 2, 4)
    assert four["parallelism"] == "blocks2x2" and four["copies"] == 2 and four["points_per_copy"] == 100
    three = bench.workload_config(args, "w", 100, 2, 3)
    assert three["parallelism"] == "replicas3"
