"""The reference arm of bench.py (`--impl reference`) on the host: one JSON line
with the contract's keys and the GPU arm's config, the reference's own CPU path
(its DoFManager, CGAssembly, DirichletBC, sparse_csr and pcg_solve) reaching a
1e-10 relative residual on a whole smaller cube of the workload, scaled to the
configured size by its measured phases, with no part of the yafel_b200 library
loaded (no GPU needed)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    env = dict(os.environ, OMP_NUM_THREADS="2")
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1",
                          "--ref-nx", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "dofs/s"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    assert d["config"] == bench_config()
    assert 1e-12 <= d["sample"]["relres_min"] and d["sample"]["relres_max"] <= 1e-10
    smp = d["sample"]
    assert smp["ran"] == "3^3 Q2 hex, full pipeline, converged" and smp["dofs"] == 3 * 7 ** 3
    # the value is the configured size's dofs over the scaled phases of the sample
    est = smp["setup_s"] * smp["scale_elements"] + smp["solve_s"] * smp["scale_entries"] * smp["scale_iterations"]
    assert abs(d["value"] - d["config"]["dofs"] / est) <= 1e-9 * d["value"]
    assert smp["scale_elements"] == 8000.0 and smp["scale_iterations"] == 20.0
    assert abs(smp["scale_entries"] - (481 / 25) ** 3) < 1e-9


def bench_config():
    sys.path.insert(0, ROOT)
    import bench
    return bench.base_config(60, 1)


def test_reference_arm_loads_no_library_of_the_product():
    code = ("import sys, bench; bench.cpu_sample(2, 2, 1e-20); "
            "m = open('/proc/self/maps').read(); "
            "sys.exit(3 if 'libyafel_b200' in m else (0 if 'libyafel_ref' in m else 4))")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300,
                         env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert out.returncode == 0, (out.returncode, out.stderr[-2000:])
