"""Benchmark: 3D linear elasticity on the unit cube, 60^3 Q2 hexahedra
(1,771,561 nodes, 5,314,683 dofs), E=1, nu=0.3, 3x3x3 Gauss-Legendre, clamped
at x=0, uniform traction (1,0,0) on x=1, FP64 3x3-block BCSR, Jacobi-PCG to a
1e-10 relative residual -- assembled and solved on one B200 per rank.

One step = GPU assembly of the tangent (pattern expansion + element kernels),
Dirichlet conditions, the traction load, and the solve to 1e-10 (relative
residual recomputed in FP64).  The DoF numbering (host, once per mesh) is set-up
and outside the step.  metric = dofs solved per second, whole job.

Timing: CUDA events on the library's stream, W untimed warm-up steps, K timed
steps bracketed by a barrier and synchronisation, max over ranks.  The matrix
(8.5 GB) is far larger than L2, so no flush is needed.  --gpus N runs N
independent replicas (the path does not shard): weak scaling, no collectives on
the data path.  --impl reference times the reference's CPU path instead.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = 60
E, NU = 1.0, 0.3
TOL = 1e-10
METRIC = "dofs solved/sec to 1e-10 (3D Q2 elasticity, Jacobi-PCG, FP64 BCSR3)"
WORKLOAD = "elasticity_q2_hex_60^3_jacobi_pcg_1e-10"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device):
        self.device, self.samples, self.proc = device, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(s[0]) for s in self.samples if len(s) >= 8 and s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if len(s) >= 8 and s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            if len(s) >= 8:
                for k, nm in enumerate(names):
                    if s[4 + k].lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def problem(nx):
    from yafel_b200 import meshgen
    return meshgen.structured_hex(nx, nx, nx, order="ccw")


def bcsr3_spmv_bytes(nnzb, n):
    """Algorithmic bytes of one FP64 BCSR 3x3 SpMV: values + block columns +
    row pointer + x read once + y written once."""
    nbrows = n // 3
    return nnzb * (8 * 9 + 4) + 4 * (nbrows + 1) + 8 * n + 8 * n


def bcsr3_spmv32_bytes(nnzb, n):
    """Algorithmic bytes of one corrected FP32-value BCSR 3x3 SpMV as the
    mixed-precision solvers run it: FP32 values + block columns + row pointer +
    the FP32 node-padded x read once (16 B a node) + y written once + the FP64
    row-sum correction (72 B a block row) + the row's own FP64 x (24 B)."""
    nbrows = n // 3
    return nnzb * (4 * 9 + 4) + 4 * (nbrows + 1) + 16 * nbrows + 8 * n + 72 * nbrows + 8 * n


TMA_CFG = {32: "64,3,4", 1: "32,4,8", 2: "32,3,8", 4: "32,2,8", 8: "32,3,12", 16: "48,3,8"}
ROW_CFG = {1: "128,2,4", 2: "128,3,4", 4: "64,2,8", 8: "64,3,8"}


def spmv_kernel_name(K, dot=1, vt="double"):
    variant, lanes = K.get_spmv(0 if vt == "double" else 1)
    if variant == 2:
        cfg = TMA_CFG.get(lanes, "64,3,4")
        xf = ",true" if vt == "float" else ",false"
        return "k_bcsr_spmv_tma<3,%s,%d,TmaCfg<3,%s,%s>%s>" % (vt, dot, vt, cfg, xf)
    if variant == 4:
        xf = ",true" if vt == "float" else ",false"
        return "k_bcsr_spmv_rows<3,%s,%d,RowCfg<3,%s,%s>%s>" % (vt, dot, vt, ROW_CFG.get(lanes, "128,2,4"), xf)
    if variant == 1:
        return "k_bcsr_spmv_staged<3,%s,%d>" % (vt, dot)
    return "k_bcsr_spmv<3,%d,%s,%d>" % (lanes, vt, dot)


def run_spmv_profile(args):
    """SpMV alone on the nx^3 Q2 elasticity matrix (BCSR3) or, with
    `--spmv-matrix poisson`, the nx^3 Q2 Poisson matrix (CSR, 27-125 entries a
    row), GPU-assembled, for roofline and ncu captures: FP64 then FP32 values,
    `--reps` launches each."""
    import yafel_b200 as yb
    poisson = args.spmv_matrix == "poisson"
    dpn = 1 if poisson else 3
    dm = yb.DoFManager(problem(args.nx), 2, dpn)
    fe = yb.FESystem(dm, 3, format=yb.CSR if poisson else yb.BCSR)
    phys = yb.PoissonEquation(3, f=0.0) if poisson else yb.LinearElasticity(3, E=E, nu=NU)
    yb.CGAssembly(phys, fe, [yb.AssemblyRequirement.Tangent])
    K = fe.getGlobalTangent()
    if args.variant is not None:
        K.set_spmv(args.variant, args.lanes)
    else:
        K.make_fp32()
        K.set_spmv(-1)  # the device autotuner, FP64 and FP32 values, as a solve runs it
    n = K.rows()
    x = yb.DeviceVector(np.random.default_rng(0).standard_normal(n), dm.ctx)
    if poisson:
        nnz = K.nnz()
        v, L = K.get_spmv()
        out = {"mesh": "%d^3 Q2 hex, Poisson" % args.nx, "dofs": n, "nnz": nnz,
               "kernel": "k_bcsr_spmv<1,%d,double,0>" % L if v == 0 else "variant %d lanes %d" % (v, L)}
        cases = ((0, "fp64", nnz * 12 + 4 * (n + 1) + 16 * n), (1, "fp32_values", nnz * 8 + 4 * (n + 1) + 16 * n))
    else:
        nnzb = K.nnz() // 9
        out = {"mesh": "%d^3 Q2 hex" % args.nx, "dofs": n, "blocks": nnzb, "kernel": spmv_kernel_name(K, 0),
               "kernel_fp32": spmv_kernel_name(K, 0, "float"), "tuned": {"fp64": K.get_spmv(0), "fp32": K.get_spmv(1)}}
        cases = ((0, "fp64", bcsr3_spmv_bytes(nnzb, n)), (3, "fp32_values", bcsr3_spmv32_bytes(nnzb, n)))
    for prec, name, nbytes in cases:
        if args.spmv_precision != "both" and name.split("_")[0] != args.spmv_precision:
            continue
        ms = K.spmv_bench(reps=args.reps, precision=prec, x=x)
        out[name] = {"ms": ms, "bytes": nbytes, "GB_s": nbytes / ms / 1e6}
    print(json.dumps(out), flush=True)


def run_gpu(args):
    import yafel_b200 as yb
    from yafel_b200 import loads
    from yafel_b200.replicas import Replicas
    rep = Replicas("nccl")
    ws, rank, local = rep.ws, rep.rank, rep.local
    ctx = yb.Context(local if ws > 1 else 0)
    lib = yb.lib()
    mesh = problem(args.nx)
    t0 = time.time()
    dm = yb.DoFManager(mesh, 2, 3, ctx=ctx)
    t_dof = time.time() - t0
    X = dm.dof_nodes
    clamp = np.nonzero(np.abs(X[:, 0]) < 1e-9)[0]
    traction = loads.hex_face_traction(dm, lambda Y: np.abs(Y[:, 0] - 1.0) < 1e-9, (1.0, 0.0, 0.0))
    phys = yb.LinearElasticity(3, E=E, nu=NU, body=(0.0, 0.0, 0.0))
    ndofs = dm.ndofs
    bcs = []
    for c in range(3):
        bc = yb.DirichletBC(dm, 0.0, c)
        bc.bc_nodes = clamp.astype(np.int64)
        bcs.append(bc)
    trac_dev = yb.DeviceVector(traction, ctx)

    phases = {"assemble": [], "bc": [], "solve": []}

    def step(precision, profile=False, record=False):
        t0 = time.perf_counter()
        fe = yb.FESystem(dm, 3, format=yb.BCSR)
        yb.CGAssembly(phys, fe)
        K, F = fe.getGlobalTangent(), fe.getGlobalResidual()
        F.axpy(1.0, trac_dev)
        for prec, pin in ((yb.PREC_FP64, args.spmv), (yb.PREC_MIXED, args.spmv32)):
            if pin:  # pinned kernels (a profiler distorts the autotuner's timings)
                K.set_spmv_for(prec, *[int(v) for v in pin.split(":")])
        ctx.synchronize()
        t1 = time.perf_counter()
        for bc in bcs:
            bc.apply(K, F)
        M = yb.JacobiPreconditioner(K)
        ctx.synchronize()
        t2 = time.perf_counter()
        x, st = yb.solve(K, F, M=M, tol=TOL, precision=precision, profile=profile)
        t3 = time.perf_counter()
        if record:
            phases["assemble"].append(t1 - t0)
            phases["bc"].append(t2 - t1)
            phases["solve"].append(t3 - t2)
        return K, x, st

    def timed(precision, steps, warmup, profile=False):
        for _ in range(warmup):
            step(precision)
        ctx.synchronize()
        rep.barrier()
        launches0 = ctx.launches
        ev = [C.c_void_p(), C.c_void_p()]
        t0 = time.perf_counter()
        stats = []
        for _ in range(steps):
            K, x, st = step(precision, profile, record=(precision == 0))
            stats.append(st)
        ctx.synchronize()
        wall = time.perf_counter() - t0
        return wall, stats, ctx.launches - launches0, K, x

    clocks = Clocks(local if ws > 1 else 0)
    # device time: each solve reports its own CUDA-event time; assembly + BC are
    # timed with host synchronisation around the step (the step ends in a sync)
    clocks.start()
    wall64, st64, launches, K, x = timed(0, args.steps, args.warmup, profile=True)
    clk = clocks.stop()
    wallmx, stmx, _, Kmx, _ = timed(1, args.steps, max(1, args.warmup // 3), profile=True)
    wallir, stir, _, _, _ = timed(2, 1, 0)
    step_s = rep.max(wall64 / args.steps)
    value = rep.job_rate(ndofs, step_s)
    # e2e: through the public API from host buffers every step: DoF numbering +
    # upload, assembly, BCs, host load vector upload, solve, solution download.
    e2e_steps = max(1, min(args.steps, 2))
    h2d = d2h = 0
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        dme = yb.DoFManager(mesh, 2, 3, ctx=ctx)
        fe = yb.FESystem(dme, 3, format=yb.BCSR)
        yb.CGAssembly(phys, fe)
        Kx, Fx = fe.getGlobalTangent(), fe.getGlobalResidual()
        Fx.axpy(1.0, yb.DeviceVector(traction, ctx))
        for c in range(3):
            bc = yb.DirichletBC(dme, 0.0, c)
            bc.bc_nodes = clamp.astype(np.int64)
            bc.apply(Kx, Fx)
        xe, ste = yb.solve(Kx, Fx, M=yb.JacobiPreconditioner(Kx), tol=TOL)
        sol = xe.numpy()
        # mesh arrays, the numbered nodes and element lists the DoFManager uploads,
        # the traction vector and the BC lists (counted, not read back)
        h2d = mesh["nodes"].nbytes + mesh["cell_nodes"].nbytes + mesh["offsets"].nbytes + \
            mesh["cell_types"].nbytes + traction.nbytes + 3 * clamp.size * 16 + \
            24 * dme.nNodes() + 4 * dme._n_el
        d2h = sol.nbytes
    e2e_s = rep.max((time.perf_counter() - t0) / e2e_steps)
    # roofline of the dominant kernel (BCSR3 SpMV inside the PCG iterations)
    rp, col, _ = None, None, None
    nnzb = K.nnz() // 9
    assert nnzb == base_config(args.nx, ws)["blocks"], nnzb
    spmv_bytes = bcsr3_spmv_bytes(nnzb, ndofs)
    spmv_ms = sum(s.spmv_ms for s in st64) / max(1, sum(s.spmv_launches for s in st64))
    spmv32_ms = sum(s.spmv_ms for s in stmx) / max(1, sum(s.spmv_launches for s in stmx))
    spmv32_bytes = bcsr3_spmv32_bytes(nnzb, ndofs)
    kname = spmv_kernel_name(K)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = spmv_bytes / (spmv_ms * 1e-3) / 1e9 if spmv_ms > 0 else None
    # DRAM bytes (read + write) of one launch of this kernel on the 60^3 matrix,
    # measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum)
    traffic = 8.729e9 if args.nx == 60 else None
    iters64 = statistics.mean(s.iterations for s in st64)
    itersmx = statistics.mean(s.iterations for s in stmx)
    mixed_step = wallmx / args.steps
    out = {
        "metric": METRIC, "value": value, "unit": "dofs/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (structured mesh, seeded nothing random)",
        "config": base_config(args.nx, ws),
        "matrix": {"nnz": K.nnz(), "blocks": nnzb, "dof_numbering": "set-up, outside the device step; inside e2e"},
        "e2e": {"value": ws * ndofs / e2e_s, "unit": "dofs/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "includes": "DoF numbering, uploads, assembly, solve, download"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "kernel": kname, "bytes_per_launch": spmv_bytes,
                     "ms_per_launch": spmv_ms, "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback",
                     "spmv_choice": {"fp64": list(K.get_spmv(0)), "fp32": list(Kmx.get_spmv(1))},
                     "fp32_values_kernel_GBs": spmv32_bytes / (spmv32_ms * 1e-3) / 1e9 if spmv32_ms > 0 else None},
        "solver": {"fp64_iterations": iters64, "fp64_relres": max(s.rel_residual for s in st64),
                   "mixed_iterations": itersmx, "mixed_relres": max(s.rel_residual for s in stmx),
                   "mixed_refinements": statistics.mean(s.refinements for s in stmx),
                   "fp64_step_ms": step_s * 1e3, "mixed_step_ms": mixed_step * 1e3,
                   "mixed_dofs_per_s": ws * ndofs / mixed_step, "mixed_speedup": step_s / mixed_step,
                   "solve_ms": statistics.mean(s.device_ms for s in st64),
                   "mixed_ir_iterations": stir[0].iterations, "mixed_ir_step_ms": wallir * 1e3,
                   "mixed_ir_relres": stir[0].rel_residual},
        "phases_ms": {k: 1e3 * statistics.mean(v) for k, v in phases.items() if v},
        "setup": {"dof_numbering_s": t_dof},
        "clocks": clk,
    }
    if ws == 1 and not args.no_extra:
        out["assembly"] = run_assembly(ctx, dm, phys, args.nx)
        out["small_poisson64"] = run_small_poisson(ctx)
        out["q3_30cubed"] = run_q3(ctx)
        out["ilu0_vs_jacobi_30cubed"] = run_ilu(ctx)
        out["gradient_recovery"] = run_gradient(ctx, dm, x, args.nx)
    if ws == 1 and not args.no_side_workloads:
        # configurations 4 and 5 (batched and served solves), one timed pass each
        del K, Kmx, x
        out["batch512"] = run_batch(args, side=True)
        out["serve"] = run_serve(args, side=True)
    if rank == 0 and not args.no_cpu_baseline and ws == 1:
        out["cpu_baseline"] = cpu_baseline(args)
    if rank == 0:
        print(json.dumps(out), flush=True)
    rep.close()


def run_small_poisson(ctx, reps=30):
    """64x64 Q1 Poisson on the unit square (4225 dofs, f=1, u=0 on the whole
    boundary, 2x2 Gauss-Legendre, FP64 CSR, Jacobi-PCG to 1e-10).  The system
    is L2-resident, so it reports latency and solves/s rather than a roofline:
    one solve = assembly + Dirichlet + Jacobi + solve, the DoF numbering done
    once.  Returns the summary dict."""
    import yafel_b200 as yb
    from yafel_b200 import meshgen
    mesh = meshgen.structured_quad(64, 64, order=meshgen.corner_order(1))
    dm = yb.DoFManager(mesh, 1, 1, ctx=ctx)
    bc = yb.DirichletBC(dm, 0.0, 0)
    bc.selectByFunction(lambda X: (X[:, 0] < 1e-9) | (X[:, 0] > 1 - 1e-9) | (X[:, 1] < 1e-9) | (X[:, 1] > 1 - 1e-9))
    phys = yb.PoissonEquation(2, f=1.0)

    def one():
        fe = yb.FESystem(dm, 2, format=yb.CSR)
        yb.CGAssembly(phys, fe)
        K, F = fe.getGlobalTangent(), fe.getGlobalResidual()
        bc.apply(K, F)
        x, st = yb.solve(K, F, M=yb.JacobiPreconditioner(K), tol=TOL)
        return K, x, st

    for _ in range(3):
        one()
    lat, solve_ms = [], []
    for _ in range(reps):
        ctx.synchronize()
        t0 = time.perf_counter()
        K, x, st = one()
        ctx.synchronize()
        lat.append(time.perf_counter() - t0)
        solve_ms.append(st.device_ms)
    lat.sort()
    return {"workload": "poisson_q1_quad_64x64_jacobi_pcg_1e-10", "dofs": dm.ndofs, "nnz": K.nnz(),
            "iterations": st.iterations, "relres": st.rel_residual, "status": st.status,
            "latency_ms_p50": 1e3 * lat[len(lat) // 2], "latency_ms_p99": 1e3 * lat[min(len(lat) - 1, int(0.99 * len(lat)))],
            "solve_device_ms_p50": sorted(solve_ms)[len(solve_ms) // 2], "solves_per_s": len(lat) / sum(lat),
            "l2": "L2-resident (%.2f MB): latency, not a roofline" % ((K.nnz() * 12 + dm.ndofs * 40) / 1e6),
            "cpu": cpu_small_poisson(mesh)}


def cpu_small_poisson(mesh, reps=5):
    """The same 64x64 Q1 Poisson solve in the reference's own code on the host
    (oracle/_ref): CGAssembly (all cores), DirichletBC::apply on the boundary
    nodes, sparse_csr(triplets) and pcg_solve with its Jacobi preconditioner
    (TOL 1e-21 on the squared preconditioned ratio).  Median latency over
    `reps` solves, DoF numbering outside the timed region as on the device."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    rd = O.RefDofManager(mesh, 1, 1)
    X = rd.nodes
    bnd = np.nonzero((X[:, 0] < 1e-9) | (X[:, 0] > 1 - 1e-9) | (X[:, 1] < 1e-9) | (X[:, 1] > 1 - 1e-9))[0]
    lat, rel = [], None
    for _ in range(reps):
        t0 = time.perf_counter()
        rs = O.RefSystem(rd, 2, O.POISSON, [1.0, 1.0], threads=os.cpu_count() or 1)
        rs.dirichlet_nodes(0, bnd, 0.0)
        A, b = rs.to_ref_csr()
        x = A.pcg_jacobi(b, np.zeros(b.size), 1e-21)
        lat.append(time.perf_counter() - t0)
        rel = A.true_relres(b, x)
    lat.sort()
    return {"latency_ms_p50": 1e3 * lat[len(lat) // 2], "relres": rel, "kind": "reference",
            "cores": os.cpu_count() or 1,
            "sample": "%d solves in the reference's own code: CGAssembly, DirichletBC, sparse_csr, "
                      "pcg_solve/Jacobi" % reps}


def run_q3(ctx, nx=30, steps=2):
    """3D elasticity, 30^3 Q3 hexes (2,260,713 dofs), clamp x=0, traction
    (1,0,0) on x=1, BCSR3, Jacobi-PCG to 1e-10 in FP64 and in mixed precision
    (FP32 matrix values, FP64 vectors, reductions and true-residual
    replacement).  Reports dofs/s of assemble+solve for each and the relative
    difference of the mixed solution from the FP64 one."""
    import yafel_b200 as yb
    from yafel_b200 import loads, meshgen
    mesh = meshgen.structured_hex(nx, nx, nx, order=meshgen.corner_order(3))
    dm = yb.DoFManager(mesh, 3, 3, ctx=ctx)
    X = dm.dof_nodes
    clamp = np.nonzero(np.abs(X[:, 0]) < 1e-9)[0].astype(np.int64)
    trac = yb.DeviceVector(loads.hex_face_traction(dm, lambda Y: np.abs(Y[:, 0] - 1.0) < 1e-9, (1.0, 0.0, 0.0)), ctx)
    phys = yb.LinearElasticity(3, E=E, nu=NU)
    out = {"workload": "elasticity_q3_hex_%d^3_jacobi_pcg_1e-10" % nx, "dofs": dm.ndofs}
    sol = {}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        times, st = [], None
        for k in range(steps + 1):
            ctx.synchronize()
            t0 = time.perf_counter()
            fe = yb.FESystem(dm, 3, format=yb.BCSR)
            yb.CGAssembly(phys, fe)
            K, F = fe.getGlobalTangent(), fe.getGlobalResidual()
            F.axpy(1.0, trac)
            for c in range(3):
                bc = yb.DirichletBC(dm, 0.0, c)
                bc.bc_nodes = clamp
                bc.apply(K, F)
            x, st = yb.solve(K, F, M=yb.JacobiPreconditioner(K), tol=TOL, precision=prec)
            ctx.synchronize()
            if k > 0:
                times.append(time.perf_counter() - t0)
        sol[name] = x.numpy()
        t = statistics.mean(times)
        out[name] = {"s_per_solve": t, "dofs_per_s": dm.ndofs / t, "iterations": st.iterations,
                     "relres": st.rel_residual, "status": st.status, "refinements": st.refinements}
        out["blocks"] = K.nnz() // 9
        del K, F, fe, x
    out["mixed_speedup"] = out["fp64"]["s_per_solve"] / out["mixed"]["s_per_solve"]
    out["mixed_rel_diff_vs_fp64"] = float(np.linalg.norm(sol["mixed"] - sol["fp64"]) / np.linalg.norm(sol["fp64"]))
    return out


def assembly_flops_per_element(nq, nen, dpn, nsd):
    """Algorithmic flops of the element-local B^T D B product per element:
    2 nq (s^2 n + s n^2) with s = 3 (2D) or 6 (3D) strain components and
    n = nen * dpn element dofs."""
    s = 3 if nsd == 2 else 6
    n = nen * dpn
    return 2 * nq * (s * s * n + s * n * n)


def assembly_executed_flops_per_element(nq, nen, nsd):
    """Flops k_assemble executes per 3D elasticity element: per quadrature point
    the Jacobian (nen*nsd^2 multiply-adds) and its inverse (~60), the physical
    gradients (nen*nsd^2 multiply-adds), and per node pair of the upper triangle
    (nen(nen+1)/2) and point the dot product (6) and the scaled weight (1) plus
    8 flops for each of the nsd^2 block entries."""
    geometry = nq * (2 * nen * nsd * nsd + 60) + nq * nen * 2 * nsd * nsd
    pairs = nen * (nen + 1) // 2
    return geometry + pairs * nq * (7 + 8 * nsd * nsd)


def assembly_scatter_bytes_per_element(nen, dpn):
    """Bytes the element scatter moves per element: every one of its nen^2 node
    blocks (dpn^2 FP64 values) read and written once."""
    return nen * nen * dpn * dpn * 8 * 2


def fp64_peak_tflops():
    """FP64 dense rate measured here: torch float64 8192^3 matmul (cuBLAS DGEMM),
    best of 5, CUDA events; None without torch CUDA."""
    try:
        import torch
        if not torch.cuda.is_available():
            return None
        a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
        b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
        torch.matmul(a, b)
        best = 1e30
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        torch.cuda.empty_cache()
        return 2 * 8192 ** 3 / (best * 1e-3) / 1e12
    except Exception:
        return None


def run_assembly(ctx, dm, phys, nx, reps=5):
    """Element kernels alone: re-assembly of the tangent's values on an existing
    pattern (CGAssembly on an FESystem that already holds K), wall time with the
    device synchronised on both sides, against the algorithmic B^T D B flops of
    the Q2 hexes (27 Gauss points, 27 nodes, 3 dofs per node)."""
    import yafel_b200 as yb
    fe = yb.FESystem(dm, 3, format=yb.BCSR)
    yb.CGAssembly(phys, fe, [yb.AssemblyRequirement.Tangent])
    ts = []
    for _ in range(reps):
        ctx.synchronize()
        t0 = time.perf_counter()
        yb.CGAssembly(phys, fe, [yb.AssemblyRequirement.Tangent])
        ctx.synchronize()
        ts.append(time.perf_counter() - t0)
    t = min(ts)
    ne = nx ** 3
    flops = assembly_flops_per_element(27, 27, 3, 3) * ne
    executed = assembly_executed_flops_per_element(27, 27, 3) * ne
    scatter = assembly_scatter_bytes_per_element(27, 3) * ne
    peak = fp64_peak_tflops()
    achieved = flops / t / 1e12
    return {"elements": ne, "ms": t * 1e3, "algorithmic_flops": flops, "achieved_TFLOPs": achieved,
            "executed_flops": executed, "executed_TFLOPs": executed / t / 1e12,
            "scatter_bytes": scatter, "scatter_GBs": scatter / t / 1e9,
            "fp64_dgemm_TFLOPs_measured": peak, "frac_of_dgemm": (achieved / peak) if peak else None,
            "executed_frac_of_dgemm": (executed / t / 1e12 / peak) if peak else None,
            "note": "algorithmic = the B^T D B count; executed = what k_assemble does (node pairs of the upper "
                    "triangle, 79 flops per pair and point, plus geometry); scatter = read-modify-write of every "
                    "element block into the value array"}


def run_ilu(ctx, nx=30):
    """ILU(0)-PCG beside Jacobi-PCG on the nx^3 Q2 elasticity problem (the
    reference's ILUPreconditioner on the scalar pattern, level-scheduled
    triangular solves): set-up (factorisation) and solve times, iterations."""
    import yafel_b200 as yb
    from yafel_b200 import loads
    dm = yb.DoFManager(problem(nx), 2, 3, ctx=ctx)
    X = dm.dof_nodes
    clamp = np.nonzero(np.abs(X[:, 0]) < 1e-9)[0].astype(np.int64)
    trac = yb.DeviceVector(loads.hex_face_traction(dm, lambda Y: np.abs(Y[:, 0] - 1.0) < 1e-9, (1.0, 0.0, 0.0)), ctx)
    fe = yb.FESystem(dm, 3, format=yb.BCSR)
    yb.CGAssembly(yb.LinearElasticity(3, E=E, nu=NU), fe)
    K, F = fe.getGlobalTangent(), fe.getGlobalResidual()
    F.axpy(1.0, trac)
    for c in range(3):
        bc = yb.DirichletBC(dm, 0.0, c)
        bc.bc_nodes = clamp
        bc.apply(K, F)
    out = {"workload": "elasticity_q2_hex_%d^3_pcg_1e-10" % nx, "dofs": dm.ndofs}
    for name, cls in (("jacobi", yb.JacobiPreconditioner), ("ilu0", yb.ILUPreconditioner)):
        ctx.synchronize()
        t0 = time.perf_counter()
        M = cls(K)
        ctx.synchronize()
        t1 = time.perf_counter()
        x, st = yb.solve(K, F, M=M, tol=TOL)
        ctx.synchronize()
        t2 = time.perf_counter()
        out[name] = {"setup_s": t1 - t0, "solve_s": t2 - t1, "iterations": st.iterations,
                     "relres": st.rel_residual, "status": st.status}
        if name == "ilu0":
            lo, up = M.levels
            out[name]["levels_forward_backward"] = [lo, up]
            out[name]["ms_per_iteration"] = 1e3 * (t2 - t1) / max(1, st.iterations)
        del M, x
    return out


def run_gradient(ctx, dm, x, nx, reps=5):
    """Gradient recovery on the benchmark's solution: LocalSmoothingGradient of
    the 60^3 Q2 elasticity displacement (nodal 3x3 gradients), and ZZ patch
    recovery of a smooth scalar field on a Q1 hex mesh of the same cell count
    (ZZ takes p = 1 scalar fields); device-synchronised wall time, best of reps."""
    import yafel_b200 as yb
    out = {}
    fe = yb.FESystem(dm, 3, format=yb.BCSR)
    fe.getSolution().axpy(1.0, x)
    ts = []
    for _ in range(reps):
        ctx.synchronize()
        t0 = time.perf_counter()
        yb.LocalSmoothingGradient(yb.LinearElasticity(3, E=E, nu=NU), fe)
        ctx.synchronize()
        ts.append(time.perf_counter() - t0)
    out["local_smoothing_q2_%dcubed" % nx] = {"cells": nx ** 3, "dofs": dm.ndofs, "ms": 1e3 * min(ts),
                                              "dofs_per_s": dm.ndofs / min(ts)}
    dm1 = yb.DoFManager(problem(nx), 1, 1, ctx=ctx)
    X = dm1.dof_nodes
    fe1 = yb.FESystem(dm1, 3)
    fe1.getSolution().upload(np.sin(2 * X[:, 0]) * np.cos(X[:, 1]) + X[:, 2] ** 2)
    ts = []
    for _ in range(reps):
        ctx.synchronize()
        t0 = time.perf_counter()
        yb.ZZGradientRecovery(yb.PoissonEquation(3), fe1)
        ctx.synchronize()
        ts.append(time.perf_counter() - t0)
    out["zz_q1_%dcubed" % nx] = {"cells": nx ** 3, "nodes": dm1.ndofs, "ms": 1e3 * min(ts),
                                 "nodes_per_s": dm1.ndofs / min(ts)}
    return out


BATCH_METRIC = "solves/sec to 1e-10 (batched 2D Poisson/elasticity, mixed precision)"


def run_batch(args, side=False):
    """Batched solves: `--problems` seeded 2D Poisson / plane elasticity problems
    (sizes log-uniform 1e3..2e5 dofs, orders 1-3, jittered tri+quad meshes, RHS
    N(0,1), u = 0 on x = 0), assembled once and held on the device.  One step
    solves all of them from x = 0 to a 1e-10 relative residual: batched in
    mixed precision (the value), batched in FP64, and one by one with the plain
    FP64 Jacobi-PCG (yg_cg) for comparison.  Wall time with the device
    synchronised on both sides (the batch loop is host-driven between graph
    replays, so device and wall time coincide up to the replay gaps).
    side=True: one warm-up and one timed step of each form, returned as an
    object of the default benchmark line instead of printed."""
    import yafel_b200 as yb
    from yafel_b200 import workloads
    ctx = yb.Context(0)
    steps, warmup = (1, 1) if side else (args.steps, args.warmup)
    specs = [workloads.problem_spec(i) for i in range(args.problems)]
    t0 = time.perf_counter()
    probs = [workloads.assemble(s, ctx) for s in specs]
    ctx.synchronize()
    t_setup = time.perf_counter() - t0
    Ks = [p[1] for p in probs]
    bs = [p[2] for p in probs]
    hb = [b.numpy() for b in bs]
    ndofs = [K.rows() for K in Ks]
    total = sum(ndofs)
    P = len(Ks)

    def sequential():
        sts = []
        for K, b in zip(Ks, bs):
            x, st = yb.solve(K, b, M=yb.JacobiPreconditioner(K), tol=TOL)
            sts.append(st)
        ctx.synchronize()
        return sts

    def make_batch(precision):
        B = yb.Batch(P, ctx)
        if args.solo_spmv_mb is not None:
            B.set_solo_bytes(int(args.solo_spmv_mb * 2 ** 20))
        xs = []
        for K, b, n in zip(Ks, bs, ndofs):
            x = yb.DeviceVector(n, ctx)
            x.fill(0.0)
            xs.append(x)
            B.add(K, b, x0=x, precision=precision)
        B.tune()
        B.run()
        return B, xs

    def batched(B, xs, e2e=False):
        if e2e:
            for b, h in zip(bs, hb):
                b.upload(h)
        for x in xs:
            x.fill(0.0)
        B.reset()
        B.run()
        if e2e:
            for x in xs:
                x.numpy()
        ctx.synchronize()

    def timed(fn, steps):
        ctx.synchronize()
        l0 = ctx.launches
        t0 = time.perf_counter()
        for _ in range(steps):
            fn()
        ctx.synchronize()
        return (time.perf_counter() - t0) / steps, ctx.launches - l0

    # plain FP64 one by one: the first pass autotunes each matrix's SpMV (untimed)
    seq_sts = sequential()
    t_seq, _ = timed(sequential, 1)
    res = {}
    clocks = Clocks(0)
    for name, prec in (("fp64", yb.PREC_FP64), ("mixed", yb.PREC_MIXED)):
        B, xs = make_batch(prec)
        for _ in range(max(0, warmup - 1)):
            batched(B, xs)
        if name == "mixed":
            clocks.start()
        t, launches = timed(lambda: batched(B, xs), steps)
        if name == "mixed":
            clk = clocks.stop()
            t_e2e, _ = timed(lambda: batched(B, xs, e2e=True), 1)
        sts = [B.stats(s) for s in range(P)]
        res[name] = {"s_per_step": t, "solves_per_s": P / t, "dofs_per_s": total / t, "launches": launches,
                     "max_relres": max(st.rel_residual for st in sts),
                     "all_converged": all(st.status == 0 for st in sts),
                     "iterations_max": max(st.iterations for st in sts),
                     "iterations_sum": sum(st.iterations for st in sts),
                     "replacements_sum": sum(st.refinements for st in sts)}
        del B, xs
    mixed = res["mixed"]
    out = {"metric": BATCH_METRIC, "value": mixed["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
           "steps": steps, "warmup": warmup, "ms_per_step": mixed["s_per_step"] * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 values, f64 vectors",
           "data": "synthetic, seeded (PCG64 seeds %d..%d)" % (workloads.BASE_SEED, workloads.BASE_SEED + P - 1),
           "config": {"workload": "batched_%d_2d_poisson_elasticity_p1-3_1e3-2e5dofs" % P, "problems": P,
                      "total_dofs": total, "min_dofs": min(ndofs), "max_dofs": max(ndofs),
                      "orders": sorted({s["order"] for s in specs}),
                      "kinds": {k: sum(1 for s in specs if s["kind"] == k) for k in ("poisson", "elasticity")},
                      "tolerance": "relative residual 1e-10 (FP64 true residual per system)",
                      "l2": "all systems together %.2f GB of matrices, larger than L2" %
                            (sum(K.nnz() for K in Ks) * 12 / 1e9)},
           "batched_mixed": mixed, "batched_fp64": res["fp64"],
           "sequential_fp64": {"s_per_step": t_seq, "solves_per_s": P / t_seq, "dofs_per_s": total / t_seq,
                               "max_relres": max(st.rel_residual for st in seq_sts),
                               "all_converged": all(st.status == 0 for st in seq_sts),
                               "iterations_sum": sum(st.iterations for st in seq_sts)},
           "speedup_vs_sequential_fp64": {"batched_mixed": t_seq / mixed["s_per_step"],
                                          "batched_fp64": t_seq / res["fp64"]["s_per_step"]},
           "e2e": {"value": P / t_e2e, "unit": "solves/s", "h2d_bytes_per_step": 8 * total,
                   "d2h_bytes_per_step": 8 * total, "includes": "RHS upload, reset, solve, solution download"},
           "gpu_launches": int(mixed["launches"] / steps),
           "setup": {"assembly_s": t_setup},
           "clocks": clk}
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_problems(specs, budget_s=10.0 if side else 30.0)
    del probs, Ks, bs
    ctx.close()
    if side:
        return out
    print(json.dumps(out), flush=True)


SERVE_METRIC = "served solves/sec to 1e-10 (continuous batching of Poisson arrivals), p50/p99 latency"


def run_serve(args, side=False):
    """Serving loop: `--requests` requests arrive as a Poisson process of rate
    `--rate` per second (seeded): 2D/3D Poisson, elasticity and SUPG
    advection-diffusion (BiCGSTAB), sizes log-uniform 1e3..1e6 dofs, orders 1-2.
    Each request carries its mesh (built by the client beforehand); the server
    side does the DoF numbering, device assembly, boundary conditions, the solve
    to a 1e-10 relative residual and the download of the solution.  Requests are
    admitted in arrival order under an HBM budget (`--budget-gb`) and solved
    together in one batch (yg_server_*), in FP64 (the value) and in mixed
    precision; the same requests served one at a time by the plain FP64
    single-system solvers give the baseline.  Latency = arrival to solution on the host.
    Requests are built on a second context of the GPU (its own stream), so their
    numbering and assembly overlap the block of iterations in flight: after each
    launch the loop builds admitted requests while the block runs (at least one,
    at most `--build-per-block`, 0 = no limit).
    side=True: `--serve-requests` requests, one-at-a-time baseline on the first
    `--serve-sequential` of them (and the server timed on that same subset),
    returned as an object of the default benchmark line instead of printed."""
    import yafel_b200 as yb
    from yafel_b200 import workloads
    ctx = yb.Context(0)
    bctx = yb.Context(0)  # builds: DoF numbering, assembly, boundary conditions
    N = args.serve_requests if side else args.requests
    specs = workloads.serving_specs(N)
    arr = workloads.arrivals(N, args.rate)
    meshes = [workloads.build_mesh(s) for s in specs]
    dofs = []
    for s in specs:
        dofs.append(s["dpn"] * (s["order"] * s["n"] + 1) ** s["dim"])
    budget = int(args.budget_gb * 1e9)

    def served(precision, idxs, clocks=None):
        S = yb.Server(budget, max_active=args.max_active, ctx=ctx)
        S.set_solo_rows(args.solo_rows)
        if args.solo_spmv_mb is not None:
            S.set_solo_spmv_bytes(int(args.solo_spmv_mb * 2 ** 20))
        idx, pending = {}, []
        lat, stats = {}, {}
        state = {"nsub": 0}
        n = len(idxs)
        l0 = ctx.launches
        ctx.synchronize()
        t0 = time.perf_counter()

        def take_arrivals():
            t = time.perf_counter() - t0
            while state["nsub"] < n and arr[idxs[state["nsub"]]] - arr[idxs[0]] <= t:
                i = idxs[state["nsub"]]
                idx[S.submit(workloads.est_bytes(specs[i], mixed=precision == yb.PREC_MIXED))] = i
                state["nsub"] += 1

        def admit_build(limit, while_running=False):
            k = 0
            while limit <= 0 or k < limit:
                if while_running and k > 0 and S.ready():
                    return
                r = S.admit()
                if r is None:
                    return
                i = idx[r]
                _, K, b, _ = workloads.assemble(specs[i], bctx, mesh=meshes[i])
                x = yb.DeviceVector(K.rows(), bctx)
                x.fill(0.0)
                pending.append((r, K, b, x, i))
                k += 1

        if clocks:
            clocks.start()
        tuned = False
        while len(lat) < n:
            take_arrivals()
            if S.info()["active"] == 0 and not pending:
                admit_build(1)
            for (r, K, b, x, i) in pending:
                S.attach(r, K, b, x, method=workloads.method(specs[i]), precision=precision)
            pending.clear()
            info = S.info()
            if info["active"] == 0:
                if state["nsub"] < n:
                    time.sleep(max(0.0, arr[idxs[state["nsub"]]] - arr[idxs[0]] - (time.perf_counter() - t0)))
                continue
            if not tuned and (info["active"] >= 32 or (info["queued"] == 0 and state["nsub"] == n)):
                S.tune()  # once, on the mix attached by then
                tuned = True
            S.launch()
            take_arrivals()
            admit_build(args.build_per_block, while_running=True)  # host work overlaps the block
            S.wait()
            for r in S.finished():
                i = idx[r]
                stats[i] = S.poll(r)
                S.solution(r).numpy()
                lat[i] = time.perf_counter() - t0 - (arr[i] - arr[idxs[0]])
                S.release(r)
        total = time.perf_counter() - t0
        clk = clocks.stop() if clocks else None
        del S
        return total, lat, stats, ctx.launches - l0, clk

    def sequential(idxs):
        lat, stats = {}, {}
        ctx.synchronize()
        t0 = time.perf_counter()
        for i in idxs:
            wait = arr[i] - arr[idxs[0]] - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            _, K, b, _ = workloads.assemble(specs[i], ctx, mesh=meshes[i])
            x, st = yb.solve(K, b, M=yb.JacobiPreconditioner(K), method=workloads.method(specs[i]), tol=TOL)
            x.numpy()
            lat[i] = time.perf_counter() - t0 - (arr[i] - arr[idxs[0]])
            stats[i] = st
            del K, b, x
        return time.perf_counter() - t0, lat, stats

    def summary(total, lat, stats, idxs):
        L = sorted(lat[i] for i in idxs)
        d = sum(dofs[i] for i in idxs)
        return {"s_total": total, "solves_per_s": len(idxs) / total, "dofs_per_s": d / total,
                "latency_s_p50": L[len(L) // 2], "latency_s_p99": L[min(len(L) - 1, int(0.99 * len(L)))],
                "latency_s_max": L[-1], "all_converged": all(stats[i].status == 0 for i in idxs),
                "max_relres": max(stats[i].rel_residual for i in idxs),
                "iterations_sum": int(sum(stats[i].iterations for i in idxs))}

    # warm-up on the smallest requests (module loading, graph capture paths)
    small = sorted(range(N), key=lambda i: dofs[i])[:max(3, args.warmup * 2)]
    served(yb.PREC_MIXED, small)
    served(yb.PREC_FP64, small)
    everything = list(range(N))
    clocks = Clocks(0)
    t64, lat64, st64, launches, clk = served(yb.PREC_FP64, everything, clocks)
    tm, latm, stm, _, _ = served(yb.PREC_MIXED, everything)
    subset = everything[:args.serve_sequential] if side else everything
    ts, lats, sts = sequential(subset)
    if side:  # the server on the same subset, for a like-for-like ratio
        t64s, lat64s, st64s, _, _ = served(yb.PREC_FP64, subset)
        tms, latms, stms, _, _ = served(yb.PREC_MIXED, subset)
    else:
        t64s, lat64s, st64s, tms, latms, stms = t64, lat64, st64, tm, latm, stm
    mixed = summary(tm, latm, stm, everything)
    fp64 = summary(t64, lat64, st64, everything)
    h2d = sum(m["nodes"].nbytes + m["cell_nodes"].nbytes + m["offsets"].nbytes + m["cell_types"].nbytes for m in meshes) + \
        8 * sum(dofs)
    out = {"metric": SERVE_METRIC, "value": fp64["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "steps": 1,
           "warmup": 2, "ms_per_step": t64 * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic, seeded (requests from seed %d)" %
           (workloads.BASE_SEED + 1_000_000),
           "config": {"workload": "serve_%d_requests_poisson_arrivals_%g_per_s" % (N, args.rate), "requests": N,
                      "offered_rate_per_s": args.rate, "total_dofs": int(sum(dofs)), "min_dofs": int(min(dofs)),
                      "max_dofs": int(max(dofs)), "budget_GB": args.budget_gb, "max_active": args.max_active,
                      "solo_rows": args.solo_rows, "build_per_block": args.build_per_block,
                      "solo_spmv_MiB": args.solo_spmv_mb,
                      "builds": "second context (own stream), overlapping the block in flight",
                      "kinds": {k: sum(1 for s in specs if s["kind"] == k) for k in ("poisson", "elasticity", "supg")},
                      "dims": {str(d): sum(1 for s in specs if s["dim"] == d) for d in (2, 3)},
                      "tolerance": "relative residual 1e-10 (FP64 true residual per request)",
                      "l2": "requests together far larger than L2"},
           "served_fp64": fp64, "served_mixed": mixed,
           "sequential_fp64": summary(ts, lats, sts, subset),
           "sequential_subset": "all requests" if not side else "the first %d requests in arrival order" % len(subset),
           "speedup_vs_sequential_fp64": {"served_mixed": ts / tms, "served_fp64": ts / t64s},
           "achieved_vs_offered": fp64["solves_per_s"] / args.rate,
           "e2e": {"value": fp64["solves_per_s"], "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                   "d2h_bytes_per_step": int(8 * sum(dofs)),
                   "includes": "DoF numbering, mesh upload, assembly, solve, solution download per request"},
           "gpu_launches": int(launches), "clocks": clk}
    if side:
        out["served_subset"] = {"served_fp64": summary(t64s, lat64s, st64s, subset),
                                "served_mixed": summary(tms, latms, stms, subset)}
    if not args.no_cpu_baseline:
        # requests in arrival order up to 1e5 dofs (the large 3D ones take minutes on the CPU)
        out["cpu_baseline"] = cpu_problems(specs, meshes, max_dofs=100000, budget_s=10.0 if side else 30.0)
    ctx.close()
    bctx.close()
    if side:
        return out
    print(json.dumps(out), flush=True)


class _NumberingView:
    """The arrays of the reference's DoFManager under the attribute names the
    traction-load routine reads (yafel_b200/loads.py is numpy only)."""

    def __init__(self, rd, p):
        self.dof_nodes, self.element_offsets, self.elements = rd.nodes, rd.offsets, rd.elements
        self.polyOrder, self.dof_per_node = p, rd.dpn
        self.ndofs = rd.n_nodes * rd.dpn


def cpu_sample(nx, threads, tol=1e-20, split=False):
    """The reference's own CPU path on an nx^3 Q2 sample of the workload, every
    step in its code compiled in place (oracle/_ref; no yafel_b200 library is
    loaded): Mesh + DoFManager(M, CG, 2, 3), CGAssembly<elasticity> on all
    cores (OpenMP), the traction load (numpy: the reference has no face
    loads), DirichletBC::apply for ux, uy, uz on x = 0, the Eigen tangent
    handed to its handmade sparse_csr(triplets), and pcg_solve with
    JacobiPreconditioner (OpenMP csr_spmv).  pcg_solve stops when
    r.z / r0.z0 < tol (a squared, preconditioned ratio).
    Returns (dofs, seconds, FP64 true relative residual, kind), and with
    `split` also the seconds up to the solve and of the solve."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as O
    from yafel_b200 import loads
    mesh = problem(nx)
    lam = (E * NU) / ((1 + NU) * (1 - 2 * NU))
    mu = E / (2 * (1 + NU))
    t0 = time.perf_counter()
    rd = O.RefDofManager(mesh, 2, 3)
    # the residual is requested too: with the tangent alone CGAssembly writes the
    # element solution through a buffer it never sized (CGAssembly.hpp:99-125)
    rs = O.RefSystem(rd, 3, O.ELASTICITY, [1.0, lam, mu, 0.0, 0.0, 0.0], tangent=True, residual=True,
                     threads=threads)
    F = loads.hex_face_traction(_NumberingView(rd, 2), lambda Y: np.abs(Y[:, 0] - 1.0) < 1e-9, (1.0, 0.0, 0.0))
    rs.set_residual(F)
    for c in range(3):
        rs.dirichlet_plane(c, 0, 0.0, 0.0)
    A, b = rs.to_ref_csr()
    t1 = time.perf_counter()
    x = A.pcg_jacobi(b, np.zeros(b.size), tol)
    t2 = time.perf_counter()
    if split:
        return b.size, t2 - t0, A.true_relres(b, x), "reference", t1 - t0, t2 - t1
    return b.size, t2 - t0, A.true_relres(b, x), "reference"


def calibrate_cpu_tol(nx, threads, target=8e-11):
    """pcg_solve's stopping test is on the preconditioned squared ratio, not
    on the true residual: one untimed solve at tol 1e-20 measures the relative
    residual reached, and tol is rescaled (the residual falls about with the
    square root of the ratio) so that the timed solves end near `target`,
    inside [5e-11, 1e-10].  Returns (tol, relres of the probe solve)."""
    _, _, rel, _ = cpu_sample(nx, threads, 1e-20)
    return 1e-20 * (target / rel) ** 2, rel


def cpu_problem(spec, mesh=None):
    """The reference's own CPU path on one seeded problem (oracle/_ref): Mesh +
    DoFManager, CGAssembly<Physics> (OpenMP), the N(0,1) right-hand side,
    DirichletBC::apply per component on x = 0, its sparse_csr(triplets), then
    pcg_solve with the Jacobi preconditioner (TOL 1e-21 on the squared
    preconditioned ratio), or for SUPG its unpreconditioned bicgstab_solve
    (whose tolerance is fixed: 1e-14 on the squared true residual).  SUPG uses
    the reference's SUPG formulas with the problem's k and h.
    Returns (dofs, seconds, FP64 relative residual)."""
    from oracle import oracle as O
    from yafel_b200 import workloads
    if mesh is None:
        mesh = workloads.build_mesh(spec)
    dim, dpn = spec["dim"], spec["dpn"]
    if spec["kind"] == "supg":
        h = 1.0 / spec["n"]
        kind, params = O.SUPG_PARAM, [h / (2.0 * spec["peclet"]), h, 1.0, 0.0]
    elif spec["kind"] == "poisson":
        kind, params = O.POISSON, [1.0, 0.0]
    else:
        lam, mu = (1.0 * 0.3) / (1.3 * 0.4), 1.0 / 2.6
        kind, params = O.ELASTICITY, [1.0, lam, mu, 0.0, 0.0, 0.0]
    t0 = time.perf_counter()
    rd = O.RefDofManager(mesh, spec["order"], dpn)
    rs = O.RefSystem(rd, dim, kind, params, threads=os.cpu_count() or 1)
    rs.set_residual(workloads.rhs(spec, rd.n_nodes * dpn))
    clamp = np.nonzero(np.abs(rd.nodes[:, 0]) < 1e-9)[0]
    for c in range(dpn):
        rs.dirichlet_nodes(c, clamp, 0.0)
    A, b = rs.to_ref_csr()
    x0 = np.zeros(b.size)
    x = A.bicgstab(b, x0) if spec["kind"] == "supg" else A.pcg_jacobi(b, x0, 1e-21)
    dt = time.perf_counter() - t0
    return b.size, dt, A.true_relres(b, x)


def cpu_problems(specs, meshes=None, budget_s=30.0, max_dofs=None):
    """The reference's CPU path over problems in order until the time budget is
    spent (a bounded sample); returns the cpu_baseline object."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    n, dofs, t, rels = 0, 0, 0.0, []
    for i, spec in enumerate(specs):
        if max_dofs and spec["dpn"] * (spec["order"] * spec["n"] + 1) ** spec["dim"] > max_dofs:
            continue
        d, dt, rel = cpu_problem(spec, meshes[i] if meshes else None)
        n, dofs, t = n + 1, dofs + d, t + dt
        rels.append(rel)
        if t > budget_s:
            break
    return {"value": n / t, "unit": "solves/s", "cores": os.cpu_count() or 1, "kind": "reference",
            "dofs_per_s": dofs / t,
            "sample": "%d problems (%d dofs), the reference's DoFManager, CGAssembly, DirichletBC and "
                      "pcg_solve/Jacobi (bicgstab_solve for SUPG) on sparse_csr, %.1f s, max relres %.1e"
                      % (n, dofs, t, max(rels))}


def cpu_baseline(args):
    """One calibrated sample of the reference's CPU path (untimed probe solve
    first) on the whole cpu_nx^3 cube, scaled to the configured size the way
    the reference arm scales its sample (phases up to the solve by the element
    count, the solve by stored entries times iterations), reported beside the
    GPU numbers."""
    threads = os.cpu_count() or 1
    nx = args.cpu_nx
    tol, _ = calibrate_cpu_tol(nx, threads)
    ndofs, dt, rel, kind, t_setup, t_solve = cpu_sample(nx, threads, tol, split=True)
    elem_ratio = (args.nx / nx) ** 3
    nnz_ratio = base_config(args.nx, 1)["blocks"] / base_config(nx, 1)["blocks"]
    iter_ratio = args.nx / nx
    est = t_setup * elem_ratio + t_solve * nnz_ratio * iter_ratio
    return {"value": base_config(args.nx, 1)["dofs"] / est, "unit": "dofs/s", "cores": threads, "kind": kind,
            "sample_rate_dofs_per_s": ndofs / dt,
            "sample": ("the reference's own code on the whole %d^3 Q2 cube (%d dofs: DoFManager, CGAssembly on "
                       "all cores, DirichletBC, sparse_csr, pcg_solve+Jacobi with TOL %.2e on r.z/r0.z0, true "
                       "relative residual %.1e): %.2f s to the solve + %.2f s of solve; scaled to %d^3 by elements "
                       "x%.1f and stored entries x%.1f times iterations x%.2f" %
                       (nx, ndofs, tol, rel, t_setup, t_solve, args.nx, elem_ratio, nnz_ratio, iter_ratio))}


def run_reference(args):
    """The reference's own CPU path (oracle/_ref: its DoFManager, CGAssembly,
    DirichletBC, sparse_csr and pcg_solve compiled in place; no yafel_b200
    library is loaded) on the benchmark's workload, on all host cores.  The
    full nx^3 = 60^3 system takes minutes per step on the CPU, so each step runs
    the same pipeline on the whole --ref-nx^3 cube (default 30^3: the same
    elements, physics, loads and tolerance) and the value is scaled to the
    configured size by the measured phases: everything up to the solve grows
    with the element count (x (nx/ref_nx)^3), and the solve with the stored
    entries times the iteration count, which grows as 1/h for this system
    (x nnz ratio x nx/ref_nx; Jacobi-PCG takes 583 and 1169 iterations to
    1e-10 at 30^3 and 60^3).  Warm-up: the tolerance probe at ref_nx^3, then
    W-1 runs at 16^3."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    rnx = args.ref_nx
    # warm-up: the first one is the tolerance probe (pcg_solve's test is on a
    # squared preconditioned ratio; the probe rescales it so that every timed
    # solve ends near a 1e-10 true relative residual, like the GPU's)
    tol, _ = calibrate_cpu_tol(rnx, threads)
    if args.warmup > 1:
        wtol, _ = calibrate_cpu_tol(16, threads)
        for _ in range(args.warmup - 2):
            cpu_sample(16, threads, wtol)
    cfg = base_config(args.nx, ws)
    elem_ratio = (args.nx / rnx) ** 3
    nnz_ratio = base_config(args.nx, ws)["blocks"] / base_config(rnx, ws)["blocks"]
    iter_ratio = args.nx / rnx
    vals, rels, setups, solves, ndofs = [], [], [], [], 0
    for _ in range(args.steps):
        ndofs, dt, rel, kind, t_setup, t_solve = cpu_sample(rnx, threads, tol, split=True)
        est = t_setup * elem_ratio + t_solve * nnz_ratio * iter_ratio
        vals.append(cfg["dofs"] / est)
        rels.append(rel)
        setups.append(t_setup)
        solves.append(t_solve)
    value = statistics.mean(vals)
    ms_step = (statistics.mean(setups) * elem_ratio + statistics.mean(solves) * nnz_ratio * iter_ratio) * 1e3
    sample_rate = ndofs / (statistics.mean(setups) + statistics.mean(solves))
    text = ("the reference's own code on the whole %d^3 Q2 cube (%d dofs: DoFManager, CGAssembly on all cores, "
            "DirichletBC, sparse_csr, pcg_solve+Jacobi with TOL %.2e on r.z/r0.z0, true relative residual %.1e): "
            "%.2f s to the solve + %.2f s of solve, %.0f dofs/s there; scaled to %d^3 by elements x%.2f "
            "(to the solve) and stored entries x%.2f times iterations x%.2f (the solve)" %
            (rnx, ndofs, tol, max(rels), statistics.mean(setups), statistics.mean(solves), sample_rate, args.nx,
             elem_ratio, nnz_ratio, iter_ratio))
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "dofs/s", "n_gpus": ws,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (structured mesh)",
           "config": cfg,
           "sample": {"ran": "%d^3 Q2 hex, full pipeline, converged" % rnx, "dofs": ndofs, "tol_rz_ratio": tol,
                      "relres_min": min(rels), "relres_max": max(rels), "setup_s": statistics.mean(setups),
                      "solve_s": statistics.mean(solves), "rate_at_sample_dofs_per_s": sample_rate,
                      "scale_elements": elem_ratio, "scale_entries": nnz_ratio, "scale_iterations": iter_ratio},
           "cpu_baseline": {"value": value, "unit": "dofs/s", "cores": threads, "kind": kind, "sample": text},
           "e2e": {"value": value, "unit": "dofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def base_config(nx, ws):
    """The workload as both arms state it.  Structured Q2 hex: (2nx+1)^3 nodes;
    a node's row holds the nodes it shares a cell with, a tensor product of the
    1-D counts, so the 3x3 blocks number (8nx+1)^3."""
    nnzb = (8 * nx + 1) ** 3
    return {"workload": "elasticity_q2_hex_%d^3_jacobi_pcg_1e-10" % nx, "mesh": "%d^3 Q2 hex" % nx,
            "dofs": 3 * (2 * nx + 1) ** 3, "blocks": nnzb, "format": "BCSR3", "preconditioner": "jacobi",
            "tolerance": "relative residual 1e-10 (FP64 true residual)",
            "l2": "inputs larger than L2 (FP64 matrix %.2f GB)" % (nnzb * 76 / 1e9),
            "step": "assemble+dirichlet+traction+solve",
            "parallelism": "replicas" if ws > 1 else "single GPU"}


def main():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1 and "OMP_NUM_THREADS" not in os.environ:
        # one process per GPU on one host: share the host cores among the ranks
        os.environ["OMP_NUM_THREADS"] = str(max(1, (os.cpu_count() or ws) // ws))
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="yafel_b200")
    ap.add_argument("--nx", type=int, default=NX)
    ap.add_argument("--cpu-nx", type=int, default=16)
    ap.add_argument("--ref-nx", type=int, default=30, help="cube the reference arm runs whole (scaled to --nx)")
    ap.add_argument("--spmv", default=None, help="pin the FP64-value SpMV as variant:lanes (default: autotuned)")
    ap.add_argument("--spmv32", default=None, help="pin the FP32-value SpMV as variant:lanes (default: autotuned)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the 64x64 Poisson, 30^3 Q3 and ILU(0) side measurements")
    ap.add_argument("--spmv-profile", action="store_true", help="time the SpMV kernel alone (roofline/ncu)")
    ap.add_argument("--variant", type=int, default=None, help="SpMV variant for --spmv-profile (0 flat, 1 staged, 2 TMA)")
    ap.add_argument("--lanes", type=int, default=32, help="SpMV lanes / TMA configuration for --spmv-profile")
    ap.add_argument("--spmv-matrix", default="elasticity", choices=["elasticity", "poisson"],
                    help="matrix of --spmv-profile: Q2 elasticity (BCSR3) or Q2 Poisson (CSR)")
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--spmv-precision", default="both", choices=["both", "fp64", "fp32"],
                    help="value precisions timed by --spmv-profile")
    ap.add_argument("--workload", default="fem", choices=["fem", "batch", "serve", "ilu"],
                    help="fem: 60^3 Q2 elasticity assemble+solve; batch: many 2D problems solved together; "
                         "serve: the serving loop; ilu: ILU(0)- beside Jacobi-PCG on the --nx^3 problem")
    ap.add_argument("--problems", type=int, default=512, help="problems in the batched workload")
    ap.add_argument("--no-side-workloads", action="store_true",
                    help="skip the batched (512 problems) and served objects of the default line")
    ap.add_argument("--serve-requests", type=int, default=1000, help="requests of the served object of the default line")
    ap.add_argument("--serve-sequential", type=int, default=200,
                    help="requests of that object also served one at a time (the first ones in arrival order)")
    ap.add_argument("--requests", type=int, default=160, help="requests in the serving workload")
    ap.add_argument("--rate", type=float, default=2000.0, help="arrival rate (req/s) of the serving workload")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="HBM budget of the serving workload")
    ap.add_argument("--max-active", type=int, default=1024, help="systems solved together by the server")
    ap.add_argument("--solo-spmv-mb", type=float, default=None,
                    help="batched and served: systems whose FP64 matrix holds at least this many MiB run their "
                         "own SpMV launch in the batch (default: the library's)")
    ap.add_argument("--build-per-block", type=int, default=0,
                    help="most requests the serving loop builds while a block runs (0 = while it runs)")
    ap.add_argument("--solo-rows", type=int, default=100000,
                    help="served systems of at least this many rows are solved alone by the single-system "
                         "solvers, whose SpMV runs at the HBM rate (0: batch all)")
    args = ap.parse_args()
    if args.spmv_profile:
        run_spmv_profile(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "ilu":
        import yafel_b200 as yb
        print(json.dumps(run_ilu(yb.Context(0), args.nx)), flush=True)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
