"""Seeded synthetic problem sets for the batched and served forms.

Every problem is a 2D (or 3D) Poisson, linear-elasticity or SUPG
advection-diffusion (element Peclet number log-uniform in [1, 100]) system on a
structured grid whose cells are quads or triangle pairs (seeded coin) with
interior nodes jittered by U(-0.2, 0.2)*h, Dirichlet u = 0 on x = 0 and an
i.i.d. N(0,1) right-hand side.  Problem i of a set uses the seed base + i
(numpy PCG64), so a set is reproducible.
"""
import math

import numpy as np

from . import meshgen

BASE_SEED = 20261203


def grid_for_dofs(target_dofs, p, dpn, dim=2):
    """Cells per side of a square (cube) grid whose order-p DoF count is close
    to target_dofs: dofs = dpn * (p*n + 1)^dim."""
    n = ((target_dofs / dpn) ** (1.0 / dim) - 1.0) / p
    return max(1, int(round(n)))


def problem_spec(i, base=BASE_SEED, lo=1e3, hi=2e5, orders=(1, 2, 3), kinds=("poisson", "elasticity"), dims=(2,)):
    rng = np.random.Generator(np.random.PCG64(base + i))
    target = math.exp(rng.uniform(math.log(lo), math.log(hi)))
    p = int(rng.choice(orders))
    kind = str(rng.choice(kinds))
    dim = int(rng.choice(dims))
    dpn = dim if kind == "elasticity" else 1
    n = grid_for_dofs(target, p, dpn, dim)
    spec = {"index": i, "seed": base + i, "target_dofs": target, "order": p, "kind": kind, "dim": dim, "dpn": dpn,
            "n": n}
    if kind == "supg":
        spec["peclet"] = math.exp(rng.uniform(math.log(1.0), math.log(100.0)))
    return spec


def method(spec):
    """Krylov method of a problem: BiCGSTAB for the non-symmetric SUPG systems."""
    return "bicgstab" if spec["kind"] == "supg" else "cg"


def physics(spec):
    """Device physics of a problem.  SUPG: U = (1,0,0), h = the cell size, and
    k = U h / (2 Pe) for the drawn element Peclet number Pe."""
    import yafel_b200 as yb
    dim = spec["dim"]
    if spec["kind"] == "poisson":
        return yb.PoissonEquation(dim, f=0.0)
    if spec["kind"] == "elasticity":
        return yb.LinearElasticity(dim, E=1.0, nu=0.3, body=(0.0, 0.0, 0.0))
    h = 1.0 / spec["n"]
    return yb.AdvectionDiffusionSUPG(dim, k=h / (2.0 * spec["peclet"]), h=h, U0=1.0, Q=0.0)


def build_mesh(spec):
    p, n = spec["order"], spec["n"]
    if spec["dim"] == 2:
        return meshgen.jittered_mixed(n, n, seed=spec["seed"], order=meshgen.corner_order(p))
    return meshgen.structured_hex(n, n, n, order=meshgen.corner_order(p))


def rhs(spec, ndofs):
    rng = np.random.Generator(np.random.PCG64(spec["seed"] + 7919))
    return rng.standard_normal(ndofs)


def clamp_dofs(X, dpn):
    nodes = np.nonzero(np.abs(X[:, 0]) < 1e-9)[0]
    return (nodes[:, None] * dpn + np.arange(dpn)[None, :]).ravel().astype(np.int64)


def assemble(spec, ctx, mesh=None):
    """Assemble problem `spec` on the device through the public API: DoF
    numbering, tangent (CSR for Poisson and SUPG, 2x2/3x3 BCSR for elasticity),
    the N(0,1) right-hand side and u = 0 on x = 0.  `mesh` may be given when it
    was built beforehand.  Returns (mesh, K, b, clamp_dofs)."""
    import yafel_b200 as yb
    if mesh is None:
        mesh = build_mesh(spec)
    dpn, dim = spec["dpn"], spec["dim"]
    dm = yb.DoFManager(mesh, spec["order"], dpn, ctx=ctx)
    fe = yb.FESystem(dm, dim, format=yb.CSR if dpn == 1 else yb.BCSR)
    yb.CGAssembly(physics(spec), fe, [yb.AssemblyRequirement.Tangent])
    K = fe.getGlobalTangent()
    b = yb.DeviceVector(rhs(spec, dm.ndofs), ctx)
    nodes = np.nonzero(np.abs(dm.dof_nodes[:, 0]) < 1e-9)[0].astype(np.int64)
    for c in range(dpn):
        bc = yb.DirichletBC(dm, 0.0, c)
        bc.bc_nodes = nodes
        bc.apply(K, b)
    return mesh, K, b, clamp_dofs(dm.dof_nodes, dpn)


def est_bytes(spec, mixed=False):
    """Upper estimate of the solver-resident device bytes of a problem, from its
    size alone (before it is built): matrix values and columns with at most
    dpn * (2p+1)^dim entries per row (plus the FP32 copy of the values when
    `mixed`), the right-hand side, the iterate and the Krylov work vectors (4 for
    PCG, 9 for BiCGSTAB), plus row data."""
    p, dim, dpn, n = spec["order"], spec["dim"], spec["dpn"], spec["n"]
    dofs = dpn * (p * n + 1) ** dim
    nnz_row = dpn * (2 * p + 1) ** dim
    vecs = (9 if spec["kind"] == "supg" else 4) + 2
    return int(dofs * ((16 if mixed else 12) * nnz_row + 8 * vecs + 16))


def serving_specs(count, base=BASE_SEED + 1_000_000, lo=1e3, hi=1e6):
    """Requests of the serving workload: sizes log-uniform in [lo, hi] dofs,
    orders 1-2, 2D/3D Poisson, elasticity and SUPG advection-diffusion."""
    return [problem_spec(i, base=base, lo=lo, hi=hi, orders=(1, 2), kinds=("poisson", "elasticity", "supg"),
                         dims=(2, 3)) for i in range(count)]


def arrivals(count, rate, seed=BASE_SEED + 2_000_000):
    """Arrival times (s) of a Poisson process of the given rate (req/s)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.cumsum(rng.exponential(1.0 / rate, count))
