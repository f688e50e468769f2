"""The serving workload's admission estimate is an upper bound of the bytes a
request holds once attached (matrix as assembled, right-hand side, iterate and
the batch's work vectors), in FP64 and with the FP32 copy of mixed precision;
checked on the oracle-assembled patterns (no GPU needed)."""
import pytest

import yafel_b200 as yb
from oracle import oracle as O
from yafel_b200 import workloads
from yafel_b200._lib import lib

SPECS = workloads.serving_specs(12, lo=1e3, hi=2e4) + [workloads.problem_spec(i, lo=1e3, hi=2e4) for i in range(6)]


@pytest.mark.parametrize("k", range(len(SPECS)))
def test_admission_estimate_bounds_the_attached_bytes(k):
    spec = SPECS[k]
    mesh = workloads.build_mesh(spec)
    odm = O.dofmanager(mesh, spec["order"])
    kind = {"poisson": O.POISSON, "elasticity": O.ELASTICITY, "supg": O.SUPG}[spec["kind"]]
    K, _ = O.assemble(odm, spec["dpn"], spec["dim"], kind, [1.0, 0.3, 0.4, 0, 0, 0], residual=False)
    dpn = spec["dpn"]
    rows = K.nrows
    nbrows, nnzb = rows // dpn, K.nnz // (dpn * dpn)
    assert nnzb * dpn * dpn == K.nnz
    method = yb.METHOD_BICGSTAB if workloads.method(spec) == "bicgstab" else yb.METHOD_CG
    attached = (nnzb * (dpn * dpn * 8 + 4) + 4 * (nbrows + 1) + 4 * nbrows + 16 * rows
                + lib().yg_batch_work_bytes(rows, method))
    assert workloads.est_bytes(spec) >= attached, spec
    assert workloads.est_bytes(spec, mixed=True) >= attached + nnzb * dpn * dpn * 4, spec
