"""solve_presolved on the GPU: presolve (host), the device-resident solve of the reduced LP,
postsolve; the original LP's KKT checker at 2·TOL and HiGHS's objective within 1e-5, in
both forms (crates/saddlepoint-cuda/tests/netlib.rs:31-74 on the presolved problem)."""
import pytest

import oracle
from conftest import TOL, netlib_lp, netlib_reference

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["afiro", "adlittle", "israel", "sctest", "shell", "etamacro", "standata",
                                  "standgub", "standmps", "25fv47", "scrs8", "stair"])
def test_presolved_netlib_solve(name, gpu_backend):
    import saddlepoint_b200 as sp

    lp = netlib_lp(name)
    status, objective = netlib_reference()[name]
    for precision in (sp.Precision.FP64, sp.Precision.Mixed):
        s = sp.solve_presolved(lp, sp.SolverParams(tolerance=TOL, precision=precision), gpu_backend)
        assert s.status == sp.Status.Optimal, (name, precision, s.status)
        oracle.check(lp, s.x, s.y).verify(2.0 * TOL)
        assert abs(s.objective - objective) / (1.0 + abs(objective)) <= 1e-5


def test_presolve_proves_woodinfe_infeasible(gpu_backend):
    import saddlepoint_b200 as sp

    s = sp.solve_presolved(netlib_lp("woodinfe"), sp.SolverParams(tolerance=TOL), gpu_backend)
    assert s.status == sp.Status.PrimalInfeasible
