"""Order of accuracy of the CUDA path on the 2-D isentropic vortex (Euler,
quads, Gauss points, c_dg correction, Rusanov, RK45, dt 1e-3, t = 1): the
BASELINE configuration's domain [-5, 5]^2 on meshes of 10^2, 20^2, 40^2 and
80^2 elements at P = 1, 2, 3.

The L2 density error is over-integrated: the solution is interpolated to the
(P + 3)-point Gauss rule of each element and compared with the exact solution
(the initial field shifted by (t, 0)) there.  Measured rates on the two
finest meshes: 2.0 (P = 1), 2.6 (P = 2), 4.1 (P = 3).

P = 2 sits between the proven DG rate P + 1/2 and the design rate P + 1.  The
reference itself gives the same: the committed fixtures order_vortex_p2_n*
are the reference's own states after the same 1000 steps on the 10^2, 20^2
and 40^2 meshes; their errors are those of this path (the states agree to
1e-11) and their rates are 2.64 and 2.59 (tests/test_oracle_golden.py checks
them on the CPU).  So the bar here is the reference's rate: P + 1 - 0.1 for
P = 1 and 3, and the reference's measured 2.5 for P = 2."""
import numpy as np
import pytest

import hifiles_b200 as H
import oracle as O
from golden_util import load, over_integrated_density_error, rel

pytestmark = pytest.mark.gpu

T_END, DT = 1.0, 1e-3
NS = (10, 20, 40, 80)
MIN_RATE = {1: 1.9, 2: 2.5, 3: 3.9}


def _run(P, n):
    s = H.Solver.box(2, P, (n, n), (-5.0, -5.0), (5.0, 5.0), viscous=False, vcjh_scheme=1, gamma=1.4)
    pos = s.geometry()["pos_upts"]
    s.set_state(np.asfortranarray(O.ic_vortex(pos)))
    s.advance(int(round(T_END / DT)), DT)
    return s.get_state(), pos


@pytest.mark.parametrize("P", [1, 2, 3])
def test_vortex_convergence_rate(P):
    errs = []
    for n in NS:
        u, pos = _run(P, n)
        errs.append(over_integrated_density_error(u, pos, P, 10.0 / n, T_END))
    rates = [np.log(errs[i] / errs[i + 1]) / np.log(NS[i + 1] / NS[i]) for i in range(len(NS) - 1)]
    print("P=%d errors %s rates %s" % (P, ["%.3e" % e for e in errs], ["%.2f" % r for r in rates]))
    assert all(np.isfinite(errs))
    assert rates[-1] > MIN_RATE[P] and rates[-2] > MIN_RATE[P], (errs, rates)


@pytest.mark.parametrize("n", [10, 20, 40])
def test_p2_states_equal_the_reference_runs(n):
    """The P = 2 convergence runs end where the reference's own runs end."""
    meta, a = load("order_vortex_p2_n%d" % n)
    u, _ = _run(2, n)
    assert rel(u, a["uN"]) <= 1e-11
