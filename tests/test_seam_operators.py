"""The product's dense operators for the per-operator path
(hifiles_b200.seam.dense_operators, built from the library's 1-D factors)
equal the oracle's opp_0 .. opp_6, which are pinned to the reference."""
import numpy as np
import pytest

import oracle as O
from hifiles_b200 import seam


@pytest.mark.parametrize("dims,P,scheme", [(2, 1, 1), (2, 3, 1), (2, 4, 2), (3, 2, 2), (3, 3, 1), (3, 3, 3)])
def test_dense_operators_equal_oracle(dims, P, scheme):
    ops = seam.dense_operators(dims, P, 0, scheme, 0.0)
    m = O.Mesh.box(dims, P, [2] * dims, [0] * dims, [1] * dims, vcjh_scheme=scheme)
    assert np.array_equal(ops["opp_0"], m.operator(0))
    assert np.array_equal(ops["opp_3"], m.operator(3))
    assert np.array_equal(ops["opp_6"], m.operator(6))
    for d in range(dims):
        for w in (1, 2, 4, 5):
            assert np.array_equal(ops["opp_%d" % w][d], m.operator(w, d)), (w, d)


def test_entry_points_refuse_bad_arguments_before_any_device_work():
    """The per-operator entry points check their arguments on the host and
    return a status, as the reference's wrappers would otherwise exit: a
    Riemann solver, dimension or boundary option that is not built gives
    FR_ERR_UNSUPPORTED, a bad size or pointer FR_ERR_ARG.  These paths touch
    no GPU."""
    import ctypes as C
    import hifiles_b200 as H
    L = seam._bind_bdy(seam._bind(H.lib()))
    ph = seam.PhysDesc(gamma=1.4, prandtl=0.72, mu_inf=0.0, rt_inf=1.0, c_sth=1.0, fix_vis=1.0, tau=1.0,
                       pen_fact=0.5)
    fake = C.c_void_p(16)                      # never dereferenced: the call returns first
    ERR_ARG, ERR_UNSUPPORTED = 1, 5
    # sparse product: sizes, flags and pointers
    assert L.fr_op_spmv_ell(0, 4, 5, 10, fake, fake, 2, fake, fake, 4, 3, 0, None) == ERR_ARG
    assert L.fr_op_spmv_ell(4, 4, 5, 10, fake, fake, 2, fake, fake, 4, 3, 2, None) == ERR_ARG
    assert L.fr_op_spmv_ell(4, 4, 5, 10, None, fake, 2, fake, fake, 4, 3, 0, None) == ERR_ARG
    assert L.fr_op_spmv_ell(300, 4, 5, 10, fake, fake, 2, fake, fake, 4, 3, 0, None) == ERR_UNSUPPORTED
    # interior common flux: Roe is 2-D only, HLLC (1) is not built; 3 dimensions need 5 fields
    args = [fake] * 9
    assert L.fr_op_int_inters_common_invFlux(4, 3, 5, 1, *args, C.byref(ph), 2, 0, None) == ERR_UNSUPPORTED
    assert L.fr_op_int_inters_common_invFlux(4, 2, 4, 1, *args, C.byref(ph), 1, 0, None) == ERR_UNSUPPORTED
    assert L.fr_op_int_inters_common_invFlux(4, 3, 4, 1, *args, C.byref(ph), 0, 0, None) == ERR_ARG
    # boundary fluxes: the same solver rules, and every table must be given
    bargs = [fake] * 7
    assert L.fr_op_bdy_inters_common_invFlux(4, 3, 5, 1, *bargs, C.byref(ph), 1.0, 2, 0, None) == ERR_UNSUPPORTED
    nulls = [fake] * 4 + [None] + [fake] * 2
    assert L.fr_op_bdy_inters_common_invFlux(4, 2, 4, 1, *nulls, C.byref(ph), 1.0, 0, 0, None) == ERR_ARG
    assert L.fr_op_bdy_inters_common_viscFlux(4, 2, 4, 1, *nulls, C.byref(ph), 1.0, None) == ERR_ARG
    # operator products: non-positive sizes and missing operators
    assert L.fr_op_extrapolate_solution(0, 4, 5, 10, fake, fake, fake, None) == ERR_ARG
    assert L.fr_op_calculate_divergence(4, 3, 5, 10, None, fake, fake, None) == ERR_ARG
    # the reason is kept for fr_last_error
    assert L.fr_op_int_inters_common_invFlux(4, 3, 5, 1, *args, C.byref(ph), 2, 0, None) == ERR_UNSUPPORTED
    assert b"2-D" in H.lib().fr_last_error()
