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
