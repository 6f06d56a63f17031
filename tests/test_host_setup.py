"""Host-side set-up of the product (no GPU): the C ABI library loads and exports
every declared entry point; its metrics, interface wiring and 1-D operator
factors agree with the oracle (which is pinned bit-exact to the reference)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import hifiles_b200 as H
import oracle as O

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for fn in os.listdir(os.path.join(REPO, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(REPO, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"\b(fr_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(H.LIB_PATH)
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


CASES = [(2, 3, (4, 5), (-5, -5), (5, 5), 0.0), (2, 2, (3, 3), (0, 0), (1, 2), 0.2),
         (3, 3, (3, 2, 2), (0, 0, 0), (6.0, 4.0, 4.0), 0.0), (3, 2, (3, 3, 3), (0, 0, 0), (1, 1, 1), 0.15),
         (3, 4, (2, 2, 2), (0, 0, 0), (2 * np.pi,) * 3, 0.1), (3, 1, (1, 1, 1), (0, 0, 0), (1, 1, 1), 0.0)]


@pytest.mark.parametrize("dims,order,n,lo,hi,jit", CASES)
def test_host_metrics_and_wiring_match_oracle(dims, order, n, lo, hi, jit):
    xv, c2v = H.box_mesh(dims, n, lo, hi, jit, seed=7)
    shift = [hi[d] - lo[d] for d in range(dims)]
    g = H.mesh_geometry(dims, xv, c2v, shift, order)
    m = O.Mesh.box(dims, order, n, lo, hi, jitter=jit, seed=7)
    og = m.geometry()
    for k in ("pos_upts", "detjac_upts", "JGinv_upts", "tdA_fpts", "norm_fpts"):
        assert np.array_equal(g[k], og[k]), k
    ol, orr = m.interfaces()
    pairs = {frozenset(p) for p in zip(g["left"].tolist(), g["right"].tolist())}
    opairs = {frozenset(p) for p in zip(ol.tolist(), orr.tolist())}
    assert pairs == opairs
    E, nf = m.n_eles, m.n_fpts
    assert len(pairs) * 2 == E * nf


def _dense_from_line(dims, P, L):
    """Rebuild opp_0, opp_2[0..D-1], opp_3 of a Gauss tensor element from the 1-D factors."""
    n = P + 1
    nu = n ** dims
    nfpf = n ** (dims - 1)
    nf = 2 * dims * nfpf

    def abc(u):
        return (u % n, (u // n) % n, u // (n * n)) if dims == 3 else (u % n, u // n, 0)

    def line(f):
        fc, r = divmod(f, nfpf)
        if dims == 2:
            j = r
            return {0: ((j, None), 1, 0), 1: ((None, j), 0, 1), 2: ((P - j, None), 1, 1), 3: ((None, P - j), 0, 0)}[fc]
        j, k = divmod(r, n)
        return {0: ((P - k, j, None), 2, 0), 1: ((k, None, j), 1, 0), 2: ((None, k, j), 0, 1),
                3: ((P - k, None, j), 1, 1), 4: ((None, P - k, j), 0, 0), 5: ((k, j, None), 2, 1)}[fc]

    o0 = np.zeros((nf, nu))
    o3 = np.zeros((nu, nf))
    for f in range(nf):
        fixed, ax, plus = line(f)
        for u in range(nu):
            c = abc(u)
            if all(fixed[d] is None or fixed[d] == c[d] for d in range(dims)):
                o0[f, u] = (L["Lp"] if plus else L["Lm"])[c[ax]]
                o3[u, f] = L["gR"][c[ax]] if plus else -L["gL"][c[ax]]
    o2 = []
    for d in range(dims):
        D = np.zeros((nu, nu))
        for k in range(nu):
            ck = abc(k)
            for u in range(nu):
                cu = abc(u)
                if all(cu[e] == ck[e] for e in range(dims) if e != d):
                    D[k, u] = L["D"][ck[d], cu[d]]
        o2.append(D)
    return o0, o2, o3


@pytest.mark.parametrize("dims,P,scheme", [(2, 1, 1), (2, 3, 1), (2, 5, 2), (3, 2, 2), (3, 3, 1), (3, 4, 3),
                                           (3, 3, 4), (2, 4, 0)])
def test_line_factors_rebuild_reference_dense_operators(dims, P, scheme):
    L = H.line_operators(P, 0, scheme, 0.3)
    m = O.Mesh.box(dims, P, [2] * dims, [0] * dims, [1] * dims, vcjh_scheme=scheme, eta=0.3)
    o0, o2, o3 = _dense_from_line(dims, P, L)
    assert np.array_equal(o0, m.operator(0))
    assert np.array_equal(o3, m.operator(3))
    for d in range(dims):
        assert np.array_equal(o2[d], m.operator(2, d))


def test_mesh_errors_are_reported_not_fatal():
    xv, c2v = H.box_mesh(3, (2, 2, 2), (0, 0, 0), (1, 1, 1))
    with pytest.raises(H.FrError) as ei:            # no periodic shift: unmatched faces
        H.mesh_geometry(3, xv, c2v, [0, 0, 0], 2)
    assert ei.value.status == 6
    with pytest.raises(H.FrError) as ei:
        H.mesh_geometry(3, xv, c2v, [1, 1, 1], 11)
    assert ei.value.status == 1
    bad = c2v.copy()
    bad[0, 0] = 10 ** 6
    with pytest.raises(H.FrError):
        H.mesh_geometry(3, xv, bad, [1, 1, 1], 2)
    flipped = c2v[:, [1, 0, 3, 2, 5, 4, 7, 6]]        # mirrored elements: negative Jacobian
    with pytest.raises(H.FrError):
        H.mesh_geometry(3, xv, flipped, [1, 1, 1], 2)


@pytest.mark.parametrize("case", ["iq_hex_tgv_p3_n3_jit", "iq_hex_tgv_p2_n3_jit_cub5", "iq_quad_vortex_p3_n6_jit_cub4"])
def test_default_volume_cubature_is_the_reference_rule(case):
    """The default rule (tensor Gauss-Legendre, full precision) is the rule the
    reference's cubature tables print to 12-15 digits, in its point order."""
    import json
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", case + ".npz"))
    meta = json.loads(str(z["meta"]))
    loc, w = H.volume_cubature(meta["dims"], meta["cub"])
    assert loc.shape == z["loc"].shape and w.shape == z["weight"].shape
    assert np.abs(loc - z["loc"]).max() <= 1e-12
    assert np.abs(w - z["weight"]).max() <= 1e-12
    assert abs(w.sum() - 2.0 ** meta["dims"]) <= 1e-13


def test_reference_cubature_table_reader(tmp_path):
    """read_reference_cubature parses the reference's data/cubature_*.dat layout."""
    loc, w = H.volume_cubature(2, 3)
    lines = ["rule=2", "locs(x)"] + ["0.1"] * 4 + ["locs(y)"] + ["0.2"] * 4 + ["weights"] + ["1.0"] * 4
    lines += ["rule=3", "locs(x)"] + ["%.15g" % x for x in loc[0]] + ["locs(y)"] + ["%.15g" % x for x in loc[1]]
    lines += ["weights"] + ["%.12g" % x for x in w]
    p = tmp_path / "cubature_quad.dat"
    p.write_text("\n".join(lines) + "\n")
    rl, rw = H.read_reference_cubature(str(p), 2, 3)
    assert np.abs(rl - loc).max() < 1e-14 and np.abs(rw - w).max() < 1e-11
    with pytest.raises(ValueError):
        H.volume_cubature(3, 13)
