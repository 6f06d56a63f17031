"""fr_residual_noalloc: the residual entry point for callers that cannot
allocate device memory when they need a residual (code recording work for
later replay, code living in someone else's memory pool, hosts that forbid
allocation after start-up).  It keeps its scratch in a fixed array inside the
library, so these checks compare it, through the C ABI, with the residual of
the allocating solver on the same mesh and state, on two calls in a row (the
second call reuses the scratch the first one left behind).

This file is collected last so that a run that stops at the first failure has
run everything else before it."""
import ctypes as C

import numpy as np
import pytest

import hifiles_b200 as H
import oracle as O
from golden_util import rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL = 1e-12     # the tolerance of the other residual parity tests


class PhysDesc(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("gamma", "prandtl", "mu_inf", "rt_inf", "c_sth", "fix_vis", "tau",
                                          "pen_fact")]


class ResidualArgs(C.Structure):
    _fields_ = [("dims", C.c_int), ("order", C.c_int), ("n_eles", C.c_int), ("viscous", C.c_int),
                ("upts_type", C.c_int), ("vcjh_scheme", C.c_int), ("eta", C.c_double), ("phys", PhysDesc),
                ("disu_upts", C.c_void_p), ("JGinv_upts", C.c_void_p), ("detjac_upts", C.c_void_p),
                ("norm_left", C.c_void_p), ("tdA_fpts", C.c_void_p), ("mate", C.c_void_p), ("side", C.c_void_p),
                ("n_int", C.c_longlong), ("face_lr", C.c_void_p), ("face_sign", C.c_void_p),
                ("div_tconf_upts", C.c_void_p)]


def _lib():
    L = H.lib()
    L.fr_residual_noalloc.restype = C.c_int
    L.fr_residual_noalloc.argtypes = [C.POINTER(ResidualArgs), C.c_void_p]
    return L


def _dev(a, dtype=torch.float64):
    a = np.asarray(a)
    return torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).to(dtype).cuda()


def _inputs(s):
    """Device copies of the solver's own set-up arrays in the ABI's layouts."""
    g = s.geometry()
    il, ir = s.interfaces()
    E, nf, D = s.n_eles, s.n_fpts, s.dims
    nrm = g["norm_fpts"].reshape(nf * E, D, order="F")
    mate = np.zeros(nf * E, dtype=np.int32)
    mate[il], mate[ir] = ir, il
    nL = np.zeros_like(nrm)
    nL[il], nL[ir] = nrm[il], nrm[il]
    n = nL[il]
    sgn = (n[:, 0] + n[:, 1]) if D == 2 else (n[:, 0] + n[:, 1] + np.sqrt(2.0) * n[:, 2])
    neg = (sgn < 0.0).astype(np.uint8)
    side = np.zeros(nf * E, dtype=np.uint8)
    side[il] = 1 | (neg << 1)
    side[ir] = neg << 1
    keep = dict(JG=_dev(g["JGinv_upts"]), dj=_dev(g["detjac_upts"]), tdA=_dev(g["tdA_fpts"]),
                nL=_dev(nL),
                mate=torch.from_numpy(mate).cuda(), side=torch.from_numpy(side).cuda(),
                face=torch.from_numpy(np.ascontiguousarray(np.stack([il, ir], axis=1).astype(np.int32))).cuda(),
                fsign=torch.from_numpy(neg).cuda())
    return keep, len(il)


def _args(s, meta, keep, n_int, u_dev, out_dev):
    ph = PhysDesc(meta["gamma"], meta["prandtl"], meta["mu_inf"], 1.0, 1.0, 1.0, meta["tau"], meta["pen_fact"])
    return ResidualArgs(s.dims, meta["order"], s.n_eles, int(meta["viscous"]), 0, meta["vcjh"], 0.0, ph,
                        u_dev.data_ptr(), keep["JG"].data_ptr(), keep["dj"].data_ptr(), keep["nL"].data_ptr(),
                        keep["tdA"].data_ptr(), keep["mate"].data_ptr(), keep["side"].data_ptr(), n_int,
                        keep["face"].data_ptr(), keep["fsign"].data_ptr(), out_dev.data_ptr())


# every (dims, order) the entry point is built for, Navier-Stokes and Euler,
# on small jittered periodic boxes
CASES = ([dict(dims=3, order=P, n=(3, 3, 2), lo=(0, 0, 0), hi=(2 * np.pi,) * 3, jitter=0.1, viscous=v, vcjh=1)
          for P in (1, 2, 3, 4) for v in (True, False)] +
         [dict(dims=2, order=P, n=(6, 5), lo=(-5, -5), hi=(5, 5), jitter=0.15, viscous=v, vcjh=2)
          for P in (1, 2, 3, 4, 5) for v in (True, False)])
IDS = ["%s_p%d_%s" % ("hex" if c["dims"] == 3 else "quad", c["order"], "ns" if c["viscous"] else "euler")
       for c in CASES]


@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_noalloc_residual_matches_solver_on_two_calls(case):
    meta = dict(case, gamma=1.4, prandtl=0.71, mu_inf=1.0 / 1600.0, tau=1.0, pen_fact=0.5)
    s = H.Solver.box(case["dims"], case["order"], case["n"], case["lo"], case["hi"], jitter=case["jitter"], seed=5,
                     viscous=case["viscous"], vcjh_scheme=case["vcjh"], gamma=1.4, prandtl=0.71,
                     mu_inf=1.0 / 1600.0, tau=1.0, pen_fact=0.5)
    pos = s.geometry()["pos_upts"]
    u = O.ic_tgv(pos) if case["dims"] == 3 else O.ic_vortex(pos)
    s.set_state(u)
    ref = s.residual()
    keep, n_int = _inputs(s)
    u_dev = _dev(u)
    L = _lib()
    for call in range(2):
        out = torch.full((u.size,), float("nan"), dtype=torch.float64, device="cuda")
        st = L.fr_residual_noalloc(C.byref(_args(s, meta, keep, n_int, u_dev, out)), None)
        assert st == 0, L.fr_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(u.shape, order="F")
        assert rel(got, ref) <= TOL, (call, rel(got, ref))


def test_noalloc_rejects_meshes_beyond_its_scratch():
    E = 2100                      # hex P=3 Navier-Stokes: ~17 kB of scratch per element
    small = torch.zeros(16, dtype=torch.float64, device="cuda")
    ints = torch.zeros(16, dtype=torch.int32, device="cuda")
    ph = PhysDesc(1.4, 0.71, 1e-3, 1.0, 1.0, 1.0, 1.0, 0.5)
    a = ResidualArgs(3, 3, E, 1, 0, 1, 0.0, ph, small.data_ptr(), small.data_ptr(), small.data_ptr(),
                     small.data_ptr(), small.data_ptr(), ints.data_ptr(), ints.data_ptr(), 1, ints.data_ptr(),
                     ints.data_ptr(), small.data_ptr())
    L = _lib()
    assert L.fr_residual_noalloc(C.byref(a), None) == 1
    assert "32 MiB" in L.fr_last_error().decode()
