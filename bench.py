#!/usr/bin/env python3
"""Throughput of the FR residual + RK45 stage on B200.

Workload: 3-D Taylor-Green vortex, compressible Navier-Stokes, periodic
[0, 2pi]^3 hex mesh of 32^3 elements at P=3 (64 solution points per element,
2.1 M points x 5 fields), Re 1600, Mach 0.1, Pr 0.71, Rusanov + LDG, c_dg
correction, low-storage RK45.  One bench step = one full RK45 step (5 stages);
the metric counts DOF updates per RK stage: n_eles * n_upts * n_fields * 5 per
step.  Data: synthetic (the analytic TGV initial field); the working set
(~1.2 GB) is larger than L2, so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--precision fp64|fp32] [--n 32] [--order 3]

Multi-GPU: one process per GPU (torchrun); every rank advances its own
replica of the mesh (weak scaling, no data-path collective); the time is the
max over ranks.  `--impl reference` times the reference's own CPU code
(oracle/_ref, built from the reference sources) on the host cores.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
for sub in ("hifiles-solver_b200", "oracle"):
    sys.path.insert(0, os.path.join(REPO, sub))

METRIC = "RK-stage DOF-updates/s (TGV P=3)"
GAMMA, MACH, RE, PR = 1.4, 0.1, 1600.0, 0.71


def tgv_state(pos):
    """TGV initial field, rho0 = U0 = 1, p0 = 1/(gamma M^2)."""
    x, y, z = pos[..., 0], pos[..., 1], pos[..., 2]
    p0 = 1.0 / (GAMMA * MACH * MACH)
    p = p0 + 1.0 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
    u = np.sin(x) * np.cos(y) * np.cos(z)
    v = -np.cos(x) * np.sin(y) * np.cos(z)
    return np.asfortranarray(np.stack([np.ones_like(x), u, v, np.zeros_like(x),
                                       p / (GAMMA - 1.0) + 0.5 * (u * u + v * v)], axis=-1))


# DRAM bytes per element of one RK stage (dram__bytes_read.sum +
# dram__bytes_write.sum of the gradient and interface/update kernels, summed
# over one stage), from the full-size ncu capture of the bench workload with
# these tiles (grad elements/CTA, threads, update elements/CTA, threads);
# profiles/dram_tgv32_p3_fp64.md gives the command and the per-kernel split.
MEASURED_TRAFFIC = {("fp64", 32, 3, (1, 64, 1, 96)): 53229}


def alg_bytes_per_element(dims, P, viscous, s=8, m=8, t=8):
    """Algorithmic HBM bytes per element per RK stage: state read+write and RK
    register read+write, metrics once (JGinv + detJ at solution points, normal +
    dA at flux points), and the face-trace exchange (each element writes its
    own traces and reads its neighbours': U at flux points, plus grad U when
    viscous)."""
    n1 = P + 1
    nu = n1 ** dims
    nf = 2 * dims * n1 ** (dims - 1)
    F = dims + 2
    v = 1 if viscous else 0
    return s * 4 * nu * F + m * (nu * (dims * dims + 1) + nf * (dims + 1)) + t * (2 * nf * F + v * 2 * nf * F * dims)


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        self.out.flush()
        rows = [r.split(",") for r in open(self.out.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.out.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for nm, flag in zip(names, r[5:9]):
                    if flag.strip().lower() in ("active", "1", "yes"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(x, world, device="cpu"):
    """Max of a per-rank scalar over all ranks (the time of the slowest rank)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_value(dof_per_step_per_rank, ms_per_step_max, world):
    """Whole-job throughput: every rank advances its own replica, the job takes
    as long as the slowest rank."""
    return dof_per_step_per_rank * world / (ms_per_step_max * 1e-3)


def peaks():
    try:
        return json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json"))), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def cpu_baseline_port(n=12, P=3, steps=2):
    """The oracle (plain-C restatement, one core) on a bounded sample of the workload."""
    import oracle as O
    m = O.Mesh.box(3, P, (n, n, n), (0, 0, 0), (2 * np.pi,) * 3, vcjh_scheme=1)
    ph = O.physics(viscous=1, gamma=GAMMA, prandtl=PR, mu_inf=1.0 / RE, tau=1.0, pen_fact=0.5)
    u0 = tgv_state(m.geometry()["pos_upts"])
    t0 = time.perf_counter()
    m.rk45(ph, u0, 1e-3, steps, norms=False)
    dt = time.perf_counter() - t0
    dof = m.n_eles * m.n_upts * m.n_fields * 5 * steps
    return {"value": dof / dt, "unit": "DOF-updates/s", "cores": 1, "kind": "port",
            "sample": "oracle (C restatement), TGV P=3 NS on %d^3 hexes, %d RK45 steps, 1 thread, %.1f s" % (n, steps, dt)}


def cpu_baseline(a):
    """The reference's own CPU code (oracle/_ref) on all host cores, bounded
    sample; the plain-C oracle on one core if the reference build is absent."""
    try:
        import bench_reference
        r = bench_reference.measure(n=10, P=a.order, steps=2)
        return {"value": r["value"], "unit": "DOF-updates/s", "cores": r["procs"], "kind": "reference",
                "sample": r["sample"]}
    except (FileNotFoundError, RuntimeError, OSError):
        return cpu_baseline_port()


BATCH_SEED, BATCH_N = 2024, 64


def batch_instances(precision):
    """The batched configuration: 64 periodic TGV instances (NS, Mach 0.1,
    Re 1600) with seeded sizes n^3, n in [8, 24], and orders P in [2, 4]."""
    rng = np.random.default_rng(BATCH_SEED)
    L = 2 * np.pi
    out = []
    for _ in range(BATCH_N):
        n, P = int(rng.integers(8, 25)), int(rng.integers(2, 5))
        out.append(dict(dims=3, order=P, n=(n, n, n), lo=(0, 0, 0), hi=(L, L, L), viscous=True, vcjh_scheme=1,
                        gamma=GAMMA, prandtl=PR, mu_inf=1.0 / RE, tau=1.0, pen_fact=0.5, precision=precision))
    return out


def box_upts(n, P, L):
    """Solution-point positions (n_upts, n_eles, 3) of the uniform periodic
    box of n^3 hexes: element i + n (j + n k), point a + (P+1)(b + (P+1) c)."""
    import hifiles_b200 as H
    loc = H.line_operators(P)["loc"]
    h = L / n
    x1 = ((np.arange(n)[:, None] + 0.5 * (loc[None, :] + 1.0)) * h)        # [cell, point]
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    e_i, e_j, e_k = i.transpose(2, 1, 0).ravel(), j.transpose(2, 1, 0).ravel(), k.transpose(2, 1, 0).ravel()
    a, b, c = np.meshgrid(np.arange(P + 1), np.arange(P + 1), np.arange(P + 1), indexing="ij")
    pa, pb, pc = a.transpose(2, 1, 0).ravel(), b.transpose(2, 1, 0).ravel(), c.transpose(2, 1, 0).ravel()
    pos = np.empty(((P + 1) ** 3, n ** 3, 3), order="F")
    pos[:, :, 0] = x1[e_i[None, :], pa[:, None]]
    pos[:, :, 1] = x1[e_j[None, :], pb[:, None]]
    pos[:, :, 2] = x1[e_k[None, :], pc[:, None]]
    return pos


def _time_steps(advance, stream, steps):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    advance(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def ke_decay(s64, s32, u0, dt, steps, every):
    """Config 2's kinetic-energy decay in the FP32 form against FP64 (the
    kinetic energy on the reference's volume cubature every `every` steps)."""
    series = {}
    for name, s in (("fp64", s64), ("fp32", s32)):
        s.set_state(u0)
        ke = [s.kinetic_energy()]
        for _ in range(steps // every):
            s.advance(every, dt)
            ke.append(s.kinetic_energy())
        series[name] = ke
    k64, k32 = np.array(series["fp64"]), np.array(series["fp32"])
    return {"steps": steps, "every": every, "dt": dt, "ke_fp64": k64.tolist(),
            "max_rel_error": float(np.max(np.abs(k32 - k64) / np.abs(k64))),
            "decay_fp64": float(1.0 - k64[-1] / k64[0]), "decay_fp32": float(1.0 - k32[-1] / k32[0])}


def measure_forms(a, dev, fp64_value, s64, u0):
    """The precision and batching forms beside the FP64 headline: the FP32
    form on the same workload with its L2 error against the FP64 path after 20
    steps, and the 64-instance batch in FP64 and FP32 (one CUDA graph per
    step, autotuned tiles per group)."""
    import torch
    import hifiles_b200 as H
    n, P, L = a.n, a.order, 2 * np.pi
    dt, steps = 1e-3, max(5, min(a.steps, 20))
    s32 = H.Solver.box(3, P, (n, n, n), (0, 0, 0), (L, L, L), viscous=True, vcjh_scheme=1, gamma=GAMMA, prandtl=PR,
                       mu_inf=1.0 / RE, rt_inf=1.0, c_sth=1.0, fix_vis=1.0, tau=1.0, pen_fact=0.5, precision=1,
                       device=dev)
    s32.set_state(u0)
    s32.autotune(3)
    st32 = torch.cuda.ExternalStream(s32.stream(), device=dev)
    s32.advance(3, dt)
    ms32 = _time_steps(lambda k: s32.advance(k, dt), st32, steps)
    dof_step = s32.n_eles * s32.n_upts * s32.n_fields * 5
    s64.set_state(u0)
    s32.set_state(u0)
    s64.advance(20, dt)
    s32.advance(20, dt)
    u64, u32 = s64.get_state(), s32.get_state()
    l2 = float(np.linalg.norm(u32 - u64) / np.linalg.norm(u64))
    ke = ke_decay(s64, s32, u0, dt, 200, 10)
    s32.close()
    out = {"fp32": {"value": dof_step / (ms32 * 1e-3), "ms_per_step": ms32, "l2_rel_vs_fp64_after_20_steps": l2,
                    "ratio_to_fp64": dof_step / (ms32 * 1e-3) / fp64_value},
           "ke_decay_fp32_vs_fp64": ke}
    for prec, name in ((0, "batched_fp64"), (1, "batched_fp32")):
        insts = batch_instances(prec)
        t0 = time.perf_counter()
        b = H.Batch(insts, device=dev)
        setup_s = time.perf_counter() - t0
        states = []
        for i, inst in enumerate(insts):
            b.set_state(i, tgv_state(box_upts(inst["n"][0], inst["order"], L)))
        b.autotune(2)
        chosen = b.merged
        stb = torch.cuda.ExternalStream(b.stream(), device=dev)
        # each launch form timed on the same state: per-group launches, merged
        # launches with registers capped for 4 and for 3 CTAs per SM
        forms = {}
        for label, on, minb in (("per_group", 0, 4), ("merged_minb4", 1, 4), ("merged_minb3", 1, 3)):
            for i, inst in enumerate(insts):
                b.set_state(i, tgv_state(box_upts(inst["n"][0], inst["order"], L)))
            b.set_merged(on, minb)
            b.advance(3, dt)
            l0 = b.launch_count()
            ms_f = _time_steps(lambda k: b.advance(k, dt), stb, steps)
            forms[label] = {"ms_per_step": ms_f, "launches_per_step": (b.launch_count() - l0) // steps}
        best = ("merged_minb%d" % chosen) if chosen else "per_group"
        msb, launches_per_step = forms[best]["ms_per_step"], forms[best]["launches_per_step"]
        v = b.dof() * 5 / (msb * 1e-3)
        out[name] = {"value": v, "ms_per_step": msb, "ratio_to_fp64": v / fp64_value, "groups": b.n_groups,
                     "launches_per_step": launches_per_step, "graphs_per_step": 1, "setup_s": setup_s,
                     "autotuned_launch_form": best, "launch_forms": forms}
        b.close()
    out["batch"] = ("%d periodic TGV instances (NS, Mach 0.1, Re 1600), sizes n^3 with n in [8, 24] and P in "
                    "[2, 4] drawn with seed %d; DOF-updates per RK stage over all instances" % (BATCH_N, BATCH_SEED))
    out["operator_path"] = measure_operator_path(a, dev, s64, u0)
    out["tgv64_p4"] = measure_tgv64_p4(dev)
    out["mixed_channel"] = {"p%d" % P: measure_mixed_channel(P) for P in (2, 3)}
    return out


# Channel flow at Mach 0.1, Re 1600 in the reference's non-dimensional units
# (what its input processing makes of Mach_free_stream 0.1, Re_free_stream
# 1600, T_wall = T_free_stream, free stream along x): the physics and the
# boundary values of bdy_inters::set_bdy_params, in that order.
CHANNEL_PHYSICS = {"gamma": 1.4, "prandtl": 0.71, "mu_inf": 0.000625, "rt_inf": 69.32142857142854,
                   "c_sth": 0.41215868109222054, "fix_vis": 1.0, "tau": 1.0, "pen_fact": 0.5}
CHANNEL_BDY = [1.0, 1.0, 0.0, 0.0, 71.4285714285714, 0.0, 0.0, 0.0, 1.0, 71.92982267888384, 1.002, 1.0, 0.0, 0.0]
CHANNEL_R_REF = 71.42857142857142


def channel_state(pos):
    """Smooth non-uniform flow at the Mach 0.1 free stream (rho = 1, u = 1,
    p = 1 / (gamma M^2)) at points pos (n, E, 3): the synthetic initial field
    of the channel runs."""
    x, y, z = pos[..., 0], pos[..., 1], pos[..., 2]
    p0 = 1.0 / (GAMMA * 0.01)
    rho = 1.0 + 0.05 * np.sin(x) * np.cos(y)
    u, v, w = 1.0 + 0.1 * np.sin(y), 0.1 * np.cos(x), 0.05 * np.sin(x + y + z)
    p = p0 * (1.0 + 0.01 * np.cos(x + y))
    q = np.stack([rho, rho * u, rho * v, rho * w, p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v + w * w)], -1)
    return np.asfortranarray(q)


def measure_mixed_channel(order, n=(40, 20, 20), steps=3, err_steps=10, dt=2e-4):
    """The mixed-element channel: 40 x 20 x 20 cells on [0, 2 pi] x [0, 2] x
    [0, pi], interior vertices jittered by up to +-0.15 h (seed 2024), the
    first and last cell layer in y extruded as prisms (two per cell), six tets
    per core cell, periodic in x and z, an isothermal wall at y = 0 and an
    adiabatic one at y = 2 on the prisms' triangular faces.  Set up by the
    library (operators, metrics, wiring: hifiles_b200.mixed) and advanced
    through the fr_op_* entry points with FP64 operator products on the FP64
    tensor cores (fp64) or the CUDA cores and BF16x3 / BF16x6 split products
    on the tcgen05 tensor cores, with their
    L2 error against FP64 after `err_steps` steps; and by the fused stage
    (fr_mixed_stage_*, FP64 tensor-core products), against the per-operator
    FP64 path."""
    import torch
    from hifiles_b200 import mixed as X
    from hifiles_b200 import seam
    t0 = time.time()
    xv, cells, period, bfaces = X.channel_mesh(n)
    M = X.MixedMesh(order, xv, cells, period, bfaces,
                    X.ElementOpts(vcjh_scheme_tet=2, vcjh_scheme_tri=1, vcjh_scheme_pri_1d=1))
    setup_s = time.time() - t0
    types, ints, bdys = M.operator_inputs({t: channel_state(m["pos_upts"]) for t, m in M.types.items()})
    m = seam.MixedOperatorMesh(types, ints, CHANNEL_PHYSICS, bdys, CHANNEL_BDY, CHANNEL_R_REF)
    u0 = {i: m.S[i]["u"].clone() for i in m.S}

    def reset():
        for i, s in m.S.items():
            s["u"].copy_(u0[i])
            s["reg"].zero_()

    res = {}
    for mode, name in ((0, "fp64"), (3, "fp64_cuda_cores"), (1, "bf16x3"), (2, "bf16x6")):
        reset()
        m.advance(1, dt, gemm_precision=mode)
        ms = _time_steps(lambda k: m.advance(k, dt, gemm_precision=mode), m.stream, steps)
        res[name] = {"value": m.dofs * 5 / (ms * 1e-3), "ms_per_step": ms}
    def l2(a, b):
        num = sum(float(torch.linalg.vector_norm(a[i] - b[i]) ** 2) for i in a)
        return (num / sum(float(torch.linalg.vector_norm(b[i]) ** 2) for i in b)) ** 0.5

    # one residual of the initial state, and the state after err_steps steps
    reset()
    m.residual(0)
    torch.cuda.synchronize()
    div0 = {i: s["div"].clone() for i, s in m.S.items()}
    m.advance(err_steps, dt, gemm_precision=0)
    torch.cuda.synchronize()
    ref = {i: s["u"].clone() for i, s in m.S.items()}
    for mode, name in ((3, "fp64_cuda_cores"), (1, "bf16x3"), (2, "bf16x6")):
        reset()
        m.residual(mode)
        torch.cuda.synchronize()
        res[name]["residual_l2_rel_vs_fp64"] = l2({i: s["div"] for i, s in m.S.items()}, div0)
        reset()
        m.advance(err_steps, dt, gemm_precision=mode)
        torch.cuda.synchronize()
        res[name]["l2_rel_vs_fp64_after_%d_steps" % err_steps] = l2({i: s["u"] for i, s in m.S.items()}, ref)
    finite = all(bool(torch.isfinite(s["u"]).all()) for s in m.S.values())
    # the fused stage (fr_mixed_stage_*): two kernels per element type and RK
    # stage, FP64 tensor-core products; launch shapes autotuned
    f = seam.FusedMixedMesh(types, ints, CHANNEL_PHYSICS, bdys, CHANNEL_BDY, CHANNEL_R_REF)
    shapes = f.autotune()
    f.residual()
    torch.cuda.synchronize()
    fres = {"residual_l2_rel_vs_operator_path": l2({i: s["div"] for i, s in f.S.items()}, div0)}
    u0f = {i: s["u"].clone() for i, s in f.S.items()}
    f.advance(1, dt)
    ms = _time_steps(lambda k: f.advance(k, dt), f.stream, steps)
    # operator-product flops of one stage (gradient kernel: [opp_4 | opp_5],
    # opp_6, [opp_1], [opp_2]; update kernel: opp_3, opp_0), 5 fields
    flops = 0.0
    for s_ in f.S.values():
        nu, nf, E = s_["nu"], s_["nf"], s_["E"]
        D = 3
        mac = 3 * nu * (nu + nf) * 5 + nf * nu * D * 5 + (nf + nu) * D * nu * 5 + 2 * nu * nf * 5
        flops += 2.0 * mac * E
    fres.update({"value": f.dofs * 5 / (ms * 1e-3), "ms_per_step": ms, "launches_per_stage": f.launches_per_stage,
                 "launch_shapes": {str(i): list(v) for i, v in shapes.items()},
                 "operator_tflops": flops * 5 / (ms * 1e-3) / 1e12,
                 "operator_flops_per_stage": flops})
    for i, s in f.S.items():
        s["u"].copy_(u0f[i])
    f.advance(err_steps, dt)
    torch.cuda.synchronize()
    fres["l2_rel_vs_operator_path_after_%d_steps" % err_steps] = l2({i: s["u"] for i, s in f.S.items()}, ref)
    res["fused_fp64"] = fres
    finite = finite and all(bool(torch.isfinite(s["u"]).all()) for s in f.S.values())
    del f
    ne = {X.TET: 0, X.PRISM: 0}
    ne.update({t: int(v["n_eles"]) for t, v in M.types.items()})
    res["workload"] = ("channel %s cells of order %d: %d tets, %d prisms, %d DOFs, jitter 0.15 h; dt %g; one step = 5 "
                       "RK stages of CalcResidual (fp64/bf16x*: the fr_op_* entry points; fused_fp64: fr_mixed_stage_*)" %
                       ("x".join(str(v) for v in n), order, ne[X.TET], ne[X.PRISM], m.dofs, dt))
    res["host_setup_s"] = setup_s
    res["finite_after_error_run"] = finite
    del m
    torch.cuda.empty_cache()
    return res


def measure_channel_fused(order, steps, warmup, n=(40, 20, 20), dt=2e-4, shapes=None):
    """The channel of measure_mixed_channel through the fused stage alone
    (fr_mixed_stage_*): launch shapes autotuned, or `shapes` ("g,u" for every
    element type) for profile captures."""
    import torch
    from hifiles_b200 import mixed as X
    from hifiles_b200 import seam
    xv, cells, period, bfaces = X.channel_mesh(n)
    # the SD-like tet correction is tabulated for orders 2 and 3; DG elsewhere
    M = X.MixedMesh(order, xv, cells, period, bfaces,
                    X.ElementOpts(vcjh_scheme_tet=2 if order in (2, 3) else 1, vcjh_scheme_tri=1,
                                  vcjh_scheme_pri_1d=1))
    types, ints, bdys = M.operator_inputs({t: channel_state(m["pos_upts"]) for t, m in M.types.items()})
    f = seam.FusedMixedMesh(types, ints, CHANNEL_PHYSICS, bdys, CHANNEL_BDY, CHANNEL_R_REF)
    if shapes:
        g, u = (int(v) for v in shapes.split(","))
        for i in f.S:
            f.set_launch(i, g, u)
    else:
        f.autotune()
    f.advance(warmup, dt)
    ms = _time_steps(lambda k: f.advance(k, dt), f.stream, steps)
    return {"workload": "channel %s order %d, fused stage" % ("x".join(str(v) for v in n), order),
            "n_eles": {str(t): int(m["n_eles"]) for t, m in M.types.items()}, "dofs": f.dofs,
            "ms_per_step": ms, "value": f.dofs * 5 / (ms * 1e-3), "unit": "DOF-updates/s",
            "launch_shapes": {str(i): list(f.launch(i)) for i in f.S}, "launches_per_stage": f.launches_per_stage}


def measure_tgv64_p4(dev, n=64, P=4, steps=100, dt=2e-4):
    """The precision sweep on TGV 64^3 hexes at P = 4 (32.8 M points x 5
    fields, 1.3 GB per FP64 state): FP64 and FP32 forms of the fused path,
    DOF-updates/s, and the L2 error of FP32 against FP64 after 100 steps."""
    import torch
    import hifiles_b200 as H
    L = 2 * np.pi
    kw = dict(viscous=True, vcjh_scheme=1, gamma=GAMMA, prandtl=PR, mu_inf=1.0 / RE, rt_inf=1.0, c_sth=1.0,
              fix_vis=1.0, tau=1.0, pen_fact=0.5, device=dev)
    out, states = {}, {}
    for prec, name in ((0, "fp64"), (1, "fp32")):
        s = H.Solver.box(3, P, (n, n, n), (0, 0, 0), (L, L, L), precision=prec, **kw)
        u0 = tgv_state(s.geometry()["pos_upts"])
        s.set_state(u0)
        s.autotune(3)
        st = torch.cuda.ExternalStream(s.stream(), device=dev)
        s.advance(3, dt)
        ms = _time_steps(lambda k: s.advance(k, dt), st, 10)
        out[name] = {"value": s.n_eles * s.n_upts * s.n_fields * 5 / (ms * 1e-3), "ms_per_step": ms}
        s.set_state(u0)
        s.advance(steps, dt)
        states[name] = s.get_state()
        s.close()
        del s
        torch.cuda.empty_cache()
    out["fp32"]["ratio_to_fp64"] = out["fp32"]["value"] / out["fp64"]["value"]
    out["fp32"]["l2_rel_vs_fp64_after_%d_steps" % steps] = float(
        np.linalg.norm(states["fp32"] - states["fp64"]) / np.linalg.norm(states["fp64"]))
    del states
    # BF16x3 operator products on the tensor cores, through the per-operator path
    from hifiles_b200 import seam
    s = H.Solver.box(3, P, (n, n, n), (0, 0, 0), (L, L, L), precision=0, **kw)
    u0 = tgv_state(s.geometry()["pos_upts"])
    phys = dict(gamma=GAMMA, prandtl=PR, mu_inf=1.0 / RE, rt_inf=1.0, c_sth=1.0, fix_vis=1.0, tau=1.0, pen_fact=0.5)
    op = seam.OperatorStage(s, phys, P, vcjh_scheme=1)
    nb = 20
    u_tc = {}
    for mode, name in ((1, "bf16x3_operator_path"), (2, "bf16x6_operator_path")):
        op.set_state(u0)
        op.advance(1, dt, gemm_precision=mode)
        ms = _time_steps(lambda k: op.advance(k, dt, gemm_precision=mode), op.stream, 2)
        out[name] = {"value": s.n_eles * s.n_upts * s.n_fields * 5 / (ms * 1e-3), "ms_per_step": ms}
        op.set_state(u0)
        op.advance(nb, dt, gemm_precision=mode)
        u_tc[name] = op.get_state()
    del op
    torch.cuda.empty_cache()
    s.set_state(u0)
    s.advance(nb, dt)
    u_ref = s.get_state()
    s.close()
    for name, u in u_tc.items():
        out[name]["l2_rel_vs_fp64_after_%d_steps" % nb] = float(np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref))
    out["workload"] = ("TGV %d^3 hex P=%d NS (Re 1600, Mach 0.1), dt %g; fused path in FP64 and FP32; BF16x3 and "
                       "BF16x6 split operator products on the tensor cores through the per-operator path (its "
                       "P = 4 operators, up to 150 x 150, take two 128-row MMA tiles)" % (n, P, dt))
    return out


def measure_operator_path(a, dev, s64, u0):
    """The reference's residual as per-operator calls (dense opp_0 .. opp_6
    over all elements, pointer-table interface kernels): FP64 operator products
    on the FP64 tensor cores (default) and on the CUDA cores against the BF16
    split products on the tcgen05 tensor cores, same workload, with the L2
    error of each form against the first after 20 steps, and the
    extrapolation product alone (opp_0 U) in every form."""
    import ctypes
    import torch
    from hifiles_b200 import seam
    dt, steps = 1e-3, 3
    phys = dict(gamma=GAMMA, prandtl=PR, mu_inf=1.0 / RE, rt_inf=1.0, c_sth=1.0, fix_vis=1.0, tau=1.0, pen_fact=0.5)
    op = seam.OperatorStage(s64, phys, a.order, vcjh_scheme=1)
    dof_step = op.E * op.nu * op.F * 5
    res = {}
    modes = ((0, "fp64"), (3, "fp64_cuda_cores"), (1, "bf16x3"), (2, "bf16x6"))
    for mode, name in modes:
        op.set_state(u0)
        op.advance(1, dt, gemm_precision=mode)
        ms = _time_steps(lambda k: op.advance(k, dt, gemm_precision=mode), op.stream, steps)
        res[name] = {"value": dof_step / (ms * 1e-3), "ms_per_step": ms}
    op.set_state(u0)
    op.advance(20, dt, gemm_precision=0)
    u_ref = op.get_state()
    for mode, name in modes[1:]:
        op.set_state(u0)
        op.advance(20, dt, gemm_precision=mode)
        u_tc = op.get_state()
        res[name]["l2_rel_vs_fp64_after_20_steps"] = float(np.linalg.norm(u_tc - u_ref) / np.linalg.norm(u_ref))
        res[name]["l2_rel_of_change_after_20_steps"] = float(np.linalg.norm(u_tc - u_ref) /
                                                             np.linalg.norm(u_ref - u0))
    # the extrapolation product opp_0 U alone (HBM-bound: U read, U_f written, FP64)
    L = op.L
    m, k, ncols = op.nf, op.nu, op.F * op.E
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for mode, name in modes:
        L.fr_op_set_gemm_precision(mode)
        for it in range(4):
            if it == 1:
                e0.record(op.stream)
            L.fr_op_extrapolate_solution(m, k, op.F, op.E, op._ops["opp_0"].data_ptr(), op.u.data_ptr(),
                                         op.ufp.data_ptr(), ctypes.c_void_p(op.stream.cuda_stream))
        e1.record(op.stream)
        e1.synchronize()
        L.fr_op_set_gemm_precision(0)
        t = e0.elapsed_time(e1) / 3 * 1e-3
        bytes_ = 8.0 * (k + m) * ncols
        flops = 2.0 * m * k * ncols * {0: 1, 3: 1, 1: 3, 2: 6}[mode]
        res[name]["opp_0_product"] = {"ms": t * 1e3, "GB/s": bytes_ / t / 1e9, "TFLOP/s": flops / t / 1e12}
    res["workload"] = ("same TGV mesh and state; one step = 5 RK stages of CalcResidual through the fr_op_* "
                       "entry points; operator products in FP64 on the FP64 tensor cores (fp64) or the CUDA "
                       "cores, or BF16x3 / BF16x6 split products on the tcgen05 tensor cores with FP32 "
                       "accumulation")
    del op
    torch.cuda.empty_cache()
    return res


def run_b200(a, rank, world, local):
    import torch
    import hifiles_b200 as H
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = local
    n, P = a.n, a.order
    L = 2 * np.pi
    s = H.Solver.box(3, P, (n, n, n), (0, 0, 0), (L, L, L), viscous=True, vcjh_scheme=1, gamma=GAMMA, prandtl=PR,
                     mu_inf=1.0 / RE, rt_inf=1.0, c_sth=1.0, fix_vis=1.0, tau=1.0, pen_fact=0.5,
                     precision=1 if a.precision == "fp32" else 0, device=dev)
    u0 = tgv_state(s.geometry()["pos_upts"])
    s.set_state(u0)
    if a.tiles:
        g, u = (int(x) for x in a.tiles.split(","))
        s.select_tiles(g, u)
        ti = s.tile_info(0, g), s.tile_info(1, u)
        tiles = (ti[0][0], ti[0][1], ti[1][0], ti[1][1])
    else:
        tiles = s.autotune(5) if not a.no_tune else None
    dt = 1e-3
    E, nu, F = s.n_eles, s.n_upts, s.n_fields
    dof_step = E * nu * F * 5
    stream = torch.cuda.ExternalStream(s.stream(), device=dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def rank_max(x):
        return max_over_ranks(x, world, "cuda:%d" % dev)

    # --- device-resident throughput (graph-replayed RK45 steps)
    s.advance(max(a.warmup, 3), dt)
    s.sync()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = s.launch_count()
    with Clocks(dev) as clk:
        torch.cuda.synchronize(dev)
        ev0.record(stream)
        s.advance(a.steps, dt)
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize(dev)
    launches = s.launch_count() - l0
    ms = ev0.elapsed_time(ev1) / a.steps
    barrier()
    ms = rank_max(ms)
    value = aggregate_value(dof_step, ms, world)

    # --- per-kernel event timing for the roofline (stage by stage, not replayed)
    ms_grad, ms_face, ms_upd = s.profile_stage(10, dt)
    stage_ms = ms_grad + ms_face + ms_upd
    pk, pk_src = peaks()
    tc = 4 if a.precision == "fp32" else 8
    b_elem = alg_bytes_per_element(3, P, True, s=8, m=tc, t=tc)
    achieved = b_elem * E / (stage_ms * 1e-3) / 1e9
    # DRAM bytes of one stage from an ncu capture of the same kernels and tiles
    # (MEASURED_TRAFFIC); null when this run's autotuner picked other tiles
    key = (a.precision, n, P, tuple(tiles) if tiles else None)
    traffic = MEASURED_TRAFFIC[key] * E if key in MEASURED_TRAFFIC else None

    # --- end to end through the public API with host buffers
    pinned = torch.empty(u0.size, dtype=torch.float64, pin_memory=True)
    host_u = pinned.numpy().reshape(u0.shape, order="F")
    host_u[...] = u0
    s.set_state(host_u)
    s.advance(1, dt, norms=True)
    torch.cuda.synchronize(dev)
    barrier()
    e2e_steps = max(1, a.steps)
    norms_pinned = torch.empty((e2e_steps, F), dtype=torch.float64, pin_memory=True).numpy()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(e2e_steps):
        # each step: its state uploaded from pinned host memory (on the copy
        # stream, overlapping the step before) and its residual norms read back
        s.set_state_async(host_u)
        s.advance_async(1, dt, norms_pinned[i])
    e1.record(stream)
    e1.synchronize()
    wall = (time.perf_counter() - t0) / e2e_steps
    if not np.isfinite(norms_pinned).all():
        raise RuntimeError("non-finite residual norms in the end-to-end run")
    e2e_ms = rank_max(max(e0.elapsed_time(e1) / e2e_steps, wall * 1e3))
    e2e = {"value": aggregate_value(dof_step, e2e_ms, world), "unit": "DOF-updates/s",
           "h2d_bytes_per_step": int(u0.size * 8), "d2h_bytes_per_step": int(F * 8),
           "ms_per_step": e2e_ms,
           "path": ("Solver.set_state_async(pinned host state) + Solver.advance_async(1 step, norms to pinned "
                    "host memory) -> C ABI; each step's upload overlaps the step before")}

    forms = measure_forms(a, dev, value / world, s, u0) if (world == 1 and not a.no_forms) else None
    cpu = cpu_baseline(a) if (rank == 0 and world == 1 and not a.no_cpu) else None
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    out = {
        "metric": METRIC, "value": value, "unit": "DOF-updates/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if a.precision == "fp64" else "f32 (f64 state/RK/reductions)",
        "data": "synthetic (analytic TGV initial field)",
        "config": {"workload": "TGV %d^3 hex P=%d Navier-Stokes (Re 1600, Mach 0.1, Pr 0.71), Rusanov+LDG, "
                               "c_dg, RK45; 1 step = 5 RK stages" % (n, P),
                   "n_eles": E, "n_upts": nu, "n_fields": F, "dof_per_stage": E * nu * F,
                   "precision": a.precision, "l2": "inputs larger than L2 (working set ~%.2f GB)" %
                                                    ((E * nu * F * 8 * 2 + E * 96 * F * tc * 2 + E * 96 * 15 * tc +
                                                      E * nu * 10 * tc) / 1e9),
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "tiles": {"grad_elements_per_cta": tiles[0], "grad_threads": tiles[1],
                             "update_elements_per_cta": tiles[2], "update_threads": tiles[3]} if tiles else None},
        "roofline": {"bound": "hbm", "kernel": "one RK stage = fr_grad_kernel + fr_face_update_kernel",
                     "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / pk["hbm_gbs"], "peak_source": pk_src,
                     "alg_bytes_per_element": b_elem, "traffic": traffic,
                     "ms_grad": ms_grad, "ms_face_update": ms_upd, "ms_stage": stage_ms,
                     "traffic_source": ("ncu capture, tiles %s" % (key[3],)) if traffic else
                     "no ncu capture of this run's tiles"},
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(),
        "forms": forms,
    }
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--n", type=int, default=32)
    ap.add_argument("--order", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--tiles", default="", help="gradient,update tile indices instead of autotuning (for captures)")
    ap.add_argument("--no-forms", action="store_true", help="skip the FP32 and batched forms")
    ap.add_argument("--channel-fused", type=int, default=0, metavar="P",
                    help="only the 40x20x20 tet/prism channel of order P through the fused stage (one JSON line)")
    ap.add_argument("--shapes", default="", help="with --channel-fused: gradient,update launch shapes")
    ap.add_argument("--channel-n", default="40,20,20", help="with --channel-fused: cells in x, y, z")
    a = ap.parse_args()
    if a.channel_fused:
        n = tuple(int(v) for v in a.channel_n.split(","))
        print(json.dumps(measure_channel_fused(a.channel_fused, a.steps, a.warmup, n=n, shapes=a.shapes or None)))
        return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if a.impl == "reference":
        if rank != 0:
            return
        import bench_reference
        bench_reference.run(a)
        return
    run_b200(a, rank, world, local)


if __name__ == "__main__":
    main()
