"""Reference arm of bench.py: the reference's own CPU code on the host cores.

Runs the unmodified reference objects (oracle/_ref/ref_harness: the
reference's set-up, CalcResidual and eles::AdvanceSolution, with a wall clock
around its time-step loop) as independent processes, one per host thread (the
reference is single-threaded and MPI is not built).  `run` (bench.py --impl
reference) times the bench configuration itself; `measure` with a smaller box
is the bounded sample behind bench.py's cpu_baseline.  Throughput is the sum
over processes of DOF updates per RK stage per second.

TEST AND CPU-BASELINE INFRASTRUCTURE ONLY: never part of the product path.
"""
import json
import os
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "_ref", "ref_harness")


def _prepare(work, n, P, dt):
    import ref_inputs as R
    L = 2 * np.pi
    xv, c2v = R.box_vertices(3, (n, n, n), (0, 0, 0), (L, L, L))
    R.write_gambit(os.path.join(work, "mesh.neu"), 3, xv, c2v, (n, n, n))
    R.write_input(os.path.join(work, "input"), order=P, viscous=1, ic_form=1, dt=dt, n_steps=1,
                  dx_cyclic=L, dy_cyclic=L, dz_cyclic=L, vcjh_scheme_hexa=1, prandtl=0.71,
                  Mach_free_stream=0.1, Re_free_stream=1600.0)


def measure(n=10, P=3, steps=4, procs=None, dt=1e-3):
    """Aggregate DOF-updates/s of `procs` concurrent reference processes."""
    if not os.path.exists(HARNESS):
        raise FileNotFoundError("oracle/_ref/ref_harness is not built (make -C oracle REF=<reference checkout> ref)")
    procs = procs or os.cpu_count() or 1
    work = tempfile.mkdtemp(prefix="fr_refbench_")
    _prepare(work, n, P, dt)
    env = dict(os.environ, HIFILES_HOME=os.path.join(HERE, "_ref"), OMP_NUM_THREADS="1")
    ps = []
    t0 = time.time()
    for i in range(procs):
        out = os.path.join(work, "out%d" % i)
        os.makedirs(out, exist_ok=True)
        ps.append(subprocess.Popen([HARNESS, "input", out, "--ic", "tgv_mach01", "--steps", str(steps), "--no-dump"],
                                   cwd=work, env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    secs = []
    for p in ps:
        txt, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("reference run failed: " + txt[-500:])
        for line in txt.splitlines():
            if line.startswith("step_loop_seconds"):
                secs.append(float(line.split()[1]))
    wall = time.time() - t0
    E, nu, F = n ** 3, (P + 1) ** 3, 5
    dof = E * nu * F * 5 * steps
    per_proc = [dof / s for s in secs]
    return {"value": float(np.sum(per_proc)), "per_process": float(np.mean(per_proc)), "procs": procs,
            "sample": "reference CPU build (oracle/_ref, g++ -O3 -D_CPU -D_NO_BLAS), TGV P=3 NS on %d^3 periodic hexes, "
                      "%d RK45 steps per process, %d concurrent single-threaded processes (wall %.1f s)" %
                      (n, steps, procs, wall),
            "seconds": secs}


def host_cpu():
    """CPU model, logical and physical core counts of this host (from /proc/cpuinfo)."""
    model, phys = "unknown", set()
    try:
        cur = {}
        for line in open("/proc/cpuinfo"):
            if ":" not in line:
                if cur:
                    phys.add((cur.get("physical id"), cur.get("core id")))
                cur = {}
                continue
            k, v = [x.strip() for x in line.split(":", 1)]
            cur[k] = v
            if k == "model name":
                model = v
        if cur:
            phys.add((cur.get("physical id"), cur.get("core id")))
    except OSError:
        pass
    return {"model": model, "logical": os.cpu_count() or 1, "physical": len(phys) or None}


def mem_available_bytes():
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except OSError:
        pass
    return None


def run(a):
    """The reference arm on the bench configuration itself (TGV n^3, P=3):
    one single-threaded reference process per host thread, as many as the
    host memory holds (about 0.7 GB per 16^3 hexes per process, measured),
    each timing a.steps (at most 2) RK45 steps of the full mesh."""
    steps = max(1, min(a.steps, 2))
    need = 0.75e9 * (a.n / 16.0) ** 3
    avail = mem_available_bytes()
    procs = os.cpu_count() or 1
    if avail:
        procs = max(1, min(procs, int(0.8 * avail // need)))
    r = measure(n=a.n, P=a.order, steps=steps, procs=procs)
    cpu = host_cpu()
    r["sample"] += "; host %s, %d logical / %s physical cores" % (cpu["model"], cpu["logical"], cpu["physical"])
    out = {
        "impl": "reference", "metric": "RK-stage DOF-updates/s (TGV P=3)", "value": r["value"],
        "unit": "DOF-updates/s", "n_gpus": 0, "steps": steps, "warmup": 0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic TGV initial field)",
        "config": {"workload": "TGV %d^3 hex P=%d Navier-Stokes (Re 1600, Mach 0.1, Pr 0.71), Rusanov+LDG, c_dg, RK45"
                               % (a.n, a.order),
                   "sample": r["sample"], "same_config": True, "host_cpu": cpu},
        "cpu_baseline": {"value": r["value"], "unit": "DOF-updates/s", "cores": r["procs"], "kind": "reference",
                         "sample": r["sample"]},
        "e2e": {"value": r["value"], "unit": "DOF-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


if __name__ == "__main__":
    print(json.dumps(measure(n=6, steps=1, procs=2)))
