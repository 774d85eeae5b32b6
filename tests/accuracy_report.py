"""Accuracy of the B200 step against the float64 oracle, for the results
table: per-field relative L2 errors (eta, u, v, T, S and the density rho)
after one step on the 720x360x50 workload and after one simulated day (48
steps) on the same option set at 180x90x50.  Prints one JSON line.

Run on a machine with the GPU (the oracle runs on the host cores):
    python tests/accuracy_report.py
"""
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from oracle import params as oparams  # noqa: E402
from oracle import step as ostep  # noqa: E402
from zhenmode_b200 import make_solver_global, workloads  # noqa: E402

FIELDS = ("u", "v", "T", "S", "eta")


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run(nx, ny, nz, nsteps):
    import torch
    grid, physics, dt, kw, T, S = workloads.make_case("plain", nx, ny, nz, dtype="float32")
    step, init, _ = make_solver_global(grid, physics, dt, **kw)
    oo = {k: v for k, v in kw.items() if k in oparams.SUPPORTED}
    oo["dtype"] = "float64"
    p = oparams.build_params(grid, physics, dt, **oo)
    st = init(T, S)
    want = {k: getattr(st, k).cpu().numpy().astype(np.float64) for k in FIELDS}
    t0 = time.time()
    for _ in range(nsteps):
        want = ostep.step(dict(want), p)
    t_cpu = time.time() - t0
    got_st = step.advance(st, nsteps)
    got = {k: getattr(got_st, k).cpu().numpy() for k in FIELDS}
    err = {k: rel(got[k], want[k]) for k in FIELDS}
    err["rho"] = rel(ostep.density_anomaly(got["T"], got["S"], p) + 1025.0,
                     ostep.density_anomaly(want["T"], want["S"], p) + 1025.0)
    err["rho_anomaly"] = rel(ostep.density_anomaly(got["T"], got["S"], p), ostep.density_anomaly(want["T"], want["S"], p))
    return {"grid": f"{nx}x{ny}x{nz}", "steps": nsteps, "rel_l2": err, "oracle_s": round(t_cpu, 1)}


if __name__ == "__main__":
    out = {"one_step_720x360x50": run(720, 360, 50, 1), "one_day_180x90x50": run(180, 90, 50, 48)}
    print(json.dumps(out))
