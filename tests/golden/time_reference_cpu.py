"""Time ZhenMode's own step code on the host cores at a given grid, next to the
float64 restatement (``oracle/``) on the same inputs, to check that the
restatement's speed stands in for the reference's in the CPU baseline.

    python tests/golden/time_reference_cpu.py --src <zhenmode-checkout>/src \
        [--grid 720x360x50] [--warmup 3] [--steps 5] [--which reference|port|both]

The reference modules run unmodified under the NumPy-backed ``jax`` stand-in
of ``tests/golden/_jaxshim`` (float64, eager; JAX is not installed here), with
the 0.5-degree plain option set of the benchmark workload.  Following the
reference's own step timing (execution/profiling.py:76-85), the first
``--warmup`` steps are discarded and the median of the next ``--steps`` is
reported.  Prints one JSON line per timed implementation.
"""
from __future__ import annotations

import dataclasses
import json
import os
import platform
import statistics
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _arg(name, default):
    return sys.argv[sys.argv.index(name) + 1] if name in sys.argv else default


def _median_step(step, state, warmup, steps):
    for _ in range(warmup):
        state = step(state)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        state = step(state)
        times.append(time.perf_counter() - t0)
    return statistics.median(times), times


def _host():
    return {"cores_available": len(os.sched_getaffinity(0)), "cpu": platform.processor() or platform.machine(),
            "threads_env": {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS")}}


def time_port(nx, ny, nz, warmup, steps):
    sys.path.insert(0, ROOT)
    from oracle import params as oparams
    from oracle import step as ostep
    from zhenmode_b200 import workloads
    grid, physics, dt, kw, T, S = workloads.make_case("plain", nx, ny, nz, dtype="float64")
    p = oparams.build_params(grid, physics, dt, **{k: v for k, v in kw.items() if k in oparams.SUPPORTED})
    st = oparams.init_state(p, T, S)
    med, times = _median_step(lambda s: ostep.step(s, p), st, warmup, steps)
    return {"impl": "port (oracle/, float64 NumPy)", "grid": f"{nx}x{ny}x{nz}", "warmup": warmup,
            "median_s_per_step": med, "steps_s": times, "host": _host()}


def time_reference(src, nx, ny, nz, warmup, steps):
    import numpy as np
    sys.path[:0] = [os.path.join(HERE, "_jaxshim"), src, ROOT]
    import zhenmode.model.config as ref_config
    from zhenmode.model.solver.factory import make_solver_global

    from zhenmode_b200 import workloads
    grid, physics, dt, kw, T, S = workloads.make_case("plain", nx, ny, nz, dtype="float64")
    phys = ref_config.PhysicsConfig(**{f.name: getattr(physics, f.name) for f in dataclasses.fields(physics)})
    step, init, _ = make_solver_global(grid, phys, dt, **kw)
    st = init(T_init=np.asarray(T), S_init=np.asarray(S))
    med, times = _median_step(step, st, warmup, steps)
    return {"impl": "reference source, NumPy shim (float64)", "grid": f"{nx}x{ny}x{nz}", "warmup": warmup,
            "median_s_per_step": med, "steps_s": times, "host": _host()}


def main():
    nx, ny, nz = (int(x) for x in _arg("--grid", "720x360x50").split("x"))
    warmup, steps = int(_arg("--warmup", "3")), int(_arg("--steps", "5"))
    which = _arg("--which", "both")
    if which in ("port", "both"):
        print(json.dumps(time_port(nx, ny, nz, warmup, steps)), flush=True)
    if which in ("reference", "both"):
        src = _arg("--src", os.environ.get("ZHENMODE_SRC"))
        if not src:
            raise SystemExit("time_reference_cpu.py: give the ZhenMode source tree with --src <path>/src")
        print(json.dumps(time_reference(src, nx, ny, nz, warmup, steps)), flush=True)


if __name__ == "__main__":
    main()
