"""The drop-in's host-side objects inside the reference's own runtime
modules, run from a ZhenMode source tree under the NumPy ``jax`` stand-in of
tests/golden/_jaxshim (no GPU needed):

* the params object that ``make_solver_global(..., return_params=True)``
  returns (zhenmode_b200.solver.B200Params) goes through the reference's
  restart fingerprint and contract (io/restart.py:34-75) and its projection
  provenance (dynamics/projection.py:53-62), as run.py:171-200 and
  io/output.py:89-96,184 use them;
* a drop-in JaxStateG of float32 host arrays (what ``step`` hands back for a
  host state) is saved and loaded by the reference's save_restart /
  load_restart (io/restart.py:153-227) with every byte kept.

The source tree is given by ``ZHENMODE_SRC`` (its ``src`` directory); the
tests are skipped without it.  Each runs in a child process so that the
stand-in ``jax`` never enters this test session.
"""
import os
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "tests", "golden", "_jaxshim")
SRC = os.environ.get("ZHENMODE_SRC")

pytestmark = pytest.mark.skipif(not SRC or not os.path.isdir(os.path.join(SRC or "", "zhenmode")),
                                reason="ZHENMODE_SRC (a ZhenMode source tree) not given")

PARAMS = textwrap.dedent("""
    import numpy as np
    from oracle import params as oparams
    from zhenmode_b200 import workloads
    from zhenmode_b200.solver import B200Params

    grid, physics, dt, kw, T, S = workloads.make_case("plain", 48, 24, 10, dtype="float32")
    okw = {k: v for k, v in kw.items() if k in oparams.SUPPORTED}
    okw["dtype"] = "float64"
    o = oparams.build_params(grid, physics, dt, **okw)
    wet3 = np.asarray(grid.wet_mask_3d, dtype=np.float32)
    params = B200Params(
        nx=48, ny=24, nz=10, dt=dt, dt_bt=dt / o.n_subcyc, mode_split=True, n_subcyc=int(o.n_subcyc),
        nu_nsub=int(o.n_subcyc), adv_nsub=int(o.adv_nsub), conv_nsub=int(o.conv_nsub), use_scan=True,
        H_sw=float(np.sum(grid.dz)), nu_h=physics.nu_h, nu_v=physics.nu_v, kappa_h=physics.kappa_h,
        kappa_v=physics.kappa_v, kappa_conv=physics.kappa_conv, nu_bi=physics.nu_bi, kappa_bi=physics.kappa_bi,
        T_ref=physics.T_ref, S_ref=physics.S_ref, r_bot=physics.r_bot, cd=physics.cd,
        bottom_friction=physics.bottom_friction, lambda_bulk=0.0, restore_coef_S=0.0, polar_cap_rows=2,
        polar_cap_taper=3, eta_relax_rate=0.0, freeze_adv_vel=False, conservative_kv=False,
        localize_conv=True, monotone_adv=False, fct_adv=True, project_adv_vel=False, projection_niter=150,
        projection_niter_source="default", projection_rtol=None, projection_preconditioner="none",
        projection_max_refinements=2, column_geometry="legacy", process_time_scheme="legacy",
        thermodynamics="linear", vertical_diffusion="explicit", dtype="float32",
        wet_mask=np.asarray(grid.wet_mask, dtype=np.float32), wet_mask_z=wet3)
""")


def _run(body, tmp_path):
    script = tmp_path / "case.py"
    script.write_text("import sys\nsys.path[:0] = [%r, %r, %r]\n" % (SHIM, SRC, ROOT) + PARAMS + body)
    proc = subprocess.run([sys.executable, str(script)], capture_output=True, text=True, timeout=300,
                          cwd=str(tmp_path))
    assert proc.returncode == 0, proc.stdout + proc.stderr
    return proc.stdout


def test_params_in_the_reference_fingerprint_and_projection_provenance(tmp_path):
    out = _run(textwrap.dedent("""
        from zhenmode.model.io.restart import fingerprint, make_restart_contract
        from zhenmode.model.solver.dynamics.projection import projection_config
        fp = fingerprint(params)
        assert fp["n_subcyc"] == params.n_subcyc and fp["wet_mask_z"]["shape"] == [48, 24, 10]
        cfg = projection_config(params)
        assert cfg["enabled"] is False and cfg["niter"] == 150 and cfg["niter_source"] == "default"
        contract = make_restart_contract(grid, params, dtype="float32", forcing={}, controls={},
                                         code_paths={}, execution={"backend": "cuda"})
        assert contract["state_shapes"]["T"] == [48, 24, 10] and contract["effective_params"] == fp
        print("ok", cfg["rtol"])
    """), tmp_path)
    assert out.startswith("ok")


def test_state_through_the_reference_restart_files(tmp_path):
    out = _run(textwrap.dedent("""
        from zhenmode.model.io.restart import load_restart, make_restart_contract, save_restart
        from zhenmode_b200 import JaxStateG
        rng = np.random.default_rng(3)
        shape = (48, 24, 10)
        state = JaxStateG(*(rng.standard_normal(shape).astype(np.float32) for _ in range(4)),
                          rng.standard_normal(shape[:2]).astype(np.float32), np.zeros(shape[:2], np.float32))
        contract = make_restart_contract(grid, params, dtype="float32", forcing={}, controls={},
                                         code_paths={}, execution={"backend": "cuda"})
        save_restart("ckpt.npz", state, contract, step=3, counters={}, cumulative={}, history={})
        back = load_restart("ckpt.npz", contract)
        for name in JaxStateG._fields:
            a, b = getattr(state, name), back.state[name]
            assert a.dtype == b.dtype and a.tobytes() == b.tobytes(), name
        print("ok")
    """), tmp_path)
    assert out.startswith("ok")
