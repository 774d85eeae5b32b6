"""Drop-in ``make_solver_global`` for the B200 global ocean step.

Mirrors ``make_solver_global`` of ``src/zhenmode/model/solver/factory.py:30-799``
for the production mode-split path: same positional/keyword arguments, the
same ``ValueError`` on invalid configurations raised before any array is
built, and the same return arity ``(step, init_state, diagnostics[, params,
terms_fn][, step_dyn])`` (factory.py:793-799).  ``step`` accepts and returns a
``JaxStateG`` whose arrays are either CUDA ``torch`` tensors (device-resident,
stream ordered on torch's current stream) or NumPy arrays (host path).

The arithmetic runs in the CUDA library ``libzm_b200.so`` (float32 fields,
float64 barotropic mode); options that path does not implement raise
:class:`UnsupportedOption` (a ``ValueError``).
"""
from __future__ import annotations

import collections
import ctypes
import dataclasses
import math
import numbers
import os

import numpy as np

from . import _native
from .config import C_P, RHO_0

JaxStateG = collections.namedtuple("JaxStateG", ["u", "v", "T", "S", "eta", "ice"])
JaxStateG.__new__.__defaults__ = (0.0,)


class UnsupportedOption(ValueError):
    """A reference option the B200 path does not implement (C-ABI status 2)."""


# Effective settings of a built step under the reference's FDPhysParams field
# names (src/zhenmode/model/solver/state.py), for the callers of
# ``make_solver_global(..., return_params=True)``: the run reporting
# (runtime/reporting.py:22-25), the output provenance (io/output.py:89-96,
# projection_config of dynamics/projection.py:53-62), the restart contract's
# fingerprint (io/restart.py:34-51, 56-75) and the budget audit
# (zhenmode_b200.ledger.make_budget_step).  Every field is a number, string,
# flag, None or host array, so the reference's fingerprint() takes it as it
# is; the step itself is attached as the attribute ``step``, outside the
# fields.
_PARAM_FIELDS = (
    "nx", "ny", "nz", "dt", "dt_bt", "mode_split", "n_subcyc", "nu_nsub", "adv_nsub", "conv_nsub", "use_scan",
    "H_sw", "nu_h", "nu_v", "kappa_h", "kappa_v", "kappa_conv", "nu_bi", "kappa_bi", "T_ref", "S_ref",
    "r_bot", "cd", "bottom_friction", "lambda_bulk", "restore_coef_S", "polar_cap_rows", "polar_cap_taper",
    "eta_relax_rate", "freeze_adv_vel", "conservative_kv", "localize_conv", "monotone_adv", "fct_adv",
    "project_adv_vel", "projection_niter", "projection_niter_source", "projection_rtol",
    "projection_preconditioner", "projection_max_refinements", "column_geometry", "process_time_scheme",
    "thermodynamics", "vertical_diffusion", "dtype", "wet_mask", "wet_mask_z")


class B200Params(collections.namedtuple("B200Params", _PARAM_FIELDS)):
    """Effective parameters of one B200 step (see _PARAM_FIELDS)."""


def _finite(name, value, *, positive=False, nonnegative=False):
    """config.py finite_number: a finite real scalar with an optional sign."""
    if isinstance(value, bool) or not isinstance(value, numbers.Real) or not math.isfinite(float(value)):
        raise ValueError(f"{name} must be a finite number")
    if positive and value <= 0:
        raise ValueError(f"{name} must be positive")
    if nonnegative and value < 0:
        raise ValueError(f"{name} must be nonnegative")


def _count(name, value, minimum=0):
    """config.py integer_count."""
    if isinstance(value, (bool, np.bool_)) or not isinstance(value, (int, np.integer)) or value < minimum:
        raise ValueError(f"{name} must be an integer >= {minimum}")


_DEFAULTS = dict(
    external_mode_scheme='forward_backward', meridional_boundary_scheme='clamped_nodes',
    pressure_continuity_scheme='centered_second', tracer_transport_scheme='centered_second',
    hydrostatic_surface_scheme='reference_plane', density_rotation_scheme='split_sources',
    vertical_tracer_scheme='donor_cell', hydrostatic_integral_scheme='trapezoidal',
    column_mean_scheme='nodal_capacity', tracer_flux_arithmetic='legacy',
    momentum_vertical_velocity_scheme='dual_face_v1', material_point_gradient_scheme='minmod_v1',
    momentum_tangent_filter_scheme='binomial_v1', column_geometry='legacy',
    process_time_scheme='legacy')

_KNOWN = dict(
    external_mode_scheme=('forward_backward', 'symmetric'),
    meridional_boundary_scheme=('clamped_nodes', 'closed_faces'),
    pressure_continuity_scheme=('centered_second', 'centered_fourth'),
    tracer_transport_scheme=('centered_second', 'product_fourth', 'paired_product_fourth'),
    hydrostatic_surface_scheme=('reference_plane', 'linear_density'),
    density_rotation_scheme=('split_sources', 'joint_shear'),
    vertical_tracer_scheme=('donor_cell', 'muscl_nodal_v1', 'muscl_endpoint_v2', 'muscl_band_v3',
                            'material_point_v4'),
    hydrostatic_integral_scheme=('trapezoidal', 'cubic_uniform_v1'),
    column_mean_scheme=('nodal_capacity', 'cubic_consistent_v1'),
    tracer_flux_arithmetic=('legacy', 'integrated_reference_v1'),
    momentum_vertical_velocity_scheme=('dual_face_v1', 'point_primitive_v1'),
    material_point_gradient_scheme=('minmod_v1', 'fourth_uniform_v1'),
    momentum_tangent_filter_scheme=('binomial_v1', 'gram_fourth_v1'),
    column_geometry=('legacy', 'nodal_dual_v1', 'fixed_partial_v1'),
    process_time_scheme=('legacy', 'consistent_split_v1', 'subcycled_rk2_v2', 'symmetric_fast_v3'))


def _validate_grid(grid):
    """grid.py:384-398 validate_grid."""
    for name in ("nx", "ny", "nz"):
        _count(name, getattr(grid, name), minimum=2)
    _finite("dy", grid.dy, positive=True)
    widths = np.asarray(grid.dx_2d, dtype=np.float64)
    depths = np.asarray(grid.z, dtype=np.float64)
    spacing = np.asarray(grid.dz, dtype=np.float64)
    if widths.shape != (grid.nx, grid.ny) or not np.all(np.isfinite(widths) & (widths > 0.)):
        raise ValueError("dx_2d must have grid shape and positive finite spacing")
    if depths.shape != (grid.nz,) or not np.all(np.isfinite(depths)) or not np.all(np.diff(depths) < 0.):
        raise ValueError("z must contain finite, strictly descending nodes")
    if (spacing.shape != (grid.nz - 1,) or not np.all(np.isfinite(spacing) & (spacing > 0.))
            or not np.allclose(spacing, -np.diff(depths), rtol=1e-12, atol=0.)):
        raise ValueError("dz must match the positive distances between z nodes")


def _f64(a, shape=None):
    out = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if shape is not None and out.shape != shape:
        raise ValueError(f"expected an array of shape {shape}, got {out.shape}")
    return out


class _Solver:
    """Owns one native solver handle and the host arrays handed to it."""

    def __init__(self, grid, physics, dt, opts):
        self.lib = _native.load()
        nx, ny, nz = int(grid.nx), int(grid.ny), int(grid.nz)
        self.shape = (nx, ny, nz)
        keep = []

        def arr(a, shape):
            if a is None:
                return None
            out = _f64(a, shape)
            keep.append(out)
            return out

        g = _native.ZmGrid()
        g.nx, g.ny, g.nz = nx, ny, nz
        g.dy = float(grid.dy)
        for name, value, shape in (("dx_2d", grid.dx_2d, (nx, ny)), ("cos_lat", grid.cos_lat, (ny,)),
                                   ("f", grid.f, (nx, ny)), ("z", grid.z, (nz,)), ("dz", grid.dz, (nz - 1,)),
                                   ("wet_mask", grid.wet_mask, (nx, ny))):
            setattr(g, name, _native.dptr(arr(value, shape)))
        wet3 = getattr(grid, "wet_mask_3d", None)
        g.wet_mask_3d = _native.dptr(arr(wet3, (nx, ny, nz))) if wet3 is not None else None

        p = _native.ZmParams()
        p.dt = float(dt)
        p.dt_bt = float(opts["dt_bt"])
        for name in ("nu_h", "nu_v", "kappa_h", "kappa_v", "kappa_conv", "nu_bi", "kappa_bi", "T_ref",
                     "S_ref", "r_bot"):
            setattr(p, name, float(getattr(physics, name)))
        p.lambda_bulk = opts["lambda_bulk"]
        p.restore_coef_S = opts["restore_coef_S"]
        p.ice_salt_flux = float(opts["ice_salt_flux"])
        p.ice_freeze_temp_c = float(opts["ice_freeze_temp_c"])
        p.nu_nsub = int(opts["nu_nsub"] or 0)
        p.polar_cap_rows = int(opts["polar_cap_rows"])
        p.polar_cap_taper = int(opts["polar_cap_taper"])
        p.limiter = 2 if opts["fct_adv"] else (1 if opts["monotone_adv"] else 0)
        p.localize_conv = int(bool(opts["localize_conv"]))
        p.conservative_kv = int(bool(opts["conservative_kv"]))
        p.freeze_adv_vel = int(bool(opts["freeze_adv_vel"]))
        p.vertical_diffusion = 1 if opts["vertical_diffusion"] == "implicit" else 0
        p.bt_kernel = _BT_KERNELS[opts["barotropic_kernel"]]
        p.autotune = 1 if opts.get("autotune") else 0
        p.project_adv_vel = int(bool(opts.get("project_adv_vel", False)))
        p.projection_niter = int(opts.get("projection_niter", 150))
        p.projection_preconditioner = 1 if opts.get("projection_preconditioner", "none") == "jacobi" else 0
        p.projection_max_refinements = int(opts.get("projection_max_refinements", 2))
        p.projection_rtol = float(opts.get("projection_rtol", 0.0))
        p.eta_relax_rate = float(opts.get("eta_relax_rate", 0.0))
        sizes = {"sponge_rate": (nx, ny), "T_clim": (nx, ny, nz), "S_clim": (nx, ny, nz), "eta_relax_mask": (nx, ny)}
        for name, shape in sizes.items():
            setattr(p, name, _native.dptr(arr(opts["fields"].get(name), shape)))
        for name in ("tau_x", "tau_y", "q_heat", "t_atm", "s_ref", "coastal_restore_coef",
                     "coastal_restore_t", "coastal_bulk_lambda", "coastal_kappa_h", "coastal_kappa_v"):
            setattr(p, name, _native.dptr(arr(opts["fields"].get(name), (nx, ny))))
        self._keep = keep
        handle = ctypes.c_void_p()
        rc = self.lib.zm_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(handle))
        if rc == _native.ZM_ERR_UNSUPPORTED:
            raise UnsupportedOption("configuration not supported by the B200 step (see stderr)")
        if rc == _native.ZM_ERR_INVALID:
            raise ValueError("invalid configuration (see stderr)")
        if rc != _native.ZM_OK:
            raise RuntimeError(f"zm_create failed with status {rc}")
        self.handle = handle
        info = (ctypes.c_int32 * 11)()
        self.lib.zm_info(handle, info, 11)
        (self.n_subcyc, self.n_nu, self.adv_nsub, self.conv_nsub, self.pitch, self.mib, _,
         self.bt_blocks, self.bt_cap_active, self.nu_halo, self.fft_lines) = list(info)

    def tuned_shapes(self):
        """(nu_h halo width, FFT lines per block) in use."""
        info = (ctypes.c_int32 * 11)()
        self.lib.zm_info(self.handle, info, 11)
        return int(info[9]), int(info[10])

    def launch_shapes(self):
        """Every launch shape the autotuner chooses, by name."""
        info = (ctypes.c_int32 * 16)()
        self.lib.zm_info(self.handle, info, 16)
        return {"nu_h_subcycles_per_pass": int(info[9]), "nu_h_warps_per_tile": int(info[15]),
                "fft_lines_per_block": int(info[10]),
                "tracer_adv_levels_per_block": int(info[11]), "linear_finish_levels_per_block": int(info[12]),
                "fz_tile_rows": int(info[13]), "pgf_tile_rows": int(info[14])}

    def kernels_per_step(self):
        info = (ctypes.c_int32 * 7)()
        self.lib.zm_info(self.handle, info, 7)
        return int(info[6])

    def profile(self, stream=None):
        """Per-class (ms, launches) of one un-graphed step of the resident state."""
        n = len(_native.KERNEL_CLASSES)
        ms = (ctypes.c_float * n)()
        cnt = (ctypes.c_int32 * n)()
        self.check(self.lib.zm_profile(self.handle, ctypes.c_void_p(stream or 0), ms, cnt, n), "zm_profile")
        return {name: (float(ms[i]), int(cnt[i])) for i, name in enumerate(_native.KERNEL_CLASSES)}

    def check(self, rc, what):
        if rc != _native.ZM_OK:
            msg = self.lib.zm_last_error(self.handle)
            raise RuntimeError(f"{what} failed (status {rc}): {msg.decode() if msg else ''}")

    def __del__(self):
        handle = getattr(self, "handle", None)
        if handle:
            self.lib.zm_destroy(handle)
            self.handle = None


def _torch_state_ptrs(state, shape):
    import torch
    nx, ny, nz = shape
    fields = []
    for name, want in (("u", shape), ("v", shape), ("T", shape), ("S", shape), ("eta", (nx, ny))):
        t = getattr(state, name)
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32
                and tuple(t.shape) == want and t.is_contiguous()):
            raise ValueError(f"state.{name} must be a contiguous CUDA float32 tensor of shape {want}")
        fields.append(t)
    return fields


_BT_KERNELS = {'auto': 0, 'resident': 1, 'streaming': 2}


@dataclasses.dataclass(frozen=True)
class BudgetDiagnostics:
    """Global tracer/volume diagnostics of one snapshot, with the fields of the
    reference's ``BudgetDiagnostics`` (diagnostics/snapshot.py:16-40)."""
    mean_T: float
    mean_S: float
    mean_T_top: float
    mean_S_top: float
    heat_content_J: float
    salt_content_kg: float
    total_volume_m3: float
    mean_depth_m: float

    def as_dict(self):
        return dataclasses.asdict(self)


def _device_fields(state, shape):
    """(CUDA float32 tensors u, v, T, S, eta; True if the state was on the host)."""
    import torch
    if isinstance(state.u, torch.Tensor):
        return _torch_state_ptrs(state, shape), False
    dev = torch.device('cuda')
    fields = [torch.as_tensor(np.ascontiguousarray(getattr(state, k), dtype=np.float32), device=dev)
              for k in ("u", "v", "T", "S", "eta")]
    return _torch_state_ptrs(JaxStateG(*fields, None), shape), True


def compute_budget_diagnostics(state, grid=None, rho0=RHO_0, cp=None, *, column_geometry="legacy",
                               thermodynamics="linear", solver):
    """Heat/salt/volume snapshot (diagnostics/snapshot.py:67-128) on the GPU.

    ``solver`` is a step returned by :func:`make_solver_global` for ``grid``;
    its grid defines the areas, node thicknesses and wet mask.  The sums are
    compensated float64 in a fixed order.
    """
    if thermodynamics != "linear":
        raise UnsupportedOption("only the linear snapshot thermodynamics is implemented on the B200 path")
    if column_geometry != "legacy":
        raise UnsupportedOption("only the legacy column geometry is implemented on the B200 path")
    return solver.budget_diagnostics(state, rho0=rho0, cp=cp)


def make_solver_global(grid, physics, dt, forcing=None,
                       T_atm=None, lambda_bulk=0.0,
                       mixed_layer_depth_m=None, mixed_layer_mask=None,
                       mixed_layer_depth_2d=None,
                       ice_freeze_temp_c=-1.8, ice_salt_flux=0.0,
                       dynamic_ice=False, ice_insulation_scale_m=1.0,
                       S_ref_surf=None, sss_restore_days=0.0,
                       coastal_restore_mask=None, coastal_restore_days=0.0,
                       coastal_bulk_mask=None, coastal_bulk_lambda=0.0,
                       coastal_kappa_h_mask=None, coastal_kappa_h=0.0,
                       coastal_kappa_v_mask=None, coastal_kappa_v=0.0,
                       coastal_restore_T=None,
                       sponge_days=0.0, sponge_cells=0,
                       T_init=None, S_init=None,
                       polar_cap_rows=2, polar_cap_taper=3, return_params=False,
                       eta_relax_days=0.0, eta_relax_box=None,
                       eta_relax_buffer=1.0, dynamic_forcing=False,
                       mode_split=False, dt_bt=150.0, nu_nsub=None,
                       dtype='float64', use_scan=False, freeze_adv_vel=False,
                       conservative_kv=False, project_adv_vel=False,
                       localize_conv=False, monotone_adv=False,
                       fct_adv=False, projection_niter=None,
                       projection_rtol=None, projection_preconditioner='none',
                       projection_max_refinements=2, column_geometry='legacy',
                       match_barotropic_transport=False, process_time_scheme='legacy',
                       eos_pressure_dbar=None, surface_pressure_pa=None,
                       vertical_diffusion='explicit', barotropic_kernel='auto', autotune=False, **schemes):
    """Build the B200 step; the argument list is the reference factory's.

    Two options are not the reference's: ``vertical_diffusion='implicit'``
    replaces the explicit L-step vertical diffusion by a per-column
    backward-Euler solve, and ``barotropic_kernel`` ('auto', 'resident',
    'streaming') picks the CUDA kernels of the barotropic subcycle (same
    arithmetic; 'auto' takes the resident kernel when the grid fits), and
    ``autotune=True`` times the launch shapes that change no result (nu_h halo
    width, FFT lines per block) at the first step and keeps the fastest.
    """
    # ---- validation, in the reference's order where it matters (factory.py:166-395)
    _finite('dt', dt, positive=True)
    _finite('dt_bt', dt_bt, positive=True)
    for name, value in schemes.items():
        if name not in _KNOWN:
            raise TypeError(f"make_solver_global() got an unexpected keyword argument '{name}'")
        if value not in _KNOWN[name]:
            raise ValueError(f"unknown {name}")
    for name in ('column_geometry', 'process_time_scheme'):
        value = locals()[name]
        if value not in _KNOWN[name]:
            raise ValueError(f"unknown {name}")
    _validate_grid(grid)
    if dtype not in {'float32', 'float64'}:
        raise ValueError('dtype must be float32 or float64')
    if physics.thermodynamics not in {'linear', 'teos10_reference'}:
        raise ValueError('unknown thermodynamics definition')
    if physics.thermodynamics == 'linear' and eos_pressure_dbar is not None:
        raise ValueError('linear EOS does not accept an unused TEOS pressure field')
    for name in ('nu_h', 'nu_v', 'nu_bi', 'kappa_h', 'kappa_v', 'kappa_bi', 'kappa_conv', 'kappa_gm',
                 'kappa_redi', 'r_bot', 'cd'):
        _finite(name, getattr(physics, name), nonnegative=True)
    for name, value in (('lambda_bulk', lambda_bulk), ('sss_restore_days', sss_restore_days),
                        ('coastal_restore_days', coastal_restore_days), ('coastal_bulk_lambda', coastal_bulk_lambda),
                        ('coastal_kappa_h', coastal_kappa_h), ('coastal_kappa_v', coastal_kappa_v),
                        ('sponge_days', sponge_days), ('eta_relax_days', eta_relax_days)):
        _finite(name, value, nonnegative=True)
    for name, value in (('polar_cap_rows', polar_cap_rows), ('polar_cap_taper', polar_cap_taper),
                        ('sponge_cells', sponge_cells)):
        _count(name, value)
    if nu_nsub is not None and not (isinstance(nu_nsub, str) and nu_nsub == 'cfl'):
        _count('nu_nsub', nu_nsub, minimum=1)
    if match_barotropic_transport and (not mode_split or column_geometry not in {'nodal_dual_v1', 'fixed_partial_v1'}):
        raise ValueError("match_barotropic_transport requires mode_split=True and reference column geometry")
    if process_time_scheme != 'legacy' and not match_barotropic_transport:
        raise ValueError(f"{process_time_scheme} requires match_barotropic_transport=True")
    if column_geometry in {'nodal_dual_v1', 'fixed_partial_v1'} and (not conservative_kv or not localize_conv):
        raise ValueError("reference column geometry requires conservative_kv=True and localize_conv=True")
    if polar_cap_rows > 0 and 2 * (polar_cap_rows + polar_cap_taper) > grid.ny:
        raise ValueError('polar cap bands must not overlap; reduce rows/taper or disable the cap')
    projection_niter_source = 'explicit'
    if projection_niter is None:
        # factory.py:368-376: the legacy environment cap, resolved once here
        legacy_cap = os.environ.get('OCEAN_PAV_NITER')
        try:
            projection_niter = 150 if legacy_cap is None else int(legacy_cap)
        except ValueError as error:
            raise ValueError('projection_niter environment value must be an integer') from error
        projection_niter_source = 'default' if legacy_cap is None else 'environment:OCEAN_PAV_NITER'
    if (isinstance(projection_niter, (bool, np.bool_)) or not isinstance(projection_niter, (int, np.integer))
            or projection_niter <= 0):
        raise ValueError('projection_niter must be a positive integer')
    if projection_rtol is not None and (not np.isfinite(projection_rtol) or projection_rtol <= 0.):
        raise ValueError('projection_rtol must be finite and positive')
    if projection_preconditioner not in {'none', 'jacobi'}:
        raise ValueError('projection_preconditioner must be none or jacobi')
    if (isinstance(projection_max_refinements, (bool, np.bool_))
            or not isinstance(projection_max_refinements, (int, np.integer))
            or not 0 <= projection_max_refinements <= 2):
        raise ValueError('projection_max_refinements must be an integer from 0 to 2')
    if mixed_layer_depth_m is not None and (not np.isfinite(mixed_layer_depth_m) or mixed_layer_depth_m < 0.):
        raise ValueError("mixed_layer_depth_m must be finite and nonnegative")
    if vertical_diffusion not in ('explicit', 'implicit'):
        raise ValueError("vertical_diffusion must be 'explicit' or 'implicit'")
    if barotropic_kernel not in _BT_KERNELS:
        raise ValueError("barotropic_kernel must be 'auto', 'resident' or 'streaming'")
    nx, ny, nz = int(grid.nx), int(grid.ny), int(grid.nz)
    if surface_pressure_pa is not None:
        load = np.asarray(surface_pressure_pa)
        if load.shape != (nx, ny) or not np.isfinite(load).all():
            raise ValueError('surface pressure must be a finite (nx, ny) Pa field')

    # ---- options outside the B200 path
    unsupported = []
    if not mode_split:
        unsupported.append('mode_split=False (monolithic free surface)')
    if dtype != 'float32':
        unsupported.append("dtype='float64' (the B200 step computes in float32)")
    if column_geometry != 'legacy' or process_time_scheme != 'legacy' or match_barotropic_transport:
        unsupported.append('non-legacy column geometry or process time scheme')
    if any(schemes.get(k, v) != v for k, v in _DEFAULTS.items() if k in schemes):
        unsupported.append('non-default numerical scheme options')
    if physics.thermodynamics != 'linear':
        unsupported.append('TEOS-10 thermodynamics')
    if physics.kappa_gm > 0 or physics.kappa_redi > 0:
        unsupported.append('GM/Redi closure')
    if physics.bottom_friction != 'linear':
        unsupported.append('quadratic bottom drag')
    if dynamic_ice:
        unsupported.append('dynamic ice')
    if (mixed_layer_depth_m or 0.0) > 0.0 or mixed_layer_depth_2d is not None:
        unsupported.append('mixed-layer heat deposition')
    if surface_pressure_pa is not None:
        unsupported.append('surface pressure load')
    if nz > 64:
        unsupported.append('more than 64 levels')
    if unsupported:
        raise UnsupportedOption('not implemented on the B200 path: ' + '; '.join(unsupported))

    # ---- derived host fields (factory.py:397-457)
    shape2 = (nx, ny)
    if forcing is None:
        tau_x = tau_y = q_heat = None
    else:
        tau_x, tau_y, q_heat = (_f64(a, shape2) for a in forcing)
    fields = dict(tau_x=tau_x, tau_y=tau_y, q_heat=q_heat)
    if T_atm is not None and lambda_bulk > 0.0:
        fields['t_atm'] = _f64(T_atm, shape2)
    else:
        lambda_bulk = 0.0
    restore_coef_S = 0.0
    if S_ref_surf is not None and sss_restore_days > 0.0:
        fields['s_ref'] = _f64(S_ref_surf, shape2)
        restore_coef_S = 1.0 / (sss_restore_days * 86400.0)

    def coastal(mask, coefficient):
        return _f64(mask, shape2) * coefficient if mask is not None and coefficient > 0.0 else None

    fields['coastal_kappa_v'] = coastal(coastal_kappa_v_mask, coastal_kappa_v)
    fields['coastal_kappa_h'] = coastal(coastal_kappa_h_mask, coastal_kappa_h)
    fields['coastal_bulk_lambda'] = coastal(coastal_bulk_mask, coastal_bulk_lambda)
    if coastal_restore_mask is not None and coastal_restore_days > 0.0 and coastal_restore_T is not None:
        fields['coastal_restore_coef'] = _f64(coastal_restore_mask, shape2) / (coastal_restore_days * 86400.0)
        fields['coastal_restore_t'] = _f64(coastal_restore_T, shape2)
    # lateral sponge: cosine taper from the polar edge rows (factory.py:456-491)
    if sponge_days > 0.0 and sponge_cells > 0:
        edge = np.minimum(np.arange(ny), ny - 1 - np.arange(ny))
        band = edge < int(sponge_cells)
        taper = np.where(band, 0.5 * (1.0 + np.cos(np.pi * edge / int(sponge_cells))), 0.0)
        fields['sponge_rate'] = np.ascontiguousarray(
            np.broadcast_to(taper[None, :] / (sponge_days * 86400.0), (nx, ny)))
        wm3 = np.asarray(getattr(grid, 'wet_mask_3d', None) if getattr(grid, 'wet_mask_3d', None) is not None
                         else np.broadcast_to(np.asarray(grid.wet_mask)[:, :, None], (nx, ny, nz)), dtype=np.float64)
        if T_init is not None:
            T_clim = np.asarray(T_init, dtype=np.float64) * wm3 + (1.0 - wm3) * physics.T_ref
            S_clim = (np.asarray(S_init, dtype=np.float64) if S_init is not None
                      else np.full((nx, ny, nz), float(physics.S_ref)))
            S_clim = S_clim * wm3 + (1.0 - wm3) * physics.S_ref
        else:  # init_state fills T_ref / S_ref: the target that leaves the sponge a no-op
            T_clim = np.full((nx, ny, nz), float(physics.T_ref))
            S_clim = np.full((nx, ny, nz), float(physics.S_ref))
        fields['T_clim'] = np.ascontiguousarray(T_clim)
        fields['S_clim'] = np.ascontiguousarray(S_clim)
    # semi-enclosed-sea eta relaxation box with a cosine buffer (factory.py:493-521)
    eta_relax_rate = 0.0
    if eta_relax_days > 0.0 and eta_relax_box is not None:
        lon0, lon1, lat0, lat1 = eta_relax_box
        lon2d, lat2d = np.meshgrid(np.asarray(grid.lon, dtype=np.float64), np.asarray(grid.lat, dtype=np.float64),
                                   indexing='ij')
        core = (lon2d >= lon0) & (lon2d <= lon1) & (lat2d >= lat0) & (lat2d <= lat1)
        d_out = np.maximum(np.maximum(np.maximum(lon0 - lon2d, lon2d - lon1), 0.0),
                           np.maximum(np.maximum(lat0 - lat2d, lat2d - lat1), 0.0))
        buf = float(eta_relax_buffer)
        mask = np.where(core, 1.0, np.where(d_out < buf, 0.5 * (1.0 + np.cos(np.pi * d_out / buf)), 0.0))
        fields['eta_relax_mask'] = mask * np.asarray(grid.wet_mask, dtype=np.float64)
        eta_relax_rate = 1.0 / (eta_relax_days * 86400.0)
    if nu_nsub == 'cfl':
        inv_dx2_max = float(np.max(np.asarray(grid.dx_2d, dtype=np.float64) ** -2))
        nu_nsub = max(1, int(np.ceil(physics.nu_h * (dt / 2.0) * (inv_dx2_max + 1.0 / float(grid.dy) ** 2) / 0.25)))
    opts = dict(dt_bt=dt_bt, lambda_bulk=float(lambda_bulk), restore_coef_S=restore_coef_S,
                ice_salt_flux=ice_salt_flux, ice_freeze_temp_c=ice_freeze_temp_c, nu_nsub=nu_nsub,
                polar_cap_rows=polar_cap_rows, polar_cap_taper=polar_cap_taper, fct_adv=fct_adv,
                monotone_adv=monotone_adv, localize_conv=localize_conv, conservative_kv=conservative_kv,
                freeze_adv_vel=freeze_adv_vel, vertical_diffusion=vertical_diffusion,
                barotropic_kernel=barotropic_kernel, autotune=bool(autotune), fields=fields,
                project_adv_vel=bool(project_adv_vel), projection_niter=int(projection_niter),
                projection_preconditioner=projection_preconditioner,
                projection_max_refinements=int(projection_max_refinements),
                projection_rtol=0.0 if projection_rtol is None else float(projection_rtol),
                eta_relax_rate=eta_relax_rate)
    solver = _Solver(grid, physics, dt, opts)
    wet3 = np.asarray(getattr(grid, 'wet_mask_3d', None) if getattr(grid, 'wet_mask_3d', None) is not None
                      else np.broadcast_to(np.asarray(grid.wet_mask)[:, :, None], (nx, ny, nz)), dtype=np.float64)
    T_ref, S_ref = float(physics.T_ref), float(physics.S_ref)

    def _run(state, nsteps):
        import torch
        if isinstance(state.u, np.ndarray):
            host = [np.ascontiguousarray(getattr(state, k), dtype=np.float32) for k in ("u", "v", "T", "S", "eta")]
            out = [np.empty_like(a) for a in host]
            sin = _native.ZmState(*[a.ctypes.data for a in host])
            sout = _native.ZmState(*[a.ctypes.data for a in out])
            solver.check(solver.lib.zm_step_host(solver.handle, None, ctypes.byref(sin), ctypes.byref(sout),
                                                 int(nsteps)), "zm_step_host")
            return JaxStateG(*out, state.ice)
        fin = _torch_state_ptrs(state, solver.shape)
        out = [torch.empty_like(t) for t in fin]
        stream = torch.cuda.current_stream(fin[0].device).cuda_stream
        sin = _native.ZmState(*[t.data_ptr() for t in fin])
        sout = _native.ZmState(*[t.data_ptr() for t in out])
        solver.check(solver.lib.zm_step(solver.handle, ctypes.c_void_p(stream), ctypes.byref(sin),
                                        ctypes.byref(sout), int(nsteps)), "zm_step")
        return JaxStateG(*out, state.ice)

    def step(state):
        """One baroclinic step (factory.py:724-726)."""
        return _run(state, 1)

    def init_state(T_init=None, S_init=None):
        """Rest state with the land/ghost T_ref/S_ref sentinel (factory.py:766-788)."""
        import torch
        shape = solver.shape
        T = np.full(shape, T_ref) if T_init is None else np.asarray(T_init, dtype=np.float64)
        S = (np.full(shape, S_ref) if S_init is None else np.asarray(S_init, dtype=np.float64)) \
            if T_init is not None else np.full(shape, S_ref)
        T = T * wet3 + (1.0 - wet3) * T_ref
        S = S * wet3 + (1.0 - wet3) * S_ref
        dev = torch.device('cuda')
        as_t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)
        zeros3 = torch.zeros(shape, dtype=torch.float32, device=dev)
        return JaxStateG(zeros3, zeros3.clone(), as_t(T), as_t(S),
                         torch.zeros(shape[:2], dtype=torch.float32, device=dev),
                         torch.zeros(shape[:2], dtype=torch.float32, device=dev))

    def diagnostics(state, surface_pressure_pa=None):
        """(rho, pressure, w) of a state (factory.py:752-760): full density,
        hydrostatic pressure with an optional (nx, ny) surface load in Pa, and
        the vertical velocity, each (nx, ny, nz) float32, on the state's side
        (CUDA tensors for a device state, NumPy arrays for a host state)."""
        import torch
        fin, host = _device_fields(state, solver.shape)
        sp = None
        if surface_pressure_pa is not None:
            sp = torch.as_tensor(np.asarray(surface_pressure_pa, dtype=np.float32)
                                 if not isinstance(surface_pressure_pa, torch.Tensor) else surface_pressure_pa,
                                 dtype=torch.float32, device=fin[0].device).contiguous()
            if tuple(sp.shape) != solver.shape[:2]:
                raise ValueError('surface pressure must be a finite (nx, ny) Pa field')
        outs = [torch.empty_like(fin[0]) for _ in range(3)]
        stream = torch.cuda.current_stream(fin[0].device).cuda_stream
        sin = _native.ZmState(*[t.data_ptr() for t in fin])
        solver.check(solver.lib.zm_diagnostics(solver.handle, ctypes.c_void_p(stream), ctypes.byref(sin),
                                               ctypes.c_void_p(sp.data_ptr() if sp is not None else None),
                                               *[ctypes.c_void_p(t.data_ptr()) for t in outs]), "zm_diagnostics")
        if host:
            return tuple(t.cpu().numpy() for t in outs)
        return tuple(outs)

    def budget_diagnostics(state, rho0=RHO_0, cp=None):
        """Heat/salt/volume snapshot of a state (diagnostics/snapshot.py:67-128)
        with compensated float64 sums on the GPU."""
        import torch
        fin, _ = _device_fields(state, solver.shape)
        out = (ctypes.c_double * 8)()
        stream = torch.cuda.current_stream(fin[0].device).cuda_stream
        solver.check(solver.lib.zm_budgets(solver.handle, ctypes.c_void_p(stream), ctypes.c_void_p(fin[2].data_ptr()),
                                           ctypes.c_void_p(fin[3].data_ptr()), float(rho0),
                                           float(C_P if cp is None else cp), out), "zm_budgets")
        return BudgetDiagnostics(*[float(x) for x in out])

    def _cur_stream():
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def set_closure(net=None, bound=8.0):
        """Turn the learned vertical-mixing closure on for the following steps
        (``net``: a :class:`zhenmode_b200.closure.ClosureMLP` or its float32
        parameters) or off (``None``).  Columns with a feature beyond
        ``bound`` take the plain closure."""
        import torch
        if net is None:
            solver.check(solver.lib.zm_set_closure(solver.handle, _cur_stream(), None, float(bound)), "zm_set_closure")
            step.closure_params = None
            return
        params = net.params if hasattr(net, "params") else net
        if not isinstance(params, torch.Tensor):
            params = torch.as_tensor(np.asarray(params, dtype=np.float32), device="cuda")
        params = params.to(device="cuda", dtype=torch.float32).contiguous()
        if params.numel() != 148032:
            raise ValueError("the closure takes 148032 float32 parameters")
        solver.check(solver.lib.zm_set_closure(solver.handle, _cur_stream(), ctypes.c_void_p(params.data_ptr()),
                                               float(bound)), "zm_set_closure")
        step.closure_params = params

    def closure_features(state):
        """Training rows of a state: (X [nx*ny][256], log10 plain kappa [nx*ny][64],
        wet-interface mask [nx*ny][64]), rows j-major with i fastest."""
        import torch
        fin, _ = _device_fields(state, solver.shape)
        n = solver.shape[0] * solver.shape[1]
        X = torch.empty((n, 256), dtype=torch.float32, device=fin[0].device)
        T = torch.empty((n, 64), dtype=torch.float32, device=fin[0].device)
        M = torch.empty((n, 64), dtype=torch.float32, device=fin[0].device)
        sin = _native.ZmState(*[t.data_ptr() for t in fin])
        solver.check(solver.lib.zm_closure_features(solver.handle, _cur_stream(), ctypes.byref(sin),
                                                    *[ctypes.c_void_p(t.data_ptr()) for t in (X, T, M)]),
                     "zm_closure_features")
        return X, T, M

    def closure_kappa(state):
        """The set closure's diffusivity for a state, [nx*ny][64] (rows as in closure_features)."""
        import torch
        fin, _ = _device_fields(state, solver.shape)
        K = torch.empty((solver.shape[0] * solver.shape[1], 64), dtype=torch.float32, device=fin[0].device)
        sin = _native.ZmState(*[t.data_ptr() for t in fin])
        solver.check(solver.lib.zm_closure_kappa(solver.handle, _cur_stream(), ctypes.byref(sin),
                                                 ctypes.c_void_p(K.data_ptr())), "zm_closure_kappa")
        return K

    def closure_stats():
        """(columns of the last step that took the plain closure, tensor-core wait errors)."""
        fb, er = ctypes.c_uint32(), ctypes.c_uint32()
        rc = solver.lib.zm_closure_stats(solver.handle, ctypes.byref(fb), ctypes.byref(er))
        if rc not in (_native.ZM_OK, _native.ZM_ERR_TIMEOUT):
            solver.check(rc, "zm_closure_stats")
        return int(fb.value), int(er.value)

    def projection_stats():
        """CG iterations of the last column projection: (first solve, refinement 1,
        refinement 2, refinement solves run)."""
        out = (ctypes.c_int32 * 4)()
        solver.check(solver.lib.zm_projection_stats(solver.handle, out, 4), "zm_projection_stats")
        return tuple(int(x) for x in out)

    def set_forcing(tau_x=None, tau_y=None, q_heat=None):
        """Replace the 2-D forcing of the following steps ((nx, ny) fields)."""
        import torch
        fs = [None if a is None else torch.as_tensor(np.asarray(a, dtype=np.float32) if not isinstance(a, torch.Tensor)
                                                    else a, dtype=torch.float32, device='cuda').contiguous()
              for a in (tau_x, tau_y, q_heat)]
        solver.check(solver.lib.zm_set_forcing(solver.handle, _cur_stream(),
                                               *[ctypes.c_void_p(t.data_ptr() if t is not None else None)
                                                 for t in fs]), "zm_set_forcing")
        step._forcing_keep = fs

    def set_forcing_seasonal(tau_x=None, tau_y=None, q_heat=None, day=0.0, blend_days=5.0):
        """Blend (12, nx, ny) monthly stacks on the device for ``day``
        (inputs/forcing/seasonal.py:86-103) into the forcing of the following
        steps; stacks left as None keep their field."""
        import torch
        fs = [None if a is None else torch.as_tensor(np.asarray(a, dtype=np.float32) if not isinstance(a, torch.Tensor)
                                                    else a, dtype=torch.float32, device='cuda').contiguous()
              for a in (tau_x, tau_y, q_heat)]
        for t in fs:
            if t is not None and tuple(t.shape) != (12,) + solver.shape[:2]:
                raise ValueError("monthly stacks are (12, nx, ny)")
        solver.check(solver.lib.zm_set_forcing_seasonal(solver.handle, _cur_stream(),
                                                        *[ctypes.c_void_p(t.data_ptr() if t is not None else None)
                                                          for t in fs], float(day), float(blend_days)),
                     "zm_set_forcing_seasonal")
        step._forcing_keep = fs

    step.solver = solver
    step.advance = _run
    step.factory_forcing = (tau_x, tau_y, q_heat)
    step.set_forcing = set_forcing
    step.set_forcing_seasonal = set_forcing_seasonal
    step.budget_diagnostics = budget_diagnostics
    step.set_closure = set_closure
    step.closure_features = closure_features
    step.closure_kappa = closure_kappa
    step.closure_stats = closure_stats
    step.projection_stats = projection_stats
    step.closure_params = None
    result = [step, init_state, diagnostics]
    if return_params:
        params = B200Params(
            nx=nx, ny=ny, nz=nz, dt=float(dt), dt_bt=float(dt) / solver.n_subcyc, mode_split=True,
            n_subcyc=solver.n_subcyc, nu_nsub=solver.n_nu, adv_nsub=solver.adv_nsub, conv_nsub=solver.conv_nsub,
            use_scan=bool(use_scan), H_sw=float(np.sum(grid.dz)), nu_h=float(physics.nu_h),
            nu_v=float(physics.nu_v), kappa_h=float(physics.kappa_h), kappa_v=float(physics.kappa_v),
            kappa_conv=float(physics.kappa_conv), nu_bi=float(physics.nu_bi), kappa_bi=float(physics.kappa_bi),
            T_ref=float(physics.T_ref), S_ref=float(physics.S_ref), r_bot=float(physics.r_bot),
            cd=float(physics.cd), bottom_friction=str(physics.bottom_friction), lambda_bulk=float(lambda_bulk),
            restore_coef_S=float(restore_coef_S), polar_cap_rows=int(polar_cap_rows),
            polar_cap_taper=int(polar_cap_taper), eta_relax_rate=float(eta_relax_rate),
            freeze_adv_vel=bool(freeze_adv_vel), conservative_kv=bool(conservative_kv),
            localize_conv=bool(localize_conv), monotone_adv=bool(monotone_adv), fct_adv=bool(fct_adv),
            project_adv_vel=bool(project_adv_vel), projection_niter=int(projection_niter),
            projection_niter_source=projection_niter_source, projection_rtol=projection_rtol,
            projection_preconditioner=projection_preconditioner,
            projection_max_refinements=int(projection_max_refinements), column_geometry=column_geometry,
            process_time_scheme=process_time_scheme, thermodynamics=str(physics.thermodynamics),
            vertical_diffusion=vertical_diffusion, dtype='float32',
            wet_mask=np.asarray(grid.wet_mask, dtype=np.float32), wet_mask_z=wet3.astype(np.float32))
        params.step = step

        def terms_fn(state):
            """(6, nx, ny, nz) float32 [adv, diff_h, diff_v, conv, gm, redi]
            temperature terms of a state (factory.py:762-764,
            dynamics/tendencies.py:74-92), on the state's side (a CUDA tensor
            for a device state, a NumPy array for a host state)."""
            import torch
            fin, host = _device_fields(state, solver.shape)
            out = torch.empty((6,) + tuple(solver.shape), dtype=torch.float32, device=fin[0].device)
            stream = torch.cuda.current_stream(fin[0].device).cuda_stream
            sin = _native.ZmState(*[t.data_ptr() for t in fin])
            solver.check(solver.lib.zm_tracer_terms(solver.handle, ctypes.c_void_p(stream), ctypes.byref(sin),
                                                    ctypes.c_void_p(out.data_ptr())), "zm_tracer_terms")
            return out.cpu().numpy() if host else out

        result += [params, terms_fn]
    if dynamic_forcing:
        def step_dyn(state, tau_x, tau_y, q_heat, T_atm_3d=None, surface_pressure_pa=None):
            """Step with runtime 2-D forcing (factory.py:735-750)."""
            import torch
            if T_atm_3d is not None or surface_pressure_pa is not None:
                raise UnsupportedOption('runtime T_atm / surface pressure are not implemented on the B200 path')
            fs = [torch.as_tensor(np.asarray(a, dtype=np.float32) if not isinstance(a, torch.Tensor) else a,
                                  dtype=torch.float32, device='cuda').contiguous() for a in (tau_x, tau_y, q_heat)]
            stream = torch.cuda.current_stream().cuda_stream
            solver.check(solver.lib.zm_set_forcing(solver.handle, ctypes.c_void_p(stream),
                                                   *[ctypes.c_void_p(t.data_ptr()) for t in fs]), "zm_set_forcing")
            return step(state)

        result.append(step_dyn)
    return tuple(result)
