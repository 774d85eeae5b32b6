"""ORACLE (test infrastructure only): float64 NumPy restatement of ZhenMode's
production baroclinic/barotropic step, ``_step_impl`` with
``mode_split=True, column_geometry='legacy', process_time_scheme='legacy'``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package; the product (``zhenmode_b200``) never does.

Every function names the reference function it restates (paths relative to
the ZhenMode source tree).  Arrays use the reference layout ``(nx, ny, nz)``
with longitude periodic on axis 0 and closed latitude walls on axis 1.
Fields are plain ``dict``s with keys ``u, v, T, S, eta``.
"""
from __future__ import annotations

import numpy as np

from .params import ALPHA_T, BETA_S, C_P, G_EARTH, OMEGA, R_EARTH, RHO_0


# ---------------------------------------------------------------- neighbours
def _east(a):
    return np.roll(a, -1, axis=0)


def _west(a):
    return np.roll(a, 1, axis=0)


def _north_held(a):
    """Row j+1 with the last row repeated (edge padding of the closed wall)."""
    ny = a.shape[1]
    return a[:, np.minimum(np.arange(ny) + 1, ny - 1)]


def _south_held(a):
    ny = a.shape[1]
    return a[:, np.maximum(np.arange(ny) - 1, 0)]


def _cos_face(p):
    return 0.5 * (p.cos_lat + np.roll(p.cos_lat, -1))


# ---------------------------------------------------------------- vertical
def bottom_index(p):
    """Deepest wet level per column (0 for land columns)."""
    if not hasattr(p, "_kbot"):
        p._kbot = np.max((p.wet_mask_z > 0.5) * np.arange(p.nz), axis=-1)
    return p._kbot


def fill_ghost_bottom(a, p):
    """numerics/vertical.py:122-135 ``_fill_ghost_bottom``: levels at and
    below the deepest wet node take that node's value."""
    idx = np.minimum(np.arange(p.nz)[None, None, :], bottom_index(p)[:, :, None])
    return np.take_along_axis(a, np.broadcast_to(idx, a.shape), axis=-1)


def d_dz(a, p):
    """numerics/vertical.py:267-272 ``_d_dz`` (derivative in signed z)."""
    z = p.z
    out = np.empty_like(a)
    out[..., 0] = (a[..., 1] - a[..., 0]) / (z[1] - z[0])
    out[..., 1:-1] = (a[..., 2:] - a[..., :-2]) / ((z[1:-1] - z[:-2]) + (z[2:] - z[1:-1]))
    out[..., -1] = (a[..., -1] - a[..., -2]) / (z[-1] - z[-2])
    return out


def d2_dz2(a, p):
    """numerics/vertical.py:275-293 ``_d2_dz2``: node form with zero-flux
    top/bottom rows on the ghost-filled column."""
    z = p.z
    a = fill_ghost_bottom(a, p)
    hm = np.abs(z[:-2] - z[1:-1])
    hp = np.abs(z[2:] - z[1:-1])
    den = hm * hp * (hm + hp) / 2.0
    out = np.empty_like(a)
    out[..., 1:-1] = (a[..., 2:] * hm + a[..., :-2] * hp - a[..., 1:-1] * (hm + hp)) / den
    out[..., 0] = 2.0 * (a[..., 1] - a[..., 0]) / abs(z[1] - z[0]) ** 2
    out[..., -1] = 2.0 * (a[..., -2] - a[..., -1]) / abs(z[-1] - z[-2]) ** 2
    return out


def _wet_interfaces(p):
    wm = p.wet_mask_z
    return (wm[..., :-1] > 0.5) & (wm[..., 1:] > 0.5)


def _interface_divergence(F, p):
    """numerics/vertical.py:296-306: (F[k-1/2]-F[k+1/2])/dz_node, zero ends."""
    zero = np.zeros_like(F[..., :1])
    up = np.concatenate([zero, F], axis=-1)
    dn = np.concatenate([F, zero], axis=-1)
    return (up - dn) / p.dz_node


def d2_dz2_flux(c, kappa, p):
    """numerics/vertical.py:317-332 ``_d2_dz2_flux`` (conservative_kv form)."""
    cf = fill_ghost_bottom(c, p)
    F = -kappa * (cf[..., 1:] - cf[..., :-1]) / p.dz_iface
    F = np.where(_wet_interfaces(p), F, 0.0)
    return _interface_divergence(F, p) * p.wet_mask_z


def kappa_v_effective(p):
    """physics/vertical.py:40-42."""
    return p.kappa_v + p.coastal_kappa_v_2d[:, :, None]


def vertical_tracer_diffusion(c, p):
    """physics/vertical.py:45-53 ``_vertical_diffusion`` with kappa_eff."""
    kappa = kappa_v_effective(p)
    if p.conservative_kv:
        return d2_dz2_flux(c, kappa, p)
    return kappa * d2_dz2(c, p)


def vertical_momentum_diffusion(a, p):
    """physics/vertical.py:56-60 (legacy geometry)."""
    return p.nu_v * d2_dz2(a, p)


# ---------------------------------------------------------------- horizontal
def laplacian_h(a, p):
    """numerics/horizontal.py:181-215 ``_laplacian_h`` (legacy branch):
    face-gated d2/dx2 + mirror-ghost face-gated d2/dy2 - (tan(lat)/R) d/dy."""
    wm = p.wet_mask_z
    d2x = ((_east(a) - a) * wm * _east(wm) - (a - _west(a)) * wm * _west(wm)) * p.inv_dx2
    d2y = ((_north_held(a) - a) * _north_held(wm) * wm
           - (a - _south_held(a)) * wm * _south_held(wm)) * p.inv_dy2
    ddy = (_north_held(a) - _south_held(a)) * (0.5 * p.inv_dy)
    sin_row = p.f[0, :] / (2.0 * OMEGA)
    tan_over_r = (sin_row / p.cos_lat) / R_EARTH
    return d2x + d2y + (-ddy * tan_over_r[None, :, None])


def biharmonic_h(a, p):
    """numerics/horizontal.py:251-253."""
    return laplacian_h(laplacian_h(a, p), p)


def horizontal_diffusion_flux(c, kappa, p):
    """numerics/horizontal.py:217-243 ``_horizontal_diffusion_flux``."""
    wm = p.wet_mask_z
    zonal = 0.5 * (kappa + _east(kappa)) * (_east(c) - c) * p.inv_dx * wm * _east(wm)
    merid = (0.5 * (kappa + _north_held(kappa)) * (_north_held(c) - c) * p.inv_dy
             * wm * _north_held(wm) * _cos_face(p)[None, :, None])
    merid[:, -1, :] = 0.0
    incoming = np.roll(merid, 1, axis=1)
    incoming[:, 0, :] = 0.0
    return ((zonal - _west(zonal)) * p.inv_dx
            + (merid - incoming) * p.inv_dy / p.cos_lat[None, :, None])


def horizontal_tracer_diffusion(c, p):
    """numerics/horizontal.py:245-249 first half."""
    kappa = p.kappa_h + p.coastal_kappa_h_2d[:, :, None]
    return horizontal_diffusion_flux(c, kappa, p)


def horizontal_biharmonic_tracer(c, p):
    """numerics/horizontal.py:245-249."""
    unit = np.ones((p.nx, p.ny, 1))
    return horizontal_diffusion_flux(horizontal_diffusion_flux(c, unit, p), unit, p)


def gradient_face_gated_3d(a, p):
    """numerics/horizontal.py:331-360 (normal=False)."""
    wm = p.wet_mask_z
    gx = p.inv_dx * 0.5 * ((_east(a) - a) * wm * _east(wm) + (a - _west(a)) * wm * _west(wm))
    gy = p.inv_dy * 0.5 * ((_north_held(a) - a) * _north_held(wm) * wm
                           + (a - _south_held(a)) * wm * _south_held(wm))
    return gx, gy


def _wall_closed_pair(wm):
    """numerics/horizontal.py:27-34 along latitude: faces through the
    truncation walls are closed."""
    pos = wm * np.roll(wm, -1, axis=1)
    neg = wm * np.roll(wm, 1, axis=1)
    pos[:, -1] = 0.0
    neg[:, 0] = 0.0
    return pos, neg


def gradient_conservative_3d(a, p):
    """numerics/horizontal.py:126-151 ``_gradient_conservative_3d`` (the
    adjoint of the conservative divergence; ``a`` may be (nx,ny,1))."""
    wm = p.wet_mask_z
    gx = p.inv_dx * 0.5 * ((_east(a) - a) * wm * _east(wm) + (a - _west(a)) * wm * _west(wm))
    pos, neg = _wall_closed_pair(wm)
    cp = 0.5 * (p.cos_lat + np.roll(p.cos_lat, -1))
    cm = 0.5 * (p.cos_lat + np.roll(p.cos_lat, 1))
    dyp = (np.roll(a, -1, axis=1) - a) * pos * cp[None, :, None]
    dym = (a - np.roll(a, 1, axis=1)) * neg * cm[None, :, None]
    gy = (p.inv_dy / p.cos_lat[None, :, None]) * 0.5 * (dyp + dym)
    return gx, gy


def gradient_conservative_2d(eta, p):
    """numerics/horizontal.py:99-124 ``_gradient_conservative``."""
    wm = p.wet_mask
    inv_dx = p.inv_dx[..., 0]
    gx = inv_dx * 0.5 * ((_east(eta) - eta) * wm * _east(wm) + (eta - _west(eta)) * wm * _west(wm))
    pos, neg = _wall_closed_pair(wm)
    cp = 0.5 * (p.cos_lat + np.roll(p.cos_lat, -1))
    cm = 0.5 * (p.cos_lat + np.roll(p.cos_lat, 1))
    dyp = (np.roll(eta, -1, axis=1) - eta) * pos * cp[None, :]
    dym = (eta - np.roll(eta, 1, axis=1)) * neg * cm[None, :]
    gy = (p.inv_dy / p.cos_lat[None, :]) * 0.5 * (dyp + dym)
    return gx, gy


def divergence_conservative_2d(ubt, vbt, p):
    """numerics/horizontal.py:69-97 ``_divergence_conservative``."""
    wm = p.wet_mask
    uface = 0.5 * (ubt + _east(ubt)) * (wm * _east(wm))
    div_x = (uface - _west(uface)) * p.inv_dx[..., 0]
    vopen = wm * np.roll(wm, -1, axis=1)
    vopen[:, -1] = 0.0
    fcos = 0.5 * (vbt + np.roll(vbt, -1, axis=1)) * vopen * _cos_face(p)[None, :]
    incoming = np.roll(fcos, 1, axis=1)
    incoming[:, 0] = 0.0
    return div_x + (fcos - incoming) * p.inv_dy / p.cos_lat[None, :]


def divergence_h(u, v, p):
    """numerics/horizontal.py:255-281 ``_divergence_h`` (face-flux form)."""
    wm = p.wet_mask_z
    Fx = 0.5 * (u + _east(u)) * wm * _east(wm)
    div_x = (Fx - _west(Fx)) * p.inv_dx
    Fy = 0.5 * (v + _north_held(v)) * wm * _north_held(wm) * _cos_face(p)[None, :, None]
    Fy[:, -1] = 0.0
    div_y = (Fy - np.roll(Fy, 1, axis=1)) * p.inv_dy / p.cos_lat[None, :, None]
    return div_x + div_y


def dealias(a, p):
    """numerics/horizontal.py:283-305 ``_dealias_h_fd`` (normal=False): 2/3
    rule along the periodic longitude, [1,4,6,4,1]/16 along latitude with
    the edge row repeated."""
    spec = np.fft.fft(a, axis=0) * p.dealias_lon_mask
    lon = np.real(np.fft.ifft(spec, axis=0))
    ny = a.shape[1]
    j = np.arange(ny)

    def row(offset):
        return lon[:, np.clip(j + offset, 0, ny - 1)]

    return (row(-2) + 4.0 * row(-1) + 6.0 * lon + 4.0 * row(1) + row(2)) / 16.0


def polar_cap_weights(ncap, ntaper):
    """numerics/horizontal.py:362-385, pole-inward order."""
    if ncap <= 0:
        return np.zeros(0)
    ramp = np.cos(np.linspace(0.0, np.pi / 2.0, ntaper + 2)[1:-1]) ** 2 if ntaper > 0 else np.zeros(0)
    return np.concatenate([np.ones(ncap), ramp])


def polar_cap(a, wm, p):
    """numerics/horizontal.py:387-451 ``_apply_polar_cap`` (legacy branch):
    wet-point zonal mean blended in with pole-inward weights on the ``nb``
    rows at each wall; land nodes of the band come back masked (zero)."""
    if p.polar_cap_rows <= 0:
        return a
    nb = p.polar_cap_rows + p.polar_cap_taper
    wts = polar_cap_weights(p.polar_cap_rows, p.polar_cap_taper)
    shape_tail = (1,) * (a.ndim - 2)

    def band(f, m, w):
        s = f * m
        count = np.maximum(np.sum(m, axis=0, keepdims=True), 1.0)
        mean = np.sum(s, axis=0, keepdims=True) / count
        mean = np.broadcast_to(mean, f.shape) * m
        wb = w.reshape((1, nb) + shape_tail)
        return wb * mean + (1.0 - wb) * s

    south = band(a[:, :nb], wm[:, :nb], wts)
    north = band(a[:, -nb:], wm[:, -nb:], wts[::-1])
    return np.concatenate([south, a[:, nb:-nb], north], axis=1)


# ---------------------------------------------------------------- transport
def vertical_transport_iface(u, v, p):
    """dynamics/transport.py:110-133: Fz[k] = sum_{m>=k} div_h[m] dz_node[m],
    Fz[nz] = 0 (downward positive)."""
    integrand = divergence_h(u, v, p) * p.dz_node
    acc = np.cumsum(integrand[..., ::-1], axis=-1)[..., ::-1]
    return np.concatenate([acc, np.zeros_like(acc[..., :1])], axis=-1)


def barotropic_velocity(u, v, p):
    """dynamics/transport.py:135-143 (legacy): layer-averaged sum over the
    full vertical span, weights dz/H."""
    ubt = np.sum(0.5 * (u[..., :-1] + u[..., 1:]) * p.dz_norm, axis=-1)
    vbt = np.sum(0.5 * (v[..., :-1] + v[..., 1:]) * p.dz_norm, axis=-1)
    return ubt, vbt


def vertical_velocity(u, v, p):
    """dynamics/transport.py:149-166 (dual-face sample)."""
    return -vertical_transport_iface(u, v, p)[..., :-1] * p.wet_mask_z


def momentum_advection(u, v, w, p):
    """dynamics/transport.py:169-197 ``_advection_flux_form`` (legacy)."""
    du_dz = d_dz(fill_ghost_bottom(u, p), p)
    dv_dz = d_dz(fill_ghost_bottom(v, p), p)
    dudx, dudy = gradient_face_gated_3d(u, p)
    dvdx, dvdy = gradient_face_gated_3d(v, p)
    adv_u = -(u * dudx + v * dudy + w * du_dz)
    adv_v = -(u * dvdx + v * dvdy + w * dv_dz)
    return dealias(adv_u, p) * p.wet_mask_z, dealias(adv_v, p) * p.wet_mask_z


def limited_slope(c, wm, axis):
    """dynamics/transport.py:199-213 minmod slope over wet neighbours."""
    if axis == 1:
        prev, nxt, pw, nw = _south_held(c), _north_held(c), _south_held(wm), _north_held(wm)
    else:
        prev, nxt, pw, nw = _west(c), _east(c), _west(wm), _east(wm)
    left, right = c - prev, nxt - c
    return 0.5 * (np.sign(left) + np.sign(right)) * np.minimum(np.abs(left), np.abs(right)) * wm * pw * nw


def horizontal_tracer_fluxes(c, u, v, p):
    """dynamics/transport.py:224-290 ``_legacy_horizontal_tracer_fluxes``."""
    wm = p.wet_mask_z
    ux = 0.5 * (u + _east(u))
    if p.fct_adv:
        sx = limited_slope(c, wm, 0)
        cx = np.where(ux >= 0.0, c + 0.5 * sx, _east(c) - 0.5 * _east(sx))
    elif p.monotone_adv:
        cx = np.where(ux >= 0.0, c, _east(c))
    else:
        cx = 0.5 * (c + _east(c))
    Fx = ux * cx * (wm * _east(wm))
    vy = 0.5 * (v + _north_held(v))
    if p.fct_adv:
        sy = limited_slope(c, wm, 1)
        cy = np.where(vy >= 0.0, c + 0.5 * sy, _north_held(c) - 0.5 * _north_held(sy))
    elif p.monotone_adv:
        cy = np.where(vy >= 0.0, c, _north_held(c))
    else:
        cy = 0.5 * (c + _north_held(c))
    Fy = vy * cy * (wm * _north_held(wm)) * _cos_face(p)[None, :, None]
    Fy[:, -1] = 0.0
    return Fx, Fy


def tracer_advection(c, u, v, Fz, p):
    """dynamics/transport.py:365-475 ``_advection_scalar`` (legacy donor-cell
    vertical flux, rigid-lid top flux Fz[0]*c[0])."""
    wm = p.wet_mask_z
    Fx, Fy = horizontal_tracer_fluxes(c, u, v, p)
    Fy_in = np.roll(Fy, 1, axis=1)
    Fy_in[:, 0] = 0.0
    hdiv = (Fx - _west(Fx)) * p.inv_dx + (Fy - Fy_in) * p.inv_dy / p.cos_lat[None, :, None]
    deep = fill_ghost_bottom(c, p)[..., 1:]
    shallow = c[..., :-1]
    wet_if = wm[..., :-1] * wm[..., 1:]
    Fzi = Fz[..., 1:-1]
    interior = Fzi * np.where(Fzi > 0.0, shallow, deep) * wet_if
    top = Fz[..., :1] * c[..., :1]
    up = np.concatenate([top, interior], axis=-1)
    dn = np.concatenate([interior, np.zeros_like(interior[..., :1])], axis=-1)
    return -(hdiv + (dn - up) / p.dz_node) * wm


# ---------------------------------------------------------------- EOS / pressure
def density_anomaly(T, S, p):
    """physics/eos.py:13-18 (linear)."""
    return RHO_0 * (-ALPHA_T * (T - p.T_ref) + BETA_S * (S - p.S_ref))


def baroclinic_pressure(T, S, p):
    """dynamics/pressure.py:32-42: trapezoid integral of the masked anomaly."""
    rho = density_anomaly(T, S, p) * p.wet_mask_z
    dp = G_EARTH * 0.5 * (rho[..., :-1] + rho[..., 1:]) * p.dz_3d
    out = np.zeros_like(T)
    out[..., 1:] = np.cumsum(dp, axis=-1)
    return out


def hydrostatic_pressure(T, S, eta, p, surface_pressure_pa=None):
    """dynamics/pressure.py:62-74 (reference-plane surface, trapezoid):
    rho0 g eta (+ the surface load) + the baroclinic integral."""
    p_bt = RHO_0 * G_EARTH * eta[:, :, None]
    if surface_pressure_pa is not None:
        p_bt = p_bt + np.asarray(surface_pressure_pa, dtype=np.float64)[..., None]
    return p_bt + baroclinic_pressure(T, S, p)


def diagnostics(state, p, surface_pressure_pa=None):
    """The diagnostics closure of factory.py:752-760: full density
    rho0 + rho', hydrostatic pressure and the dual-face vertical velocity."""
    rho = RHO_0 + density_anomaly(state["T"], state["S"], p)
    pres = hydrostatic_pressure(state["T"], state["S"], state["eta"], p, surface_pressure_pa)
    w = vertical_velocity(state["u"], state["v"], p)
    return rho, pres, w


def pressure_gradient(T, S, eta, p):
    """dynamics/pressure.py:62-97: -grad(rho0 g eta + p_bc)/rho0."""
    pres = RHO_0 * G_EARTH * eta[:, :, None] + baroclinic_pressure(T, S, p)
    gx, gy = gradient_conservative_3d(pres, p)
    return -gx / RHO_0, -gy / RHO_0


def bt_rho_pgf(T, S, p):
    """dynamics/pressure.py:144-180 (legacy): wet-interface layer average of
    the 3-D baroclinic gradient, normalised by rho0 H_sw."""
    gx, gy = gradient_conservative_3d(baroclinic_pressure(T, S, p), p)
    wm = p.wet_mask_z
    wet_if = wm[..., :-1] * wm[..., 1:]
    lx = 0.5 * (gx[..., :-1] + gx[..., 1:])
    ly = 0.5 * (gy[..., :-1] + gy[..., 1:])
    fx = -np.sum(lx * wet_if * p.dz_3d, axis=-1) / (RHO_0 * p.H_sw)
    fy = -np.sum(ly * wet_if * p.dz_3d, axis=-1) / (RHO_0 * p.H_sw)
    return fx, fy


# ---------------------------------------------------------------- convection
def convective_gates(T, S, p):
    """physics/vertical.py:63-82 ``_convective_mask`` (linear EOS)."""
    rho = density_anomaly(T, S, p) * p.wet_mask_z
    unstable = (rho[..., :-1] > rho[..., 1:]) & _wet_interfaces(p)
    return np.any(unstable, axis=-1, keepdims=True), unstable


def convective_tendency(c, column_gate, kappa, p, iface_gate):
    """physics/vertical.py:13-37 ``_conv_flux_tendency``."""
    if kappa <= 0.0:
        return np.zeros_like(c)
    cf = fill_ghost_bottom(c, p)
    F = -kappa * (cf[..., 1:] - cf[..., :-1]) / p.dz_iface
    allow = column_gate & _wet_interfaces(p)
    if iface_gate is not None:
        allow = allow & iface_gate
    F = np.where(allow, F, 0.0)
    return _interface_divergence(F, p) * p.wet_mask_z


# ---------------------------------------------------------------- tendencies
def _surface_heat_factor(p):
    """physics/surface.py:8-20 default branch / (rho0 cp)."""
    return p.surface_mask * p.wet_mask_z / p.dz_surface / (RHO_0 * C_P)


def tracer_tendency(u, v, T, S, p, rec=None):
    """dynamics/tendencies.py:94-219 ``_compute_tracer_tendency`` (no GM/Redi,
    no dynamic ice, default mixed layer); with a ledger recorder ``rec`` the
    hooks of tendencies.py:211-214 (the surface flux Fz[0] c[0] of the
    advection, transport.py:459-475, averaged over the substeps like the rate)."""
    Fz = vertical_transport_iface(u, v, p)
    na = int(p.adv_nsub)
    if na > 1:
        dts = p.dt / na
        tT, tS = T, S
        aT_list, aS_list, tops_T, tops_S = [], [], [], []
        for _ in range(na):
            aT = tracer_advection(tT, u, v, Fz, p)
            aS = tracer_advection(tS, u, v, Fz, p)
            aT_list.append(aT)
            aS_list.append(aS)
            tops_T.append(Fz[..., 0] * tT[..., 0])
            tops_S.append(Fz[..., 0] * tS[..., 0])
            tT, tS = tT + aT * dts, tS + aS * dts
        adv_T = np.mean(np.stack(aT_list), axis=0)
        adv_S = np.mean(np.stack(aS_list), axis=0)
        top_T = sum(tops_T) / na
        top_S = sum(tops_S) / na
    else:
        adv_T = tracer_advection(T, u, v, Fz, p)
        adv_S = tracer_advection(S, u, v, Fz, p)
        top_T, top_S = Fz[..., 0] * T[..., 0], Fz[..., 0] * S[..., 0]
    dh_T = horizontal_tracer_diffusion(T, p)
    dh_S = horizontal_tracer_diffusion(S, p)
    dv_T = vertical_tracer_diffusion(T, p)
    dv_S = vertical_tracer_diffusion(S, p)
    column, unstable = convective_gates(T, S, p)
    gate = unstable if p.localize_conv else None
    nc = int(p.conv_nsub)
    if nc > 1:
        kappa_c = p.kappa_conv / nc
        hc = p.dt / nc
        tT, tS = T, S
        cT_list, cS_list = [], []
        for _ in range(nc):
            cT = convective_tendency(tT, column, kappa_c, p, gate)
            cS = convective_tendency(tS, column, kappa_c, p, gate)
            cT_list.append(cT)
            cS_list.append(cS)
            tT, tS = tT + cT * hc, tS + cS * hc
        conv_T = np.mean(np.stack(cT_list), axis=0)
        conv_S = np.mean(np.stack(cS_list), axis=0)
    else:
        conv_T = convective_tendency(T, column, p.kappa_conv, p, gate)
        conv_S = convective_tendency(S, column, p.kappa_conv, p, gate)
    hf = _surface_heat_factor(p)
    sst = T[..., 0:1]
    heat_T = p.Q_heat_2d[:, :, None] * hf
    bulk_T = p.lambda_bulk * (p.T_atm_3d - sst) * hf
    cbulk_T = p.coastal_bulk_lambda_2d[:, :, None] * (p.T_atm_3d - sst) * hf
    rest_S = p.restore_coef_S * (p.S_ref_2d[:, :, None] - S[..., 0:1]) * p.surface_mask
    ice_salt = p.ice_salt_flux * (sst <= p.ice_freeze_temp_c) * p.surface_mask
    rest_T = p.coastal_restore_coef_2d[:, :, None] * (p.coastal_restore_T_2d[:, :, None] - sst) * p.surface_mask
    dT = adv_T + dh_T + dv_T + heat_T + bulk_T + cbulk_T + conv_T + rest_T
    dS = adv_S + dh_S + dv_S + conv_S + rest_S + ice_salt
    if rec is not None:
        zero = np.zeros_like(adv_T)
        rec.surface_sources((heat_T, bulk_T, cbulk_T, rest_T, rest_S, ice_salt))
        rec.nonlinear_terms(((adv_T, adv_S), (conv_T, conv_S), (zero, zero), (zero, zero)))
        rec.advection_boundary_fluxes(top_T, top_S)
    return dT * p.wet_mask_z, dS * p.wet_mask_z


def tracer_terms(st, p):
    """dynamics/tendencies.py:74-92 ``_tracer_terms`` (what ``terms_fn`` of
    factory.py:762-764 returns): the (6, nx, ny, nz) stack [adv, diff_h,
    diff_v, conv, gm, redi] of land-masked temperature terms at the state,
    one advection evaluation (no substeps) and one convective evaluation
    with kappa_conv; GM and Redi are zero (kappa_gm = kappa_redi = 0)."""
    T, S, u, v = st["T"], st["S"], st["u"], st["v"]
    Fz = vertical_transport_iface(u, v, p)
    adv = tracer_advection(T, u, v, Fz, p)
    dh = horizontal_tracer_diffusion(T, p)
    dv = vertical_tracer_diffusion(T, p)
    column, unstable = convective_gates(T, S, p)
    conv = convective_tendency(T, column, p.kappa_conv, p, unstable if p.localize_conv else None)
    zero = np.zeros_like(T)
    return np.stack([t * p.wet_mask_z for t in (adv, dh, dv, conv, zero, zero)], axis=0)


def tracer_residual(u, v, T, S, p, rec=None):
    """dynamics/tendencies.py:227-245: tendency minus the L-step linear terms."""
    dT, dS = tracer_tendency(u, v, T, S, p, rec)
    dT = dT - horizontal_tracer_diffusion(T, p)
    dS = dS - horizontal_tracer_diffusion(S, p)
    dT = dT - vertical_tracer_diffusion(T, p)
    dS = dS - vertical_tracer_diffusion(S, p)
    return dT, dS


def momentum_tendency(u, v, T, S, eta, p):
    """dynamics/tendencies.py:39-72 (linear drag)."""
    w = vertical_velocity(u, v, p)
    adv_u, adv_v = momentum_advection(u, v, w, p)
    f3 = p.f[:, :, None]
    pgf_x, pgf_y = pressure_gradient(T, S, eta, p)
    wind = 1.0 / (RHO_0 * p.dz_surface)
    du = (adv_u + f3 * v + pgf_x + p.nu_h * laplacian_h(u, p) + vertical_momentum_diffusion(u, p)
          + p.tau_x_2d[:, :, None] * wind * p.surface_mask - p.r_bot * u * p.bottom_mask)
    dv = (adv_v - f3 * u + pgf_y + p.nu_h * laplacian_h(v, p) + vertical_momentum_diffusion(v, p)
          + p.tau_y_2d[:, :, None] * wind * p.surface_mask - p.r_bot * v * p.bottom_mask)
    return du * p.wet_mask_z, dv * p.wet_mask_z


def momentum_residual(u, v, T, S, eta, p):
    """dynamics/tendencies.py:247-319 (legacy geometry, mode split)."""
    du, dv = momentum_tendency(u, v, T, S, eta, p)
    du = du - p.nu_h * laplacian_h(u, p) - vertical_momentum_diffusion(u, p)
    dv = dv - p.nu_h * laplacian_h(v, p) - vertical_momentum_diffusion(v, p)
    f3 = p.f[:, :, None]
    du = du - f3 * v
    dv = dv + f3 * u
    ex, ey = gradient_conservative_3d(eta[:, :, None], p)
    du = du + G_EARTH * ex
    dv = dv + G_EARTH * ey
    fx, fy = bt_rho_pgf(T, S, p)
    du = du - fx[:, :, None] - (p.tau_x_2d / (RHO_0 * p.H_sw))[:, :, None]
    dv = dv - fy[:, :, None] - (p.tau_y_2d / (RHO_0 * p.H_sw))[:, :, None]
    return du * p.wet_mask_z, dv * p.wet_mask_z


# ---------------------------------------------------------------- implicit column solve
def implicit_vertical_solve(rhs, kappa, dt, p):
    """Extension (not a reference option): backward-Euler ``(I - dt K D2) x =
    rhs`` per column with the node-form operator of ``d2_dz2`` on the wet
    levels 0..kbot (rows below kbot pass ``rhs`` through).  Each column's
    tridiagonal matrix is assembled in full and solved directly
    (numpy.linalg.solve, LU in float64), columns in batches."""
    z = p.z
    nz = p.nz
    kbot = bottom_index(p)
    kap = np.broadcast_to(np.asarray(kappa, dtype=np.float64), rhs.shape[:2] + (1,))[..., 0]
    out = np.array(rhs, dtype=np.float64, copy=True)
    hm = np.abs(np.diff(z))            # hm[k-1] = |z[k-1]-z[k]|
    kb = kbot.reshape(-1).astype(np.int64)
    s = (dt * kap).reshape(-1)
    flat = out.reshape(-1, nz)
    cols = np.nonzero(kb > 0)[0]
    kk = np.arange(nz)
    for lo in range(0, cols.size, 8192):
        c_idx = cols[lo:lo + 8192]
        m = c_idx.size
        kbc, sc = kb[c_idx][:, None], s[c_idx][:, None]
        live = kk[None, :] <= kbc                     # rows 0..kb of the system
        a = np.zeros((m, nz))
        b = np.ones((m, nz))
        c = np.zeros((m, nz))
        h0 = hm[0]
        b[:, 0] += sc[:, 0] * 2.0 / h0 ** 2
        c[:, 0] -= sc[:, 0] * 2.0 / h0 ** 2
        if nz > 1:
            hb = hm[-1]
            a[:, nz - 1] -= sc[:, 0] * 2.0 / hb ** 2
            b[:, nz - 1] += sc[:, 0] * 2.0 / hb ** 2
        for k in range(1, nz - 1):
            up, dn = hm[k - 1], hm[k]
            den = up * dn * (up + dn) / 2.0
            a[:, k] -= sc[:, 0] * dn / den
            b[:, k] += sc[:, 0] * (up + dn) / den
            interior = k < kbc[:, 0]
            c[:, k] = np.where(interior, c[:, k] - sc[:, 0] * up / den, c[:, k])
            b[:, k] = np.where(interior, b[:, k], b[:, k] - sc[:, 0] * up / den)
        # rows beyond kb pass the right-hand side through (identity rows)
        a = np.where(live, a, 0.0)
        c = np.where(live, c, 0.0)
        b = np.where(live, b, 1.0)
        a[:, 0] = 0.0
        c = np.where(kk[None, :] < kbc, c, 0.0)       # no coupling from row kb to kb + 1
        mat = np.zeros((m, nz, nz))
        mat[:, kk, kk] = b
        mat[:, kk[1:], kk[:-1]] = a[:, 1:]
        mat[:, kk[:-1], kk[1:]] = c[:, :-1]
        flat[c_idx] = np.linalg.solve(mat, flat[c_idx][..., None])[..., 0]
    return out


# ---------------------------------------------------------------- linear half step
def linear_half_step(st, p, dt_half, rec=None):
    """timestepping/step.py:76-187 ``_linear_half_step`` (legacy, mode split);
    ledger hooks of step.py:138-161."""
    u0, v0, T0, S0 = st["u"], st["v"], st["T"], st["S"]
    wm = p.wet_mask_z
    n_nu = max(1, int(p.n_subcyc if p.nu_nsub is None else p.nu_nsub))
    dts = dt_half / n_nu
    u, v = u0, v0
    for _ in range(n_nu):
        u, v = u + p.nu_h * laplacian_h(u, p) * dts, v + p.nu_h * laplacian_h(v, p) * dts
    T = T0 + horizontal_tracer_diffusion(T0, p) * dt_half
    S = S0 + horizontal_tracer_diffusion(S0, p) * dt_half
    if p.nu_bi > 0.0:
        u = u - p.nu_bi * biharmonic_h(u0, p) * dt_half
        v = v - p.nu_bi * biharmonic_h(v0, p) * dt_half
    if p.kappa_bi > 0.0:
        T = T - p.kappa_bi * horizontal_biharmonic_tracer(T0, p) * dt_half
        S = S - p.kappa_bi * horizontal_biharmonic_tracer(S0, p) * dt_half
    if p.vertical_diffusion == "implicit":
        u = implicit_vertical_solve(u, p.nu_v, dt_half, p)
        v = implicit_vertical_solve(v, p.nu_v, dt_half, p)
        T = implicit_vertical_solve(T, kappa_v_effective(p), dt_half, p)
        S = implicit_vertical_solve(S, kappa_v_effective(p), dt_half, p)
    else:
        u = u + vertical_momentum_diffusion(u0, p) * dt_half
        v = v + vertical_momentum_diffusion(v0, p) * dt_half
        T = T + vertical_tracer_diffusion(T0, p) * dt_half
        S = S + vertical_tracer_diffusion(S0, p) * dt_half
    u = u * wm + u0 * (1.0 - wm)
    v = v * wm + v0 * (1.0 - wm)
    T = T * wm + T0 * (1.0 - wm)
    S = S * wm + S0 * (1.0 - wm)
    diffused = dict(u=u, v=v, T=T, S=S, eta=st["eta"])
    if rec is not None:
        rec.stage("linear_diffusion", st, diffused)
    decay = np.exp(-p.sponge_rate * dt_half)
    u = u * decay
    v = v * decay
    T = p.T_clim_3d + (T - p.T_clim_3d) * decay
    S = p.S_clim_3d + (S - p.S_clim_3d) * decay
    if rec is not None:
        rec.stage("sponge", diffused, dict(u=u, v=v, T=T, S=S, eta=st["eta"]))
        rec.sponge_sources(diffused, decay)
    angle = p.f[:, :, None] * dt_half
    ca, sa = np.cos(angle), np.sin(angle)
    return dict(u=ca * u + sa * v, v=-sa * u + ca * v, T=T, S=S, eta=st["eta"])


# ---------------------------------------------------------------- nonlinear full step
# ---------------------------------------------------------------- column projection
def column_divergence(u, v, p):
    """dynamics/transport.py:45-57 (legacy): sum_k div_h[k] dz_node[k] on wet columns."""
    return np.sum(divergence_h(u, v, p) * p.dz_node, axis=-1) * p.wet_mask


def column_projection_diagonal(p):
    """dynamics/projection.py:10-51 (legacy branch): the exact diagonal of the
    projection operator."""
    wet = p.wet_mask_z
    pos_x = wet * np.roll(wet, -1, axis=0)
    neg_x = wet * np.roll(wet, 1, axis=0)
    dxg = 0.25 * p.inv_dx[..., :1] ** 2 * ((pos_x - neg_x) ** 2 + pos_x ** 2 + neg_x ** 2)
    if p.nx <= 2:
        dxg = np.zeros_like(wet)
    c = p.cos_lat[None, :, None]
    cn = np.roll(c, -1, axis=1)
    cs = np.roll(c, 1, axis=1)
    pos_y = wet * np.roll(wet, -1, axis=1)
    pos_y[:, -1, :] = 0.0
    neg_y = wet * np.roll(wet, 1, axis=1)
    neg_y[:, 0, :] = 0.0
    pos_y = pos_y * 0.5 * (c + cn)
    neg_y = neg_y * 0.5 * (c + cs)
    dyg = 0.25 * p.inv_dy ** 2 * ((pos_y - neg_y) ** 2 / c ** 2 + pos_y ** 2 / (c * cn) + neg_y ** 2 / (c * cs))
    area = p.dx_2d * p.dy * p.wet_mask
    return area * np.sum((dxg + dyg) * p.dz_node, axis=-1)


def conjugate_gradient(A, b, tol, maxiter, M=None, atol=0.0):
    """Preconditioned CG with the loop of jax.scipy.sparse.linalg.cg (jax 0.11.2,
    the reference's pinned version; the dependency is absent here): x0 = 0,
    stop when the squared residual norm (<r, z> without a preconditioner,
    <r, r> with one) is at most max(tol^2 <b, b>, atol^2) or after maxiter
    iterations."""
    identity = M is None
    prec = (lambda r: r) if identity else M
    x = np.zeros_like(b)
    atol2 = max(tol * tol * float(np.vdot(b, b)), atol * atol)
    r = b - A(x)
    z = prec(r)
    pdir = z
    gamma = float(np.vdot(r, z))
    k = 0
    while (gamma if identity else float(np.vdot(r, r))) > atol2 and k < maxiter:
        Ap = A(pdir)
        alpha = gamma / float(np.vdot(pdir, Ap))
        x = x + alpha * pdir
        r = r - alpha * Ap
        z = prec(r)
        gamma_new = float(np.vdot(r, z))
        pdir = z + (gamma_new / gamma) * pdir
        gamma = gamma_new
        k += 1
    return x


def project_column_divergence(u, v, p, dt):
    """dynamics/projection.py:64-127: remove the column-integrated horizontal
    divergence by the Euler correction -dt g grad(psi) of the potential that
    solves the area-weighted problem with the exact column divergence, then up
    to projection_max_refinements corrective solves while the actual surface
    transport stays above its threshold."""
    g = G_EARTH
    area = p.dx_2d * p.dy * p.wet_mask
    rhs = -(column_divergence(u, v, p) / (dt * g)) * area

    def matvec(psi):
        gx, gy = gradient_conservative_3d(psi[:, :, None], p)
        return -column_divergence(gx, gy, p) * area

    M = None
    if p.projection_preconditioner == "jacobi":
        diag = column_projection_diagonal(p)
        inv = 1.0 / np.where(diag > 0.0, diag, 1.0)
        M = lambda r: r * inv  # noqa: E731

    def correct(vel, psi):
        gx, gy = gradient_conservative_3d(psi[..., None], p)
        return vel[0] - (dt * g) * gx, vel[1] - (dt * g) * gy

    tol = p.projection_rtol
    psi = conjugate_gradient(matvec, rhs, tol, p.projection_niter, M)
    corrected = correct((u, v), psi)
    if p.projection_max_refinements == 0:
        return corrected

    def transport_norm_squared(vel):
        top = vertical_transport_iface(vel[0], vel[1], p)[..., 0]
        return float(np.sum(top ** 2 * p.dx_2d * p.dy * p.wet_mask))

    threshold = p.projection_transport_rtol ** 2 * transport_norm_squared((u, v))
    floor = tol * float(np.linalg.norm(rhs))
    for _ in range(p.projection_max_refinements):
        if transport_norm_squared(corrected) > threshold:
            residual = -(column_divergence(corrected[0], corrected[1], p) / (dt * g)) * area
            delta = conjugate_gradient(matvec, residual, tol, p.projection_niter, M, atol=floor)
            corrected = correct(corrected, delta)
    return corrected


def explicit_full_step(st, p, rec=None):
    """timestepping/step.py:249-320 ``_explicit_full_step`` (legacy RK2 with
    the exact linear-drag decay of the mode-split path)."""
    u, v, T, S, eta = st["u"], st["v"], st["T"], st["S"], st["eta"]
    dt = p.dt
    dT1, dS1 = tracer_residual(u, v, T, S, p, rec)
    Tp, Sp = T + dT1 * dt, S + dS1 * dt
    du1, dv1 = momentum_residual(u, v, Tp, Sp, eta, p)
    bm = p.bottom_mask * p.wet_mask_z
    du1 = du1 + p.r_bot * u * bm
    dv1 = dv1 + p.r_bot * v * bm
    up, vp = u + du1 * dt, v + dv1 * dt
    if p.freeze_adv_vel:
        dT2, dS2 = tracer_residual(u, v, Tp, Sp, p, rec)
    else:
        if p.project_adv_vel:   # step.py:292-303
            ua, va = project_column_divergence(up, vp, p, dt)
            if rec is not None:
                rec.column_projection(vertical_transport_iface(up, vp, p)[..., 0],
                                      vertical_transport_iface(ua, va, p)[..., 0])
            up, vp = ua, va
        dT2, dS2 = tracer_residual(up, vp, Tp, Sp, p, rec)
    Tn = T + 0.5 * (dT1 + dT2) * dt
    Sn = S + 0.5 * (dS1 + dS2) * dt
    du2, dv2 = momentum_residual(u, v, Tn, Sn, eta, p)
    du2 = du2 + p.r_bot * u * bm
    dv2 = dv2 + p.r_bot * v * bm
    decay = np.exp(-p.r_bot * dt * bm)
    un = (u + 0.5 * (du1 + du2) * dt) * decay
    vn = (v + 0.5 * (dv1 + dv2) * dt) * decay
    return dict(u=un, v=vn, T=Tn, S=Sn, eta=eta)


# ---------------------------------------------------------------- barotropic subcycle
def filter_barotropic_eta(eta, p, duration):
    """dynamics/barotropic.py:22-41: sponge and relaxation decays with the
    removed volume refilled uniformly, then the polar cap."""
    area = p.dx_2d * p.dy
    ocean_area = max(float(np.sum(area * p.wet_mask)), 1.0)

    def refill(now, before):
        dV = np.sum(area * (now - before))
        return now + (-dV / ocean_area) * p.wet_mask

    decayed = refill(eta * np.exp(-p.sponge_rate_2d * duration), eta)
    relaxed = refill(decayed * np.exp(-p.eta_relax_rate * duration * p.eta_relax_mask), decayed)
    return polar_cap(relaxed, p.wet_mask, p)


def free_surface_step(eta, ubt, vbt, p, F_rho_x, F_rho_y, dt_bt):
    """dynamics/barotropic.py:86-265 ``_free_surface_step_fd``, mode-split
    legacy branch: forward-backward gravity step, backward-Euler Coriolis,
    implicit linear drag, wet mask, sponge decay, polar cap."""
    wm = p.wet_mask
    Fx = F_rho_x + p.tau_x_2d / (RHO_0 * p.H_sw)
    Fy = F_rho_y + p.tau_y_2d / (RHO_0 * p.H_sw)
    drag = 1.0 / (1.0 + p.r_bot * dt_bt)
    div = divergence_conservative_2d(ubt * wm, vbt * wm, p)
    eta_new = (eta - dt_bt * p.H_sw * div) * wm
    sponge = np.exp(-p.sponge_rate_2d * dt_bt)
    eta_new = filter_barotropic_eta(eta_new, p, dt_bt)
    gx, gy = gradient_conservative_2d(eta_new, p)
    us = ubt + dt_bt * (-G_EARTH * gx + Fx)
    vs = vbt + dt_bt * (-G_EARTH * gy + Fy)
    fd = p.f * dt_bt
    den = 1.0 + fd * fd
    un = (us + fd * vs) / den * drag * wm * sponge
    vn = (vs - fd * us) / den * drag * wm * sponge
    return eta_new, polar_cap(un, wm, p), polar_cap(vn, wm, p)


# ---------------------------------------------------------------- full step
def step(st, p, rec=None):
    """timestepping/step.py:341-458 ``_step_impl``: L(dt/2) N(dt) L(dt/2), the
    barotropic subcycle and its uniform projection, polar cap, land hold and
    the no-flux wall on v; with a ledger recorder the stage hooks of
    step.py:366-368, 425-427 and 452-455."""
    dt_half = p.dt / 2.0
    held = {k: st[k] for k in ("u", "v", "T", "S")}
    s = linear_half_step(st, p, dt_half, rec)
    n_start = s
    s = explicit_full_step(s, p, rec)
    if rec is not None:
        rec.stage("nonlinear", n_start, s)
    s = linear_half_step(s, p, dt_half, rec)
    fx, fy = bt_rho_pgf(s["T"], s["S"], p)
    ubt0, vbt0 = barotropic_velocity(s["u"], s["v"], p)
    eta, ubt, vbt = s["eta"], ubt0, vbt0
    for _ in range(int(p.n_subcyc)):
        eta, ubt, vbt = free_surface_step(eta, ubt, vbt, p, fx, fy, p.dt_bt)
    u = s["u"] + (ubt - ubt0)[:, :, None]
    v = s["v"] + (vbt - vbt0)[:, :, None]
    after_bt = dict(u=u, v=v, T=s["T"], S=s["S"], eta=eta)
    if rec is not None:
        rec.stage("free_surface", s, after_bt)
    wm = p.wet_mask_z
    out = {}
    for key, field in (("u", u), ("v", v), ("T", s["T"]), ("S", s["S"])):
        capped = polar_cap(field, wm, p)
        out[key] = capped * wm + held[key] * (1.0 - wm)
    out["v"] = out["v"] * p.interior_mask_z
    out["eta"] = eta
    if rec is not None:
        rec.stage("polar_cap_and_masks", after_bt, out)
        rec.stage("dynamic_ice", out, out)
    return out


def run(st, p, nsteps):
    for _ in range(nsteps):
        st = step(st, p)
    return st
