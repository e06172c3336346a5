"""CPU oracle for gradients: the reverse-mode derivative (vector-Jacobian product) of the
numpy restatement of one simulate.step, and of a rollout with curvature actuation.

TEST INFRASTRUCTURE ONLY, like ``ref_numpy``: the CUDA adjoint kernels are checked
against it, and it is itself checked against central finite differences of
``ref_numpy`` in float64.

It follows the derivative conventions ``jax.grad`` applies to the reference:

* the Peskin stencil positions are ``jax.lax.stop_gradient``-ed
  (src/microcosmos/solver/fluid.py:237-239): the IB weights, indices, coverage and
  its inverse are constants of the derivative;
* ``floor`` has derivative 0, ``mod`` (jnp.mod) derivative 1 in its first argument;
* ``max(a, b)`` / ``min(a, b)`` pass the cotangent to the selected argument and split
  it evenly on a tie (lax.max / lax.min JVP rules);
* the steric potential is differentiated through the deposit weights, the spectral
  filter (a symmetric circular convolution, its own adjoint), the bilinear samples
  (weights and values) and the analytic neighbour term.

The cotangents of the outputs ``steric`` and ``fluid_velocity`` are taken as zero (they
are diagnostics of the step, not inputs to the next one).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import ref_numpy as R

E = R.E
WGT = R.WGT
OPP = R.OPP


def dmax(x, c):
    """d max(x, c) / dx with the even split on ties."""
    return np.where(x > c, 1.0, np.where(x == c, 0.5, 0.0)).astype(np.result_type(x))


def clamp_vjp(x, y, vmax, gx, gy):
    """Cotangent of (x, y) through (x c, y c), c = min(1, vmax / (sqrt(x^2+y^2+eps)+eps))
    (src/microcosmos/solver/fluid.py:272-274, 300-303, 312-314)."""
    dt = np.result_type(x)
    eps = dt.type(R.EPSIL32)
    mag = np.sqrt(x * x + y * y + eps)
    a = dt.type(vmax) / (mag + eps)
    c = np.minimum(dt.type(1.0), a)
    sel = np.where(a < 1.0, 1.0, np.where(a == 1.0, 0.5, 0.0)).astype(dt)
    gc = x * gx + y * gy
    da = -dt.type(vmax) / ((mag + eps) * (mag + eps))
    k = gc * sel * da / mag
    return c * gx + k * x, c * gy + k * y


def actuation(act, t, dtype):
    c, amp, om, ph = (np.asarray(a, dtype) for a in act)
    return c + amp * np.sin(om * dtype(t) + ph)


# ----------------------------------------------------------------------------- tape
@dataclasses.dataclass
class Tape:
    s: R.State                  # step input
    rest: np.ndarray            # rest angles used by the step
    pred0: np.ndarray
    V: np.ndarray | None
    pbd_pos: list               # PBD iteration inputs pos_0 .. pos_{C-1}, then the final pos_C
    pbd_theta: list             # theta_0 .. theta_C
    vel1: np.ndarray
    ib: dict | None


def _ib_tape(H, W, pos, vel, f_grid, cfg, dtstep, ib_positions, pairs=None):
    """ib_lbm with its intermediates kept (same arithmetic as ref_numpy.ib_lbm).  With
    synthetic_node_width > 0 the IB points are the synthetic pairs, built from the
    stop_gradient-ed stencil positions (constants of the derivative, fluid.py:259), each
    carrying its node's velocity; a node's reaction is the mean of its two points'."""
    dt = f_grid.dtype
    t = dt.type
    h, w = f_grid.shape[1], f_grid.shape[2]  # the fluid lattice; (H, W) is the domain grid
    scale = np.array([w / H, h / W], dtype=dt)
    vmax = cfg.max_fluid_velocity * 0.5 * (w / H + h / W)
    eps = t(R.EPSIL32)
    node_vel = vel * scale * t(dtstep)
    gpos = (pos if ib_positions is None else ib_positions) * scale
    nn = pos.shape[0]
    syn = cfg.synthetic_node_width > 0.0
    if syn:
        gpos = R.synthetic_ib_positions(H, W, pos if ib_positions is None else ib_positions, pairs, gpos,
                                        cfg.synthetic_node_width, 0.5 * (w / H + h / W))
        node_vel = np.concatenate([node_vel, node_vel], axis=0)
    f0 = np.maximum(f_grid, eps)
    rho_raw = f0[0]
    for i in range(1, 9):
        rho_raw = rho_raw + f0[i]
    rho, ux, uy = R.macroscopic(f0)
    c1 = R.velocity_clamp_factor(ux, uy, vmax)
    vx, vy = ux * c1, uy * c1
    idx, wts = R.peskin_weights(h, w, gpos, cfg.ibm_kernel_size)
    flat = idx.reshape(-1)
    wflat = wts.reshape(-1)
    cov = np.zeros(h * w, dt)
    np.add.at(cov, flat, wflat)
    inv = t(1.0) / np.maximum(cov, t(1.0))
    ucx = vx.reshape(-1).copy()
    ucy = vy.reshape(-1).copy()
    nst = wts.shape[1]
    sraw = []
    for _ in range(cfg.ibm_iterations):
        gx = ucx[idx] * wts
        gy = ucy[idx] * wts
        ix_ = np.zeros(gx.shape[0], dt)
        iy_ = np.zeros(gx.shape[0], dt)
        for k in range(nst):
            ix_ = ix_ + gx[:, k]
            iy_ = iy_ + gy[:, k]
        sx = (node_vel[:, 0] - ix_) * t(cfg.ibm_relaxation)
        sy = (node_vel[:, 1] - iy_) * t(cfg.ibm_relaxation)
        sraw.append((sx, sy))
        mag = np.sqrt(sx * sx + sy * sy + eps)
        cf = np.minimum(t(1.0), t(vmax) / (mag + eps))
        dx = np.zeros(h * w, dt)
        dy = np.zeros(h * w, dt)
        np.add.at(dx, flat, np.repeat(sx * cf, nst) * wflat)
        np.add.at(dy, flat, np.repeat(sy * cf, nst) * wflat)
        ucx = ucx + dx * inv
        ucy = ucy + dy * inv
    uc5x, uc5y = ucx.reshape(h, w), ucy.reshape(h, w)
    c2 = R.velocity_clamp_factor(uc5x, uc5y, vmax)
    ucx_c, ucy_c = uc5x * c2, uc5y * c2
    Fx = (ucx_c - vx) * rho
    Fy = (ucy_c - vy) * rho
    Fraw = None
    if cfg.enable_force_clamp:
        # the optional force clamp (fluid.py:336-339), same factor form as the velocity clamp
        Fraw = (Fx, Fy)
        c3 = R.velocity_clamp_factor(Fx, Fy, vmax)
        Fx = Fx * c3
        Fy = Fy * c3
    wp, wm = R.trt_rates(cfg, dt)
    fpost, usx, usy = R.collide(f0, rho, vx, vy, Fx, Fy, wp, wm)
    fnew = R.stream(fpost)
    Ff = (Fx.reshape(-1), Fy.reshape(-1))
    nf = []
    for comp in Ff:
        g = comp[idx] * wts
        acc = np.zeros(g.shape[0], dt)
        for k in range(nst):
            acc = acc + g[:, k]
        if syn:
            acc = t(0.5) * (acc[:nn] + acc[nn:])
        nf.append(acc)
    sdt = scale * t(dtstep)
    vel_out = np.stack([vel[:, 0] - (nf[0] / t(cfg.node_mass)) / sdt[0],
                        vel[:, 1] - (nf[1] / t(cfg.node_mass)) / sdt[1]], axis=-1)
    tape = dict(syn=syn, nn=nn, Fraw=Fraw, scale=scale, vmax=vmax, f=f_grid, f0=f0, rho_raw=rho_raw, rho=rho, ux=ux, uy=uy, vx=vx, vy=vy,
                idx=idx, wts=wts, inv=inv, sraw=sraw, uc5=(uc5x, uc5y), ucc=(ucx_c, ucy_c), F=(Fx, Fy),
                fpost=fpost, wp=wp, wm=wm, sdt=sdt)
    return vel_out, fnew, np.stack([usx, usy]), tape


def step_tape(s: R.State, cfg: R.Config, dtstep: float, rest_angles, ib_positions=None):
    """ref_numpy.step with every intermediate the derivative needs."""
    dt = s.position.dtype
    t = dt.type
    H, W = s.H, s.W
    rest = s.bending_rest_angles if rest_angles is None else np.asarray(rest_angles, dt)
    prev = s.position
    pred0 = prev + s.velocity * t(cfg.damping) * t(dtstep)
    pred = pred0
    V = None
    if cfg.enable_steric:
        V, fst = R.steric_force(H, W, pred0, cfg)
        pred = pred0 + fst * t(cfg.steric_strength) * t(dtstep)
    pos, theta = pred, s.theta
    pp, tt = [pos], [theta]
    for _ in range(cfg.cycles_per_step):
        if cfg.solver_type == "cosserat":
            pos, theta = R.cosserat_iteration(H, W, pos, pred, theta, s.pairs, s.bending_pairs, s.rest_lengths,
                                              rest, s.bending_stiffness, cfg)
        else:
            pos, theta = R.pbd_iteration(H, W, pos, theta, s.pairs, s.bending_pairs, s.rest_lengths, rest,
                                         s.bending_stiffness, cfg)
        pp.append(pos)
        tt.append(theta)
    vel1 = (pos - prev) / t(dtstep)
    out = s.copy()
    out.bending_rest_angles = rest
    ib = None
    vel = vel1
    if cfg.enable_fluid:
        vel, fnew, fluid_u, ib = _ib_tape(H, W, pos, vel1, s.f_grid, cfg, dtstep, ib_positions, s.pairs)
        out.f_grid = fnew
        out.fluid_velocity = fluid_u
    if V is not None:
        out.steric = V
    out.position = R.periodic_boundary(H, W, pos)
    out.velocity = vel
    out.theta = theta
    return out, Tape(s=s, rest=rest, pred0=pred0, V=V, pbd_pos=pp, pbd_theta=tt, vel1=vel1, ib=ib)


# ----------------------------------------------------------------------------- pieces
def collide_vjp(f0, rho, vx, vy, Fx, Fy, wp, wm, g_out):
    """Cotangents of (f0, rho, vx, vy, Fx, Fy) through ref_numpy.collide's first output."""
    dt = f0.dtype
    t = dt.type
    half = t(0.5)
    usx = vx + half * Fx / rho
    usy = vy + half * Fy / rho
    feq = R.equilibrium(rho, usx, usy)
    udF = usx * Fx + usy * Fy
    usq = usx * usx + usy * usy
    raw = []
    for i in range(9):
        eu = t(E[i, 0]) * usx + t(E[i, 1]) * usy
        eF = t(E[i, 0]) * Fx + t(E[i, 1]) * Fy
        raw.append(t(WGT[i]) * (t(3.0) * (eF - udF) + t(9.0) * eu * eF))
    raw = np.stack(raw)
    post = f0 - wp * (half * (f0 + f0[OPP]) - half * (feq + feq[OPP])) - wm * (half * (f0 - f0[OPP]) - half * (feq - feq[OPP]))
    src = (t(1.0) - half * wp) * (half * (raw + raw[OPP])) + (t(1.0) - half * wm) * (half * (raw - raw[OPP]))
    g = g_out * dmax(post + src, t(R.EPSIL32))
    gp = half * (g + g[OPP])
    gm = half * (g - g[OPP])
    lf = g - wp * gp - wm * gm
    lfeq = wp * gp + wm * gm
    lraw = (t(1.0) - half * wp) * gp + (t(1.0) - half * wm) * gm
    lrho = np.zeros_like(rho)
    lusx = np.zeros_like(rho)
    lusy = np.zeros_like(rho)
    lFx = np.zeros_like(rho)
    lFy = np.zeros_like(rho)
    for i in range(9):
        ex, ey = t(E[i, 0]), t(E[i, 1])
        wi = t(WGT[i])
        eu = ex * usx + ey * usy
        eF = ex * Fx + ey * Fy
        lrho = lrho + lfeq[i] * wi * (t(1.0) + t(3.0) * eu + t(4.5) * eu * eu - t(1.5) * usq)
        a = lfeq[i] * rho * wi
        lusx = lusx + a * (t(3.0) * ex + t(9.0) * eu * ex - t(3.0) * usx)
        lusy = lusy + a * (t(3.0) * ey + t(9.0) * eu * ey - t(3.0) * usy)
        b = lraw[i] * wi
        lusx = lusx + b * (-t(3.0) * Fx + t(9.0) * eF * ex)
        lusy = lusy + b * (-t(3.0) * Fy + t(9.0) * eF * ey)
        lFx = lFx + b * (t(3.0) * ex - t(3.0) * usx + t(9.0) * eu * ex)
        lFy = lFy + b * (t(3.0) * ey - t(3.0) * usy + t(9.0) * eu * ey)
    lvx, lvy = lusx, lusy
    lFx = lFx + half * lusx / rho
    lFy = lFy + half * lusy / rho
    lrho = lrho - half * (lusx * Fx + lusy * Fy) / (rho * rho)
    return lf, lrho, lvx, lvy, lFx, lFy


def _gather_sum(field_flat, idx, wts):
    g = field_flat[idx] * wts
    acc = np.zeros(g.shape[0], g.dtype)
    for k in range(g.shape[1]):
        acc = acc + g[:, k]
    return acc


def _scatter(n_cells, idx, wts, node_vals):
    out = np.zeros(n_cells, wts.dtype)
    np.add.at(out, idx.reshape(-1), (node_vals[:, None] * wts).reshape(-1))
    return out


def ib_vjp(H, W, cfg, dtstep, tp, lvel_out, lf_new):
    """Cotangents of (vel1, f_grid) through _ib_tape's (vel_out, f_new).  Everything here
    lives on the fluid lattice, whose shape is the tape's f_grid's."""
    dt = lf_new.dtype
    t = dt.type
    eps = t(R.EPSIL32)
    idx, wts, inv = tp["idx"], tp["wts"], tp["inv"]
    H, W = tp["f"].shape[1], tp["f"].shape[2]
    HW = H * W
    # node reaction: vel_out = vel1 - (nf / m) / sdt
    lvel1 = lvel_out.copy()
    lnf = [-lvel_out[:, 0] / t(cfg.node_mass) / tp["sdt"][0], -lvel_out[:, 1] / t(cfg.node_mass) / tp["sdt"][1]]
    if tp["syn"]:
        # a node's reaction is 0.5 (point + its pair): each point gets half the cotangent
        lnf = [np.concatenate([t(0.5) * a, t(0.5) * a]) for a in lnf]
    lFx = _scatter(HW, idx, wts, lnf[0]).reshape(H, W)
    lFy = _scatter(HW, idx, wts, lnf[1]).reshape(H, W)
    # stream: f_new_i[y+cy, x+cx] = max(fpost_i[y, x], eps)
    fpost = tp["fpost"]
    lpost = np.empty_like(lf_new)
    for i in range(9):
        cx, cy = int(E[i, 0]), int(E[i, 1])
        g = lf_new[i] * dmax(np.roll(fpost[i], shift=(cy, cx), axis=(0, 1)), eps)
        lpost[i] = np.roll(g, shift=(-cy, -cx), axis=(0, 1))
    rho, vx, vy = tp["rho"], tp["vx"], tp["vy"]
    Fx, Fy = tp["F"]
    lf0, lrho, lvx, lvy, cFx, cFy = collide_vjp(tp["f0"], rho, vx, vy, Fx, Fy, tp["wp"], tp["wm"], lpost)
    lFx = lFx + cFx
    lFy = lFy + cFy
    if tp["Fraw"] is not None:
        lFx, lFy = clamp_vjp(tp["Fraw"][0], tp["Fraw"][1], tp["vmax"], lFx, lFy)
    # F = (ucc - v) rho
    uccx, uccy = tp["ucc"]
    luccx, luccy = lFx * rho, lFy * rho
    lvx = lvx - lFx * rho
    lvy = lvy - lFy * rho
    lrho = lrho + lFx * (uccx - vx) + lFy * (uccy - vy)
    uc5x, uc5y = tp["uc5"]
    lux_, luy_ = clamp_vjp(uc5x, uc5y, tp["vmax"], luccx, luccy)
    lucx, lucy = lux_.reshape(-1).copy(), luy_.reshape(-1).copy()
    # multi-direct forcing iterations, last first
    lnode_vel = np.zeros((idx.shape[0], 2), dt)
    relax = t(cfg.ibm_relaxation)
    for k in reversed(range(cfg.ibm_iterations)):
        sx, sy = tp["sraw"][k]
        lsx = _gather_sum(inv * lucx, idx, wts)
        lsy = _gather_sum(inv * lucy, idx, wts)
        lrx, lry = clamp_vjp(sx, sy, tp["vmax"], lsx, lsy)
        lnode_vel[:, 0] += relax * lrx
        lnode_vel[:, 1] += relax * lry
        lucx = lucx + _scatter(HW, idx, wts, -relax * lrx)
        lucy = lucy + _scatter(HW, idx, wts, -relax * lry)
    lvx = lvx + lucx.reshape(H, W)
    lvy = lvy + lucy.reshape(H, W)
    lux, luy = clamp_vjp(tp["ux"], tp["uy"], tp["vmax"], lvx, lvy)
    # macroscopic: rho = max(sum f, 0.1), u = m / rho
    ux, uy = tp["ux"], tp["uy"]
    lrho = lrho - (lux * ux + luy * uy) / rho
    lraw = lrho * dmax(tp["rho_raw"], t(0.1))
    for i in range(9):
        lf0[i] = lf0[i] + lraw + (t(E[i, 0]) * lux + t(E[i, 1]) * luy) / rho
    lf = lf0 * dmax(tp["f"], eps)
    if tp["syn"]:
        nn = tp["nn"]
        lnode_vel = lnode_vel[:nn] + lnode_vel[nn:]
    lvel1 = lvel1 + lnode_vel * tp["scale"] * t(dtstep)
    return lvel1, lf


def _sample_parts(V, yy, xx):
    """Bilinear wrap sample pieces: the four (cell, weight) pairs and d/dy, d/dx."""
    dt = V.dtype
    H, W = V.shape
    ly, lx = np.floor(yy), np.floor(xx)
    ty, tx = yy - ly, xx - lx
    iy, ix = ly.astype(np.int64), lx.astype(np.int64)
    iy0, iy1 = np.mod(iy, H), np.mod(iy + 1, H)
    ix0, ix1 = np.mod(ix, W), np.mod(ix + 1, W)
    one = dt.type(1.0)
    v00, v01, v10, v11 = V[iy0, ix0], V[iy0, ix1], V[iy1, ix0], V[iy1, ix1]
    dsdx = (one - ty) * (v01 - v00) + ty * (v11 - v10)
    dsdy = (one - tx) * (v10 - v00) + tx * (v11 - v01)
    cells = [(iy0, ix0, (one - ty) * (one - tx)), (iy0, ix1, (one - ty) * tx),
             (iy1, ix0, ty * (one - tx)), (iy1, ix1, ty * tx)]
    return cells, dsdy, dsdx


def gaussian_filter_adjoint(g, sigma):
    """The spectral filter is real, even in frequency: it is its own adjoint."""
    return R.gaussian_filter(g, sigma)


def steric_vjp(H, W, cfg, dtstep, pred0, V, lpred1):
    """Cotangent of pred0 through pred1 = pred0 + steric_force(pred0) * strength * dt."""
    dt = pred0.dtype
    t = dt.type
    lf = lpred1 * t(cfg.steric_strength) * t(dtstep)
    lpred0 = lpred1.copy()
    p = R.periodic_boundary(H, W, pred0)
    x, y = p[:, 0], p[:, 1]
    e = t(0.5)
    lV = np.zeros((H, W), dt)
    lp = np.zeros_like(p)
    # raw = -[(S(y, x+e) - S(y, x-e)) / 1, (S(y+e, x) - S(y-e, x)) / 1]
    den = t(1.0)
    for (yy, xx, coef_x, coef_y) in ((y, x + e, -lf[:, 0] / den, None), (y, x - e, lf[:, 0] / den, None),
                                      (y + e, x, None, -lf[:, 1] / den), (y - e, x, None, lf[:, 1] / den)):
        coef = coef_x if coef_x is not None else coef_y
        cells, dsdy, dsdx = _sample_parts(V, yy, xx)
        for (cy, cx, wgt) in cells:
            np.add.at(lV, (cy, cx), coef * wgt)
        lp[:, 0] += coef * dsdx
        lp[:, 1] += coef * dsdy
    # analytic neighbour term: fst -= (s / sigma^2) sum_o valid K(r) r
    n = cfg.steric_neighbor_skip
    N = p.shape[0]
    if n > 0:
        sigma = cfg.steric_sigma
        s2 = t(sigma * sigma)
        inv2s2 = t(2.0 * sigma * sigma)
        norm = t(2.0 * np.pi * sigma * sigma)
        pre = t(cfg.steric_scatter_value / (sigma * sigma))
        for o in range(-n, n + 1):
            j = np.arange(N) + o
            valid = ((j >= 0) & (j < N)).astype(dt)
            js = np.clip(j, 0, N - 1)
            r = R.displacement(H, W, p, p[js])
            d2 = r[:, 0] * r[:, 0] + r[:, 1] * r[:, 1]
            K = np.exp(-d2 / inv2s2) / norm * valid
            # d(K r)/dr = K (I - r r^T / sigma^2); cotangent of (K r) is -pre * lf
            gx, gy = -pre * lf[:, 0], -pre * lf[:, 1]
            rg = (r[:, 0] * gx + r[:, 1] * gy) / s2
            lrx = K * (gx - r[:, 0] * rg)
            lry = K * (gy - r[:, 1] * rg)
            lp[:, 0] += lrx
            lp[:, 1] += lry
            np.add.at(lp[:, 0], js, -lrx)
            np.add.at(lp[:, 1], js, -lry)
    lpred0 += lp
    # V = G * deposit(pred0)
    ldep = gaussian_filter_adjoint(lV, cfg.steric_sigma)
    fx, fy = np.floor(x), np.floor(y)
    x0 = np.mod(fx.astype(np.int64), W)
    y0 = np.mod(fy.astype(np.int64), H)
    x1, y1 = (x0 + 1) % W, (y0 + 1) % H
    dx, dy = x - fx, y - fy
    one = t(1.0)
    sv = t(cfg.steric_scatter_value)
    d00, d10, d01, d11 = ldep[y0, x0], ldep[y0, x1], ldep[y1, x0], ldep[y1, x1]
    lpred0[:, 0] += sv * (-(one - dy) * d00 + (one - dy) * d10 - dy * d01 + dy * d11)
    lpred0[:, 1] += sv * (-(one - dx) * d00 - dx * d10 + (one - dx) * d01 + dx * d11)
    return lpred0


def pbd_iteration_vjp(H, W, cfg, s, rest, pos, theta, lpos_out, ltheta_out):
    """Cotangents of (pos, theta, rest, rest_lengths, bending_stiffness) through one
    ref_numpy.pbd_iteration."""
    dt = pos.dtype
    t = dt.type
    Ecount = theta.shape[0]
    N = pos.shape[0]
    src, tgt = s.pairs[:, 0], s.pairs[:, 1]
    ein, eout = s.bending_pairs[:, 0], s.bending_pairs[:, 1]
    kb = s.bending_stiffness
    L0 = s.rest_lengths
    edeg = np.zeros(Ecount, dt)
    np.add.at(edeg, ein, t(1.0))
    np.add.at(edeg, eout, t(1.0))
    edeg = np.maximum(edeg, t(1.0))
    pi = t(np.pi)
    diff = np.mod(theta[eout] - theta[ein] + pi, t(2 * np.pi)) - pi
    corr = (diff - rest) * kb * t(0.5)
    delta = np.zeros(Ecount, dt)
    np.add.at(delta, ein, corr)
    np.add.at(delta, eout, -corr)
    theta_new = theta + delta / edeg * t(1.8)
    ndeg = np.zeros(N, dt)
    np.add.at(ndeg, src, t(1.0))
    np.add.at(ndeg, tgt, t(1.0))
    ndeg = np.maximum(ndeg, t(1.0))
    cur = R.displacement(H, W, pos[tgt], pos[src])
    L = np.sqrt(cur[:, 0] * cur[:, 0] + cur[:, 1] * cur[:, 1])
    m = np.maximum(L, t(1e-8))
    ks, kst = t(cfg.stiffness_shear), t(cfg.stiffness_stretch)
    # position pass
    ldisp = lpos_out / ndeg[:, None]
    h = (ldisp[src] - ldisp[tgt]) * kst * t(0.5)
    lstretch = (t(1.0) - ks) * h
    lcur = ks * h
    ltarget = -ks * h
    # stretch = cur (L - L0) / m
    a = (L - L0) / m
    dL = dmax(L, t(1e-8))
    # d a / d cur = cur / L * (1/m - (L - L0) dL / m^2)
    da = (t(1.0) / m - (L - L0) * dL / (m * m)) / L
    sdot = cur[:, 0] * lstretch[:, 0] + cur[:, 1] * lstretch[:, 1]
    lcur = lcur + a[:, None] * lstretch + (sdot * da)[:, None] * cur
    lL0 = -sdot / m
    c, sn = np.cos(theta_new), np.sin(theta_new)
    lL0 = lL0 + c * ltarget[:, 0] + sn * ltarget[:, 1]
    ltheta_new = ltheta_out + L0 * (-sn * ltarget[:, 0] + c * ltarget[:, 1])
    lpos = lpos_out.copy()
    np.add.at(lpos, tgt, lcur)
    np.add.at(lpos, src, -lcur)
    # theta pass: theta_new = theta + (sum_in corr - sum_out corr) / edeg * 1.8
    lcorr = t(1.8) * (ltheta_new[ein] / edeg[ein] - ltheta_new[eout] / edeg[eout])
    ltheta = ltheta_new.copy()
    g = lcorr * kb * t(0.5)
    np.add.at(ltheta, eout, g)
    np.add.at(ltheta, ein, -g)
    lrest = -g
    lkb = lcorr * (diff - rest) * t(0.5)
    return lpos, ltheta, lrest, lL0, lkb


def cosserat_iteration_vjp(H, W, cfg, s, rest, pos, y, theta, lpos_out, ltheta_out):
    """Cotangents of (pos, y, theta, rest, rest_lengths, bending_stiffness) through one
    ref_numpy.cosserat_iteration (y: the inertial prediction the iteration pulls toward).
    mod has derivative 1 (so the pull's wrap passes its cotangent through), and
    d atan2(r_y, r_x) = (r_x dr_y - r_y dr_x) / |r|^2."""
    dt = pos.dtype
    t = dt.type
    Ecount = theta.shape[0]
    N = pos.shape[0]
    src, tgt = s.pairs[:, 0], s.pairs[:, 1]
    ein, eout = s.bending_pairs[:, 0], s.bending_pairs[:, 1]
    kb = s.bending_stiffness
    L0 = s.rest_lengths
    edeg = np.zeros(Ecount, dt)
    np.add.at(edeg, ein, t(1.0))
    np.add.at(edeg, eout, t(1.0))
    edeg = np.maximum(edeg, t(1.0))
    pi = t(np.pi)
    twopi = t(2 * np.pi)
    diff = np.mod(theta[eout] - theta[ein] + pi, twopi) - pi
    corr = (diff - rest) * kb * t(0.5)
    delta = np.zeros(Ecount, dt)
    np.add.at(delta, ein, corr)
    np.add.at(delta, eout, -corr)
    th1 = theta + delta / edeg
    seg = R.displacement(H, W, pos[tgt], pos[src])
    alpha = np.arctan2(seg[:, 1], seg[:, 0])
    thn = th1 + (np.mod(alpha - th1 + pi, twopi) - pi) * t(0.05)
    ks = t(cfg.stiffness_stretch)
    w = t(1.0 / (cfg.dt ** 2))
    cs, sn = np.cos(thn), np.sin(thn)
    f_edge = (ks / L0)[:, None] * (seg / L0[:, None] - np.stack([cs, sn], axis=-1))
    f_node = w * (y - pos)
    h_node = np.full(N, w, dt)
    np.add.at(f_node, src, f_edge)
    np.add.at(f_node, tgt, -f_edge)
    np.add.at(h_node, src, ks / (L0 * L0))
    np.add.at(h_node, tgt, ks / (L0 * L0))
    # x_new = pos + f_node / h_node
    lf = lpos_out / h_node[:, None]
    lh = -np.sum(lpos_out * f_node, axis=1) / (h_node * h_node)
    lpos = lpos_out - w * lf
    ly = w * lf
    lfe = lf[src] - lf[tgt]
    # f_edge = (ks / L0) (seg / L0 - d(thn)), h_edge = ks / L0^2
    lseg = (ks / L0 / L0)[:, None] * lfe
    lthn = ltheta_out + (ks / L0) * (lfe[:, 0] * sn - lfe[:, 1] * cs)
    lL0 = (np.sum(lfe * (-(ks / (L0 * L0))[:, None] * (seg / L0[:, None] - np.stack([cs, sn], axis=-1))
                         - (ks / L0)[:, None] * seg / (L0 * L0)[:, None]), axis=1)
           + (lh[src] + lh[tgt]) * (-t(2.0) * ks / (L0 * L0 * L0)))
    # thn = th1 + wrap(alpha - th1) * 0.05
    lth1 = lthn - t(0.05) * lthn
    lalpha = t(0.05) * lthn
    r2 = seg[:, 0] * seg[:, 0] + seg[:, 1] * seg[:, 1]
    lseg = lseg + np.stack([-seg[:, 1] * lalpha / r2, seg[:, 0] * lalpha / r2], axis=-1)
    np.add.at(lpos, tgt, lseg)
    np.add.at(lpos, src, -lseg)
    # th1 = theta + (sum_in corr - sum_out corr) / edeg
    lcorr = lth1[ein] / edeg[ein] - lth1[eout] / edeg[eout]
    ltheta = lth1.copy()
    g = lcorr * kb * t(0.5)
    np.add.at(ltheta, eout, g)
    np.add.at(ltheta, ein, -g)
    lrest = -g
    lkb = lcorr * (diff - rest) * t(0.5)
    return lpos, ly, ltheta, lrest, lL0, lkb


@dataclasses.dataclass
class StepCot:
    position: np.ndarray
    velocity: np.ndarray
    theta: np.ndarray
    f_grid: np.ndarray | None
    rest: np.ndarray | None = None
    rest_lengths: np.ndarray | None = None
    bending_stiffness: np.ndarray | None = None


def step_vjp(cfg: R.Config, dtstep: float, tape: Tape, cot: StepCot) -> StepCot:
    """Cotangents of the step input (position, velocity, theta, f_grid) and of the rest
    angles, rest lengths and bending stiffness, given those of the step output."""
    s = tape.s
    H, W = s.H, s.W
    dt = s.position.dtype
    t = dt.type
    lvel_out = cot.velocity
    lf = cot.f_grid          # without the fluid the lattice passes through unchanged
    if cfg.enable_fluid:
        lvel1, lf = ib_vjp(H, W, cfg, dtstep, tape.ib, lvel_out, cot.f_grid)
    else:
        lvel1 = lvel_out
    # vel1 = (pos_C - prev) / dt; position output = mod(pos_C)
    lposC = cot.position + lvel1 / t(dtstep)
    lprev = -lvel1 / t(dtstep)
    lpos, ltheta = lposC, cot.theta.copy()
    lrest = np.zeros_like(tape.rest)
    lL0 = np.zeros_like(s.rest_lengths)
    lkb = np.zeros_like(s.bending_stiffness)
    ly = np.zeros_like(lpos)
    for k in reversed(range(cfg.cycles_per_step)):
        if cfg.solver_type == "cosserat":
            lpos, lyk, ltheta, lr, ll, lk = cosserat_iteration_vjp(H, W, cfg, s, tape.rest, tape.pbd_pos[k],
                                                                   tape.pbd_pos[0], tape.pbd_theta[k], lpos, ltheta)
            ly = ly + lyk
        else:
            lpos, ltheta, lr, ll, lk = pbd_iteration_vjp(H, W, cfg, s, tape.rest, tape.pbd_pos[k],
                                                         tape.pbd_theta[k], lpos, ltheta)
        lrest += lr
        lL0 += ll
        lkb += lk
    # the Cosserat iterations start from the prediction and are pulled toward it
    lpos = lpos + ly
    if cfg.enable_steric:
        lpred0 = steric_vjp(H, W, cfg, dtstep, tape.pred0, tape.V, lpos)
    else:
        lpred0 = lpos
    return StepCot(position=lprev + lpred0, velocity=lpred0 * t(cfg.damping) * t(dtstep), theta=ltheta, f_grid=lf,
                   rest=lrest, rest_lengths=lL0, bending_stiffness=lkb)


# ----------------------------------------------------------------------------- rollout
def rollout(s, cfg, dtstep, num_steps, act=None, ib_positions=None, t0=0):
    """Forward rollout in the state's dtype; returns the final state and the tapes.
    ``ib_positions`` (list, one array per step) hold the Peskin stencil positions."""
    dt = s.position.dtype
    tapes = []
    for k in range(num_steps):
        ra = None if act is None else actuation(act, t0 + k, dt.type)
        s, tp = step_tape(s, cfg, dtstep, ra, None if ib_positions is None else ib_positions[k])
        tapes.append(tp)
    return s, tapes


def ib_positions_of(tapes):
    """The Peskin stencil positions a rollout used (its PBD outputs), for freezing them."""
    return [tp.pbd_pos[-1].copy() for tp in tapes]


def rollout_vjp(cfg, dtstep, tapes, cot: StepCot, act=None, t0=0):
    """Cotangents of the initial state and, with actuation (c, amp, omega, phase) per
    bending pair, of c, amp and phase; else of the static rest angles."""
    dt = tapes[0].s.position.dtype
    tt = dt.type
    lrest_static = np.zeros_like(tapes[0].rest)
    lc = np.zeros_like(tapes[0].rest)
    lamp = np.zeros_like(lc)
    lph = np.zeros_like(lc)
    lom = np.zeros_like(lc)
    lL0 = np.zeros_like(tapes[0].s.rest_lengths)
    lkb = np.zeros_like(tapes[0].s.bending_stiffness)
    for k in reversed(range(len(tapes))):
        cot = step_vjp(cfg, dtstep, tapes[k], cot)
        lL0 += cot.rest_lengths
        lkb += cot.bending_stiffness
        if act is None:
            lrest_static += cot.rest
        else:
            c, amp, om, ph = (np.asarray(a, dt) for a in act)
            arg = om * tt(t0 + k) + ph
            lc += cot.rest
            lamp += cot.rest * np.sin(arg)
            lph += cot.rest * amp * np.cos(arg)
            lom += cot.rest * amp * np.cos(arg) * tt(t0 + k)
    out = dict(position=cot.position, velocity=cot.velocity, theta=cot.theta, f_grid=cot.f_grid,
               rest_lengths=lL0, bending_stiffness=lkb)
    if act is None:
        out["rest"] = lrest_static
    else:
        out.update(act_c=lc, act_amp=lamp, act_omega=lom, act_phase=lph)
    return out
