"""CPU oracle: a numpy restatement of microcosmos's per-step physics hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``microcosmos_b200``) imports
this module; it is the checker that the CUDA path is compared against, and the
CPU baseline that ``bench.py`` times.  It is pinned against golden vectors that
were produced by executing the reference's own source on numpy (see
``tests/golden/make_golden.py``), because the reference's tests hold no numeric
known-answer vectors.

Every function cites the reference lines it restates (paths relative to the
reference project root).  ``dtype`` selects float32 (the reference's arithmetic,
x64 disabled) or float64 (used to state the error of float32 results); ``EPSIL``
stays float32 epsilon in both, as in ``src/microcosmos/utils.py:9``.

Summation orders are fixed and sequential (population sums in index order, stencil
sums in stencil order, scatter-adds in update order as ``np.add.at`` applies them)
so that the CUDA kernels can reproduce them; XLA's own reduction order is
unspecified, which is why the golden comparisons carry a small tolerance.
"""
from __future__ import annotations

import dataclasses

import numpy as np

EPSIL32 = float(np.finfo(np.float32).eps)

# D2Q9 lattice (src/microcosmos/solver/fluid.py:15-23)
E = np.array([[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1],
              [1, 1], [-1, 1], [-1, -1], [1, -1]], dtype=np.int64)
WGT = np.array([4 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 36, 1 / 36, 1 / 36, 1 / 36])
OPP = np.array([0, 3, 4, 1, 2, 7, 8, 5, 6])


@dataclasses.dataclass(frozen=True)
class Config:
    """The scalar fields of ConstraintSolverConfig used by the PBD path
    (src/microcosmos/solver/config.py:9-97); defaults are the benchmark overrides of
    PBD_SCHEME (viscosity 0.1, 4-point kernel, steric on, stretch/shear 1.0/0.1)."""
    cycles_per_step: int = 20
    stiffness_stretch: float = 1.0
    stiffness_shear: float = 0.1
    damping: float = 1.0
    enable_fluid: bool = True
    viscosity: float = 0.1
    max_fluid_velocity: float = 0.2
    ibm_iterations: int = 5
    synthetic_node_width: float = 0.0
    ibm_kernel_size: int = 4
    ibm_relaxation: float = 0.3
    node_mass: float = 1.0
    lambda_trt: float = 0.25
    enable_force_clamp: bool = False
    enable_steric: bool = True
    steric_strength: float = 1.0
    steric_sigma: float = 1.5
    steric_neighbor_skip: int = 5
    steric_scatter_value: float = 1.0
    # rod solver: "pbd" (solver/pbd.py) or "cosserat" (solver/stable_cosserat.py), whose
    # inertia weight is 1 / dt**2 with this dt (solver/config.py:29-31)
    solver_type: str = "pbd"
    dt: float = 0.05


@dataclasses.dataclass
class State:
    """Nodes/Edges/Fields of one rollout (structs/*.py), numpy arrays."""
    H: int
    W: int
    position: np.ndarray
    velocity: np.ndarray
    pairs: np.ndarray
    theta: np.ndarray
    rest_lengths: np.ndarray
    bending_pairs: np.ndarray
    bending_rest_angles: np.ndarray
    bending_stiffness: np.ndarray
    f_grid: np.ndarray
    steric: np.ndarray
    fluid_velocity: np.ndarray

    def copy(self):
        return dataclasses.replace(self, **{f.name: (getattr(self, f.name).copy()
                                                     if isinstance(getattr(self, f.name), np.ndarray)
                                                     else getattr(self, f.name))
                                            for f in dataclasses.fields(self)})

    def astype(self, dt):
        kw = {}
        for f in dataclasses.fields(self):
            v = getattr(self, f.name)
            if isinstance(v, np.ndarray) and np.issubdtype(v.dtype, np.floating):
                v = v.astype(dt)
            kw[f.name] = v
        return State(**kw)


def state_from_scenario(sc, dtype=np.float32):
    return State(H=sc.H, W=sc.W, position=sc.position.copy(), velocity=sc.velocity.copy(),
                 pairs=sc.pairs.copy(), theta=sc.theta.copy(), rest_lengths=sc.rest_lengths.copy(),
                 bending_pairs=sc.bending_pairs.copy(),
                 bending_rest_angles=sc.bending_rest_angles.copy(),
                 bending_stiffness=sc.bending_stiffness.copy(), f_grid=sc.f_grid.copy(),
                 steric=sc.steric.copy(), fluid_velocity=sc.fluid_velocity.copy()).astype(dtype)


# ----------------------------------------------------------------------------- utils
def fmod_floor(x, y):
    """JAX/numpy floored modulo for floats (src/microcosmos/utils.py:18-33 use jnp.mod)."""
    return np.mod(x, y)


def displacement(H, W, x, y):
    """Minimum-image x - y; size (H, W) is flipped to (W, H) for (x, y) positions
    (src/microcosmos/utils.py:18-23)."""
    dt = np.result_type(x)
    L = np.array([W, H], dtype=dt)
    half = L / dt.type(2.0)
    return np.mod(x - y + half, L) - half


def periodic_boundary(H, W, p):
    """Floored wrap into [0, W) x [0, H) (src/microcosmos/utils.py:29-33)."""
    dt = np.result_type(p)
    return np.mod(p, np.array([W, H], dtype=dt))


def gaussian_filter(data, sigma):
    """real(ifft2(fft2(rho) * exp(-2 pi^2 sigma^2 (r^2 + c^2)))) with fftfreq abscissae
    (src/microcosmos/utils.py:35-49)."""
    dt = data.dtype
    rows, cols = data.shape
    r = np.fft.fftfreq(rows).astype(dt)
    c = np.fft.fftfreq(cols).astype(dt)
    r, c = np.meshgrid(r, c, indexing="ij")
    kf = np.exp(dt.type(-2 * np.pi ** 2 * sigma ** 2) * (r ** 2 + c ** 2))
    return np.fft.ifft2(np.fft.fft2(data) * kf).real.astype(dt)


# ----------------------------------------------------------------------------- steric
def steric_deposit(H, W, pos, scatter_value):
    """Cloud-in-cell deposit before the filter (src/microcosmos/forces.py:84-115):
    four scatter-adds, all (y0,x0) updates first, then (y0,x1), (y1,x0), (y1,x1)."""
    dt = pos.dtype
    p = periodic_boundary(H, W, pos)
    x = p[:, 0]
    y = p[:, 1]
    fx = np.floor(x)
    fy = np.floor(y)
    x0 = np.mod(fx.astype(np.int64), W)
    y0 = np.mod(fy.astype(np.int64), H)
    x1 = (x0 + 1) % W
    y1 = (y0 + 1) % H
    dx = x - fx
    dy = y - fy
    one = dt.type(1.0)
    s = dt.type(scatter_value)
    w00 = (one - dx) * (one - dy) * s
    w10 = dx * (one - dy) * s
    w01 = (one - dx) * dy * s
    w11 = dx * dy * s
    g = np.zeros((H, W), dt)
    np.add.at(g, (y0, x0), w00)
    np.add.at(g, (y0, x1), w10)
    np.add.at(g, (y1, x0), w01)
    np.add.at(g, (y1, x1), w11)
    return g


def update_steric_potential(H, W, pos, sigma, scatter_value):
    """CIC deposit + spectral Gaussian (src/microcosmos/forces.py:84-118)."""
    return gaussian_filter(steric_deposit(H, W, pos, scatter_value), sigma)


def sample_bilinear_wrap(V, yy, xx):
    """jax.scipy.ndimage.map_coordinates(V, [yy, xx], order=1, mode="wrap"): nodes
    floor/floor+1 per axis, weights (1-t, t), indices wrapped by floored modulo, the four
    terms in (y-major) product order, added left to right (src/microcosmos/forces.py:30-34)."""
    dt = V.dtype
    H, W = V.shape
    ly = np.floor(yy)
    lx = np.floor(xx)
    ty = yy - ly
    tx = xx - lx
    wy = (dt.type(1.0) - ty, ty)
    wx = (dt.type(1.0) - tx, tx)
    iy = ly.astype(np.int64)
    ix = lx.astype(np.int64)
    iys = (np.mod(iy, H), np.mod(iy + 1, H))
    ixs = (np.mod(ix, W), np.mod(ix + 1, W))
    acc = None
    for a in range(2):
        for b in range(2):
            term = (wy[a] * wx[b]) * V[iys[a], ixs[b]]
            acc = term if acc is None else acc + term
    return acc


def force_interp(pos, V, fd_eps=0.5):
    """-grad V by central differences (eps=0.5) of bilinear samples
    (src/microcosmos/forces.py:20-38)."""
    dt = V.dtype
    y = pos[:, 1]
    x = pos[:, 0]
    e = dt.type(fd_eps)
    den = dt.type(2.0 * fd_eps)
    gx = (sample_bilinear_wrap(V, y, x + e) - sample_bilinear_wrap(V, y, x - e)) / den
    gy = (sample_bilinear_wrap(V, y + e, x) - sample_bilinear_wrap(V, y - e, x)) / den
    return -np.stack([gx, gy], axis=-1)


def steric_force(H, W, pred, cfg):
    """compute_field_steric_force_corrected (src/microcosmos/forces.py:41-81).
    Returns (steric potential field, corrected force).  The analytic neighbour term uses
    global node indices i-n..i+n with only a 0<=j<N mask, so it reaches across filament
    boundaries exactly like the reference."""
    dt = pred.dtype
    sigma = cfg.steric_sigma
    V = update_steric_potential(H, W, pred, sigma, cfg.steric_scatter_value)
    pos = periodic_boundary(H, W, pred)
    raw = force_interp(pos, V)
    N = pos.shape[0]
    n = cfg.steric_neighbor_skip
    if n <= 0:
        return V, raw
    inv2s2 = dt.type(2.0 * sigma * sigma)
    norm = dt.type(2.0 * np.pi * sigma * sigma)
    acc = np.zeros((N, 2), dt)
    for o in range(-n, n + 1):
        j = np.arange(N) + o
        valid = ((j >= 0) & (j < N)).astype(dt)
        js = np.clip(j, 0, N - 1)
        r = displacement(H, W, pos, pos[js])
        d2 = r[:, 0] * r[:, 0] + r[:, 1] * r[:, 1]
        K = np.exp(-d2 / inv2s2) / norm
        acc = acc + (K * valid)[:, None] * r
    contrib = dt.type(cfg.steric_scatter_value / (sigma * sigma)) * acc
    return V, raw - contrib


# ----------------------------------------------------------------------------- PBD
def pbd_iteration(H, W, pos, theta, pairs, bpairs, rest_len, rest_ang, k_bend, cfg):
    """One Jacobi iteration of pbd_rod_constraint (src/microcosmos/solver/pbd.py:14-91):
    theta pass over bending pairs (SOR 1.8, divided by edge bending degree), then the
    position pass over edges (stretch + shear*k_shear)*k_stretch/2 divided by node degree.
    Scatter order: all e_in (src) updates, then all e_out (tgt) updates."""
    dt = pos.dtype
    Ecount = theta.shape[0]
    N = pos.shape[0]
    src, tgt = pairs[:, 0], pairs[:, 1]
    ein, eout = bpairs[:, 0], bpairs[:, 1]
    edeg = np.zeros(Ecount, dt)
    np.add.at(edeg, ein, dt.type(1.0))
    np.add.at(edeg, eout, dt.type(1.0))
    edeg = np.maximum(edeg, dt.type(1.0))
    diff = theta[eout] - theta[ein]
    pi = dt.type(np.pi)
    diff = np.mod(diff + pi, dt.type(2 * np.pi)) - pi
    corr = (diff - rest_ang) * k_bend * dt.type(0.5)
    delta = np.zeros(Ecount, dt)
    np.add.at(delta, ein, corr)
    np.add.at(delta, eout, -corr)
    delta = delta / edeg * dt.type(1.8)
    theta = theta + delta

    ndeg = np.zeros(N, dt)
    np.add.at(ndeg, src, dt.type(1.0))
    np.add.at(ndeg, tgt, dt.type(1.0))
    ndeg = np.maximum(ndeg, dt.type(1.0))
    d = np.stack([np.cos(theta), np.sin(theta)], axis=-1)
    target = d * rest_len[:, None]
    cur = displacement(H, W, pos[tgt], pos[src])
    L = np.sqrt(cur[:, 0] * cur[:, 0] + cur[:, 1] * cur[:, 1])[:, None]
    dirs = cur / np.maximum(L, dt.type(1e-8))
    stretch = dirs * (L - rest_len[:, None])
    shear = (cur - target) - stretch
    forces = (stretch + shear * dt.type(cfg.stiffness_shear)) * dt.type(cfg.stiffness_stretch) * dt.type(0.5)
    disp = np.zeros((N, 2), dt)
    np.add.at(disp, src, forces)
    np.add.at(disp, tgt, -forces)
    disp = disp / ndeg[:, None]
    return pos + disp, theta


def cosserat_iteration(H, W, pos, y, theta, pairs, bpairs, rest_len, rest_ang, k_bend, cfg):
    """One iteration of stable_cosserat_constraint (src/microcosmos/solver/stable_cosserat.py:13-119).
    Phase 1: the bending pass of pbd.py without the 1.8 over-relaxation, then a pull of
    theta toward the segment direction, wrap(atan2(r) - theta) * 0.05.  Phase 2: one
    implicit position update with the inertia weight w = 1/dt**2 (cfg.dt):
    x += (w (y - x) + sum of +-(k_s/l)(r/l - d(theta))) / (w + sum of k_s/l**2), with the
    scatter order of the reference (all src updates, then all tgt updates)."""
    dt = pos.dtype
    t = dt.type
    Ecount = theta.shape[0]
    N = pos.shape[0]
    src, tgt = pairs[:, 0], pairs[:, 1]
    ein, eout = bpairs[:, 0], bpairs[:, 1]
    edeg = np.zeros(Ecount, dt)
    np.add.at(edeg, ein, t(1.0))
    np.add.at(edeg, eout, t(1.0))
    edeg = np.maximum(edeg, t(1.0))
    pi = t(np.pi)
    twopi = t(2 * np.pi)
    diff = theta[eout] - theta[ein]
    diff = np.mod(diff + pi, twopi) - pi
    corr = (diff - rest_ang) * k_bend * t(0.5)
    delta = np.zeros(Ecount, dt)
    np.add.at(delta, ein, corr)
    np.add.at(delta, eout, -corr)
    theta_new = theta + delta / edeg
    seg = displacement(H, W, pos[tgt], pos[src])
    alpha = np.arctan2(seg[:, 1], seg[:, 0])
    pull = np.mod(alpha - theta_new + pi, twopi) - pi
    theta_new = theta_new + pull * t(0.05)

    ks = t(cfg.stiffness_stretch)
    w = t(1.0 / (cfg.dt ** 2))
    d = np.stack([np.cos(theta_new), np.sin(theta_new)], axis=-1)
    c = seg / rest_len[:, None] - d
    f_edge = (ks / rest_len)[:, None] * c
    h_edge = ks / (rest_len * rest_len)
    f_node = w * (y - pos)
    h_node = np.full(N, w, dt)
    np.add.at(f_node, src, f_edge)
    np.add.at(f_node, tgt, -f_edge)
    np.add.at(h_node, src, h_edge)
    np.add.at(h_node, tgt, h_edge)
    return pos + f_node / h_node[:, None], theta_new


def synthetic_ib_positions(H, W, pos, pairs, gpos, width, mean_scale):
    """Synthetic IB node pairs (src/microcosmos/solver/fluid.py:241-263): the chain tangent
    at each node is the sum of its edges' min-image vectors (all src updates, then all tgt
    updates), normalised by sqrt(|t|^2 + EPSIL); the points are gpos +- width*perp*mean_scale,
    perp = (-t_y, t_x), the + set first."""
    dt = pos.dtype
    t = dt.type
    src, tgt = pairs[:, 0], pairs[:, 1]
    ev = displacement(H, W, pos[tgt], pos[src])
    raw = np.zeros_like(pos)
    np.add.at(raw, src, ev)
    np.add.at(raw, tgt, ev)
    nrm = np.sqrt(raw[:, 0] * raw[:, 0] + raw[:, 1] * raw[:, 1] + t(EPSIL32))[:, None]
    tan = raw / nrm
    perp = np.stack([-tan[:, 1], tan[:, 0]], axis=-1)
    off = t(width) * perp * t(mean_scale)
    return np.concatenate([gpos + off, gpos - off], axis=0)


# ----------------------------------------------------------------------------- IB + LBM
def peskin_weights(H, W, gpos, K):
    """Per-point K x K stencil (src/microcosmos/solver/fluid.py:31-87): start at
    floor(x) - (K-1)//2, phi(r) = 0.25(1 + cos(pi |r| / (2h))) for |r|/h <= 2 with h = K/2,
    w = phi(dx) phi(dy) normalised by (sum + EPSIL).  ``dy, dx = meshgrid(offsets, offsets)``
    ('xy' indexing) makes dy vary fastest: stencil entry s = a*K + b has dx = a, dy = b.
    Flat index = (y % H) * W + (x % W)."""
    dt = gpos.dtype
    half = (K - 1) // 2
    hw = dt.type(K / 2.0)
    x = gpos[:, 0]
    y = gpos[:, 1]
    sx = np.floor(x) - dt.type(half)
    sy = np.floor(y) - dt.type(half)
    offs = np.arange(K).astype(dt)
    dy_, dx_ = np.meshgrid(offs, offs)
    dxf = dx_.reshape(-1)
    dyf = dy_.reshape(-1)
    nx = sx[:, None] + dxf[None, :]
    ny = sy[:, None] + dyf[None, :]

    def phi(r):
        ra = np.abs(r) / hw
        return np.where(ra <= dt.type(2.0), dt.type(0.25) * (dt.type(1.0) + np.cos(dt.type(np.pi) * ra / dt.type(2.0))),
                        dt.type(0.0))
    w = phi(nx - x[:, None]) * phi(ny - y[:, None])
    s = np.zeros(w.shape[0], dt)
    for k in range(w.shape[1]):
        s = s + w[:, k]
    w = w / (s + dt.type(EPSIL32))[:, None]
    ix = np.mod(nx.astype(np.int64), W)
    iy = np.mod(ny.astype(np.int64), H)
    return iy * W + ix, w


def macroscopic(f):
    """density = max(sum f, 0.1); u = sum e_i f_i / density (src/microcosmos/solver/fluid.py:136-142),
    sums taken sequentially over i."""
    dt = f.dtype
    rho = f[0]
    for i in range(1, 9):
        rho = rho + f[i]
    rho = np.maximum(rho, dt.type(0.1))
    ux = ((((f[1] - f[3]) + f[5]) - f[6]) - f[7]) + f[8]
    uy = ((((f[2] - f[4]) + f[5]) + f[6]) - f[7]) - f[8]
    return rho, ux / rho, uy / rho


def equilibrium(rho, ux, uy):
    """feq = rho w_i (1 + 3 e.u + 4.5 (e.u)^2 - 1.5 u^2) (src/microcosmos/solver/fluid.py:145-151)."""
    dt = rho.dtype
    usq = ux * ux + uy * uy
    out = []
    for i in range(9):
        eu = dt.type(E[i, 0]) * ux + dt.type(E[i, 1]) * uy
        out.append(rho * dt.type(WGT[i]) * (((dt.type(1.0) + dt.type(3.0) * eu) + dt.type(4.5) * (eu * eu))
                                            - dt.type(1.5) * usq))
    return np.stack(out)


def trt_rates(cfg, dt=np.float32):
    """omega+ = clip(1/(3 nu + 0.5), 0, 1.9); omega- from the magic parameter
    (src/microcosmos/solver/fluid.py:155-161, 342-344)."""
    t = np.dtype(dt).type
    wp = t(min(max(1.0 / (3.0 * cfg.viscosity + 0.5), 0.0), 1.9))
    eps = t(EPSIL32)
    off = t(1.0) / np.maximum(wp, eps) - t(0.5)
    wm = t(1.0) / (t(cfg.lambda_trt) / np.maximum(off, eps) + t(0.5))
    return wp, wm


def velocity_clamp_factor(ux, uy, vmax):
    """min(1, vmax / (sqrt(ux^2+uy^2+EPSIL) + EPSIL)) (src/microcosmos/solver/fluid.py:272-274)."""
    dt = ux.dtype
    eps = dt.type(EPSIL32)
    mag = np.sqrt(ux * ux + uy * uy + eps)
    return np.minimum(dt.type(1.0), dt.type(vmax) / (mag + eps))


def collide(f, rho, vx, vy, Fx, Fy, wp, wm):
    """TRT collision at u* = u + F/(2 rho) with the TRT-aware Guo source, then the EPSIL
    floor (src/microcosmos/solver/fluid.py:164-199, 346-350)."""
    dt = f.dtype
    half = dt.type(0.5)
    usx = vx + half * Fx / rho
    usy = vy + half * Fy / rho
    feq = equilibrium(rho, usx, usy)
    udF = usx * Fx + usy * Fy
    raw = []
    for i in range(9):
        eu = dt.type(E[i, 0]) * usx + dt.type(E[i, 1]) * usy
        eF = dt.type(E[i, 0]) * Fx + dt.type(E[i, 1]) * Fy
        raw.append(dt.type(WGT[i]) * (dt.type(3.0) * (eF - udF) + dt.type(9.0) * eu * eF))
    raw = np.stack(raw)
    fo = f[OPP]
    feqo = feq[OPP]
    rawo = raw[OPP]
    post = f - wp * (half * (f + fo) - half * (feq + feqo)) - wm * (half * (f - fo) - half * (feq - feqo))
    src = (dt.type(1.0) - half * wp) * (half * (raw + rawo)) + (dt.type(1.0) - half * wm) * (half * (raw - rawo))
    return np.maximum(post + src, dt.type(EPSIL32)), usx, usy


def stream(fpost):
    """Push streaming f_new[y+cy, x+cx] = f_post[y, x] (jnp.roll, solver/fluid.py:352-357)."""
    out = np.empty_like(fpost)
    for i in range(9):
        out[i] = np.roll(fpost[i], shift=(int(E[i, 1]), int(E[i, 0])), axis=(0, 1))
    return np.maximum(out, fpost.dtype.type(EPSIL32))


@dataclasses.dataclass
class IBResult:
    velocity: np.ndarray
    fluid_velocity: np.ndarray
    f_grid: np.ndarray
    force_field: np.ndarray
    density: np.ndarray
    vel_before: np.ndarray


def ib_lbm(H, W, grid_shape, pos, vel, f_grid, cfg, dtstep, ib_positions=None, pairs=None):
    """immersed_boundary_interaction (src/microcosmos/solver/fluid.py:202-386):
    macroscopic + clamp, multi-direct forcing
    (ibm_iterations x interpolate/clamp/spread), post clamp, F = (u_corr - u) rho,
    TRT+Guo collide, stream, node reaction.  ``grid_shape`` is the domain grid; the
    scale keeps the reference's axis order scale = (w / grid_shape[0], h / grid_shape[1]).

    ``ib_positions`` (default: ``pos``) are the positions the Peskin stencils are built
    from.  The reference wraps them in ``jax.lax.stop_gradient`` (fluid.py:239), so a
    finite-difference check of its gradients holds them at the unperturbed trajectory's
    values.  With ``synthetic_node_width > 0`` the IB points are the synthetic pairs
    (``synthetic_ib_positions``, needs ``pairs``) carrying their node's velocity, and each
    node's reaction is the mean of its two points' forces (fluid.py:371-374)."""
    dt = f_grid.dtype
    t = dt.type
    h, w = f_grid.shape[1], f_grid.shape[2]
    scale = np.array([w / grid_shape[0], h / grid_shape[1]], dtype=dt)
    mean_scale = 0.5 * (w / grid_shape[0] + h / grid_shape[1])
    vmax = cfg.max_fluid_velocity * mean_scale
    eps = t(EPSIL32)
    node_vel = vel * scale * t(dtstep)
    gpos = (pos if ib_positions is None else ib_positions) * scale
    nn = pos.shape[0]
    if cfg.synthetic_node_width > 0.0:
        gpos = synthetic_ib_positions(grid_shape[0], grid_shape[1], pos if ib_positions is None else ib_positions,
                                      pairs, gpos, cfg.synthetic_node_width, mean_scale)
        node_vel = np.concatenate([node_vel, node_vel], axis=0)
    f = np.maximum(f_grid, eps)
    rho, ux, uy = macroscopic(f)
    c1 = velocity_clamp_factor(ux, uy, vmax)
    vx = ux * c1
    vy = uy * c1
    idx, wts = peskin_weights(h, w, gpos, cfg.ibm_kernel_size)
    flat = idx.reshape(-1)
    wflat = wts.reshape(-1)
    cov = np.zeros(h * w, dt)
    np.add.at(cov, flat, wflat)
    inv = t(1.0) / np.maximum(cov, t(1.0))
    ucx = vx.reshape(-1).copy()
    ucy = vy.reshape(-1).copy()
    nst = wts.shape[1]
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
        mag = np.sqrt(sx * sx + sy * sy + eps)
        cf = np.minimum(t(1.0), t(vmax) / (mag + eps))
        sx = sx * cf
        sy = sy * cf
        dx = np.zeros(h * w, dt)
        dy = np.zeros(h * w, dt)
        np.add.at(dx, flat, np.repeat(sx, nst) * wflat)
        np.add.at(dy, flat, np.repeat(sy, nst) * wflat)
        ucx = ucx + dx * inv
        ucy = ucy + dy * inv
    ucx = ucx.reshape(h, w)
    ucy = ucy.reshape(h, w)
    c2 = velocity_clamp_factor(ucx, ucy, vmax)
    ucx = ucx * c2
    ucy = ucy * c2
    Fx = (ucx - vx) * rho
    Fy = (ucy - vy) * rho
    if cfg.enable_force_clamp:
        c3 = velocity_clamp_factor(Fx, Fy, vmax)
        Fx = Fx * c3
        Fy = Fy * c3
    wp, wm = trt_rates(cfg, dt)
    fpost, usx, usy = collide(f, rho, vx, vy, Fx, Fy, wp, wm)
    fnew = stream(fpost)
    Fxf = Fx.reshape(-1)
    Fyf = Fy.reshape(-1)
    gx = Fxf[idx] * wts
    gy = Fyf[idx] * wts
    nfx = np.zeros(gx.shape[0], dt)
    nfy = np.zeros(gx.shape[0], dt)
    for k in range(nst):
        nfx = nfx + gx[:, k]
        nfy = nfy + gy[:, k]
    if cfg.synthetic_node_width > 0.0:
        nfx = t(0.5) * (nfx[:nn] + nfx[nn:])
        nfy = t(0.5) * (nfy[:nn] + nfy[nn:])
    sdt = scale * t(dtstep)
    dvx = (nfx / t(cfg.node_mass)) / sdt[0]
    dvy = (nfy / t(cfg.node_mass)) / sdt[1]
    vel_out = np.stack([vel[:, 0] - dvx, vel[:, 1] - dvy], axis=-1)
    return IBResult(velocity=vel_out, fluid_velocity=np.stack([usx, usy]), f_grid=fnew,
                    force_field=np.stack([Fx, Fy]), density=rho, vel_before=np.stack([vx, vy]))


# ----------------------------------------------------------------------------- step / simulate
def step(s: State, cfg: Config, dtstep: float, rest_angles=None, ib_positions=None):
    """One simulate.step (src/microcosmos/simulate.py:37-100) with the PBD or the
    stable-Cosserat rod solver (cfg.solver_type; the Cosserat inertial prediction is the
    position after the steric displacement, simulate.py:70-71).
    ``rest_angles`` overrides edges.bending_rest_angles for this step (the caller-side
    curvature actuation); ``ib_positions`` see ``ib_lbm``."""
    dt = s.position.dtype
    t = dt.type
    H, W = s.H, s.W
    s = s.copy()
    if rest_angles is not None:
        s.bending_rest_angles = np.asarray(rest_angles, dt)
    prev = s.position
    vel = s.velocity * t(cfg.damping)
    pred = prev + vel * t(dtstep)
    if cfg.enable_steric:
        V, fst = steric_force(H, W, pred, cfg)
        s.steric = V
        pred = pred + fst * t(cfg.steric_strength) * t(dtstep)
    pos, theta = pred, s.theta
    for _ in range(cfg.cycles_per_step):
        if cfg.solver_type == "cosserat":
            pos, theta = cosserat_iteration(H, W, pos, pred, theta, s.pairs, s.bending_pairs, s.rest_lengths,
                                            s.bending_rest_angles, s.bending_stiffness, cfg)
        else:
            pos, theta = pbd_iteration(H, W, pos, theta, s.pairs, s.bending_pairs, s.rest_lengths,
                                       s.bending_rest_angles, s.bending_stiffness, cfg)
    vel = (pos - prev) / t(dtstep)
    if cfg.enable_fluid:
        r = ib_lbm(H, W, (H, W), pos, vel, s.f_grid, cfg, dtstep, ib_positions, pairs=s.pairs)
        vel = r.velocity
        s.f_grid = r.f_grid
        s.fluid_velocity = r.fluid_velocity
    s.position = periodic_boundary(H, W, pos)
    s.velocity = vel
    s.theta = theta
    return s


def resize_linear(x, shape):
    """jax.image.resize(x, shape, method="linear") as the reference records u* on the domain
    grid when the fluid lattice differs (simulate.py:24-29): along each axis whose size
    changes (m -> n), output o = sum_i w[i, o] x[i] with the triangle kernel at
    sample (o + 0.5) m/n - 0.5, widened by max(m/n, 1) (antialiasing), weights normalised
    by their sum and zero outside [-0.5, m - 0.5].  Restated from JAX's published resize;
    sums in index order (JAX's einsum order is unspecified)."""
    out = np.asarray(x, np.float32)
    for d, (m, n) in enumerate(zip(out.shape, shape)):
        if m == n:
            continue
        inv = np.float32(1.0 / (n / m))
        ks = max(inv, np.float32(1.0))
        sf = (np.arange(n, dtype=np.float32) + np.float32(0.5)) * inv - np.float32(0.5)
        w = np.maximum(np.float32(0.0), np.float32(1.0) - np.abs(sf[None, :] - np.arange(m, dtype=np.float32)[:, None]) / ks)
        tot = w.sum(axis=0, keepdims=True)
        w = np.where(np.abs(tot) > np.float32(1000.0 * EPSIL32), w / np.where(tot != 0, tot, 1), 0)
        w = np.where(((sf >= -0.5) & (sf <= m - 0.5))[None, :], w, 0).astype(np.float32)
        out = np.moveaxis(np.tensordot(np.moveaxis(out, d, -1), w, axes=([-1], [0])), -1, d).astype(np.float32)
    return out


def actuation(act, t):
    """rest[b](t) = c[b] + A sin(omega t + phase) (caller-side actuation closed form)."""
    c, amp, om, ph = act
    arg = (om * np.float32(t) + ph).astype(np.float32)
    return (c + amp * np.sin(arg)).astype(np.float32)


def simulate(s: State, cfg: Config, dtstep: float, num_steps: int, act=None, record=False,
             t0=0):
    """lax.scan of step (src/microcosmos/simulate.py:15-35).  With ``record`` the per-step
    node positions/velocities and steric/fluid_velocity fields are returned like the
    reference's timeseries."""
    ts = {"position": [], "velocity": [], "steric": [], "fluid_velocity": []} if record else None
    for k in range(num_steps):
        ra = None if act is None else actuation(act, t0 + k).astype(s.position.dtype)
        s = step(s, cfg, dtstep, ra)
        if record:
            ts["position"].append(s.position)
            ts["velocity"].append(s.velocity)
            ts["steric"].append(s.steric)
            u = s.fluid_velocity
            ts["fluid_velocity"].append(u if u.shape[1:] == (s.H, s.W) else resize_linear(u, (2, s.H, s.W)))
    if record:
        ts = {k: np.stack(v) for k, v in ts.items()}
    return s, ts


def config_from_npz(z):
    kw = {}
    for f in dataclasses.fields(Config):
        key = "cfg_" + f.name
        if key in z:
            v = z[key]
            kw[f.name] = type(f.default)(v.item()) if not isinstance(f.default, bool) else bool(v.item())
    return Config(**kw)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
