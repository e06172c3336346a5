"""Generate golden input/output vectors by running the reference's own source.

Run in an environment that has the reference checkout (it is not needed anywhere
else)::

    python tests/golden/make_golden.py /root/reference

JAX is not installed here, so ``numpy_jax_shim`` is installed as ``jax`` first; the
reference modules (``src/microcosmos/{utils,forces,simulate}.py``,
``solver/{fluid,pbd,config}.py``, ``structs/*.py``, ``graph.py``) are then imported
from the checkout unmodified and executed on numpy float32.  Each case writes one
``.npz`` with its inputs, its parameters and the reference outputs.
"""
from __future__ import annotations

import dataclasses
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, REPO)

import numpy_jax_shim  # noqa: E402


def load_reference(ref_root):
    numpy_jax_shim.install()
    sys.path.insert(0, os.path.join(ref_root, "src"))
    import microcosmos.simulate as simulate_mod
    import microcosmos.forces as forces_mod
    import microcosmos.utils as utils_mod
    import microcosmos.solver.fluid as fluid_mod
    import microcosmos.solver.pbd as pbd_mod
    import microcosmos.solver.config as config_mod
    import microcosmos.solver.stable_cosserat as cosserat_mod
    import microcosmos.graph as graph_mod
    from microcosmos.structs.nodes import Nodes
    from microcosmos.structs.edges import Edges
    from microcosmos.structs.fields import Fields
    for cls in (Nodes, Edges, Fields):
        if not hasattr(cls, "__replace__"):
            cls.__replace__ = lambda self, **kw: dataclasses.replace(self, **kw)
    return dict(simulate=simulate_mod, forces=forces_mod, utils=utils_mod, fluid=fluid_mod,
                pbd=pbd_mod, stable_cosserat=cosserat_mod, config=config_mod, graph=graph_mod, Nodes=Nodes, Edges=Edges,
                Fields=Fields)


def A(x):
    return np.asarray(x).view(np.ndarray).copy()


def baseline_config(cfg_mod, **over):
    """PBD_SCHEME with the benchmark overrides (viscosity 0.1 -> tau+=0.8, Lambda=1/4,
    4-point IB kernel, steric on, stretch/bend/"twist"=shear 1.0/0.1/0.1)."""
    base = dict(viscosity=0.1, lambda_trt=0.25, ibm_kernel_size=4, enable_steric=True,
                stiffness_stretch=1.0, stiffness_shear=0.1)
    base.update(over)
    return dataclasses.replace(cfg_mod.PBD_SCHEME, **base)


CFG_KEYS = ["cycles_per_step", "stiffness_stretch", "stiffness_shear", "damping", "enable_fluid",
            "viscosity", "max_fluid_velocity", "ibm_iterations", "synthetic_node_width",
            "ibm_kernel_size", "ibm_relaxation", "node_mass", "lambda_trt", "enable_force_clamp",
            "enable_steric", "steric_strength", "steric_sigma", "steric_neighbor_skip",
            "steric_scatter_value"]
# written only by the fixtures whose config uses them (stable-Cosserat solver)
CFG_KEYS_SOLVER = ["solver_type", "dt"]


def cfg_arrays(cfg, solver=False):
    keys = CFG_KEYS + (CFG_KEYS_SOLVER if solver else [])
    return {"cfg_" + k: np.asarray(getattr(cfg, k)) for k in keys}


def state_arrays(prefix, nodes, edges, fields):
    out = {}
    if nodes is not None:
        out[prefix + "position"] = A(nodes.position)
        out[prefix + "velocity"] = A(nodes.velocity)
    if edges is not None:
        out[prefix + "theta"] = A(edges.theta)
        out[prefix + "pairs"] = A(edges.pairs)
        out[prefix + "rest_lengths"] = A(edges.rest_lengths)
        out[prefix + "bending_pairs"] = A(edges.bending_pairs)
        out[prefix + "bending_rest_angles"] = A(edges.bending_rest_angles)
        out[prefix + "bending_stiffness"] = A(edges.bending_stiffness)
    if fields is not None:
        out[prefix + "steric"] = A(fields.steric)
        out[prefix + "fluid_velocity"] = A(fields.fluid_velocity)
        if fields.f_grid is not None:
            out[prefix + "f_grid"] = A(fields.f_grid)
    return out


def to_ref(R, sc):
    jnp = sys.modules["jax"].numpy
    nodes = R["Nodes"](position=jnp.array(sc.position), velocity=jnp.array(sc.velocity),
                       color_bend=jnp.zeros(sc.N), debug_vector=jnp.zeros((sc.N, 2)))
    edges = R["Edges"](pairs=jnp.array(sc.pairs), theta=jnp.array(sc.theta),
                       rest_lengths=jnp.array(sc.rest_lengths),
                       bending_pairs=jnp.array(sc.bending_pairs),
                       bending_rest_angles=jnp.array(sc.bending_rest_angles),
                       bending_stiffness=jnp.array(sc.bending_stiffness))
    fields = R["Fields"](grid_shape=(sc.H, sc.W), steric=jnp.array(sc.steric),
                         fluid_velocity=jnp.array(sc.fluid_velocity), f_grid=jnp.array(sc.f_grid))
    return nodes, edges, fields


def save(name, **arrs):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrs)
    print("wrote", path, sum(v.nbytes for v in arrs.values()), "bytes")


GROUPS = ("base", "cosserat", "synthetic", "gym", "render", "fluidgrid", "worm", "env")


def main(ref_root, groups=GROUPS):
    R = load_reference(ref_root)
    if "base" in groups:
        base_cases(R)
    if "cosserat" in groups:
        cosserat_cases(R)
    if "synthetic" in groups:
        synthetic_cases(R)
    if "gym" in groups:
        gym_cases(R)
    if "render" in groups:
        render_cases(R)
    if "fluidgrid" in groups:
        fluidgrid_cases(R)
    if "worm" in groups:
        worm_case(R)
    if "env" in groups:
        env_cases(R)


def env_cases(R):
    """MicrocosmosEnv (src/microcosmos/env.py): the chain and loop factories, then the
    env's rollout (PBD_SCHEME, dt 0.05) and one step of the fluid-free preset."""
    import microcosmos.env as E
    specs = [("env_chain_32x40", E.MicrocosmosEnv(grid_shape=(32, 40), num_steps=5), "chain", 10, 2.0, "rollout"),
             ("env_loop_48x48", E.MicrocosmosEnv(grid_shape=(48, 48), num_steps=4), "loop", 16, 1.5, "rollout"),
             ("env_loop_nofluid_24x24", E.MicrocosmosEnv.no_fluid(grid_shape=(24, 24), num_steps=3), "loop", 9, 2.0,
              "step")]
    for name, env, kind, n, spacing, run in specs:
        nodes, edges = (env.make_chain if kind == "chain" else env.make_loop)(n, spacing=spacing)
        out = dict(H=np.int32(env.grid_shape[0]), W=np.int32(env.grid_shape[1]), dt=np.float32(env.dt),
                   num_steps=np.int32(env.num_steps), num_nodes=np.int32(n), spacing=np.float32(spacing),
                   no_fluid=np.bool_(not env.solver_config.enable_fluid),
                   in_color_bend=A(nodes.color_bend), **state_arrays("in_", nodes, edges, env.fields))
        if run == "rollout":
            nts, fts = env.rollout(nodes, edges)
            out.update(ts_position=A(nts.position), ts_velocity=A(nts.velocity), ts_steric=A(fts.steric),
                       ts_fluid_velocity=A(fts.fluid_velocity))
        else:
            n1, e1, f1 = env.step(nodes, edges)
            out.update(**state_arrays("out_", n1, e1, f1))
        save(name, **out)


def base_cases(R):
    from microcosmos_b200 import scenarios as S
    U = R["utils"]
    jnp = sys.modules["jax"].numpy
    rng = np.random.default_rng(1234)

    # ---- utils: displacement, periodic_boundary, gaussian_filter (utils.py:18-49)
    for (H, W) in [(16, 16), (12, 20)]:
        x = rng.uniform(-30, 50, size=(64, 2)).astype(np.float32)
        y = rng.uniform(-30, 50, size=(64, 2)).astype(np.float32)
        data = rng.uniform(0, 1, size=(H, W)).astype(np.float32)
        save(f"utils_{H}x{W}", H=np.int32(H), W=np.int32(W), x=x, y=y, data=data,
             sigma=np.float32(1.5),
             displacement=A(U.displacement((H, W), jnp.array(x), jnp.array(y))),
             periodic_boundary=A(U.periodic_boundary((H, W), jnp.array(x))),
             gaussian_filter=A(U.gaussian_filter(jnp.array(data), sigma=1.5)))

    cfg_mod = R["config"]

    # ---- steric: deposit + filter + corrected force (forces.py:41-118)
    for (H, W, F, n, seed) in [(20, 28, 3, 9, 5), (32, 32, 2, 14, 6)]:
        sc = S.make_scenario(H, W, F, n, seed=seed, amp=0.2)
        nodes, edges, fields = to_ref(R, sc)
        pred = jnp.array(sc.position + rng.normal(0, 0.3, size=sc.position.shape).astype(np.float32)
                         + np.float32(W) * (rng.uniform(size=sc.position.shape) < 0.1))
        nodes = nodes.__replace__(position=pred)
        fields2, f_st = R["forces"].compute_field_steric_force_corrected(
            nodes, fields, sigma=1.5, neighbor_skip=5, scatter_value=1.0)
        save(f"steric_{H}x{W}", H=np.int32(H), W=np.int32(W), position=A(pred), sigma=np.float32(1.5),
             neighbor_skip=np.int32(5), scatter_value=np.float32(1.0),
             steric=A(fields2.steric), force=A(f_st))

    # ---- PBD: one iteration and a 20-iteration fori_loop (solver/pbd.py:14-91)
    for (H, W, F, n, seed) in [(20, 28, 3, 9, 7), (64, 64, 2, 24, 8)]:
        sc = S.make_scenario(H, W, F, n, seed=seed, amp=0.3)
        nodes, edges, fields = to_ref(R, sc)
        pos = jnp.array(sc.position + rng.normal(0, 0.2, size=sc.position.shape).astype(np.float32))
        th = jnp.array(sc.theta + rng.normal(0, 0.3, size=sc.theta.shape).astype(np.float32))
        nodes = nodes.__replace__(position=pos)
        edges = edges.__replace__(theta=th)
        cfg = baseline_config(cfg_mod)
        n1, e1 = R["pbd"].pbd_rod_constraint(0, (nodes, edges), cfg, (H, W))
        carry = (nodes, edges)
        for i in range(cfg.cycles_per_step):
            carry = R["pbd"].pbd_rod_constraint(i, carry, cfg, (H, W))
        n20, e20 = carry
        save(f"pbd_{H}x{W}", H=np.int32(H), W=np.int32(W), **cfg_arrays(cfg),
             **state_arrays("in_", nodes, edges, None),
             pos_1=A(n1.position), theta_1=A(e1.theta), pos_20=A(n20.position), theta_20=A(e20.theta))

    # ---- IB + LBM: immersed_boundary_interaction (solver/fluid.py:202-386)
    for (H, W, F, n, ks, seed, ustd) in [(24, 24, 2, 10, 4, 9, 1e-3), (24, 24, 2, 10, 2, 10, 1e-3),
                                         (20, 28, 2, 8, 4, 11, 1e-3), (16, 16, 1, 10, 4, 12, 0.15)]:
        sc = S.make_scenario(H, W, F, n, seed=seed, u0_std=ustd)
        nodes, edges, fields = to_ref(R, sc)
        vel = jnp.array(rng.normal(0, 5.0, size=sc.position.shape).astype(np.float32))
        nodes = nodes.__replace__(velocity=vel)
        cfg = baseline_config(cfg_mod, ibm_kernel_size=ks)
        dt = 0.01
        n2, f2, fnew = R["fluid"].immersed_boundary_interaction(nodes, edges, fields, fields.f_grid, dt, cfg)
        save(f"ib_{H}x{W}_k{ks}" + ("_clamp" if ustd > 0.01 else ""), H=np.int32(H), W=np.int32(W),
             dt=np.float32(dt), **cfg_arrays(cfg), **state_arrays("in_", nodes, edges, fields),
             velocity_out=A(n2.velocity), fluid_velocity_out=A(f2.fluid_velocity), f_grid_out=A(fnew))

    # ---- full step / simulate (simulate.py:15-100)
    for (H, W, F, n, seed, steps, name) in [(24, 32, 2, 10, 13, 6, "sim_24x32"),
                                            (32, 32, 3, 12, 14, 6, "sim_32x32")]:
        sc = S.make_scenario(H, W, F, n, seed=seed, amp=0.2, period=20.0)
        nodes, edges, fields = to_ref(R, sc)
        cfg = baseline_config(cfg_mod)
        dt = 0.01
        # a) simulate() with fixed rest angles: reference-shaped timeseries
        nts, fts = R["simulate"].simulate(nodes, edges, fields, dt, steps, cfg)
        # b) step() loop with the caller-side curvature actuation
        nd, ed, fd = nodes, edges, fields
        traj = []
        for t in range(steps):
            ed = ed.__replace__(bending_rest_angles=jnp.array(S.actuation_rest_angles(sc, t)))
            nd, ed, fd = R["simulate"].step(nd, ed, fd, dt, cfg)
            traj.append(A(nd.position))
        save(name, H=np.int32(H), W=np.int32(W), dt=np.float32(dt), steps=np.int32(steps),
             **cfg_arrays(cfg), **state_arrays("in_", nodes, edges, fields),
             act_c=sc.act_c, act_amp=sc.act_amp, act_omega=sc.act_omega, act_phase=sc.act_phase,
             ts_position=A(nts.position), ts_velocity=A(nts.velocity), ts_steric=A(fts.steric),
             ts_fluid_velocity=A(fts.fluid_velocity),
             act_position=np.stack(traj), act_velocity=A(nd.velocity), act_theta=A(ed.theta),
             act_f_grid=A(fd.f_grid), act_steric=A(fd.steric), act_fluid_velocity=A(fd.fluid_velocity))

    # ---- the reference test scenario: closed loop of 10 nodes (tests/conftest.py:9-59),
    #      PBD_SCHEME defaults (2-point kernel, steric off), one step on a 32x32 grid
    G = R["graph"]
    num = 10
    pairs, dep = G.make_edges(num, graph="loop", num_instances=1)
    bp, _ = G.compute_bending_pairs(pairs, dep, num)
    radius = 3.0 / (2.0 * np.sin(np.pi / num))
    ang = np.linspace(0, 2 * np.pi, num, endpoint=False)
    pos = (np.array([16.0, 16.0]) + radius * np.stack([np.cos(ang), np.sin(ang)], 1)).astype(np.float32)
    d = U.displacement((32, 32), jnp.array(pos)[A(pairs)[:, 1]], jnp.array(pos)[A(pairs)[:, 0]])
    th = np.arctan2(A(d)[:, 1], A(d)[:, 0]).astype(np.float32)
    sc = S.make_scenario(32, 32, 1, num, seed=15)
    sc.position = pos
    sc.velocity = rng.normal(0, 1.0, size=pos.shape).astype(np.float32)
    sc.pairs = A(pairs)
    sc.theta = th
    sc.rest_lengths = np.full(num, 3.0, np.float32)
    sc.bending_pairs = A(bp)
    sc.bending_rest_angles = np.full(bp.shape[0], 2 * np.pi / num, np.float32)
    sc.bending_stiffness = np.full(bp.shape[0], 0.5, np.float32)
    nodes, edges, fields = to_ref(R, sc)
    cfg = cfg_mod.PBD_SCHEME
    nd, ed, fd = R["simulate"].step(nodes, edges, fields, 0.01, cfg)
    nd2, ed2, fd2 = R["simulate"].step(nd, ed, fd, 0.01, cfg)
    save("loop_32x32", H=np.int32(32), W=np.int32(32), dt=np.float32(0.01), **cfg_arrays(cfg),
         **state_arrays("in_", nodes, edges, fields), **state_arrays("out_", nd2, ed2, fd2))


def cosserat_cases(R):
    """The stable-Cosserat plugin (solver/stable_cosserat.py:13-119): the constraint alone
    (one iteration and a cycles_per_step loop with the inertial prediction in
    debug_vector, as simulate.step sets it), and full steps with and without fluid."""
    from microcosmos_b200 import scenarios as S
    jnp = sys.modules["jax"].numpy
    cfg_mod = R["config"]
    rng = np.random.default_rng(4321)
    for (H, W, F, n, seed) in [(20, 28, 3, 9, 21), (64, 64, 2, 24, 22)]:
        sc = S.make_scenario(H, W, F, n, seed=seed, amp=0.3)
        nodes, edges, fields = to_ref(R, sc)
        y = sc.position + rng.normal(0, 0.2, size=sc.position.shape).astype(np.float32)
        pos = jnp.array(y + rng.normal(0, 0.1, size=sc.position.shape).astype(np.float32))
        th = jnp.array(sc.theta + rng.normal(0, 0.3, size=sc.theta.shape).astype(np.float32))
        nodes = nodes.__replace__(position=pos, debug_vector=jnp.array(y))
        edges = edges.__replace__(theta=th)
        cfg = cfg_mod.COSSERAT_SCHEME_NO_FLUID
        con = R["stable_cosserat"].stable_cosserat_constraint
        n1, e1 = con(0, (nodes, edges), cfg, (H, W))
        carry = (nodes, edges)
        for i in range(cfg.cycles_per_step):
            carry = con(i, carry, cfg, (H, W))
        n20, e20 = carry
        save(f"cosserat_{H}x{W}", H=np.int32(H), W=np.int32(W), **cfg_arrays(cfg, solver=True),
             **state_arrays("in_", nodes, edges, None), in_y=A(y),
             pos_1=A(n1.position), theta_1=A(e1.theta), pos_20=A(n20.position), theta_20=A(e20.theta))
    # full steps: no fluid at the preset's dt; with fluid and steric at dt = 0.01 with the
    # stiffness scaled to the inertia weight (k_s / l^2 = 1 / dt^2 for unit rest lengths)
    cases = [("sim_cosserat_nofluid_24x32", 24, 32, 2, 10, 23, 0.05,
              dataclasses.replace(cfg_mod.COSSERAT_SCHEME_NO_FLUID)),
             ("sim_cosserat_fluid_32x32", 32, 32, 3, 12, 24, 0.01,
              dataclasses.replace(cfg_mod.COSSERAT_SCHEME, dt=0.01, stiffness_stretch=10000.0,
                                  stiffness_shear=10000.0, viscosity=0.1, ibm_kernel_size=4,
                                  enable_steric=True))]
    for (name, H, W, F, n, seed, dt, cfg) in cases:
        sc = S.make_scenario(H, W, F, n, seed=seed, amp=0.2, period=20.0)
        sc.velocity = rng.normal(0, 0.5, size=sc.velocity.shape).astype(np.float32)
        nodes, edges, fields = to_ref(R, sc)
        steps = 6
        nd, ed, fd = nodes, edges, fields
        traj = []
        for t in range(steps):
            ed = ed.__replace__(bending_rest_angles=jnp.array(S.actuation_rest_angles(sc, t)))
            nd, ed, fd = R["simulate"].step(nd, ed, fd, dt, cfg)
            traj.append(A(nd.position))
        save(name, H=np.int32(H), W=np.int32(W), dt=np.float32(dt), steps=np.int32(steps),
             **cfg_arrays(cfg, solver=True), **state_arrays("in_", nodes, edges, fields),
             act_c=sc.act_c, act_amp=sc.act_amp, act_omega=sc.act_omega, act_phase=sc.act_phase,
             act_position=np.stack(traj), act_velocity=A(nd.velocity), act_theta=A(ed.theta),
             act_f_grid=A(fd.f_grid), act_steric=A(fd.steric), act_fluid_velocity=A(fd.fluid_velocity))


def synthetic_cases(R):
    """Synthetic IB node pairs (solver/fluid.py:241-263, 371-374): one
    immersed_boundary_interaction with synthetic_node_width > 0, and full steps."""
    from microcosmos_b200 import scenarios as S
    jnp = sys.modules["jax"].numpy
    cfg_mod = R["config"]
    rng = np.random.default_rng(5678)
    for (H, W, F, n, ks, width, seed) in [(24, 24, 2, 10, 4, 1.0, 31), (20, 28, 2, 8, 2, 0.5, 32)]:
        sc = S.make_scenario(H, W, F, n, seed=seed, u0_std=1e-3)
        nodes, edges, fields = to_ref(R, sc)
        vel = jnp.array(rng.normal(0, 5.0, size=sc.position.shape).astype(np.float32))
        nodes = nodes.__replace__(velocity=vel)
        cfg = baseline_config(cfg_mod, ibm_kernel_size=ks, synthetic_node_width=width)
        dt = 0.01
        n2, f2, fnew = R["fluid"].immersed_boundary_interaction(nodes, edges, fields, fields.f_grid, dt, cfg)
        save(f"ib_syn_{H}x{W}_k{ks}", H=np.int32(H), W=np.int32(W), dt=np.float32(dt), **cfg_arrays(cfg),
             **state_arrays("in_", nodes, edges, fields),
             velocity_out=A(n2.velocity), fluid_velocity_out=A(f2.fluid_velocity), f_grid_out=A(fnew))
    sc = S.make_scenario(32, 32, 3, 12, seed=33, amp=0.2, period=20.0)
    nodes, edges, fields = to_ref(R, sc)
    cfg = baseline_config(cfg_mod, synthetic_node_width=1.0)
    dt = 0.01
    steps = 6
    nd, ed, fd = nodes, edges, fields
    traj = []
    for t in range(steps):
        ed = ed.__replace__(bending_rest_angles=jnp.array(S.actuation_rest_angles(sc, t)))
        nd, ed, fd = R["simulate"].step(nd, ed, fd, dt, cfg)
        traj.append(A(nd.position))
    save("sim_syn_32x32", H=np.int32(32), W=np.int32(32), dt=np.float32(dt), steps=np.int32(steps),
         **cfg_arrays(cfg), **state_arrays("in_", nodes, edges, fields),
         act_c=sc.act_c, act_amp=sc.act_amp, act_omega=sc.act_omega, act_phase=sc.act_phase,
         act_position=np.stack(traj), act_velocity=A(nd.velocity), act_theta=A(ed.theta),
         act_f_grid=A(fd.f_grid), act_steric=A(fd.steric), act_fluid_velocity=A(fd.fluid_velocity))


def gym_cases(R):
    """The reference's gym environments (src/microcosmos/gym/*.py): reset, then three steps
    with seeded actions (energy source on, walk off, max_steps = 3)."""
    jax = sys.modules["jax"]
    jnp = jax.numpy
    import microcosmos.gym as G
    rng = np.random.default_rng(999)
    common = dict(energy_amplitude=1.0, max_steps=3)
    specs = [("gym_line", G.LineEnv, dict(num_nodes=12, grid_shape=(48, 48), energy_size=6.0)),
             ("gym_ring", G.RingEnv, dict(num_nodes=12, grid_shape=(48, 48), energy_size=6.0)),
             ("gym_tadpole", G.TadpoleEnv, dict(head_nodes=8, tail_nodes=6, grid_shape=(48, 64))),
             ("gym_multi", G.MultiAgentEnv, dict(creatures=(G.LineTopology(num_nodes=10), G.RingTopology(num_nodes=12)),
                                                 grid_shape=(64, 64), energy_size=8.0)),
             ("gym_line_ring", G.LineRingEnv, dict(line_nodes=10, ring_nodes=12, centered_line=True,
                                                   grid_shape=(64, 64), energy_size=8.0))]
    for name, cls, kw in specs:
        env = cls(**kw, **common)
        key = jax.random.PRNGKey(0)
        obs0, st = env.reset(key)
        out = dict(H=np.int32(env.grid_shape[0]), W=np.int32(env.grid_shape[1]), dt=np.float32(env.dt),
                   max_steps=np.int32(env.max_steps), energy_size=np.float32(env.energy_size),
                   energy_amplitude=np.float32(env.energy_amplitude), obs0=A(obs0),
                   center0=A(st.energy_center), **state_arrays("in_", st.nodes, st.edges, st.fields))
        acts_r, acts_b, obs, rew, done = [], [], [], [], []
        for t in range(3):
            a = {"d_rest_length": jnp.array(rng.normal(0, 0.1, env.num_edges).astype(np.float32)),
                 "d_bending_angle": jnp.array(rng.normal(0, 0.1, env.num_bending_pairs).astype(np.float32))}
            key, sub = jax.random.split(key)
            o, st, r, d, info = env.step(sub, st, a)
            acts_r.append(A(a["d_rest_length"]))
            acts_b.append(A(a["d_bending_angle"]))
            obs.append(A(o))
            rew.append(np.float32(A(r)))
            done.append(bool(A(d)))
        out.update(act_rest=np.stack(acts_r), act_bend=np.stack(acts_b), obs=np.stack(obs), reward=np.array(rew),
                   done=np.array(done), time=np.int32(A(st.time)), center=A(st.energy_center),
                   **state_arrays("out_", st.nodes, st.edges, st.fields))
        if hasattr(env, "fitness_per_creature"):
            out["fitness"] = A(env.fitness_per_creature(st))
            out["segments"] = np.array([s.start for s in env.node_slices] + [env.node_slices[-1].stop], np.int32)
        save(name, **out)


def render_cases(R):
    """rendering.render (src/microcosmos/rendering.py:20-80) on small recorded timeseries:
    nodes inside, outside and on top of each other, debug vectors, steric values below 0
    and above 1; square and non-square grids, up- and down-sampling sizes, uniform colour
    and no particles.  The module's display imports (cv2, matplotlib) are stubbed: render()
    does not use them."""
    import types
    for name in ("matplotlib", "matplotlib.pyplot", "matplotlib.cm", "cv2"):
        if name not in sys.modules:
            sys.modules[name] = types.ModuleType(name)
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    sys.modules["matplotlib"].cm = sys.modules["matplotlib.cm"]
    import microcosmos.rendering as rendering
    jnp = sys.modules["jax"].numpy
    rng = np.random.default_rng(77)
    cases = [("render_32x32", 32, 32, 3, 20, [(64, True, False), (16, True, False), (32, True, True), (48, False, False)]),
             ("render_24x40", 24, 40, 2, 15, [(50, True, False), (20, True, False)])]
    for name, H, W, T, N, variants in cases:
        pos = rng.uniform(-3, [W + 3, H + 3], size=(T, N, 2)).astype(np.float32)
        pos[:, 1] = pos[:, 0]  # a pixel hit by two nodes
        dbg = rng.normal(0, 2.0, size=(T, N, 2)).astype(np.float32)
        dbg[:, ::3] = 0.0      # debug pixels on top of their node
        color = (np.arange(N) % 3).astype(np.int32)
        steric = rng.uniform(-0.3, 1.4, size=(T, H, W)).astype(np.float32)
        nodes = R["Nodes"](position=jnp.array(pos), velocity=jnp.zeros_like(jnp.array(pos)),
                           color_bend=jnp.array(np.broadcast_to(color, (T, N)).copy()), debug_vector=jnp.array(dbg))
        fields = R["Fields"](grid_shape=(H, W), steric=jnp.array(steric), fluid_velocity=jnp.zeros((T, 2, H, W)),
                             f_grid=None)
        out = dict(H=np.int32(H), W=np.int32(W), position=pos, debug_vector=dbg, color_bend=color, steric=steric)
        for sz, particles, uniform in variants:
            img = rendering.render(nodes, fields, sz, render_particles=particles, uniform_color=uniform)
            out[f"frames_{sz}_{int(particles)}{int(uniform)}"] = A(img)
        save(name, **out)


def _on_lattice(sc, h, w, rng, u0_std=1e-3):
    """The scenario's fluid moved to an h x w lattice: feq(1, u0) with fresh u0."""
    from microcosmos_b200 import scenarios as S
    ux = rng.normal(0, u0_std, (h, w)).astype(np.float32)
    uy = rng.normal(0, u0_std, (h, w)).astype(np.float32)
    sc.f_grid = S.equilibrium(np.ones((h, w), np.float32), ux, uy)
    sc.fluid_velocity = np.zeros((2, h, w), np.float32)
    return sc


def fluidgrid_cases(R):
    """A fluid lattice different from the domain grid (solver/fluid.py:221-235: IB points
    at position * (w / H, h / W), lattice velocities, velocity clamp and node reaction
    scaled; simulate.py:24-29: recorded u* resized to the domain grid)."""
    from microcosmos_b200 import scenarios as S
    jnp = sys.modules["jax"].numpy
    cfg_mod = R["config"]
    rng = np.random.default_rng(2468)
    for (H, W, h, w, F, n, ks, seed) in [(24, 24, 48, 48, 2, 10, 4, 41), (32, 32, 24, 24, 2, 12, 2, 42),
                                         (20, 28, 30, 42, 2, 8, 4, 43)]:
        sc = _on_lattice(S.make_scenario(H, W, F, n, seed=seed), h, w, rng)
        nodes, edges, fields = to_ref(R, sc)
        vel = jnp.array(rng.normal(0, 5.0, size=sc.position.shape).astype(np.float32))
        nodes = nodes.__replace__(velocity=vel)
        cfg = baseline_config(cfg_mod, ibm_kernel_size=ks)
        n2, f2, fnew = R["fluid"].immersed_boundary_interaction(nodes, edges, fields, fields.f_grid, 0.01, cfg)
        save(f"ib_lat_{H}x{W}_on_{h}x{w}", H=np.int32(H), W=np.int32(W), dt=np.float32(0.01), **cfg_arrays(cfg),
             **state_arrays("in_", nodes, edges, fields),
             velocity_out=A(n2.velocity), fluid_velocity_out=A(f2.fluid_velocity), f_grid_out=A(fnew))
    for (H, W, h, w, seed, name) in [(32, 32, 64, 64, 44, "sim_lat_32_on_64"), (40, 40, 30, 30, 45, "sim_lat_40_on_30")]:
        sc = _on_lattice(S.make_scenario(H, W, 3, 12, seed=seed, amp=0.2, period=20.0), h, w, rng)
        nodes, edges, fields = to_ref(R, sc)
        cfg = baseline_config(cfg_mod)
        dt, steps = 0.01, 6
        nts, fts = R["simulate"].simulate(nodes, edges, fields, dt, steps, cfg)
        nd, ed, fd = nodes, edges, fields
        traj = []
        for t in range(steps):
            ed = ed.__replace__(bending_rest_angles=jnp.array(S.actuation_rest_angles(sc, t)))
            nd, ed, fd = R["simulate"].step(nd, ed, fd, dt, cfg)
            traj.append(A(nd.position))
        save(name, H=np.int32(H), W=np.int32(W), dt=np.float32(dt), steps=np.int32(steps),
             **cfg_arrays(cfg), **state_arrays("in_", nodes, edges, fields),
             act_c=sc.act_c, act_amp=sc.act_amp, act_omega=sc.act_omega, act_phase=sc.act_phase,
             ts_position=A(nts.position), ts_velocity=A(nts.velocity), ts_steric=A(fts.steric),
             ts_fluid_velocity=A(fts.fluid_velocity),
             act_position=np.stack(traj), act_velocity=A(nd.velocity), act_theta=A(ed.theta),
             act_f_grid=A(fd.f_grid), act_steric=A(fd.steric), act_fluid_velocity=A(fd.fluid_velocity))


def worm_case(R):
    """The swimmer of the reference's end-to-end test (tests/test_worm.py): 20 nodes on a
    sine wave over a 50x50 grid, rest angles from a phase advancing 0.1 rad per step, 200
    steps of step() under PBD_SCHEME; the state after 50 and after 200 steps."""
    jnp = sys.modules["jax"].numpy
    G, U = R["graph"], R["utils"]
    n, H, W = 20, 50, 50
    pairs, dep = G.make_edges(n, graph="line", num_instances=1)
    bp, _ = G.compute_bending_pairs(pairs, dep, n)
    xs = jnp.linspace(W * 0.1, W * 0.9, n)
    amp = H * 0.3
    k = 2 * jnp.pi * 2 / (xs[-1] - xs[0])
    pos = jnp.stack([xs, H / 2 + amp * jnp.sin(k * xs)], axis=1)
    d = U.displacement((H, W), pos[pairs[:, 1]], pos[pairs[:, 0]])

    def rest(phase):
        tt = jnp.arctan(amp * k * jnp.cos(k * xs + phase))
        return tt[1:-1] - tt[:-2]

    nodes = R["Nodes"](position=pos, velocity=jnp.zeros_like(pos), color_bend=jnp.arange(n) % 3,
                       debug_vector=jnp.zeros((n, 2)))
    edges = R["Edges"](pairs=pairs, theta=jnp.arctan2(d[:, 1], d[:, 0]), rest_lengths=jnp.full(n - 1, 2.0),
                       bending_pairs=bp, bending_rest_angles=rest(0.0), bending_stiffness=jnp.ones(n - 2) * 0.5)
    w9 = jnp.array([4 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 36, 1 / 36, 1 / 36, 1 / 36])
    fields = R["Fields"](grid_shape=(H, W), steric=jnp.zeros((H, W)), fluid_velocity=jnp.zeros((2, H, W)),
                         f_grid=jnp.zeros((9, H, W)).at[:].set(w9[:, None, None]))
    out = dict(H=np.int32(H), W=np.int32(W), **state_arrays("in_", nodes, edges, fields))
    rests = []
    phase = 0.0
    for t in range(200):
        ra = rest(phase)
        rests.append(A(ra))
        edges = edges.__replace__(bending_rest_angles=ra)
        nodes, edges, fields = R["simulate"].step(nodes, edges, fields, 0.01, R["config"].PBD_SCHEME)
        if t == 49:
            out["pos_50"] = A(nodes.position)
        phase += 0.1
    out.update(rest_angles=np.stack(rests), pos_200=A(nodes.position), vel_200=A(nodes.velocity),
               f_grid_200=A(fields.f_grid))
    save("worm_50x50", **out)


if __name__ == "__main__":
    # usage: make_golden.py [reference root] [group,group,...]  (groups: GROUPS)
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    main(root, tuple(sys.argv[2].split(",")) if len(sys.argv) > 2 else GROUPS)
