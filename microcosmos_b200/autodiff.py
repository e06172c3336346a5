"""Gradients of a rollout: the reverse-mode derivative of ``simulate`` through hand-written
adjoint kernels (C ABI ``mc_grad_*``), as a ``torch.autograd.Function``.

The reference differentiates ``simulate`` with ``jax.grad`` / ``jax.value_and_grad``
(tests/test_differentiability.py:45,65).  Here the forward rollout runs the same CUDA
kernels as ``simulate.run`` while keeping a checkpoint of the state every
``checkpoint_every`` steps (default ceil(sqrt(T))); the backward pass recomputes each
segment from its checkpoint and runs the adjoint steps of stream+collide, IB, PBD and
steric in reverse.  The derivative follows the reference's conventions: the Peskin
stencil positions are ``stop_gradient``-ed (src/microcosmos/solver/fluid.py:239), floor
has derivative 0, mod derivative 1, max/min split ties evenly.  Cotangents of the
``steric`` and ``fluid_velocity`` outputs are zero (they are returned as
non-differentiable outputs).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .engine import _require_cuda, mc_config

_F32 = torch.float32


class GradPlan:
    """One rollout's gradient plan: topology, config, dt, step count and checkpoint interval."""

    def __init__(self, H, W, N, pairs, bending_pairs, cfg, dt, num_steps, checkpoint_every=0, device="cuda",
                 fluid_shape=None):
        """(H, W) the domain grid; ``fluid_shape`` = (h, w) of the fluid lattice when it
        differs from the domain grid (f_grid is then (9, h, w))."""
        _require_cuda()
        lib = _lib.load()
        self.pairs = np.ascontiguousarray(pairs, np.int32).reshape(-1, 2)
        self.bpairs = np.ascontiguousarray(bending_pairs, np.int32).reshape(-1, 2)
        self.H, self.W, self.N = int(H), int(W), int(N)
        self.lH, self.lW = (self.H, self.W) if fluid_shape is None else (int(fluid_shape[0]), int(fluid_shape[1]))
        self.E, self.B = self.pairs.shape[0], self.bpairs.shape[0]
        self.num_steps = int(num_steps)
        dims = _lib.McDims(self.H, self.W, self.N, self.E, self.B)
        if (self.lH, self.lW) != (self.H, self.W):
            dims.fluid_H, dims.fluid_W = self.lH, self.lW
        c = mc_config(cfg)
        h = ctypes.c_void_p()
        _lib.check(lib.mc_grad_plan_create(ctypes.byref(dims), ctypes.byref(c), float(dt),
                                           self.pairs.ctypes.data_as(_lib.c_int_p),
                                           self.bpairs.ctypes.data_as(_lib.c_int_p), self.num_steps,
                                           int(checkpoint_every), ctypes.byref(h)))
        self._h = h
        self.checkpoint_every = int(lib.mc_grad_plan_checkpoint_every(h))
        nbytes = lib.mc_grad_plan_workspace_bytes(h)
        self.workspace = torch.empty(nbytes + 256, dtype=torch.uint8, device=device)
        ptr = (self.workspace.data_ptr() + 255) // 256 * 256
        self.workspace_bytes = nbytes
        s = torch.cuda.current_stream().cuda_stream
        _lib.check(lib.mc_grad_plan_bind(h, ctypes.c_void_p(ptr), nbytes, ctypes.c_void_p(s)))
        self.has_act = False

    def forward(self, state, actuation=None):
        """Run the rollout in place on a ``DeviceState``; ``actuation`` (engine.Actuation, t0 = 0)."""
        lib = _lib.load()
        st = state.struct()
        act = None
        if actuation is not None:
            act = actuation.struct()
        self.has_act = act is not None
        s = torch.cuda.current_stream().cuda_stream
        _lib.check(lib.mc_grad_forward(self._h, ctypes.byref(st), ctypes.byref(act) if act is not None else None,
                                       ctypes.c_void_p(s)))

    def backward(self, d_position=None, d_velocity=None, d_theta=None, d_f_grid=None, device="cuda"):
        """Cotangents of the final state in, gradients of the initial state and parameters out."""
        lib = _lib.load()
        z = lambda *shape: torch.empty(shape, dtype=_F32, device=device)  # noqa: E731
        seeds = [_c(d_position), _c(d_velocity), _c(d_theta), _c(d_f_grid)]  # alive until the call returns
        fin = _lib.McStateCot(*[t.data_ptr() if t is not None else None for t in seeds])
        out = {"position": z(self.N, 2), "velocity": z(self.N, 2), "theta": z(self.E),
               "f_grid": z(9, self.lH, self.lW), "rest_lengths": z(self.E), "bending_stiffness": z(self.B)}
        if self.has_act:
            out.update(act_c=z(self.B), act_amp=z(self.B), act_omega=z(self.B), act_phase=z(self.B))
        else:
            out["bending_rest_angles"] = z(self.B)
        ini = _lib.McStateCot(out["position"].data_ptr(), out["velocity"].data_ptr(), out["theta"].data_ptr(),
                              out["f_grid"].data_ptr())
        g = _lib.McParamGrads(out["bending_rest_angles"].data_ptr() if not self.has_act else None,
                              out["act_c"].data_ptr() if self.has_act else None,
                              out["act_amp"].data_ptr() if self.has_act else None,
                              out["act_phase"].data_ptr() if self.has_act else None,
                              out["rest_lengths"].data_ptr(), out["bending_stiffness"].data_ptr(),
                              out["act_omega"].data_ptr() if self.has_act else None)
        s = torch.cuda.current_stream().cuda_stream
        _lib.check(lib.mc_grad_backward(self._h, ctypes.byref(fin), ctypes.byref(ini), ctypes.byref(g),
                                        ctypes.c_void_p(s)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().mc_grad_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _c(t):
    if t is None:
        return None
    return t.detach().to(_F32).contiguous()


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, position, velocity, theta, f_grid, rest_lengths, bending_stiffness, bending_rest_angles,
                act_c, act_amp, act_omega, act_phase, spec):
        from .engine import Actuation, DeviceState
        H, W, pairs, bpairs, cfg, dt, num_steps, ckpt = spec
        fluid_shape = (int(f_grid.shape[1]), int(f_grid.shape[2]))
        st = DeviceState.from_arrays(H, W, position.detach(), velocity.detach(), pairs, theta.detach(),
                                     rest_lengths.detach(), bpairs, bending_rest_angles.detach(),
                                     bending_stiffness.detach(), f_grid.detach(), device=position.device)
        act = None
        if act_c is not None:
            dev = position.device
            act = Actuation(*[_c(torch.as_tensor(a, device=dev)) for a in (act_c, act_amp, act_omega, act_phase)], 0)
        plan = GradPlan(H, W, st.N, pairs, bpairs, cfg, dt, num_steps, ckpt, device=position.device,
                        fluid_shape=fluid_shape)
        plan.forward(st, act)
        ctx.plan = plan
        ctx.has_act = act is not None
        ctx.mark_non_differentiable(st.steric, st.fluid_velocity)
        return st.position, st.velocity, st.theta, st.f_grid, st.steric, st.fluid_velocity

    @staticmethod
    def backward(ctx, gpos, gvel, gth, gf, _gs, _gu):
        g = ctx.plan.backward(gpos, gvel, gth, gf)
        if ctx.has_act:
            gr, gc, ga, go, gp = None, g["act_c"], g["act_amp"], g["act_omega"], g["act_phase"]
        else:
            gr, gc, ga, go, gp = g["bending_rest_angles"], None, None, None, None
        grads = (g["position"], g["velocity"], g["theta"], g["f_grid"], g["rest_lengths"], g["bending_stiffness"],
                 gr, gc, ga, go, gp)
        # inputs given as arrays (e.g. a fixed omega) take no gradient
        return tuple(x if need else None for x, need in zip(grads, ctx.needs_input_grad)) + (None,)


def rollout(position, velocity, theta, f_grid, rest_lengths, bending_stiffness, bending_rest_angles, pairs,
            bending_pairs, cfg, dt, num_steps, actuation=None, checkpoint_every=0, grid_shape=None):
    """Differentiable rollout (torch): returns (position, velocity, theta, f_grid, steric,
    fluid_velocity) after ``num_steps`` steps.  ``actuation`` = (c, amp, omega, phase) per
    bending pair (rest[b](t) = c + amp sin(omega t + phase)); gradients flow to every
    float tensor argument.  ``f_grid`` is (9, h, w) on the fluid lattice; ``grid_shape`` =
    (H, W) of the domain when it differs from the lattice (Fields.grid_shape)."""
    f_grid = f_grid.reshape(9, *f_grid.shape[-2:])
    H, W = (int(f_grid.shape[1]), int(f_grid.shape[2])) if grid_shape is None else map(int, grid_shape)
    pairs_h = np.ascontiguousarray(pairs.detach().cpu().numpy() if isinstance(pairs, torch.Tensor) else pairs,
                                   np.int32).reshape(-1, 2)
    bp_h = np.ascontiguousarray(bending_pairs.detach().cpu().numpy() if isinstance(bending_pairs, torch.Tensor)
                                else bending_pairs, np.int32).reshape(-1, 2)
    c = amp = om = ph = None
    if actuation is not None:
        c, amp, om, ph = actuation
    spec = (H, W, pairs_h, bp_h, cfg, float(dt), int(num_steps), int(checkpoint_every))
    return _Rollout.apply(position, velocity, theta, f_grid, rest_lengths, bending_stiffness, bending_rest_angles,
                          c, amp, om, ph, spec)
