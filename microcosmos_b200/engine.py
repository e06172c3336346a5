"""Host-side engine over the C ABI: plans, device workspaces and device-resident
rollout state.

A ``Plan`` holds one or more rollouts (any grid and filament sizes) that step
together; the single-instance path is a plan of one.  The C library allocates nothing
on the device: the workspace is a torch tensor owned by the ``Plan``.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import torch

from . import _lib
from .config import ConstraintSolverConfig, pbd_rod_constraint, stable_cosserat_constraint

_F32 = torch.float32


def _require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("microcosmos_b200 needs a CUDA device; there is no CPU fallback")


SOLVERS = {"pbd": 0, "cosserat": 1}


def mc_config(cfg: ConstraintSolverConfig) -> _lib.McConfig:
    """The C-ABI mirror of a ConstraintSolverConfig.  The plugin slot must hold one of the
    two device solvers, matching ``solver_type`` (simulate.py:68-71 switches on it)."""
    plugin = {pbd_rod_constraint: "pbd", stable_cosserat_constraint: "cosserat"}.get(cfg.bending_constraint)
    if plugin is None:
        raise NotImplementedError("bending_constraint must be pbd_rod_constraint or stable_cosserat_constraint; "
                                  "a host-side Python constraint cannot run inside the device step")
    if cfg.solver_type not in SOLVERS or cfg.solver_type != plugin:
        raise ValueError(f"solver_type {cfg.solver_type!r} does not match the {plugin} bending_constraint")
    c = _lib.McConfig()
    c.solver_type = SOLVERS[cfg.solver_type]
    c.solver_dt = float(cfg.dt)
    c.cycles_per_step = int(cfg.cycles_per_step)
    c.stiffness_stretch = float(cfg.stiffness_stretch)
    c.stiffness_shear = float(cfg.stiffness_shear)
    c.damping = float(cfg.damping)
    c.enable_fluid = int(bool(cfg.enable_fluid))
    c.viscosity = float(cfg.viscosity)
    c.max_fluid_velocity = float(cfg.max_fluid_velocity)
    c.ibm_iterations = int(cfg.ibm_iterations)
    c.synthetic_node_width = float(cfg.synthetic_node_width)
    c.ibm_kernel_size = int(cfg.ibm_kernel_size)
    c.ibm_relaxation = float(cfg.ibm_relaxation)
    c.node_mass = float(cfg.node_mass)
    c.lambda_trt = float(cfg.lambda_trt)
    c.enable_force_clamp = int(bool(cfg.enable_force_clamp))
    c.enable_steric = int(bool(cfg.enable_steric))
    c.steric_strength = float(cfg.steric_strength)
    c.steric_sigma = float(cfg.steric_sigma)
    c.steric_neighbor_skip = int(cfg.steric_neighbor_skip)
    c.steric_scatter_value = float(cfg.steric_scatter_value)
    return c


def _dev(x, dtype=_F32, device="cuda"):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=device)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


@dataclasses.dataclass
class DeviceState:
    """Device-resident Nodes/Edges/Fields of one rollout (float32, contiguous)."""
    H: int
    W: int
    position: torch.Tensor
    velocity: torch.Tensor
    theta: torch.Tensor
    rest_lengths: torch.Tensor
    bending_rest_angles: torch.Tensor
    bending_stiffness: torch.Tensor
    steric: torch.Tensor
    fluid_velocity: torch.Tensor
    f_grid: torch.Tensor
    pairs: np.ndarray          # host int32 topology
    bending_pairs: np.ndarray

    @property
    def N(self):
        return self.position.shape[0]

    @property
    def lH(self):
        """Rows of the fluid lattice (f_grid)."""
        return int(self.f_grid.shape[1])

    @property
    def lW(self):
        return int(self.f_grid.shape[2])

    @property
    def E(self):
        return int(self.pairs.shape[0])

    @property
    def B(self):
        return int(self.bending_pairs.shape[0])

    @classmethod
    def from_arrays(cls, H, W, position, velocity, pairs, theta, rest_lengths, bending_pairs,
                    bending_rest_angles, bending_stiffness, f_grid, steric=None, fluid_velocity=None,
                    device="cuda"):
        pairs_h = np.ascontiguousarray(
            pairs.detach().cpu().numpy() if isinstance(pairs, torch.Tensor) else pairs, dtype=np.int32).reshape(-1, 2)
        bp_h = np.ascontiguousarray(
            bending_pairs.detach().cpu().numpy() if isinstance(bending_pairs, torch.Tensor) else bending_pairs,
            dtype=np.int32).reshape(-1, 2)
        # f_grid (9, h, w) on its own lattice; a flat array is taken on the domain grid
        fg = _dev(f_grid, device=device)
        fg = (fg if fg.dim() == 3 else fg.reshape(9, H, W)).clone()
        return cls(
            H=int(H), W=int(W),
            position=_dev(position, device=device).reshape(-1, 2).clone(),
            velocity=_dev(velocity, device=device).reshape(-1, 2).clone(),
            theta=_dev(theta, device=device).reshape(-1).clone(),
            rest_lengths=_dev(rest_lengths, device=device).reshape(-1).clone(),
            bending_rest_angles=_dev(bending_rest_angles, device=device).reshape(-1).clone(),
            bending_stiffness=_dev(bending_stiffness, device=device).reshape(-1).clone(),
            steric=(_dev(steric, device=device).clone() if steric is not None
                    else torch.zeros((H, W), dtype=_F32, device=device)),
            fluid_velocity=(_dev(fluid_velocity, device=device).clone() if fluid_velocity is not None
                            else torch.zeros((2,) + tuple(fg.shape[1:]), dtype=_F32, device=device)),
            f_grid=fg, pairs=pairs_h, bending_pairs=bp_h)

    @classmethod
    def from_scenario(cls, sc, device="cuda"):
        return cls.from_arrays(sc.H, sc.W, sc.position, sc.velocity, sc.pairs, sc.theta, sc.rest_lengths,
                               sc.bending_pairs, sc.bending_rest_angles, sc.bending_stiffness, sc.f_grid,
                               sc.steric, sc.fluid_velocity, device=device)

    def struct(self) -> _lib.McState:
        s = _lib.McState()
        s.position = self.position.data_ptr()
        s.velocity = self.velocity.data_ptr()
        s.theta = self.theta.data_ptr()
        s.rest_lengths = self.rest_lengths.data_ptr()
        s.bending_rest_angles = self.bending_rest_angles.data_ptr()
        s.bending_stiffness = self.bending_stiffness.data_ptr()
        s.steric = self.steric.data_ptr()
        s.fluid_velocity = self.fluid_velocity.data_ptr()
        s.f_grid = self.f_grid.data_ptr()
        return s

    def host(self):
        """Copy to numpy (synchronises)."""
        return {k: getattr(self, k).detach().cpu().numpy() for k in
                ("position", "velocity", "theta", "bending_rest_angles", "steric", "fluid_velocity", "f_grid")}


@dataclasses.dataclass
class Actuation:
    """rest[b](t) = c[b] + amp[b] sin(omega[b] t + phase[b]) on the device."""
    c: torch.Tensor
    amp: torch.Tensor
    omega: torch.Tensor
    phase: torch.Tensor
    t0: int = 0

    @classmethod
    def from_scenario(cls, sc, device="cuda", t0=0):
        if sc.act_amp is None:
            return None
        return cls(_dev(sc.act_c, device=device), _dev(sc.act_amp, device=device),
                   _dev(sc.act_omega, device=device), _dev(sc.act_phase, device=device), t0)

    def struct(self):
        a = _lib.McActuation()
        a.c, a.amp, a.omega, a.phase = (self.c.data_ptr(), self.amp.data_ptr(), self.omega.data_ptr(),
                                        self.phase.data_ptr())
        a.t0 = int(self.t0)
        return a


@dataclasses.dataclass
class Record:
    position: torch.Tensor | None = None
    velocity: torch.Tensor | None = None
    steric: torch.Tensor | None = None
    fluid_velocity: torch.Tensor | None = None
    every: int = 1

    @classmethod
    def allocate(cls, state: DeviceState, num_steps: int, every: int = 1, fields=True, device="cuda"):
        T = num_steps // every
        N, H, W = state.N, state.H, state.W
        return cls(position=torch.empty((T, N, 2), dtype=_F32, device=device),
                   velocity=torch.empty((T, N, 2), dtype=_F32, device=device),
                   steric=torch.empty((T, H, W), dtype=_F32, device=device) if fields else None,
                   fluid_velocity=torch.empty((T, 2, H, W), dtype=_F32, device=device) if fields else None,
                   every=every)

    def struct(self):
        r = _lib.McRecord()
        r.position = self.position.data_ptr() if self.position is not None else None
        r.velocity = self.velocity.data_ptr() if self.velocity is not None else None
        r.steric = self.steric.data_ptr() if self.steric is not None else None
        r.fluid_velocity = self.fluid_velocity.data_ptr() if self.fluid_velocity is not None else None
        r.every = int(self.every)
        return r


class Plan:
    """A bound plan for a list of rollouts (dims + config + dt + topology each)."""

    def __init__(self, specs, device="cuda", lbm_shape=None, steric_method=0, fft_values=0, bin_threads=0,
                 bin_sort_capacity=0, ib_cluster=0, lbm_stages=None):
        """specs: list of (H, W, N, pairs(E,2) int32, bending_pairs(B,2) int32, cfg, dt[, (fluid_H, fluid_W)]).
        ``lbm_shape`` = (cells_per_lane, rows_per_cta) of the dense pass (default: the
        library's choice; ``microcosmos_b200.autotune`` picks one by timing).
        ``steric_method``: 0 = per rollout (direct convolution where it applies, else
        FFT), 1 = FFT, 2 = direct convolution.  ``fft_values``: values per thread of the
        power-of-two FFT kernels (4, 8, 16; 0 = the library's choice).  ``bin_threads``:
        threads per CTA of the contribution-sorting tile kernel (64, 128, 256; 0 = 128).
        ``bin_sort_capacity``: contributions per tile sorted in shared memory (0 = 2048).
        ``ib_cluster``: CTAs per rollout cluster for the IB iterations (0 = separate launches).
        ``lbm_stages``: 2..6 runs the staged dense pass (row bands copied into shared
        memory by bulk copies, that many in flight per CTA), 0 the tiled kernel of
        ``lbm_shape``; None keeps the library's choice (a given ``lbm_shape`` selects the
        tiled kernel)."""
        _require_cuda()
        lib = _lib.load()
        n = len(specs)
        dims = (_lib.McDims * n)()
        cfgs = (_lib.McConfig * n)()
        dts = (ctypes.c_float * n)()
        self._keep = []
        pp = (_lib.c_int_p * n)()
        bp = (_lib.c_int_p * n)()
        for i, spec in enumerate(specs):
            H, W, N, pairs, bpairs, cfg, dt = spec[:7]
            fh, fw = spec[7] if len(spec) > 7 else (0, 0)
            pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
            bpairs = np.ascontiguousarray(bpairs, dtype=np.int32).reshape(-1, 2)
            self._keep += [pairs, bpairs]
            dims[i] = _lib.McDims(int(H), int(W), int(N), pairs.shape[0], bpairs.shape[0], int(fh), int(fw))
            cfgs[i] = mc_config(cfg)
            dts[i] = float(dt)
            pp[i] = pairs.ctypes.data_as(_lib.c_int_p)
            bp[i] = bpairs.ctypes.data_as(_lib.c_int_p)
        h = ctypes.c_void_p()
        _lib.check(lib.mc_plan_create(n, dims, cfgs, dts, pp, bp, ctypes.byref(h)))
        self._h = h
        self.n = n
        self.specs = specs
        if lbm_shape is not None:
            _lib.check(lib.mc_plan_set_lbm_shape(h, int(lbm_shape[0]), int(lbm_shape[1])))
        if lbm_stages is not None:
            _lib.check(lib.mc_plan_set_lbm_staging(h, int(lbm_stages)))
        if steric_method:
            _lib.check(lib.mc_plan_set_steric_method(h, int(steric_method)))
        if fft_values:
            _lib.check(lib.mc_plan_set_fft_values_per_thread(h, int(fft_values)))
        if bin_threads:
            _lib.check(lib.mc_plan_set_bin_threads(h, int(bin_threads)))
        if bin_sort_capacity:
            _lib.check(lib.mc_plan_set_bin_sort_capacity(h, int(bin_sort_capacity)))
        nbytes = lib.mc_plan_workspace_bytes(h)
        self.workspace = torch.empty(nbytes + 256, dtype=torch.uint8, device=device)
        base = self.workspace.data_ptr()
        self._ws_ptr = (base + 255) // 256 * 256
        self.workspace_bytes = nbytes
        stream = torch.cuda.current_stream().cuda_stream
        _lib.check(lib.mc_plan_bind(h, ctypes.c_void_p(self._ws_ptr), nbytes, ctypes.c_void_p(stream)))
        if ib_cluster:
            _lib.check(lib.mc_plan_set_ib_cluster(h, int(ib_cluster)))

    @classmethod
    def for_states(cls, states, cfgs, dts, device="cuda", lbm_shape=None, steric_method=0, fft_values=0,
                   bin_threads=0, bin_sort_capacity=0, ib_cluster=0, lbm_stages=None):
        specs = [(s.H, s.W, s.N, s.pairs, s.bending_pairs, c, d, (s.lH, s.lW)) for s, c, d in zip(states, cfgs, dts)]
        return cls(specs, device=device, lbm_shape=lbm_shape, steric_method=steric_method, fft_values=fft_values,
                   bin_threads=bin_threads, bin_sort_capacity=bin_sort_capacity, ib_cluster=ib_cluster,
                   lbm_stages=lbm_stages)

    def bin_threads(self):
        return int(_lib.load().mc_plan_bin_threads(self._h))

    def fft_values(self):
        """Values per thread of the power-of-two FFT kernels."""
        return int(_lib.load().mc_plan_fft_values_per_thread(self._h))

    def steric_method(self):
        """1: FFT, 2: direct convolution, 3: mixed across rollouts, 0: no steric."""
        return int(_lib.load().mc_plan_steric_method(self._h))

    def lbm_stages(self):
        """Bands in flight per CTA of the staged dense pass (0: the tiled kernel)."""
        return int(_lib.load().mc_plan_lbm_staging(self._h))

    def lbm_shape(self):
        """(cells_per_lane, rows_per_cta) of the tiled dense-pass kernel."""
        a, b = ctypes.c_int32(), ctypes.c_int32()
        _lib.check(_lib.load().mc_plan_get_lbm_shape(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def _arrays(self, states, actuations, records):
        n = self.n
        if len(states) != n:
            raise ValueError(f"plan has {n} rollouts, got {len(states)} states")
        st = (_lib.McState * n)()
        for i, s in enumerate(states):
            st[i] = s.struct()
        act_arr = None
        if actuations is not None and any(a is not None for a in actuations):
            structs = [a.struct() if a is not None else None for a in actuations]
            self._act_structs = structs
            act_arr = (ctypes.POINTER(_lib.McActuation) * n)(
                *[ctypes.pointer(s) if s is not None else ctypes.POINTER(_lib.McActuation)() for s in structs])
        rec_arr = None
        if records is not None and any(r is not None for r in records):
            structs = [r.struct() if r is not None else None for r in records]
            self._rec_structs = structs
            rec_arr = (ctypes.POINTER(_lib.McRecord) * n)(
                *[ctypes.pointer(s) if s is not None else ctypes.POINTER(_lib.McRecord)() for s in structs])
        self._st = st
        return st, act_arr, rec_arr

    @staticmethod
    def _stream(stream):
        return ctypes.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)

    def rollout(self, states, num_steps, actuations=None, records=None, use_graph=True, stream=None):
        """Run num_steps steps of every rollout (mc_rollout)."""
        st, act_arr, rec_arr = self._arrays(states, actuations, records)
        _lib.check(_lib.load().mc_rollout(self._h, st, int(num_steps), act_arr, rec_arr, int(bool(use_graph)),
                                          self._stream(stream)))

    def begin(self, states, actuations=None, records=None, stream=None):
        st, act_arr, rec_arr = self._arrays(states, actuations, records)
        _lib.check(_lib.load().mc_rollout_begin(self._h, st, act_arr, rec_arr, self._stream(stream)))

    def advance(self, num_steps, use_graph=True, last=False, stream=None):
        _lib.check(_lib.load().mc_rollout_advance(self._h, int(num_steps), int(bool(use_graph)), int(bool(last)),
                                                  self._stream(stream)))

    def end(self, stream=None):
        _lib.check(_lib.load().mc_rollout_end(self._h, self._stream(stream)))

    def set_fused_ib(self, enable=True):
        _lib.check(_lib.load().mc_plan_set_fused_ib(self._h, int(bool(enable))))

    def uses_fused_ib(self):
        return bool(_lib.load().mc_plan_uses_fused_ib(self._h))

    def set_ib_cluster(self, ctas):
        """Run each rollout's IB iterations in one cluster of `ctas` CTAs (0: separate launches)."""
        _lib.check(_lib.load().mc_plan_set_ib_cluster(self._h, int(ctas)))

    def ib_cluster(self):
        return int(_lib.load().mc_plan_ib_cluster(self._h))

    def profile(self, enable=True):
        _lib.check(_lib.load().mc_plan_profile(self._h, int(bool(enable))))

    def profile_reset(self):
        _lib.check(_lib.load().mc_plan_profile_reset(self._h))

    def profile_read(self):
        """{kernel: (total_ms, launches)} of the per-kernel event timing."""
        lib = _lib.load()
        out = {}
        for name in lib.mc_profile_kernel_names().decode().split(","):
            ms = ctypes.c_double()
            cnt = ctypes.c_int64()
            _lib.check(lib.mc_plan_profile_read(self._h, name.encode(), ctypes.byref(ms), ctypes.byref(cnt)))
            out[name] = (ms.value, cnt.value)
        return out

    def read_flags(self, clear=False):
        lib = _lib.load()
        out = (ctypes.c_uint32 * self.n)()
        s = torch.cuda.current_stream().cuda_stream
        _lib.check(lib.mc_plan_read_flags(self._h, out, int(bool(clear)), ctypes.c_void_p(s)))
        return list(out)

    def last_launch_count(self):
        return int(_lib.load().mc_plan_last_launch_count(self._h))

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().mc_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
