"""C ABI checks that need no GPU: the in-tree library loads, exports every function that
include/microcosmos_b200.h declares, and validates plans on the host (mc_plan_create
touches no device)."""
import ctypes
import os
import re

import numpy as np
import pytest

from microcosmos_b200 import _lib, baseline_config, scenarios

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(REPO, "include", "microcosmos_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mc_[a-z_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from microcosmos_b200 import build
    build.build()
    return _lib.load()


def test_exports_every_declared_symbol(lib):
    names = header_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
    assert set(_lib.SIGNATURES) == set(names)


def test_version(lib):
    assert b"sm_100a" in lib.mc_version()


def _create(specs):
    lib = _lib.load()
    from microcosmos_b200.engine import mc_config
    n = len(specs)
    dims = (_lib.McDims * n)()
    cfgs = (_lib.McConfig * n)()
    dts = (ctypes.c_float * n)()
    pp = (_lib.c_int_p * n)()
    bp = (_lib.c_int_p * n)()
    keep = []
    for i, (H, W, N, pairs, bpairs, cfg, dt) in enumerate(specs):
        pairs = np.ascontiguousarray(pairs, np.int32).reshape(-1, 2)
        bpairs = np.ascontiguousarray(bpairs, np.int32).reshape(-1, 2)
        keep += [pairs, bpairs]
        dims[i] = _lib.McDims(H, W, N, pairs.shape[0], bpairs.shape[0])
        cfgs[i] = mc_config(cfg)
        dts[i] = dt
        pp[i] = pairs.ctypes.data_as(_lib.c_int_p)
        bp[i] = bpairs.ctypes.data_as(_lib.c_int_p)
    h = ctypes.c_void_p()
    st = lib.mc_plan_create(n, dims, cfgs, dts, pp, bp, ctypes.byref(h))
    return st, h


def test_plan_create_and_workspace_size(lib):
    sc = scenarios.make_scenario(64, 64, 3, 20, seed=0)
    st, h = _create([(64, 64, sc.N, sc.pairs, sc.bending_pairs, baseline_config(), 0.01)])
    assert st == _lib.MC_OK, lib.mc_last_error()
    nbytes = lib.mc_plan_workspace_bytes(h)
    # two population buffers dominate: 2 * 9 * 64 * 64 * 4 bytes
    assert nbytes > 2 * 9 * 64 * 64 * 4
    lib.mc_plan_destroy(h)


def test_plan_rejects_bad_topology(lib):
    sc = scenarios.make_scenario(32, 32, 1, 10, seed=0)
    bad = sc.pairs.copy()
    bad[3, 1] = sc.N + 5
    st, _ = _create([(32, 32, sc.N, bad, sc.bending_pairs, baseline_config(), 0.01)])
    assert st == _lib.MC_ERR_INVALID
    assert b"outside" in lib.mc_last_error()
    badb = sc.bending_pairs.copy()
    badb[0, 0] = -1
    st, _ = _create([(32, 32, sc.N, sc.pairs, badb, baseline_config(), 0.01)])
    assert st == _lib.MC_ERR_INVALID


def test_plan_rejects_unsupported_config(lib):
    sc = scenarios.make_scenario(32, 32, 1, 10, seed=0)
    import dataclasses
    st, _ = _create([(32, 32, sc.N, sc.pairs, sc.bending_pairs,
                      dataclasses.replace(baseline_config(), synthetic_node_width=-1.0), 0.01)])
    assert st == _lib.MC_ERR_INVALID
    st, h = _create([(32, 32, sc.N, sc.pairs, sc.bending_pairs,
                      dataclasses.replace(baseline_config(), synthetic_node_width=1.0), 0.01)])
    assert st == _lib.MC_OK
    lib.mc_plan_destroy(h)
    # 34 x 34: no FFT plan (prime factor 17) and too small for the direct filter (radius 17)
    st, _ = _create([(34, 34, sc.N, sc.pairs, sc.bending_pairs, baseline_config(), 0.01)])
    assert st == _lib.MC_ERR_UNSUPPORTED
    st, _ = _create([(34, 34, sc.N, sc.pairs, sc.bending_pairs,
                      dataclasses.replace(baseline_config(), enable_steric=False), 0.01)])
    assert st == _lib.MC_OK
    # 51 x 51 has no FFT plan: the direct filter
    st, h = _create([(51, 51, sc.N, sc.pairs, sc.bending_pairs, baseline_config(), 0.01)])
    assert st == _lib.MC_OK
    assert lib.mc_plan_steric_method(h) == 2
    assert lib.mc_plan_set_steric_method(h, 1) == _lib.MC_ERR_UNSUPPORTED
    lib.mc_plan_destroy(h)
    st, _ = _create([(32, 32, sc.N, sc.pairs, sc.bending_pairs, baseline_config(), 0.0)])
    assert st == _lib.MC_ERR_INVALID


def test_rod_solver_selection(lib):
    """Both device rod solvers build plans; a foreign plugin, a solver_type that does not
    match the plugin, and a non-positive Cosserat dt are rejected."""
    import dataclasses
    from microcosmos_b200 import COSSERAT_SCHEME, COSSERAT_SCHEME_NO_FLUID, PBD_SCHEME
    from microcosmos_b200.engine import mc_config
    c = mc_config(COSSERAT_SCHEME)
    assert c.solver_type == 1 and c.solver_dt == 0.05
    assert mc_config(PBD_SCHEME).solver_type == 0
    with pytest.raises(NotImplementedError):
        mc_config(dataclasses.replace(PBD_SCHEME, bending_constraint=lambda *a, **k: a))
    with pytest.raises(ValueError):
        mc_config(dataclasses.replace(PBD_SCHEME, solver_type="cosserat"))
    sc = scenarios.make_scenario(32, 32, 1, 10, seed=0)
    for cfg in (COSSERAT_SCHEME, COSSERAT_SCHEME_NO_FLUID):
        st, h = _create([(32, 32, sc.N, sc.pairs, sc.bending_pairs, cfg, 0.05)])
        assert st == _lib.MC_OK
        lib.mc_plan_destroy(h)
    st, _ = _create([(32, 32, sc.N, sc.pairs, sc.bending_pairs, dataclasses.replace(COSSERAT_SCHEME, dt=0.0), 0.05)])
    assert st == _lib.MC_ERR_INVALID


def test_gradient_plan_scope(lib):
    """mc_grad_plan_create (host-only) takes both rod solvers, synthetic IB pairs and a
    fluid lattice other than the domain grid; a half-given lattice shape is refused."""
    import dataclasses
    from microcosmos_b200 import COSSERAT_SCHEME, PBD_SCHEME
    from microcosmos_b200.engine import mc_config
    sc = scenarios.make_scenario(32, 32, 2, 10, seed=0)
    pairs = np.ascontiguousarray(sc.pairs, np.int32)
    bpairs = np.ascontiguousarray(sc.bending_pairs, np.int32)

    def create(cfg, fluid=(0, 0)):
        dims = _lib.McDims(32, 32, sc.N, pairs.shape[0], bpairs.shape[0])
        dims.fluid_H, dims.fluid_W = fluid
        c = mc_config(cfg)
        h = ctypes.c_void_p()
        st = lib.mc_grad_plan_create(ctypes.byref(dims), ctypes.byref(c), 0.01, pairs.ctypes.data_as(_lib.c_int_p),
                                     bpairs.ctypes.data_as(_lib.c_int_p), 10, 0, ctypes.byref(h))
        if st == _lib.MC_OK:
            lib.mc_grad_plan_destroy(h)
        return st

    assert create(PBD_SCHEME) == _lib.MC_OK
    assert create(COSSERAT_SCHEME) == _lib.MC_OK
    assert create(dataclasses.replace(COSSERAT_SCHEME, dt=0.0)) == _lib.MC_ERR_INVALID
    assert create(dataclasses.replace(PBD_SCHEME, synthetic_node_width=0.5)) == _lib.MC_OK
    assert create(dataclasses.replace(COSSERAT_SCHEME, synthetic_node_width=0.5)) == _lib.MC_OK
    assert create(PBD_SCHEME, fluid=(16, 16)) == _lib.MC_OK
    assert create(PBD_SCHEME, fluid=(48, 40)) == _lib.MC_OK
    assert create(PBD_SCHEME, fluid=(16, 0)) == _lib.MC_ERR_INVALID


def test_batch_plan_of_uneven_rollouts(lib):
    scs = [scenarios.make_scenario(s, s, f, n, seed=i) for i, (s, f, n) in
           enumerate([(128, 3, 16), (192, 1, 100), (64, 5, 30)])]
    st, h = _create([(s.H, s.W, s.N, s.pairs, s.bending_pairs, baseline_config(), 0.01) for s in scs])
    assert st == _lib.MC_OK, lib.mc_last_error()
    lib.mc_plan_destroy(h)


def test_lbm_shape_setter_validates_and_reports(lib):
    sc = scenarios.make_scenario(64, 96, 2, 12, seed=0)
    st, h = _create([(64, 96, sc.N, sc.pairs, sc.bending_pairs, baseline_config(), 0.01)])
    assert st == _lib.MC_OK
    a, b = ctypes.c_int32(), ctypes.c_int32()
    assert lib.mc_plan_get_lbm_shape(h, ctypes.byref(a), ctypes.byref(b)) == _lib.MC_OK
    assert (a.value, b.value) == (2, 4)  # the library's default for a small plan
    assert lib.mc_plan_set_lbm_shape(h, 2, 32) == _lib.MC_OK
    lib.mc_plan_get_lbm_shape(h, ctypes.byref(a), ctypes.byref(b))
    assert (a.value, b.value) == (2, 32)
    assert lib.mc_plan_set_lbm_shape(h, 3, 0) == _lib.MC_ERR_INVALID
    assert lib.mc_plan_set_lbm_shape(h, 0, 12) == _lib.MC_ERR_INVALID
    assert lib.mc_plan_set_lbm_shape(h, 0, 64) == _lib.MC_ERR_INVALID
    lib.mc_plan_destroy(h)
    # 4 cells per lane must divide W
    sc2 = scenarios.make_scenario(64, 66, 1, 10, seed=0)
    st, h2 = _create([(64, 66, sc2.N, sc2.pairs, sc2.bending_pairs, baseline_config(), 0.01)])
    assert st == _lib.MC_OK
    assert lib.mc_plan_set_lbm_shape(h2, 4, 4) == _lib.MC_ERR_UNSUPPORTED
    lib.mc_plan_destroy(h2)


def test_autotune_candidates_respect_widths():
    from microcosmos_b200 import autotune

    class S:
        def __init__(self, W):
            self.W = W

    assert autotune.candidates([S(64), S(128)]) == [(v, r) for v in (1, 2, 4) for r in (4, 8, 16, 32)]
    assert autotune.candidates([S(64), S(66)]) == [(v, r) for v in (1, 2) for r in (4, 8, 16, 32)]
    assert autotune.candidates([S(63)]) == [(1, r) for r in (4, 8, 16, 32)]


def test_tile_kernel_threads_setter(lib):
    sc = scenarios.make_scenario(64, 64, 2, 12, seed=0)
    st, h = _create([(64, 64, sc.N, sc.pairs, sc.bending_pairs, baseline_config(), 0.01)])
    assert st == _lib.MC_OK
    assert lib.mc_plan_bin_threads(h) == 128
    assert lib.mc_plan_set_bin_threads(h, 128) == _lib.MC_OK and lib.mc_plan_bin_threads(h) == 128
    assert lib.mc_plan_set_bin_threads(h, 96) == _lib.MC_ERR_INVALID
    assert lib.mc_plan_set_fft_values_per_thread(h, 8) == _lib.MC_OK and lib.mc_plan_fft_values_per_thread(h) == 8
    assert lib.mc_plan_set_fft_values_per_thread(h, 5) == _lib.MC_ERR_INVALID
    # default 2048, capped by the plan's bin capacity (1024 for this sparse rollout)
    assert lib.mc_plan_bin_sort_capacity(h) == 1024
    assert lib.mc_plan_set_bin_sort_capacity(h, 512) == _lib.MC_OK and lib.mc_plan_bin_sort_capacity(h) == 512
    assert lib.mc_plan_set_bin_sort_capacity(h, 300) == _lib.MC_ERR_INVALID
    lib.mc_plan_destroy(h)
    dense = scenarios.make_scenario(32, 32, 8, 60, seed=0)  # 480 nodes on 4 tiles: deep bins
    st, h = _create([(32, 32, dense.N, dense.pairs, dense.bending_pairs, baseline_config(), 0.01)])
    assert st == _lib.MC_OK and lib.mc_plan_bin_sort_capacity(h) == 2048
    lib.mc_plan_destroy(h)


def test_plan_limits(lib):
    """Sort keys hold 24-bit contribution indices: N * K^2 >= 2^24 IB contributions are
    refused (synthetic pairs double them); a lattice more than 7x the domain grid is refused."""
    import dataclasses
    N = 1 << 20
    empty = np.zeros((0, 2), np.int32)
    st, _ = _create([(4096, 4096, N, empty, empty, baseline_config(), 0.01)])
    assert st == _lib.MC_ERR_UNSUPPORTED and b"24-bit" in lib.mc_last_error()
    st, h = _create([(4096, 4096, N // 2 - 1, empty, empty, baseline_config(), 0.01)])
    assert st == _lib.MC_OK
    lib.mc_plan_destroy(h)
    st, _ = _create([(4096, 4096, N // 2, empty, empty, baseline_config(synthetic_node_width=1.0), 0.01)])
    assert st == _lib.MC_ERR_UNSUPPORTED
    from microcosmos_b200.engine import mc_config
    dims = _lib.McDims(32, 32, 0, 0, 0, 32 * 8, 32)
    cfg = (_lib.McConfig * 1)(mc_config(baseline_config()))
    h = ctypes.c_void_p()
    dt = (ctypes.c_float * 1)(0.01)
    nul = (_lib.c_int_p * 1)()
    assert lib.mc_plan_create(1, ctypes.byref(dims), cfg, dt, nul, nul, ctypes.byref(h)) == _lib.MC_ERR_INVALID
    dims = _lib.McDims(32, 32, 0, 0, 0, 64, 96)
    assert lib.mc_plan_create(1, ctypes.byref(dims), cfg, dt, nul, nul, ctypes.byref(h)) == _lib.MC_OK
    lib.mc_plan_destroy(h)


def test_env_and_render_entry_points_validate_on_the_host(lib):
    """The gym and frame entry points reject bad tables / sizes before touching a device."""
    env = (_lib.McEnv * 1)()
    dummy = ctypes.c_void_p(256)
    assert lib.mc_env_table_bytes(3) == 3 * ctypes.sizeof(_lib.McEnv)
    assert lib.mc_env_table_upload(env, 0, dummy, None) == _lib.MC_ERR_INVALID
    assert lib.mc_env_table_upload(env, 1, dummy, None) == _lib.MC_ERR_INVALID  # N = 0
    env[0].N, env[0].E, env[0].B, env[0].H, env[0].W = 4, 3, 2, 16, 16
    assert lib.mc_env_table_upload(env, 1, dummy, None) == _lib.MC_ERR_INVALID  # null buffers
    assert b"null" in lib.mc_last_error()
    assert lib.mc_env_act(None, 1, None) == _lib.MC_ERR_INVALID
    assert lib.mc_env_observe(None, 1, 1, None) == _lib.MC_ERR_INVALID
    assert lib.mc_render_scratch_bytes(2, 8, 10) == 2 * 8 * 10 * 4
    assert lib.mc_render_frames(None, None, None, None, 0, 1, 8, 8, 16, 1, 0, None, None, None) == _lib.MC_ERR_INVALID
    assert lib.mc_render_frames(None, None, None, dummy, 1, 4, 8, 8, 16, 1, 0, None, dummy, None) == _lib.MC_ERR_INVALID
    assert lib.mc_render_frames(None, None, None, dummy, 1, 0, 8, 100, 1, 0, 0, None, dummy, None) == _lib.MC_ERR_INVALID
