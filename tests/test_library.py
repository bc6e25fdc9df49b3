"""The C ABI library: it loads, exports every entry point declared in
include/tandav_gpu.h, and fails cleanly (no crash, an error code) where no
GPU is present. No compute call is made here."""
import ctypes as C
import re
from pathlib import Path

import pytest

import tandav_b200
from tandav_b200 import gravity

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "tandav_gpu.h").read_text()
    return sorted(set(re.findall(r"\b(tvg_[a-z_0-9]+)\s*\(", text)))


def test_header_and_exports_agree():
    assert set(declared_symbols()) == set(tandav_b200.EXPORTS)


def test_library_exports_every_symbol():
    lib = tandav_b200.lib()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_version_string():
    assert b"sm_100a" in tandav_b200.lib().tvg_version()


def test_init_rejects_bad_config():
    lib = tandav_b200.lib()
    ctx = C.c_void_p()
    cfg = gravity.Config(3, 0, 0.0, 1.0, 0.01, 0.25, 0.005, 64, 0, 100)
    assert lib.tvg_init(0, C.byref(cfg), C.byref(ctx)) == 5      # TVG_E_BADINPUT
    cfg = gravity.Config(4, 1, 0.0, 1.0, 0.01, 0.25, 0.005, 64, 0, 100)
    assert lib.tvg_init(0, C.byref(cfg), C.byref(ctx)) == 5      # periodic without box


def test_init_without_gpu_reports_cuda_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = tandav_b200.lib()
    ctx = C.c_void_p()
    cfg = gravity.Config(4, 0, 0.0, 1.0, 0.01, 0.25, 0.005, 64, 0, 100)
    assert lib.tvg_init(0, C.byref(cfg), C.byref(ctx)) == 1      # TVG_E_CUDA
    with pytest.raises(gravity.TvgError):
        gravity.GravityContext(100)


def test_init_rejects_capacity_beyond_32bit_indices():
    lib = tandav_b200.lib()
    ctx = C.c_void_p()
    cfg = gravity.Config(4, 0, 0.0, 1.0, 0.01, 0.25, 0.005, 64, 0, (1 << 30) - 4095)
    assert lib.tvg_init(0, C.byref(cfg), C.byref(ctx)) == 5      # > TVG_MAX_PARTICLES


def test_host_register_rejects_null_or_empty_ranges():
    lib = tandav_b200.lib()
    buf = (C.c_char * 64)()
    assert lib.tvg_host_register(None, C.c_size_t(64)) == 5
    assert lib.tvg_host_register(buf, C.c_size_t(0)) == 5
    assert lib.tvg_host_unregister(None) == 5


def test_step_entry_points_reject_a_null_context():
    """The whole-step calls check their arguments before any CUDA call, so
    they answer TVG_E_BADINPUT without a GPU."""
    lib = tandav_b200.lib()
    p = gravity.Particles()
    i32, u32, i64 = C.c_int32, C.c_uint32, C.c_int64
    assert lib.tvg_force_step(None, i32(1), i32(0), u32(1), i32(0)) == 5
    assert lib.tvg_force_step_host(None, i64(10), C.byref(p), u32(gravity.F_POS), C.byref(p), u32(0),
                                   i32(1), i32(0), u32(1), i32(0)) == 5
    # a context is required, and so are the input and output descriptions
    fake = C.c_void_p(1)
    assert lib.tvg_force_step_host(fake, i64(10), None, u32(gravity.F_POS), C.byref(p), u32(0),
                                   i32(1), i32(0), u32(1), i32(0)) == 5
    assert lib.tvg_force_step_host(fake, i64(10), C.byref(p), u32(gravity.F_POS), None, u32(0),
                                   i32(1), i32(0), u32(1), i32(0)) == 5
    assert lib.tvg_kick_first_halfstep(None) == 5
    assert lib.tvg_kick_second_halfstep(None) == 5
    assert lib.tvg_drift_to_sync_point(None) == 5
    assert lib.tvg_set_new_timesteps(None) == 5
    assert lib.tvg_time_for_domain_update(None, C.c_double(0.1), None) == 5
