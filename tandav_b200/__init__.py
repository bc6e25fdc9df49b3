"""tandav_b200 -- B200-native (sm_100a) gravity hot path of the Tandav N-body code.

The product is the CUDA library ``libtandav_gpu.so`` behind the C ABI in
``include/tandav_gpu.h``. This package loads it (``lib()``) and offers a thin
Python view of the same entry points (``gravity.GravityContext``) used by the
tests and by bench.py. There is no CPU fallback: without the built library or
without a CUDA device the calls raise.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libtandav_gpu.so"

_lib = None

# every exported entry point of include/tandav_gpu.h
EXPORTS = (
    "tvg_init", "tvg_finalize", "tvg_last_error", "tvg_version", "tvg_upload", "tvg_download",
    "tvg_set_domain", "tvg_peano_keys", "tvg_sort_particles", "tvg_reverse_keys",
    "tvg_top_nodes", "tvg_set_domain_decomposition", "tvg_decomposition_rounds", "tvg_tree_build", "tvg_download_tree", "tvg_ewald_init",
    "tvg_download_ewald_table", "tvg_upload_ewald_table", "tvg_walk", "tvg_save_last_accel", "tvg_zero_accel",
    "tvg_force_step", "tvg_force_step_host", "tvg_phase_times", "tvg_walk_counters", "tvg_walk_quad_interactions", "tvg_set_active", "tvg_timer",
    "tvg_launch_count", "tvg_host_alloc", "tvg_host_free",
    "tvg_host_register", "tvg_host_unregister", "tvg_fp32_peak",
    "tvg_sort_keys_noalloc", "tvg_forcetest", "tvg_set_opening",
    "tvg_set_ewald_opening", "tvg_set_walk_limit", "tvg_timeline_init", "tvg_download_kick_drift_table",
    "tvg_kick_drift_factors", "tvg_set_new_timesteps", "tvg_kick_first_halfstep",
    "tvg_kick_second_halfstep", "tvg_drift_to_sync_point", "tvg_timeline_get", "tvg_timeline_set",
    "tvg_rung_histogram", "tvg_compute_acceleration", "tvg_step_graph", "tvg_step_graph_reset",
    "tvg_ewald_mlp_train",
    "tvg_ewald_mlp_weights", "tvg_ewald_mlp_grad", "tvg_ewald_mlp_eval", "tvg_ewald_mlp_validate",
    "tvg_autotune", "tvg_write_snapshot", "tvg_write_snapshot_host",
    "tvg_read_snapshot_header", "tvg_read_snapshot_host", "tvg_read_snapshot",
    "tvg_find_domain", "tvg_time_for_domain_update",
)


def lib() -> C.CDLL:
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python tandav_b200/build.py`")
        _lib = C.CDLL(str(LIB_PATH))
        _lib.tvg_last_error.restype = C.c_char_p
        _lib.tvg_version.restype = C.c_char_p
    return _lib
