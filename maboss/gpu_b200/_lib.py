"""ctypes declarations of the C ABI (include/maboss_b200.h) and the in-tree build."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libmaboss_b200.so")
CSRC = os.path.join(PKG_DIR, "csrc")

_lib = None


class EngineError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[status {status}] {message}")
        self.status = status


def build(jobs: int = 8) -> str:
    """Build libmaboss_b200.so and the MaBoSS.GPU front-end in place."""
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", CSRC], check=True)
    return LIB_PATH


def _declare(L: C.CDLL) -> None:
    vp, i32, u64, i64, f32, sz = C.c_void_p, C.c_int, C.c_ulonglong, C.c_longlong, C.c_float, C.c_size_t
    P = C.POINTER
    sigs = {
        "mb_version": (C.c_char_p, []),
        "mb_last_error": (C.c_char_p, []),
        "mb_model_parse_files": (i32, [C.c_char_p, C.c_char_p, P(vp)]),
        "mb_model_parse_text": (i32, [C.c_char_p, C.c_char_p, P(vp)]),
        "mb_model_free": (i32, [vp]),
        "mb_model_num_nodes": (i32, [vp, P(i32)]),
        "mb_model_node_name": (i32, [vp, i32, C.c_char_p, sz, P(sz)]),
        "mb_model_node_info": (i32, [vp, i32, P(f32), P(i32)]),
        "mb_model_set_istate": (i32, [vp, i32, f32]),
        "mb_model_get_constant": (i32, [vp, C.c_char_p, P(f32)]),
        "mb_model_set_constant": (i32, [vp, C.c_char_p, f32]),
        "mb_model_get_variable": (i32, [vp, C.c_char_p, P(f32)]),
        "mb_model_set_variable": (i32, [vp, C.c_char_p, f32]),
        "mb_model_num_variables": (i32, [vp, P(i32)]),
        "mb_model_variable_name": (i32, [vp, i32, C.c_char_p, sz, P(sz)]),
        "mb_model_num_constants": (i32, [vp, P(i32)]),
        "mb_model_constant_name": (i32, [vp, i32, C.c_char_p, sz, P(sz)]),
        "mb_model_generate_code": (i32, [vp, C.c_char_p, sz, P(sz)]),
        "mb_device_malloc": (i32, [vp, sz, P(vp)]),
        "mb_device_free": (i32, [vp, vp]),
        "mb_memcpy": (i32, [vp, vp, vp, vp, sz]),
        "mb_memset_async": (i32, [vp, vp, vp, i32, sz]),
        "mb_synchronize": (i32, [vp]),
        "mb_module_context": (i32, [vp, P(vp)]),
        "mb_stats_create_sections": (i32, [vp, f32, f32, i32, P(i32), i32, i64, C.c_uint, P(vp)]),
        "mb_partition_scratch_size": (sz, [i32]),
        "mb_launch_partition": (i32, [vp, vp, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
        "mb_run_module": (i32, [vp, vp, vp, P(vp)]),
        "mb_result_format": (i32, [vp, i32, i32, P(C.c_char_p), i32, C.c_char_p, sz, P(sz)]),
        "mb_result_create": (i32, [vp, P(vp)]),
        "mb_result_sparse_size": (i32, [vp, P(i64), P(i64), P(C.c_uint)]),
        "mb_result_windows_sparse": (i32, [vp, P(i32)]),
        "mb_result_write_final_csv": (i32, [vp, vp, C.c_char_p]),
        "mb_model_apply_cfg_overrides": (i32, [vp]),
        "mb_result_sparse_windows": (i32, [vp, vp, vp, vp, vp]),
        "mb_result_sparse_final": (i32, [vp, vp, vp]),
        "mb_batch_set_options": (i32, [vp, i32, i32]),
        "mb_batch_set_specialize": (i32, [vp, i32]),
        "mb_autotune": (i32, [vp, vp, P(f32), P(i32), P(f32), i32, P(i32)]),
        "mb_batch_info": (i32, [vp, P(i32), P(i32), P(C.c_uint), P(C.c_uint), P(i32)]),
        "mb_batch_tuning": (i32, [vp, i32, P(i32), P(i32), P(i32), P(f32)]),
        "mb_result_info": (i32, [vp, P(i64), P(i32), P(f32), P(f32), vp]),
        "mb_result_merge": (i32, [P(vp), i32, P(vp)]),
        "mb_context_create": (i32, [i32, P(vp)]),
        "mb_context_free": (i32, [vp]),
        "mb_context_stream": (i32, [vp, P(vp)]),
        "mb_context_sm_count": (i32, [vp, P(i32)]),
        "mb_module_compile": (i32, [vp, C.c_char_p, P(vp)]),
        "mb_module_compile_model": (i32, [vp, vp, P(vp)]),
        "mb_module_free": (i32, [vp]),
        "mb_jit_check": (i32, [C.c_char_p, P(sz), C.c_char_p, sz]),
        "mb_module_state_size": (i32, [vp, P(i32), P(i32)]),
        "mb_module_log": (i32, [vp, C.c_char_p, sz, P(sz)]),
        "mb_rand_state_size": (sz, []),
        "mb_launch_initialize_random": (i32, [vp, vp, i32, u64, u64, vp]),
        "mb_launch_initialize_initial_state": (i32, [vp, vp, i32, i32, vp, vp, vp, vp]),
        "mb_launch_simulate": (i32, [vp, vp, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp]),
        "mb_stats_create": (i32, [vp, f32, f32, i32, P(i32), i32, i64, P(vp)]),
        "mb_stats_free": (i32, [vp]),
        "mb_launch_window_average_stats": (i32, [vp, vp, i32, i32, i32, vp, vp, vp]),
        "mb_launch_final_states_stats": (i32, [vp, vp, i32, i32, vp, vp]),
        "mb_launch_fixed_states_stats": (i32, [vp, vp, i32, i32, vp, vp]),
        "mb_stats_finalize": (i32, [vp, i64, P(vp)]),
        "mb_run_config_default": (i32, [vp, vp]),
        "mb_run": (i32, [vp, vp, P(vp)]),
        "mb_runner_create": (i32, [vp, vp, P(vp)]),
        "mb_runner_launch": (i32, [vp, vp]),
        "mb_runner_result": (i32, [vp, vp, P(vp)]),
        "mb_runner_kernel_launches": (i32, [vp, P(C.c_uint)]),
        "mb_runner_free": (i32, [vp]),
        "mb_batch_create": (i32, [vp, P(vp)]),
        "mb_batch_free": (i32, [vp]),
        "mb_batch_add_model": (i32, [vp, vp, P(i32)]),
        "mb_batch_add_variant": (i32, [vp, i32, P(C.c_char_p), P(f32), i32, i64, u64, P(i32)]),
        "mb_batch_run": (i32, [vp, u64, P(f32)]),
        "mb_batch_result": (i32, [vp, i32, P(vp)]),
        "mb_batch_add_variant_grad": (i32, [vp, i32, P(C.c_char_p), P(f32), i32, i64, u64, P(C.c_char_p), i32,
                                            P(i32)]),
        "mb_batch_add_mutant": (i32, [vp, i32, P(C.c_char_p), P(f32), i32, i64, u64, P(C.c_char_p), P(i32), i32,
                                      P(i32)]),
        "mb_batch_set_variables": (i32, [vp, i32, P(C.c_char_p), P(f32), i32]),
        "mb_batch_run_gradient": (i32, [vp, u64, P(C.c_void_p), i32, P(f32)]),
        "mb_batch_gradient": (i32, [vp, i32, P(C.c_double), i32, P(i32)]),
        "mb_gradient": (i32, [vp, vp, P(C.c_char_p), P(f32), i32, i64, u64, vp, vp, P(vp)]),
        "mb_fixed_states_noalloc": (i32, [vp, i32, i32, i32, vp, vp, vp, vp, i32, P(i32)]),
        "mb_result_free": (i32, [vp]),
        "mb_result_dims": (i32, [vp, P(i32), P(i32), P(i32), P(i32), P(i32)]),
        "mb_result_transitions": (i32, [vp, P(u64)]),
        "mb_result_timing": (i32, [vp, P(f32), P(f32), P(i32)]),
        "mb_result_window_probs": (i32, [vp, vp]),
        "mb_result_window_entropy": (i32, [vp, vp]),
        "mb_result_window_raw": (i32, [vp, vp, vp, vp, P(i32), P(i32)]),
        "mb_result_final_counts": (i32, [vp, vp]),
        "mb_result_num_fixed": (i32, [vp, P(i32), P(C.c_uint)]),
        "mb_result_fixed": (i32, [vp, i32, vp, P(C.c_uint)]),
        "mb_result_write_csv": (i32, [vp, vp, C.c_char_p]),
        "mb_result_visualize": (i32, [vp, vp, C.c_char_p, sz, P(sz)]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def lib() -> C.CDLL:
    """The loaded engine library. Raises if it has not been built: there is no fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing; build it with `make -C {CSRC}` or maboss.gpu_b200.build()")
        L = C.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != 0:
        raise EngineError(status, lib().mb_last_error().decode(errors="replace"))


def read_string(fn, *args) -> str:
    n = C.c_size_t()
    check(fn(*args, None, 0, C.byref(n)))
    buf = C.create_string_buffer(n.value + 1)
    check(fn(*args, buf, n.value + 1, C.byref(n)))
    return buf.value.decode()
