"""ctypes declarations of include/pr_gpu.h (libgapbs_pr.so)."""
from __future__ import annotations

from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_size_t, c_void_p

P = c_void_p

PR_GPU_OK = 0
PR_GPU_EINVAL = -1
PR_GPU_ECUDA = -2
PR_GPU_ENOMEM = -3
PR_GPU_ENOGRAPH = -4
PR_GPU_EGRAPH = -5
PR_GPU_ERANGE = -6

PR_GPU_SWEEP_AUTO = 0
PR_GPU_SWEEP_GATHER = 1
PR_GPU_SWEEP_BLOCKED = 2

# Every symbol include/pr_gpu.h declares.
SYMBOLS = (
    "pr_gpu_create", "pr_gpu_upload", "pr_gpu_upload_sg", "pr_gpu_generate", "pr_gpu_download_csr",
    "pr_gpu_run", "pr_gpu_run_device", "pr_gpu_bfs", "pr_gpu_bfs_device",
    "pr_gpu_connected_components",
    "pr_gpu_connected_components_device",
    "pr_gpu_adjoint", "pr_gpu_adjoint_device", "pr_gpu_set_stream",
    "pr_gpu_set_batch_tile", "pr_gpu_get_batch_tile", "pr_gpu_set_sweep_layout",
    "pr_gpu_sweep_layout_info", "pr_gpu_sweep_kernel_times", "pr_gpu_last_timing",
    "pr_gpu_set_edge_weights_device", "pr_gpu_set_batch_schedule", "pr_gpu_get_batch_schedule",
    "pr_gpu_verify", "pr_gpu_graph_info", "pr_gpu_measure_gather_rate",
    "pr_gpu_measure_row_gather_rate", "pr_gpu_run_noalloc", "pr_gpu_destroy", "pr_gpu_last_error",
)


def declare(lib):
    lib.pr_gpu_create.argtypes = [POINTER(P), c_int]
    lib.pr_gpu_create.restype = c_int
    lib.pr_gpu_upload.argtypes = [P, c_int64, c_int64, P, P, P, P, P]
    lib.pr_gpu_upload.restype = c_int
    lib.pr_gpu_bfs.argtypes = [P, c_int64, P, P, c_int, POINTER(c_int)]
    lib.pr_gpu_bfs.restype = c_int
    lib.pr_gpu_bfs_device.argtypes = [P, c_int64, P, P, c_int, POINTER(c_int)]
    lib.pr_gpu_bfs_device.restype = c_int
    lib.pr_gpu_connected_components.argtypes = [P, P]
    lib.pr_gpu_connected_components.restype = c_int
    lib.pr_gpu_connected_components_device.argtypes = [P, P]
    lib.pr_gpu_connected_components_device.restype = c_int
    lib.pr_gpu_upload_sg.argtypes = [P, c_char_p]
    lib.pr_gpu_upload_sg.restype = c_int
    lib.pr_gpu_generate.argtypes = [P, c_int, c_int, c_int, P, POINTER(c_int64), POINTER(c_int64)]
    lib.pr_gpu_generate.restype = c_int
    lib.pr_gpu_download_csr.argtypes = [P, P, P]
    lib.pr_gpu_download_csr.restype = c_int
    lib.pr_gpu_run.argtypes = [P, c_int, c_double, c_float, c_int, P, P, P, P]
    lib.pr_gpu_run.restype = c_int
    lib.pr_gpu_run_device.argtypes = [P, c_int, c_double, c_float, c_int, P, P, P, P]
    lib.pr_gpu_run_device.restype = c_int
    lib.pr_gpu_adjoint.argtypes = [P, c_int, c_double, c_float, P, P, P, P, P]
    lib.pr_gpu_adjoint.restype = c_int
    lib.pr_gpu_adjoint_device.argtypes = [P, c_int, c_double, c_float, P, P, P, P, P]
    lib.pr_gpu_adjoint_device.restype = c_int
    lib.pr_gpu_set_batch_tile.argtypes = [P, c_int]
    lib.pr_gpu_set_batch_tile.restype = c_int
    lib.pr_gpu_get_batch_tile.argtypes = [P, POINTER(c_int)]
    lib.pr_gpu_get_batch_tile.restype = c_int
    lib.pr_gpu_set_sweep_layout.argtypes = [P, c_int, c_int, c_int]
    lib.pr_gpu_set_sweep_layout.restype = c_int
    lib.pr_gpu_sweep_layout_info.argtypes = [P, POINTER(c_int), POINTER(c_int), POINTER(c_int),
                                             POINTER(c_int64), POINTER(c_int64), POINTER(c_int64),
                                             POINTER(c_int)]
    lib.pr_gpu_sweep_layout_info.restype = c_int
    lib.pr_gpu_sweep_kernel_times.argtypes = [P, c_int, c_double, POINTER(c_double), c_int,
                                              POINTER(c_int), POINTER(c_int32)]
    lib.pr_gpu_sweep_kernel_times.restype = c_int
    lib.pr_gpu_verify.argtypes = [P, P, c_float, POINTER(c_double)]
    lib.pr_gpu_verify.restype = c_int
    lib.pr_gpu_set_batch_schedule.argtypes = [P, c_int, c_int]
    lib.pr_gpu_set_batch_schedule.restype = c_int
    lib.pr_gpu_get_batch_schedule.argtypes = [P, POINTER(c_int), POINTER(c_int), POINTER(c_int)]
    lib.pr_gpu_get_batch_schedule.restype = c_int
    lib.pr_gpu_set_edge_weights_device.argtypes = [P, c_void_p]
    lib.pr_gpu_set_edge_weights_device.restype = c_int
    lib.pr_gpu_set_stream.argtypes = [P, P]
    lib.pr_gpu_set_stream.restype = c_int
    lib.pr_gpu_last_timing.argtypes = [P, POINTER(c_double), POINTER(c_double), POINTER(c_int64)]
    lib.pr_gpu_last_timing.restype = c_int
    lib.pr_gpu_graph_info.argtypes = [P, POINTER(c_int64), POINTER(c_int64), POINTER(c_int64),
                                      POINTER(c_int64), c_int]
    lib.pr_gpu_graph_info.restype = c_int
    lib.pr_gpu_measure_gather_rate.argtypes = [c_int, c_int64, POINTER(c_double)]
    lib.pr_gpu_measure_gather_rate.restype = c_int
    lib.pr_gpu_measure_row_gather_rate.argtypes = [c_int, c_int64, c_int, POINTER(c_double)]
    lib.pr_gpu_measure_row_gather_rate.restype = c_int
    lib.pr_gpu_run_noalloc.argtypes = [c_int, c_int64, c_int64, P, P, P, c_int, c_double, c_float,
                                       P, P, P, P, c_char_p, c_size_t]
    lib.pr_gpu_run_noalloc.restype = c_int
    lib.pr_gpu_destroy.argtypes = [P]
    lib.pr_gpu_destroy.restype = None
    lib.pr_gpu_last_error.argtypes = [P]
    lib.pr_gpu_last_error.restype = c_char_p
