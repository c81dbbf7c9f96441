"""ctypes declarations of include/dmolp_b200.h."""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_uint64, c_void_p

DMOLP_OK = 0
DMOLP_ERR_ARG = 1
DMOLP_ERR_CUDA = 2
DMOLP_ERR_NOMEM = 3
DMOLP_ERR_STATE = 4
DMOLP_ERR_BAD_LABELS = 5
DMOLP_ERR_NO_GPU = 6
MODE_REF = 0
MODE_FIXED = 1
CAP_REF = 0
CAP_FULL = 1
MAX_K = 1024

# every function the header declares (checked by the CPU test suite against the built library)
EXPORTS = [
    "dmolp_last_error", "dmolp_create", "dmolp_destroy", "dmolp_graph_upload", "dmolp_phase1", "dmolp_lp_run",
    "dmolp_metrics", "dmolp_labels_get", "dmolp_labels_set", "dmolp_window_select", "dmolp_lp_apply",
    "dmolp_lp_history", "dmolp_device_labels", "dmolp_kernel_launches", "dmolp_adjtext_load",
    "dmolp_adjtext_error", "dmolp_host_graph_nv", "dmolp_host_graph_narcs", "dmolp_host_graph_offsets",
    "dmolp_host_graph_indices", "dmolp_host_graph_raw_degree", "dmolp_host_graph_free", "dmolp_stream",
    "dmolp_labels_save", "dmolp_labels_restore", "dmolp_set_profiling", "dmolp_kernel_profile",
    "dmolp_set_wait_limit",
    "dmolp_set_symmetry_test",
    "dmolp_graph_symmetric",
    "dmolp_find_seeds", "dmolp_expand_partitions", "dmolp_current_device", "dmolp_device_code_version", "dmolp_metrics_noalloc",
    "dmolp_batch_create", "dmolp_batch_destroy", "dmolp_batch_upload", "dmolp_batch_labels_set",
    "dmolp_batch_labels_get", "dmolp_batch_device_labels", "dmolp_batch_stream", "dmolp_batch_lp_run",
    "dmolp_batch_autotune", "dmolp_batch_counts", "dmolp_batch_labels_save", "dmolp_batch_labels_restore",
    "dmolp_mpnn_num_params", "dmolp_mpnn_create", "dmolp_mpnn_destroy", "dmolp_mpnn_set_wait_limit", "dmolp_mpnn_set_params",
    "dmolp_mpnn_get_params", "dmolp_mpnn_features", "dmolp_mpnn_set_features", "dmolp_mpnn_forward",
    "dmolp_mpnn_prepare_training", "dmolp_mpnn_backward", "dmolp_mpnn_train_step", "dmolp_mpnn_decode",
    "dmolp_batch_propose", "dmolp_mpnn_gate", "dmolp_mpnn_train_gate", "dmolp_batch_phase1",
    "dmolp_graph_upload_adjtext", "dmolp_graph_load_adjtext", "dmolp_graph_size", "dmolp_graph_get",
    "dmolp_graph_upload_adjtext_device", "dmolp_find_hubs_pairs", "dmolp_degree_order", "dmolp_find_hubs",
]
BATCH_MAX_K = 64


class Phase1Info(ctypes.Structure):
    _fields_ = [("initial_edge_cut", c_int64), ("initial_vertex_balance", c_double),
                ("initial_edge_balance", c_double), ("num_seeds_found", c_int32), ("rounds", c_int32),
                ("num_hubs", c_int64), ("traversed_edges", c_uint64), ("gpu_ms", c_double),
                ("hubs_ms", c_double), ("seeds_ms", c_double), ("expand_ms", c_double)]


class LpConfig(ctypes.Structure):
    _fields_ = [("mode", c_int32), ("iterations", c_int32), ("cap", c_int32), ("flags", c_int32)]


class LpResult(ctypes.Structure):
    _fields_ = [("edge_cut", c_int64), ("vertex_balance", c_double), ("edge_balance", c_double),
                ("iterations_run", c_int32), ("stop_reason", c_int32), ("traversed_edges", c_uint64),
                ("total_vertices", c_int64), ("total_edges", c_int64), ("gpu_ms", c_double)]


class LpRecord(ctypes.Structure):
    _fields_ = [("iteration", c_int32), ("window", c_int32), ("candidates", c_int32), ("changes", c_int32),
                ("boundary", c_int32), ("reserved", c_int32), ("edge_cut", c_int64), ("te_prev", c_uint64),
                ("te_cand", c_uint64), ("te_sel", c_uint64), ("te_stats", c_uint64), ("arcs_read", c_uint64),
                ("window_sum", c_uint64)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("block_threads", c_int32), ("thread_row_max", c_int32), ("blocks_per_sm", c_int32),
                ("reserved", c_int32)]


class BatchResult(ctypes.Structure):
    _fields_ = [("edge_cut", c_int64), ("traversed_edges", c_uint64), ("arcs_read", c_uint64),
                ("vertex_visits", c_uint64), ("vertex_balance", c_double), ("edge_balance", c_double), ("iterations_run", c_int32),
                ("stop_reason", c_int32), ("status", c_int32), ("changes", c_int32)]


class IngestInfo(ctypes.Structure):
    _fields_ = [("num_vertices", c_int64), ("num_arcs", c_int64), ("num_tokens", c_int64),
                ("rows_sorted_on_device", c_int64), ("read_ms", c_double), ("parse_ms", c_double),
                ("total_ms", c_double), ("kernels", c_int64), ("count_ms", c_double), ("emit_ms", c_double),
                ("setup_ms", c_double)]


class BatchP1Result(ctypes.Structure):
    _fields_ = [("num_seeds_found", c_int32), ("rounds", c_int32), ("traversed_edges", c_uint64)]


def bind(lib: ctypes.CDLL) -> ctypes.CDLL:
    vp = c_void_p
    lib.dmolp_last_error.restype = c_char_p
    lib.dmolp_last_error.argtypes = []
    lib.dmolp_current_device.argtypes = []
    lib.dmolp_device_code_version.argtypes = [c_int, POINTER(c_int)]
    lib.dmolp_create.argtypes = [c_int, POINTER(vp)]
    lib.dmolp_destroy.argtypes = [vp]
    lib.dmolp_graph_upload.argtypes = [vp, c_int64, c_int64, vp, vp, vp]
    lib.dmolp_graph_upload_adjtext.argtypes = [vp, c_char_p, c_int64, POINTER(IngestInfo)]
    lib.dmolp_graph_load_adjtext.argtypes = [vp, c_char_p, POINTER(IngestInfo)]
    lib.dmolp_graph_upload_adjtext_device.argtypes = [vp, vp, c_int64, POINTER(IngestInfo)]
    lib.dmolp_graph_size.argtypes = [vp, POINTER(c_int64), POINTER(c_int64)]
    lib.dmolp_find_hubs_pairs.argtypes = [c_int64, vp, vp, vp, POINTER(c_int64)]
    lib.dmolp_degree_order.argtypes = [c_int64, vp, vp]
    lib.dmolp_find_hubs.argtypes = [c_int64, vp, vp, POINTER(c_int64), POINTER(c_int32), POINTER(c_int32)]
    lib.dmolp_graph_get.argtypes = [vp, vp, vp, vp]
    lib.dmolp_phase1.argtypes = [vp, c_int, c_int, vp, vp, vp, POINTER(Phase1Info)]
    lib.dmolp_lp_run.argtypes = [vp, c_int, POINTER(LpConfig), POINTER(LpResult), vp, c_int]
    lib.dmolp_metrics.argtypes = [vp, c_int, POINTER(c_int64), vp, vp]
    lib.dmolp_labels_get.argtypes = [vp, vp]
    lib.dmolp_labels_set.argtypes = [vp, vp]
    lib.dmolp_window_select.argtypes = [vp, c_int, c_int, vp, vp, c_int64, vp, POINTER(c_int64)]
    lib.dmolp_lp_apply.argtypes = [vp, c_int, c_int, vp, vp, c_int64, vp, vp, POINTER(c_int64)]
    lib.dmolp_lp_history.argtypes = [vp, c_int, c_int, vp, vp]
    lib.dmolp_device_labels.argtypes = [vp, POINTER(vp)]
    lib.dmolp_kernel_launches.argtypes = [vp]
    lib.dmolp_kernel_launches.restype = c_int64
    lib.dmolp_adjtext_load.argtypes = [c_char_p, POINTER(vp)]
    lib.dmolp_adjtext_error.restype = c_char_p
    lib.dmolp_adjtext_error.argtypes = []
    for f in ("dmolp_host_graph_nv", "dmolp_host_graph_narcs"):
        getattr(lib, f).argtypes = [vp]
        getattr(lib, f).restype = c_int64
    for f in ("dmolp_host_graph_offsets", "dmolp_host_graph_indices", "dmolp_host_graph_raw_degree"):
        getattr(lib, f).argtypes = [vp]
        getattr(lib, f).restype = vp
    lib.dmolp_host_graph_free.argtypes = [vp]
    lib.dmolp_host_graph_free.restype = None
    lib.dmolp_stream.argtypes = [vp]
    lib.dmolp_stream.restype = vp
    lib.dmolp_labels_save.argtypes = [vp]
    lib.dmolp_labels_restore.argtypes = [vp]
    lib.dmolp_set_profiling.argtypes = [vp, c_int]
    lib.dmolp_set_wait_limit.argtypes = [vp, ctypes.c_uint32]
    lib.dmolp_set_symmetry_test.argtypes = [vp, ctypes.c_int]
    lib.dmolp_graph_symmetric.argtypes = [vp, POINTER(c_int)]
    lib.dmolp_find_seeds.argtypes = [vp, c_int, c_int32, vp, c_int64, vp, POINTER(c_int32)]
    lib.dmolp_expand_partitions.argtypes = [vp, c_int, c_int, vp, c_int32, POINTER(c_int32)]
    lib.dmolp_metrics_noalloc.argtypes = [c_int, c_int64, vp, vp, vp, c_int, vp, POINTER(c_int64), vp, vp]
    lib.dmolp_kernel_profile.argtypes = [vp, c_int, POINTER(c_double), POINTER(c_int64), POINTER(c_double)]
    lib.dmolp_batch_create.argtypes = [c_int, POINTER(vp)]
    lib.dmolp_batch_destroy.argtypes = [vp]
    lib.dmolp_batch_upload.argtypes = [vp, c_int32, vp, vp, vp, vp]
    lib.dmolp_batch_labels_set.argtypes = [vp, vp]
    lib.dmolp_batch_labels_get.argtypes = [vp, vp]
    lib.dmolp_batch_device_labels.argtypes = [vp, POINTER(vp)]
    lib.dmolp_batch_stream.argtypes = [vp]
    lib.dmolp_batch_stream.restype = vp
    lib.dmolp_batch_lp_run.argtypes = [vp, POINTER(LpConfig), POINTER(BatchTuning), vp, POINTER(c_double)]
    lib.dmolp_batch_autotune.argtypes = [vp, POINTER(LpConfig), POINTER(BatchTuning), POINTER(c_double)]
    lib.dmolp_batch_counts.argtypes = [vp, c_int32, vp, vp]
    lib.dmolp_batch_labels_save.argtypes = [vp]
    lib.dmolp_batch_labels_restore.argtypes = [vp]
    lib.dmolp_mpnn_num_params.argtypes = []
    lib.dmolp_mpnn_num_params.restype = c_int64
    lib.dmolp_mpnn_create.argtypes = [c_int, POINTER(vp)]
    lib.dmolp_mpnn_destroy.argtypes = [vp]
    lib.dmolp_mpnn_set_wait_limit.argtypes = [vp, ctypes.c_uint32]
    lib.dmolp_mpnn_set_params.argtypes = [vp, vp]
    lib.dmolp_mpnn_get_params.argtypes = [vp, vp]
    lib.dmolp_mpnn_features.argtypes = [vp, vp, vp]
    lib.dmolp_mpnn_set_features.argtypes = [vp, vp, vp]
    lib.dmolp_mpnn_forward.argtypes = [vp, vp, vp]
    lib.dmolp_mpnn_prepare_training.argtypes = [vp, vp]
    lib.dmolp_mpnn_backward.argtypes = [vp, vp, vp, vp]
    lib.dmolp_mpnn_train_step.argtypes = [vp, vp, vp, ctypes.c_float, POINTER(c_double)]
    lib.dmolp_mpnn_decode.argtypes = [vp, vp, vp, vp]
    lib.dmolp_batch_propose.argtypes = [vp, vp, vp]
    lib.dmolp_mpnn_gate.argtypes = [vp, vp, vp]
    lib.dmolp_batch_phase1.argtypes = [vp, c_int, vp, vp, vp, POINTER(c_double)]
    lib.dmolp_mpnn_train_gate.argtypes = [vp, vp, vp, ctypes.c_float, POINTER(c_double)]
    return lib
