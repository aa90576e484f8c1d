"""ctypes binding of lib/libbp.so (include/bp.h and include/graph.h).

Nothing here computes: every call goes to the CUDA library, which fails
loudly (an exception naming the C status) when there is no GPU, when the
library is missing, or when a kernel reports an error.  There is no CPU
fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libbp.so")
MAX_STATES = 10

BP_MEM_HOST, BP_MEM_DEVICE = 0, 1
BP_SCHEDULE_NODE, BP_SCHEDULE_EDGE = 0, 1
BP_DELTA_AUTO, BP_DELTA_SERIAL_F32, BP_DELTA_F64 = 0, 1, 2
BP_SYNC_EAGER, BP_SYNC_LAZY = 0, 1
BP_GRAPH_REORDER_BY_OUT_DEGREE = 1
STATUS = {0: "BP_OK", 1: "BP_ERR_INVALID", 2: "BP_ERR_SHAPE", 3: "BP_ERR_CUDA", 4: "BP_ERR_NOMEM",
          5: "BP_ERR_NO_DEVICE", 6: "BP_ERR_GRAPH", 7: "BP_ERR_STATE", 8: "BP_ERR_TIMEOUT"}


class BPError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class GraphDesc(C.Structure):
    _fields_ = [("num_nodes", C.c_uint32), ("num_edges", C.c_uint32), ("uniform_states", C.c_uint32),
                ("node_num_states", C.c_void_p), ("edge_src", C.c_void_p), ("edge_dst", C.c_void_p),
                ("edge_joint", C.c_void_p), ("joint_row_stride", C.c_uint32),
                ("joint_edge_stride", C.c_uint64), ("dest_node_list", C.c_void_p),
                ("dest_edge_list", C.c_void_p), ("src_node_list", C.c_void_p),
                ("src_edge_list", C.c_void_p), ("memory", C.c_int32), ("flags", C.c_int32)]


class LoopyOptions(C.Structure):
    _fields_ = [("tolerance", C.c_float), ("max_iterations", C.c_uint32), ("check_every", C.c_uint32),
                ("schedule", C.c_int32), ("delta_mode", C.c_int32), ("verbose", C.c_int32),
                ("graph_chunk", C.c_uint32), ("kernel_variant", C.c_int32)]


class LoopyResult(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("executed", C.c_uint32), ("converged", C.c_int32),
                ("delta", C.c_float), ("previous_delta", C.c_float), ("delta_f64", C.c_double),
                ("elapsed_ms", C.c_float), ("serial_sums", C.c_uint32), ("serial_refines", C.c_uint32),
                ("kernel_used", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchOptions(C.Structure):
    _fields_ = [("tolerance", C.c_float), ("max_iterations", C.c_uint32), ("delta_mode", C.c_int32),
                ("block_threads", C.c_uint32), ("init_messages", C.c_int32), ("reserved", C.c_int32)]


class BatchResult(C.Structure):
    _fields_ = [("num_networks", C.c_uint32), ("converged", C.c_uint32), ("max_executed", C.c_uint32),
                ("elapsed_ms", C.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TreeResult(C.Structure):
    _fields_ = [("num_levels", C.c_uint32), ("num_waves", C.c_uint32), ("elapsed_ms", C.c_float)]


class StructGraph(C.Structure):
    """struct graph of include/graph.h (the reference's layout + bp_device)."""
    _fields_ = [("total_num_vertices", C.c_uint), ("total_num_edges", C.c_uint),
                ("current_num_vertices", C.c_uint), ("current_num_edges", C.c_uint),
                ("max_degree", C.c_uint),
                ("edges_src_index", C.POINTER(C.c_uint)), ("edges_dest_index", C.POINTER(C.c_uint)),
                ("edges_x_dim", C.POINTER(C.c_uint)), ("edges_y_dim", C.POINTER(C.c_uint)),
                ("edges_joint_probabilities", C.POINTER(C.c_float)),
                ("edges_messages", C.POINTER(C.c_float)), ("last_edges_messages", C.POINTER(C.c_float)),
                ("current_edge_messages", C.POINTER(C.POINTER(C.c_float))),
                ("previous_edge_messages", C.POINTER(C.POINTER(C.c_float))),
                ("node_states", C.POINTER(C.c_float)), ("node_num_vars", C.POINTER(C.c_uint)),
                ("src_nodes_to_edges_node_list", C.POINTER(C.c_uint)),
                ("src_nodes_to_edges_edge_list", C.POINTER(C.c_uint)),
                ("dest_nodes_to_edges_node_list", C.POINTER(C.c_uint)),
                ("dest_nodes_to_edges_edge_list", C.POINTER(C.c_uint)),
                ("levels_to_nodes", C.POINTER(C.c_uint)), ("num_levels", C.c_uint),
                ("diameter", C.c_int), ("visited", C.c_void_p), ("node_names", C.c_void_p),
                ("variable_names", C.c_void_p), ("observed_nodes", C.c_void_p),
                ("graph_name", C.c_char * 50), ("node_hash_table_created", C.c_char),
                ("node_hash_table", C.c_void_p), ("src_node_to_edge_table", C.c_void_p),
                ("dest_node_to_edge_table", C.c_void_p), ("edge_tables_created", C.c_char),
                ("bp_device", C.c_void_p)]


# every symbol include/bp.h and include/graph.h declare
BP_SYMBOLS = [
    "bp_status_string", "bp_last_error", "bp_version", "bp_graph_create", "bp_graph_destroy",
    "bp_graph_info", "bp_set_stream", "bp_synchronize", "bp_graph_device_bytes", "bp_set_beliefs",
    "bp_get_beliefs", "bp_set_messages", "bp_get_messages", "bp_set_latest_slot", "bp_get_latest_slot",
    "bp_loopy_default_options", "bp_init_messages", "bp_loopy", "bp_tree_build_levels",
    "bp_tree_set_levels", "bp_tree_start", "bp_tree_level", "bp_tree_reset_visited",
    "bp_tree_marginalize", "bp_tree", "bp_set_visited", "bp_get_visited", "bp_set_sync_mode",
    "bp_sync_host", "bp_graph_of", "bp_loopy_noalloc", "bp_release_cached_memory", "bp_reserve_cached_memory", "bp_batch_create", "bp_batch_destroy",
    "bp_batch_layout", "bp_batch_set_beliefs", "bp_batch_get_beliefs", "bp_batch_get_messages",
    "bp_batch_default_options", "bp_batch_autotune", "bp_batch_get_block_threads", "bp_batch_get_groups", "bp_batch_loopy",
    "bp_batch_network_results", "bp_unrolled_create", "bp_unrolled_destroy", "bp_unrolled_set_stream",
    "bp_unrolled_forward", "bp_unrolled_backward",
]
GRAPH_SYMBOLS = [
    "create_graph", "graph_add_node", "graph_add_and_set_node_state", "graph_set_node_state",
    "graph_add_edge", "set_up_src_nodes_to_edges", "set_up_dest_nodes_to_edges", "init_levels_to_nodes",
    "calculate_diameter", "initialize_node", "node_set_state", "init_edge", "send_message",
    "fill_in_node_table", "find_node_by_name", "fill_in_node_hash_table", "fill_in_leaf_nodes_in_index",
    "visit_node", "graph_vertex_count", "graph_edge_count", "graph_destroy",
    "propagate_using_levels_start", "propagate_using_levels", "reset_visited", "init_previous_edge",
    "loopy_propagate_one_iteration", "loopy_propagate_until", "loopy_propagate_until_edge",
    "loopy_progagate_until_acc", "loopy_progagate_until_edge_acc", "marginalize", "print_node",
    "print_edge", "print_nodes", "print_edges", "print_src_nodes_to_edges", "print_dest_nodes_to_edges",
    "print_levels_to_nodes",
]

_lib = None


def load(path=LIB_PATH):
    """Load libbp.so (built by build.py).  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with belief-propagation_b200/build.py")
    L = C.CDLL(path)
    vp, u32, i32 = C.c_void_p, C.c_uint32, C.c_int
    sig = {
        "bp_status_string": ([i32], C.c_char_p), "bp_last_error": ([], C.c_char_p), "bp_version": ([], i32),
        "bp_graph_create": ([C.POINTER(vp), C.POINTER(GraphDesc), vp], i32),
        "bp_graph_destroy": ([vp], None),
        "bp_graph_info": ([vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)], i32),
        "bp_set_stream": ([vp, vp], i32), "bp_synchronize": ([vp], i32),
        "bp_graph_device_bytes": ([vp, C.POINTER(C.c_uint64)], i32),
        "bp_set_beliefs": ([vp, vp, u32, i32], i32), "bp_get_beliefs": ([vp, vp, u32, i32], i32),
        "bp_set_messages": ([vp, i32, vp, u32, i32], i32), "bp_get_messages": ([vp, i32, vp, u32, i32], i32),
        "bp_set_latest_slot": ([vp, i32], i32), "bp_get_latest_slot": ([vp, C.POINTER(i32)], i32),
        "bp_loopy_default_options": ([C.POINTER(LoopyOptions)], None),
        "bp_init_messages": ([vp], i32),
        "bp_loopy": ([vp, C.POINTER(LoopyOptions), C.POINTER(LoopyResult)], i32),
        "bp_tree_build_levels": ([vp, vp, C.POINTER(u32)], i32),
        "bp_tree_set_levels": ([vp, vp, u32], i32), "bp_tree_start": ([vp], i32),
        "bp_tree_level": ([vp, u32], i32), "bp_tree_reset_visited": ([vp], i32),
        "bp_tree_marginalize": ([vp], i32), "bp_tree": ([vp, C.POINTER(TreeResult)], i32),
        "bp_set_visited": ([vp, vp], i32), "bp_get_visited": ([vp, vp], i32),
        "bp_set_sync_mode": ([vp, i32], i32), "bp_sync_host": ([vp], i32),
        "bp_graph_of": ([vp, C.POINTER(vp)], i32), "bp_release_cached_memory": ([], i32), "bp_reserve_cached_memory": ([C.c_uint64], i32),
        "bp_loopy_noalloc": ([u32, u32, u32, vp, vp, vp, vp, vp, i32, i32, C.c_float, u32, vp,
                              C.POINTER(LoopyResult), C.POINTER(i32)], i32),
        "bp_batch_create": ([C.POINTER(vp), u32, C.POINTER(GraphDesc), vp], i32),
        "bp_batch_destroy": ([vp], None),
        "bp_batch_layout": ([vp, vp, vp], i32),
        "bp_batch_set_beliefs": ([vp, vp, i32], i32), "bp_batch_get_beliefs": ([vp, vp, i32], i32),
        "bp_batch_get_messages": ([vp, vp, i32], i32),
        "bp_batch_default_options": ([C.POINTER(BatchOptions)], None),
        "bp_batch_autotune": ([vp, C.POINTER(BatchOptions)], i32),
        "bp_batch_get_block_threads": ([vp, vp, vp, C.POINTER(u32)], i32),
        "bp_batch_get_groups": ([vp, vp, vp, vp, vp, C.POINTER(u32)], i32),
        "bp_batch_loopy": ([vp, C.POINTER(BatchOptions), C.POINTER(BatchResult)], i32),
        "bp_batch_network_results": ([vp, vp, vp, vp, vp], i32),
        "bp_unrolled_create": ([C.POINTER(vp), u32, u32, u32, u32, vp, vp, vp, u32, u32, vp], i32),
        "bp_unrolled_destroy": ([vp], None), "bp_unrolled_set_stream": ([vp, vp], i32),
        "bp_unrolled_forward": ([vp, vp, vp, vp], i32), "bp_unrolled_backward": ([vp, vp, vp, vp], i32),
        "bp_serial_sum_f32": ([vp, C.c_uint64, vp, i32, vp], i32),
        "bp_nll_f32": ([vp, vp, u32, u32, vp, vp, vp], i32),
        "bp_nll_grad_f32": ([vp, u32, u32, vp, vp, vp], i32),
        "bp_serial_sum_bounds": ([vp, C.c_uint64, vp, vp], i32),
        # graph.h
        "create_graph": ([C.c_uint, C.c_uint], C.POINTER(StructGraph)),
        "graph_add_node": ([vp, C.c_uint, C.c_char_p], None),
        "graph_add_and_set_node_state": ([vp, C.c_uint, C.c_char_p, vp], None),
        "graph_set_node_state": ([vp, C.c_uint, C.c_uint, vp], None),
        "graph_add_edge": ([vp, C.c_uint, C.c_uint, C.c_uint, C.c_uint, vp], None),
        "set_up_src_nodes_to_edges": ([vp], None), "set_up_dest_nodes_to_edges": ([vp], None),
        "init_levels_to_nodes": ([vp], None), "calculate_diameter": ([vp], None),
        "graph_destroy": ([vp], None), "propagate_using_levels_start": ([vp], None),
        "propagate_using_levels": ([vp, C.c_uint], None), "reset_visited": ([vp], None),
        "init_previous_edge": ([vp], None), "loopy_propagate_one_iteration": ([vp], None),
        "loopy_propagate_until": ([vp, C.c_float, C.c_uint], C.c_uint),
        "loopy_propagate_until_edge": ([vp, C.c_float, C.c_uint], C.c_uint),
        "loopy_progagate_until_acc": ([vp, C.c_float, C.c_uint], C.c_uint),
        "loopy_progagate_until_edge_acc": ([vp, C.c_float, C.c_uint], C.c_uint),
        "marginalize": ([vp], None), "find_node_by_name": ([C.c_char_p, vp], C.c_uint),
        "graph_vertex_count": ([vp], i32), "graph_edge_count": ([vp], i32),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(status):
    if status != 0:
        msg = _lib.bp_last_error().decode(errors="replace") if _lib else ""
        raise BPError(status, msg)
    return status


def ptr(a):
    """Address of a numpy array or a torch tensor (host or device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()
