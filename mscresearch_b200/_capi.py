"""ctypes declarations for the engine's C ABI (include/maxflow_b200.h).

The shared library is built in-tree (mscresearch_b200/libmfb200.so) by
``mscresearch_b200.build.build()``.  There is no fallback: if the library is
missing or cannot be loaded, importing this module raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# MF_LIB_VARIANT=chk selects the self-check build (traces + index checks)
LIB_PATH = os.path.join(_HERE, "libmfb200_chk.so" if os.environ.get("MF_LIB_VARIANT") == "chk"
                        else "libmfb200.so")

i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
u8p = C.POINTER(C.c_uint8)
f64p = C.POINTER(C.c_double)


class MfOpts(C.Structure):
    _fields_ = [
        ("kernel_cycles", C.c_int),
        ("gr_freq", C.c_int),
        ("gr_work_alpha", C.c_double),
        ("prune_mode", C.c_int),
        ("path_push_switch", C.c_int),
        ("max_path_len", C.c_int),
        ("use_path_push", C.c_int),
        ("use_hot_sweep", C.c_int),
        ("hot_regions", C.c_int),
        ("use_rm", C.c_int),
        ("rm_freq", C.c_int),
        ("h_cut", C.c_int),
        ("stagnate_rounds", C.c_int),
        ("force_rm", C.c_int),
        ("force_path_push", C.c_int),
        ("iter_max", C.c_longlong),
        ("group_ctas", C.c_int),
        ("threads", C.c_int),
        ("certify", C.c_int),
        ("verbose", C.c_int),
        ("use_kept_cache", C.c_int),
        ("schedule", C.c_int),
        ("relabel_early_stop", C.c_int),
        ("local_relabel", C.c_int),
    ]


class MfStats(C.Structure):
    _fields_ = [
        ("flow", C.c_longlong),
        ("status", C.c_int),
        ("mask_vertices", C.c_int),
        ("mask_arcs", C.c_longlong),
        ("rounds", C.c_longlong),
        ("global_relabels", C.c_longlong),
        ("arcs_examined", C.c_longlong),
        ("vertices_examined", C.c_longlong),
        ("pushes", C.c_longlong),
        ("rm_fixed", C.c_longlong),
        ("path_push_rounds", C.c_longlong),
        ("hot_sweeps", C.c_longlong),
        ("deficit_phases", C.c_longlong),
        ("cut_capacity", C.c_longlong),
        ("time_ms", C.c_double),
        ("service_ms", C.c_double),
        ("finish_ms", C.c_double),
        ("prune_ms", C.c_double),
        ("relabel_ms", C.c_double),
        ("rounds_ms", C.c_double),
        ("relabel_arcs", C.c_longlong),
        ("hub_arcs", C.c_longlong),
        ("hub_passes", C.c_longlong),
        ("hub_relabels", C.c_longlong),
        ("levels", C.c_longlong),
        ("levels_bottom_up", C.c_longlong),
        ("levels_solo", C.c_longlong),
        ("local_relabels", C.c_longlong),
    ]


# name -> (restype, argtypes); every symbol the header declares.
SIGNATURES = {
    "mf_opts_default": (None, [C.POINTER(MfOpts)]),
    "mf_last_error_string": (C.c_char_p, []),
    "mf_version": (C.c_char_p, []),
    "mf_graph_create_from_edges": (C.c_int, [C.c_int, C.c_longlong, i32p, i32p, i64p, C.c_int, C.POINTER(C.c_void_p)]),
    "mf_graph_create_from_device_edges": (C.c_int, [C.c_int, C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "mf_graph_load_file": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]),
    "mf_graph_save": (C.c_int, [C.c_void_p, C.c_char_p]),
    "mf_graph_load_binary": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "mf_graph_destroy": (C.c_int, [C.c_void_p]),
    "mf_graph_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_int)]),
    "mf_graph_export": (C.c_int, [C.c_void_p, i32p, i32p, i64p, i32p, i32p, i32p, f64p, i32p]),
    "mf_graph_repartition": (C.c_int, [C.c_void_p, C.c_int]),
    "mf_graph_scc": (C.c_int, [C.c_void_p, i32p, C.POINTER(C.c_int32), C.POINTER(C.c_longlong)]),
    "mf_graph_scc_contracted": (C.c_int, [C.c_void_p, i32p, i32p, i64p, C.c_longlong]),
    "mf_solve": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(MfOpts), i64p, C.POINTER(MfStats)]),
    "mf_solve_batch": (C.c_int, [C.c_void_p, C.c_int, i32p, i32p, C.POINTER(MfOpts), i64p, C.POINTER(MfStats)]),
    "mf_solve_batch_override": (C.c_int, [C.c_void_p, C.c_int, i32p, i32p, C.c_longlong, i32p, i32p, i64p, C.POINTER(MfOpts), i64p, C.POINTER(MfStats)]),
    "mf_last_device_ms": (C.c_double, [C.c_void_p]),
    "mf_debug_prune_mask": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(MfOpts), u8p, C.POINTER(C.c_int)]),
    "mf_debug_initial_heights": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(MfOpts), i32p]),
    "mf_solve_residual": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(MfOpts), i64p, i64p, C.POINTER(MfStats)]),
    "mf_certify": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(MfOpts), i64p, C.POINTER(MfStats)]),
    "mf_debug_alloc_fail_after": (C.c_int, [C.c_longlong]),
    "mf_debug_alloc_live": (C.c_int, [C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "mf_solve_csr_noalloc": (C.c_int, [C.c_int, C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.POINTER(MfOpts), C.c_void_p, i64p, C.POINTER(MfStats)]),
    "mf_update_caps": (C.c_int, [C.c_void_p, C.c_int, i32p, i32p, i64p, C.POINTER(C.c_int)]),
    "mf_session_create": (C.c_int, [C.c_void_p, C.c_int, i32p, i32p, C.POINTER(MfOpts), C.POINTER(C.c_void_p)]),
    "mf_session_solve": (C.c_int, [C.c_void_p, i64p, C.POINTER(MfStats)]),
    "mf_session_update": (C.c_int, [C.c_void_p, C.c_int, i32p, i32p, i64p, i64p, C.POINTER(MfStats)]),
    "mf_session_destroy": (C.c_int, [C.c_void_p]),
    "mf_server_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(MfOpts), C.c_int, C.POINTER(C.c_void_p)]),
    "mf_server_slots": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "mf_server_submit": (C.c_int, [C.c_void_p, C.c_int, C.c_int32, C.c_int32, C.POINTER(C.c_longlong)]),
    "mf_server_update": (C.c_int, [C.c_void_p, C.c_int, C.c_int, i32p, i32p, i64p, C.POINTER(C.c_longlong)]),
    "mf_server_poll": (C.c_int, [C.c_void_p, C.c_longlong, C.POINTER(C.c_int), i64p, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "mf_server_drain": (C.c_int, [C.c_void_p]),
    "mf_server_destroy": (C.c_int, [C.c_void_p]),
    "mf_autotune": (C.c_int, [C.c_void_p, C.c_int, i32p, i32p, C.POINTER(MfOpts), C.POINTER(MfOpts), C.POINTER(C.c_int)]),
    "mf_gen_uniform": (C.c_int, [C.c_int, C.c_longlong, C.c_longlong, C.c_longlong, C.c_ulonglong, i32p, i32p, i64p]),
    "mf_gen_rmat": (C.c_int, [C.c_int, C.c_longlong, C.c_double, C.c_double, C.c_double, C.c_longlong, C.c_longlong, C.c_ulonglong, i32p, i32p, i64p, C.POINTER(C.c_longlong)]),
    "mf_gen_grid": (C.c_int, [C.c_int, C.c_int, C.c_ulonglong, i32p, i32p, i64p, C.POINTER(C.c_longlong)]),
    "mf_gen_queries_hub": (C.c_int, [C.c_int, C.c_longlong, i32p, i32p, C.c_int, C.c_int, C.c_ulonglong, i32p, i32p]),
    "mf_write_graph_txt": (C.c_int, [C.c_char_p, C.c_int, C.c_longlong, i32p, i32p, i64p]),
    "mf_write_test_txt": (C.c_int, [C.c_char_p, C.c_int, i32p, i32p]),
    "mf_read_graph_txt": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong), i32p, i32p, i64p, C.c_longlong]),
    "mf_graph_txt_header": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
}


def load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "mscresearch_b200: %s is missing; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` or `make -C mscresearch_b200/csrc`"
            % LIB_PATH)
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError = the library lacks a declared entry point
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load()
