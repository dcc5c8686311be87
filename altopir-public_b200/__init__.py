"""B200 AltoPIR answer engine: Python host binding of libaltopir_gpu.so.

The package directory is ``altopir-public_b200``; it is loaded under the module name ``altopir_b200`` (see
``load()`` in ``__graft_entry__.py``).  ``engine`` mirrors the reference's Rust engine wrapper (src/engine.rs) and
``service`` its service glue (src/service.rs): parameters, the request codec and the synthetic database.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaltopir_gpu.so")

_lib = None


def lib():
    """The loaded engine library.  Raises when it has not been built: there is no fallback path."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python {os.path.join(HERE, 'build.py')}`")
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    c = ctypes
    P, S, I, U64, D = c.c_void_p, c.c_size_t, c.c_int, c.c_uint64, c.POINTER(c.c_double)
    PP = c.POINTER(c.c_void_p)
    sigs = {
        "sw_amx_init": (I, []),
        "sw_alloc_zeroed": (P, [S]),
        "sw_alloc": (P, [S]),
        "sw_free": (None, [P]),
        "sw_tile_db": (None, [P, P, S, S, S, I]),
        "sw_pack_build": (None, [P, PP, PP, P, P, S, S, S, S, U64, I]),
        "alto_engine_new": (P, [P, P, S, S, S, P, S, S, PP, S, S, U64, I, PP, P, U64, I]),
        "alto_engine_free": (None, [P]),
        "alto_request_len": (S, [P]),
        "alto_response_len": (S, [P]),
        "alto_answer": (I, [P, PP, c.POINTER(S), S, PP, c.POINTER(I), I, D]),
        "alto_last_error": (c.c_char_p, []),
        "alto_answer_device": (I, [P, P, S, S, P, S, c.POINTER(I), D]),
        "alto_last_launches": (I, [P]),
        "alto_enqueue_device": (I, [P, P, S, S, P, S, P]),
        "alto_engine_sync": (I, [P]),
        "alto_engine_stream": (P, [P]),
        "alto_kernel_times": (I, [P, c.POINTER(c.c_double), c.POINTER(c.c_longlong), I]),
        "alto_engine_set_graphs": (I, [P, I]),
        "alto_engine_set_lanes": (I, [P, I]),
        "alto_engine_fence": (I, [P]),
        "alto_engine_set_tuning": (I, [P, P, S]),
        "alto_answer_device_noalloc": (I, [P, P, S, S, P, S, P]),
        "alto_answer_device_parts": (I, [P, P, S, S, PP, S, S, S, c.POINTER(I)]),
        "alto_ipc_export": (I, [P, P, c.POINTER(S)]),
        "alto_ipc_import": (P, [P]),
        "alto_ipc_release": (I, [P]),
        "alto_server_new": (P, [P, S, S, I]),
        "alto_server_new_keyed": (P, [P, S, S, I, S]),
        "alto_server_log": (I, [P, c.POINTER(c.c_double), S]),
        "alto_server_new_loopback": (P, [S, S, S, S, I, c.c_double]),
        "alto_server_submit": (c.c_longlong, [P, P, S]),
        "alto_server_wait": (I, [P, c.c_longlong, P, S, I, c.POINTER(c.c_double)]),
        "alto_server_stats": (I, [P, c.POINTER(c.c_double), S]),
        "alto_server_free": (None, [P]),
        "alto_engine_new_empty": (P, [S, S, P, S, S, PP, S, S, U64, I, PP, P, U64, I]),
        "alto_engine_load_records": (I, [P, P, S, S, S]),
        "alto_engine_load_file": (I, [P, c.c_char_p, S]),
        "alto_synthetic_db_col": (None, [P, S, S, S, S, I]),
        "alto_synthetic_db_col_device": (I, [P, S, S, S, S]),
        "alto_engine_fill_synthetic": (I, [P]),
        "alto_hint_ring": (I, [P, P, P, I]),
        "alto_engine_offline": (I, [P, P, P, P, P, P, P, P, c.POINTER(c.c_double)]),
        "alto_synthetic_requests_device": (I, [P, S, S, S, S, S, U64, U64]),
        "alto_fill_uniform_u32": (None, [P, S, U64, U64, I]),
        "alto_fill_uniform_u64": (None, [P, S, U64, U64, I]),
        "alto_fill_bytes": (None, [P, S, U64, I]),
        "alto_synthetic_request": (None, [P, S, S, U64, U64]),
        "alto_pack_encode": (None, [P, P, S, S, I]),
        "alto_rescale_digest": (U64, [U64, U64, U64, I]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def last_error():
    return lib().alto_last_error().decode()


# Symbols the header include/altopir_gpu.h declares (checked by the tests against the built library).
EXPORTS = (
    "sw_amx_init", "sw_alloc_zeroed", "sw_alloc", "sw_free", "sw_tile_db", "sw_pack_build", "alto_engine_new",
    "alto_engine_free", "alto_request_len", "alto_response_len", "alto_answer", "alto_last_error",
    "alto_answer_device", "alto_last_launches", "alto_enqueue_device", "alto_engine_sync", "alto_engine_stream",
    "alto_kernel_times", "alto_engine_set_graphs", "alto_engine_set_lanes", "alto_engine_fence",
    "alto_engine_set_tuning", "alto_answer_device_noalloc",
    "alto_answer_device_parts", "alto_ipc_export", "alto_ipc_import", "alto_ipc_release", "alto_server_new",
    "alto_server_new_keyed", "alto_server_log",
    "alto_server_new_loopback",
    "alto_server_submit", "alto_server_wait", "alto_server_stats", "alto_server_free", "alto_engine_new_empty",
    "alto_engine_load_records", "alto_engine_load_file", "alto_synthetic_db_col", "alto_synthetic_db_col_device",
    "alto_engine_fill_synthetic", "alto_synthetic_requests_device", "alto_hint_ring",
    "alto_engine_offline",
    "alto_fill_uniform_u32", "alto_fill_uniform_u64", "alto_fill_bytes", "alto_synthetic_request",
    "alto_pack_encode", "alto_rescale_digest",
)
