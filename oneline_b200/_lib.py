"""ctypes binding of liboneline_cuda.so (the C ABI in include/oneline_cuda.h).

The library is loaded from this package directory. There is no CPU fallback: if
the library is missing or no CUDA device is present, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboneline_cuda.so")

OL_OK = 0
STATUS_NAMES = {
    1: "OL_ERR_INVALID_ARG", 2: "OL_ERR_INPUT_TOO_LARGE", 3: "OL_ERR_BAD_PATTERN", 4: "OL_ERR_TOO_DEEP",
    5: "OL_ERR_OOM", 6: "OL_ERR_ADMISSION", 7: "OL_ERR_TIMEOUT", 8: "OL_ERR_CUDA", 9: "OL_ERR_NOT_FOUND",
}

# Every symbol include/oneline_cuda.h declares, with (restype, argtypes).
_P = ctypes.c_void_p
_U8P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_I32 = ctypes.c_int32
_S = ctypes.c_int32
_PP = ctypes.POINTER(ctypes.c_void_p)
_U32P = ctypes.POINTER(ctypes.c_uint32)
_U64P = ctypes.POINTER(ctypes.c_uint64)

SIGNATURES: dict[str, tuple] = {
    "ol_ctx_create": (_S, [_I32, _PP]),
    "ol_ctx_destroy": (None, [_P]),
    "ol_last_error": (ctypes.c_char_p, [_P]),
    "ol_ctx_device_name": (_S, [_P, ctypes.c_char_p, ctypes.c_size_t]),
    "ol_ctx_sync": (_S, [_P]),
    "ol_ctx_stream": (_P, [_P]),
    "ol_ctx_inject": (_S, [_P, _U32]),
    "ol_launch_count": (_U64, []),
    "ol_profile_begin": (_S, [_P]),
    "ol_profile_end": (_S, [_P, _P]),
    "ol_doc_upload": (_S, [_P, _U8P, _U64, _PP]),
    "ol_doc_upload_device": (_S, [_P, _U8P, _U64, _PP]),
    "ol_doc_free": (None, [_P]),
    "ol_doc_line_count": (_U64, [_P]),
    "ol_doc_text_len": (_U64, [_P]),
    "ol_doc_max_depth": (_U64, [_P]),
    "ol_doc_reparse_async": (_S, [_P, _P]),
    "ol_doc_read_offsets": (_S, [_P, _P, _P, _U64]),
    "ol_doc_read_kinds": (_S, [_P, _P, _P, _U64]),
    "ol_doc_read_nodes": (_S, [_P, _P, _P, _U64]),
    "ol_doc_device_views": (_S, [_P, _PP, _PP, _PP, _PP]),
    "ol_doc_save_olb": (_S, [_P, _P, ctypes.c_char_p]),
    "ol_doc_load_olb": (_S, [_P, ctypes.c_char_p, _U32, _PP]),
    "ol_parse_raw": (_S, [_P, _U8P, _U64, _P, _P, _U64, _U64P]),
    "ol_scan_line_offsets": (_S, [_P, _U8P, _U64, _P, _U64, _U64P]),
    "ol_parse_with_offsets": (_S, [_P, _U8P, _U64, _P, _U64, _P]),
    "ol_tree_build": (_S, [_P, _P, _U32, _PP]),
    "ol_tree_build_reusing": (_S, [_P, _P, _P, _U32, _PP]),
    "ol_tree_rebuild_async": (_S, [_P, _P, _P]),
    "ol_tree_free": (None, [_P]),
    "ol_tree_line_count": (_U64, [_P]),
    "ol_tree_read": (_S, [_P, _P, _P, _P, _P, _P, _U64]),
    "ol_search": (_S, [_P, _P, _U8P, _U32, _U32, _U32P, _P]),
    "ol_search_raw": (_S, [_P, _U8P, _U64, _U8P, _U32, _U32, _U32P, _P]),
    "ol_search_async": (_S, [_P, _P, _U8P, _U32, _U32, _P, _P]),
    "ol_search_multi": (_S, [_P, _P, _P, _P, _U32, _P, _P, _P]),
    "ol_search_multi_async": (_S, [_P, _P, _P, _P, _U32, _P, _P, _P]),
    "ol_query_document": (_S, [_P, _P, _U32, _U32, _U32, _U32P, _P]),
    "ol_query_subtree": (_S, [_P, _P, _P, _U64, _U32, _U32, _U32, _U32P, _P]),
    "ol_query_raw": (_S, [_P, _U8P, _U64, _U32, _U32, _U32, _U32P, _P]),
    "ol_query": (_S, [_P, _U8P, _U64, _P, _U64, _U32, _U32, _U32, _U32P, _P]),
    "ol_pipeline_capture": (_S, [_P, _P, _P, _P, _P, _U32, _P, _P, _P, _PP]),
    "ol_pipeline_launch": (_S, [_P]),
    "ol_pipeline_sync": (_S, [_P]),
    "ol_pipeline_stream": (_P, [_P]),
    "ol_pipeline_kernels": (_U32, [_P]),
    "ol_pipeline_free": (None, [_P]),
    "ol_tuning_get": (_S, [_P, _P]),
    "ol_tuning_set": (_S, [_P, _P]),
    "ol_autotune": (_S, [_P, _P, _P, _P, _P, _U32, ctypes.c_char_p, _P]),
    "ol_tuning_load": (_S, [_P, ctypes.c_char_p]),
    "ol_dict_stats": (_S, [_P, _P]),
    "ol_patset_compile": (_S, [_P, _P, _P, _P, _U32, _PP]),
    "ol_patset_free": (None, [_P]),
    "ol_patset_len": (_U32, [_P]),
    "ol_patset_unique": (_U32, [_P]),
    "ol_search_many": (_S, [_P, _P, _P, _U64, _P, _U64P, _P]),
    "ol_search_many_device": (_S, [_P, _P, _P, _U64, _U32, _P, _U64P, _P]),
    "ol_search_many_u64": (_S, [_P, _P, _P, _U64, _P, _U64P, _P, _P]),
    "ol_search_many_device_u64": (_S, [_P, _P, _P, _U64, _U32, _P, _U64P, _P, _P]),
    "ol_batch_upload": (_S, [_P, _U8P, _P, _U32, _PP]),
    "ol_batch_free": (None, [_P]),
    "ol_batch_docs": (_U32, [_P]),
    "ol_batch_text_len": (_U64, [_P]),
    "ol_batch_doc_info": (_S, [_P, _U32, _U64P, _U64P, _U64P, _U64P]),
    "ol_batch_build_trees": (_S, [_P, _P]),
    "ol_batch_read_doc": (_S, [_P, _P, _U32, _P, _P, _P, _P, _P, _P, _U64]),
    "ol_batch_search_many": (_S, [_P, _P, _P, _U64, _U32, _P, _U64P, _P]),
    "ol_server_create": (_S, [_I32, _U32, _U64, _U64, _PP]),
    "ol_server_create_ex": (_S, [_I32, _U32, _U64, _U64, _U32, _PP]),
    "ol_server_submit_parse_to": (_S, [_P, _U8P, _U64, _P, _U64P]),
    "ol_server_submit_search_to": (_S, [_P, _U64, _P, _P, _U32, _P, _U64P]),
    "ol_server_pause": (_S, [_P, _U32]),
    "ol_server_steps": (_S, [_P, _U64P, _U64P, _U64P]),
    "ol_server_destroy": (None, [_P]),
    "ol_server_submit_parse": (_S, [_P, _U8P, _U64, _U64P]),
    "ol_server_submit_search": (_S, [_P, _U64, _P, _P, _U32, _U64P]),
    "ol_server_wait": (_S, [_P, _U64, _P]),
    "ol_server_stats": (_S, [_P, _U64P, _U64P, _U64P, _U64P]),
    "ol_search_noalloc": (_S, [_U8P, _U64, _U64, _U8P, _U32, _U32, _P, _P, _P, ctypes.c_char_p, _U32]),
}

_lib = None


def load(build_if_missing: bool = True) -> ctypes.CDLL:
    """Load the CUDA library (building it first when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise OSError(f"{LIB_PATH} is missing; run oneline_b200.build.build_cuda()")
        from .build import build_cuda
        build_cuda()
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return _lib


class OnelineError(RuntimeError):
    """A non-OK status from the C ABI."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def check(status: int, ctx=None) -> None:
    if status != OL_OK:
        msg = load().ol_last_error(ctx).decode(errors="replace") if ctx else ""
        raise OnelineError(status, msg)
