"""ctypes bindings for the C ABI in include/pentago_b200.h.

The shared library is built in-tree by ``python -m pentago_b200.build`` into
pentago_b200/_lib/libpentago_b200.so.  Loading fails loudly if it is missing:
there is no CPU fallback behind these entry points.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libpentago_b200.so")

PG_OK = 0
PG_ERR_ARG = -1
PG_ERR_CUDA = -2
PG_ERR_BOUNDS = -3
PG_ERR_TIMEOUT = -4
PG_ERR_FORMAT = -5
PG_ERR_CAPACITY = -6
PG_ERR_IO = -7
PG_LOOKUP_MISSING = -2

PG_LINE_STORE = 0
PG_LINE_OR = 1


class PentagoError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"pentago_b200 error {code}: {message}")
        self.code = code


class pg_line_t(ctypes.Structure):
    _fields_ = [
        ("section", ctypes.c_uint64),
        ("dimension", ctypes.c_uint8),
        ("length", ctypes.c_uint8),
        ("block_base", ctypes.c_uint8 * 3),
        ("flags", ctypes.c_uint8),
        ("reserved", ctypes.c_uint8 * 2),
        ("input", ctypes.c_void_p),
        ("output", ctypes.c_void_p),
        ("input_block_offsets", ctypes.POINTER(ctypes.c_int64)),
        ("output_block_offsets", ctypes.POINTER(ctypes.c_int64)),
        ("input_block_stride", ctypes.c_int64),
        ("output_block_stride", ctypes.c_int64),
    ]


class pg_line_info_t(ctypes.Structure):
    _fields_ = [
        ("input_nodes", ctypes.c_int64),
        ("output_nodes", ctypes.c_int64),
        ("input_blocks", ctypes.c_int32),
        ("block_stride", ctypes.c_int32),
        ("child_section", ctypes.c_uint64),
        ("child_dimension", ctypes.c_int32),
        ("input_shape", ctypes.c_int32 * 4),
        ("output_shape", ctypes.c_int32 * 4),
    ]


class pg_block_ref_t(ctypes.Structure):
    _fields_ = [("section", ctypes.c_uint64), ("block", ctypes.c_int32 * 4)]


class pg_mid_value_t(ctypes.Structure):
    _fields_ = [("raw", ctypes.c_uint64), ("value", ctypes.c_int32), ("pad", ctypes.c_int32)]


class pg_mid_values_t(ctypes.Structure):
    _fields_ = [("size", ctypes.c_int32), ("pad", ctypes.c_int32), ("entries", pg_mid_value_t * 163)]


MID_VALUES_BYTES = 8 + 16 * 163


class pg_shard_block_t(ctypes.Structure):
    _fields_ = [("section", ctypes.c_int32), ("block", ctypes.c_uint8 * 4), ("block_size", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("node_offset", ctypes.c_int64)]


class pg_supertensor_header_t(ctypes.Structure):
    _fields_ = [("version", ctypes.c_uint32), ("valid", ctypes.c_uint32), ("stones", ctypes.c_uint32),
                ("block_size", ctypes.c_uint32), ("section", ctypes.c_uint64), ("shape", ctypes.c_uint16 * 4),
                ("blocks", ctypes.c_uint16 * 4), ("filter", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("index", ctypes.c_uint64 * 3)]

# Every exported symbol of include/pentago_b200.h with its ctypes signature.
_P = ctypes.c_void_p
_I = ctypes.c_int
_U64 = ctypes.c_uint64
_I64 = ctypes.c_int64
SIGNATURES = {
    "pg_last_error": (ctypes.c_char_p, []),
    "pg_init": (_I, []),
    "pg_line_info": (_I, [ctypes.POINTER(pg_line_t), ctypes.POINTER(pg_line_info_t)]),
    "pg_end_compute_lines": (_I, [ctypes.POINTER(pg_line_t), _I, _P]),
    "pg_end_check": (_I, [_P]),
    "pg_end_plan_create": (_I, [ctypes.POINTER(pg_line_t), _I, ctypes.POINTER(_P)]),
    "pg_end_plan_run": (_I, [_P, _P]),
    "pg_end_plan_streams": (_I, [_P]),
    "pg_end_plan_destroy": (_I, [_P]),
    "pg_section_shape": (_I, [_U64, ctypes.POINTER(ctypes.c_int32)]),
    "pg_section_standardize": (_I, [_U64, ctypes.POINTER(_U64), ctypes.POINTER(ctypes.c_int32)]),
    "pg_debug_super": (_I, [_I, _P, _P, _P, _I, _P]),
    "pg_selftest_super_host": (_I, [_I, _P, _P, _P, _I]),
    "pg_selftest_end_lines_host": (_I, [ctypes.POINTER(pg_line_t), _I]),
    "pg_selftest_table": (ctypes.c_void_p, [ctypes.c_char_p, ctypes.POINTER(_I)]),
    "pg_slice_layout": (_I, [_P, _I, _P]),
    "pg_descendent_sections": (_I, [_U64, _I, _P, _I]),
    "pg_end_sweep_slice": (_I, [_P, _I, _P, _P, _I, _P, _P]),
    "pg_end_sweep_slice_child": (_I, [_P, _I, _P, _U64, _P, _P]),
    "pg_section_counts": (_I, [_P, _I, _P, _P, _P]),
    "pg_serve_open": (_I, [_I64, ctypes.POINTER(_P)]),
    "pg_serve_submit": (_I64, [_P, _U64]),
    "pg_serve_poll": (_I, [_P, _I64, _P]),
    "pg_serve_close": (_I, [_P]),
    "pg_serve_state": (_I, [_P]),
    "pg_rans_bound": (_I64, [_I64]),
    "pg_rans_encode_batch": (_I, [_P, _P, _I, _P, _P, _P, _P]),
    "pg_rans_decode_batch": (_I, [_P, _P, _P, _I, _P, _P, _P, _P, _P]),
    "pg_node_symbols": (_I, [_P, _I64, _I, _P, _P]),
    "pg_symbols_nodes": (_I, [_P, _I64, _I, _P, _P]),
    "pg_pack_streams": (_I, [_P, _P, _P, _I, _P, _P, _P]),
    "pg_store_bound": (_I64, [_I64]),
    "pg_store_table": (_I, [_P, _P, _P, _I, _I, _P, _P]),
    "pg_store_encode": (_I, [_P, _P, _P, _I, _I, _P, _P, _P, _P, _P]),
    "pg_store_decode": (_I, [_P, _P, _P, _P, _P, _I, _I, _P, _P, _P, _P]),
    "pg_learned_model_bytes": (_I64, []),
    "pg_rans_learned_bound": (_I64, [_I64]),
    "pg_rans_learned_encode": (_I, [_P, _P, _I, _P, _P, _P, _P, _P, _P]),
    "pg_rans_learned_decode": (_I, [_P, _P, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    "pg_learned_freqs": (_I, [_P, _P, _I, _P, _P, _P, _I64, _P, _P]),
    "pg_learned_samples": (_I, [_P, _I64, ctypes.c_uint64, _I64, _I64, _P, _P]),
    "pg_learned_grad": (_I, [_P, _P, _I, _P, _P, _P, _I64, _P, _P, _P]),
    "pg_learned_adam": (_I, [_P, _P, _P, _P, _I64, ctypes.c_float, ctypes.c_float, _P]),
    "pg_learned_export": (_I, [_P, _P]),
    "pg_midsolve_workspace_size": (_I, [_I]),
    "pg_selftest_midsolve_host": (_I, [_P, _I, _P, _P]),
    "pg_selftest_midsolve_groups_host": (_I, [_P, _I, _I, _P]),
    "pg_debug_barrier_timeout": (_I, [ctypes.c_uint, ctypes.POINTER(_I)]),
    "pg_midsolve_scratch_bytes": (_I, [_P, _I, ctypes.POINTER(_I64)]),
    "pg_midsolve_batch": (_I, [_P, _I, _P, _P, _I64, _P]),
    "pg_midsolve_batch_noalloc": (_I, [_P, _I, _P, _P]),
    "pg_supertensor_header_pack": (_I, [ctypes.POINTER(pg_supertensor_header_t), _P]),
    "pg_supertensor_header_unpack": (_I, [_P, ctypes.POINTER(pg_supertensor_header_t)]),
    "pg_supertensor_filter": (_I, [_P, _I64, _I, _I, _P, _P]),
    "pg_supertensor_unfilter": (_I, [_P, _I64, _I, _I, _P, _P]),
    "pg_supertensor_open": (_I, [ctypes.c_char_p, ctypes.POINTER(_P)]),
    "pg_supertensor_header": (_I, [_P, _I, ctypes.POINTER(pg_supertensor_header_t)]),
    "pg_supertensor_block_blob": (_I, [_P, _I, _P, _P]),
    "pg_supertensor_read_blocks_host": (_I, [_P, _I, _P, _P, _P, _P, _I]),
    "pg_supertensor_read_blocks": (_I, [_P, _I, _P, _P, _P, _P, _I, _I, _P]),
    "pg_supertensor_close": (_I, [_P]),
    "pg_supertensor_create": (_I, [ctypes.c_char_p, _P, _I, _I, _I, _I, _I, ctypes.POINTER(_P)]),
    "pg_supertensor_write_blocks_host": (_I, [_P, _I, _P, _P, _P, _P, _I]),
    "pg_supertensor_write_blocks": (_I, [_P, _I, _P, _P, _P, _P, _I, _I, _P]),
    "pg_supertensor_finalize": (_I, [_P, _I]),
    "pg_supertensor_writer_close": (_I, [_P]),
    "pg_shard_sections": (_I, [_I, _P, _I]),
    "pg_shard_total": (_I64, [_I]),
    "pg_shard_size": (_I64, [_I, _I, _I]),
    "pg_shard_permute": (_I, [_I, _P, _I64, _I, _P, _P]),
    "pg_shard_boards": (_I, [_I, _P, _I64, _P, _P]),
    "pg_shard_scatter": (_I, [_I, _I, _I, _I, _P, _I, _P, _I, _P, _P, _P]),
    "pg_selftest_shard_host": (_I, [_I, _I, _P, _I64, _P]),
    "pg_lookup_open": (_I, [ctypes.POINTER(ctypes.c_char_p), _I, _I64, ctypes.POINTER(_P)]),
    "pg_lookup_values": (_I, [_P, _P, _I64, _P, _P]),
    "pg_lookup_close": (_I, [_P]),
    "pg_lookup_stats": (_I, [_P, _P]),
    "pg_selftest_lookup_locate_host": (_I, [_P, _I64, _P, _P, _P, _P]),
}

_lib = None


def lib():
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m pentago_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code):
    """Raise PentagoError for a negative return code."""
    if code < 0:
        raise PentagoError(code, lib().pg_last_error().decode(errors="replace"))
    return code


def ptr(x):
    """Raw address of a torch tensor or numpy array (or None)."""
    if x is None:
        return None
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    return x.ctypes.data


def stream_handle(stream=None):
    """cudaStream_t of a torch stream (default: the current stream)."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
