"""Loader for the CPU checkers under oracle/ (test infrastructure only).

``oracle()``     the C restatement (oracle/_build/liboracle.so), built on demand.
``reference()``  the reference engine compiled in place (oracle/_ref/libpentago_ref.so),
                 or None when it has not been built (it needs the reference sources).
Both export the same function names behind ``or_`` / ``ref_`` prefixes; ``Checker``
hides the prefix so a test can run against either.
"""
import ctypes
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "_build", "liboracle.so")
REF_LIB = os.path.join(ORACLE_DIR, "_ref", "libpentago_ref.so")

_u64 = ctypes.c_uint64
_p = ctypes.c_void_p
_i = ctypes.c_int
_i64 = ctypes.c_int64
SIGS = {
    "table": (ctypes.c_void_p, [ctypes.c_char_p, ctypes.POINTER(_i)]),
    "rmax": (None, [_p, _p, _i]),
    "super_wins": (None, [_p, _p, _i]),
    "transform_super": (None, [_p, _p, _p, _i]),
    "symmetry_product": (None, [_p, _p, _p, _i]),
    "halfsuper_wins": (None, [_p, _p, _p, _i]),
    "halfsuper_rmax": (None, [_p, _p, _i]),
    "line_sizes": (_i, [_u64, _i, _i, _p, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "compute_line": (_i, [_u64, _i, _i, _p, _p, _p, _i]),
    "count_block_wins": (None, [_u64, _p, _p, _p]),
    "descendent_sections": (_i, [_u64, _i, _p, _i]),
    "midsolve": (_i, [_u64, _p, _p]),
    "midsolve_internal": (None, [_u64, _p]),
    "midsolve_workspace_size": (_i, [_i]),
    "lookup_locate": (None, [_u64, _p, _p, _p, _p]),
    "lookup_values": (None, [_p, _i64, _p, _i, _p, _p, _p]),
    "st_filter": (None, [_p, _i64, _i, _i, _p]),
    "st_unfilter": (None, [_p, _i64, _i, _i, _p]),
    "rans_encode": (_i64, [_p, _i64, _p, _i64]),
    "rans_decode": (_i64, [_p, _i64, _p, _i64]),
    "lm_nodes": (_i64, [_u64, _p]),
    "lm_freqs": (_i, [_p, _u64, _p, _p, _p, _i64, _p]),
    "lm_encode": (_i64, [_p, _u64, _p, _p, _p, _i64]),
    "lm_decode": (_i64, [_p, _u64, _p, _p, _i64, _p, _i64]),
    "lm_grad": (ctypes.c_double, [_p, _u64, _p, _p, _p, _i64, _p]),
    "store_bound": (_i64, [_i64]),
    "store_table": (None, [_p, _p, _p, _i, _i, _p]),
    "store_encode_block": (_i64, [_p, _i, _i, _p, _p]),
    "store_decode_block": (_i64, [_p, _i64, _i, _i, _p, _p]),
}


class Checker:
    def __init__(self, path, prefix):
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix
        self.path = path
        for name, (res, args) in SIGS.items():
            f = getattr(self.lib, prefix + name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
            setattr(self, name, f)
        if prefix == "or_":
            self.lib.or_init()
        else:
            # the reference's thread pool starts when a call needs it; its idle
            # workers spin, so callers release it when they are done
            self.lib.ref_threads.restype = _i
            self.lib.ref_release_threads.restype = _i

    def release_threads(self):
        """Stop the reference's thread pool (no-op for the C restatement)."""
        f = getattr(self.lib, "ref_release_threads", None)
        if f is not None:
            f()

    def get_table(self, name, dtype):
        import numpy as np
        n = _i()
        p = self.table(name.encode(), ctypes.byref(n))
        return np.frombuffer((ctypes.c_char * n.value).from_address(p), dtype=dtype).copy()


_oracle = None
_ref = None


def build_oracle():
    """Compile oracle/pentago_oracle.c (fast; plain gcc)."""
    subprocess.check_call(["make", "-s", "-C", ORACLE_DIR, "oracle"], stdout=subprocess.DEVNULL)


def oracle():
    global _oracle
    if _oracle is None:
        build_oracle()  # make rebuilds it only when a source changed
        _oracle = Checker(ORACLE_LIB, "or_")
    return _oracle


def reference():
    global _ref
    if _ref is None and os.path.exists(REF_LIB):
        _ref = Checker(REF_LIB, "ref_")
    return _ref


def P(a):
    return ctypes.c_void_p(a.ctypes.data)
