"""End-engine block lines: the host-side mirror of the reference's line interface.

``Line`` mirrors ``line_t`` (pentago/end/line.h:15-33); ``line_info`` mirrors
``line_data_t`` (pentago/end/compute.cc:24-46); ``compute_lines`` is the GPU
form of ``schedule_compute_line`` (pentago/end/compute.h:122-123) and writes
each line's parent nodes into its output buffer, or ORs them in (the
``accumulate`` of pentago/end/block_store.cc:173-226).
"""
import ctypes
from dataclasses import dataclass, field
from typing import Optional, Sequence

from . import capi


def section_sig(counts):
    """section_t::sig() (pentago/base/section.h:35-42) of [[b0,w0],...,[b3,w3]]."""
    s = 0
    for q in range(4):
        for k in range(2):
            s |= int(counts[q][k]) << (16 * q + 8 * k)
    return s


def section_counts(sig):
    return [[(sig >> (16 * q + 8 * k)) & 0xFF for k in range(2)] for q in range(4)]


def section_shape(sig):
    out = (ctypes.c_int32 * 4)()
    capi.check(capi.lib().pg_section_shape(ctypes.c_uint64(sig), out))
    return list(out)


def section_standardize(sig):
    std = ctypes.c_uint64()
    g = ctypes.c_int32()
    capi.check(capi.lib().pg_section_standardize(ctypes.c_uint64(sig), ctypes.byref(std), ctypes.byref(g)))
    return std.value, g.value


def section_sum(sig):
    return sum(sum(c) for c in section_counts(sig))


@dataclass
class Line:
    """One block line: ``length`` blocks of ``section`` along ``dimension``."""
    section: int
    dimension: int
    block_base: Sequence[int]
    length: Optional[int] = None
    flags: int = capi.PG_LINE_STORE
    # Buffers: torch tensors (uint64 on the device) or raw device addresses
    input: object = None
    output: object = None
    input_block_offsets: Optional[Sequence[int]] = None
    output_block_offsets: Optional[Sequence[int]] = None
    input_block_stride: int = 0
    output_block_stride: int = 0
    _keep: list = field(default_factory=list, repr=False)

    def __post_init__(self):
        if self.length is None:
            self.length = (section_shape(self.section)[self.dimension] + 7) // 8

    def to_c(self):
        c = capi.pg_line_t()
        c.section = self.section
        c.dimension = self.dimension
        c.length = self.length
        for i in range(3):
            c.block_base[i] = int(self.block_base[i])
        c.flags = self.flags
        c.input = _addr(self.input)
        c.output = _addr(self.output)
        self._keep = []
        for name in ("input_block_offsets", "output_block_offsets"):
            v = getattr(self, name)
            if v is not None:
                arr = (ctypes.c_int64 * len(v))(*[int(x) for x in v])
                self._keep.append(arr)
                setattr(c, name, ctypes.cast(arr, ctypes.POINTER(ctypes.c_int64)))
        c.input_block_stride = self.input_block_stride
        c.output_block_stride = self.output_block_stride
        return c


def _addr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return capi.ptr(x)


@dataclass
class LineInfo:
    input_nodes: int
    output_nodes: int
    input_blocks: int
    block_stride: int
    child_section: int
    child_dimension: int
    input_shape: list
    output_shape: list


def line_info(line: Line) -> LineInfo:
    info = capi.pg_line_info_t()
    c = line.to_c()
    capi.check(capi.lib().pg_line_info(ctypes.byref(c), ctypes.byref(info)))
    return LineInfo(info.input_nodes, info.output_nodes, info.input_blocks, info.block_stride,
                    info.child_section, info.child_dimension, list(info.input_shape), list(info.output_shape))


def _array(lines):
    arr = (capi.pg_line_t * len(lines))()
    for i, l in enumerate(lines):
        arr[i] = l.to_c()
    return arr


def compute_lines(lines: Sequence[Line], stream=None):
    """Launch the line kernel for ``lines`` on ``stream`` (default: torch's current stream)."""
    arr = _array(lines)
    capi.check(capi.lib().pg_end_compute_lines(arr, len(lines), capi.stream_handle(stream)))


class Plan:
    """Lines planned once (the host work of line_details_t) and run many
    times; the lines' buffers must stay alive while the plan is used."""

    def __init__(self, lines: Sequence[Line]):
        self._arr = _array(lines)
        self._lines = list(lines)
        self._h = ctypes.c_void_p()
        capi.check(capi.lib().pg_end_plan_create(self._arr, len(lines), ctypes.byref(self._h)))

    def run(self, stream=None):
        capi.check(capi.lib().pg_end_plan_run(self._h, capi.stream_handle(stream)))

    @property
    def streams(self):
        """Streams a run uses: one per dimension when the dimensions' lines
        are independent, else 1."""
        return capi.check(capi.lib().pg_end_plan_streams(self._h))

    def close(self):
        if self._h:
            capi.lib().pg_end_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def check_errors(stream=None):
    """Synchronize and raise if a device-side bounds check fired."""
    capi.check(capi.lib().pg_end_check(capi.stream_handle(stream)))


def selftest_lines_host(lines: Sequence[Line]):
    """Run the kernel's own microline code sequentially on the CPU, on host
    buffers (numpy).  For CPU tests of the kernel arithmetic only."""
    arr = _array(lines)
    capi.check(capi.lib().pg_selftest_end_lines_host(arr, len(lines)))
