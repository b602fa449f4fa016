/* pentago_b200: B200-native (sm_100a) kernels for pentago's backward solve.
 *
 * C ABI.  All pointers marked "device" are CUDA device pointers on the current
 * device; `stream` is a cudaStream_t (NULL = legacy default stream).  Every
 * entry point returns 0 on success or a negative PG_ERR_* code and never
 * aborts; pg_last_error() describes the last failure on the calling thread.
 *
 * Data formats are the reference's own (github.com/girving/pentago):
 *   - a super is 4 little-endian uint64 words, bit r = i0 + 4 i1 + 16 i2 + 64 i3
 *     (pentago/base/superscore.h:29-44);
 *   - an end-engine node is [we-win super, we-win-or-tie super] = 64 bytes
 *     (pentago/end/block_store.h:22-43);
 *   - nodes of a section are ordered by rotation-minimal quadrant index in
 *     8x8x8x8 blocks, each block row-major in its own shape
 *     (pentago/end/compute.h:21-27, pentago/base/section.h:26-27);
 *   - a halfsuper is 2 little-endian uint64 (pentago/mid/halfsuper_c.h:9-19).
 */
#ifndef PENTAGO_B200_H
#define PENTAGO_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PG_OK 0
#define PG_ERR_ARG -1      /* invalid argument (bad section, dimension, size...) */
#define PG_ERR_CUDA -2     /* a CUDA call failed */
#define PG_ERR_BOUNDS -3   /* a device-side bounds check failed */
#define PG_ERR_TIMEOUT -4  /* a bounded device wait ran out */
#define PG_ERR_FORMAT -5   /* malformed encoded stream */
#define PG_ERR_CAPACITY -6 /* output buffer too small / budget exceeded */
#define PG_ERR_IO -7       /* a file could not be opened, read or written */

const char* pg_last_error(void);

/* Build host tables and upload them to the current device.  Called implicitly
 * by every entry point; exposed so callers can pay the cost up front. */
int pg_init(void);

/* ---------------------------------------------------------------------------
 * End engine.
 *
 * pg_line_t mirrors the reference's line_t (pentago/end/line.h:15-33) plus the
 * buffers that line_details_t owns (pentago/end/compute.h:48-108).  The child
 * line holds input_blocks blocks of the standardized child section
 * section.child(dimension).standardize<8>() along the child dimension; the
 * output line holds `length` blocks of `section` along `dimension`.
 * ------------------------------------------------------------------------- */

#define PG_LINE_STORE 0 /* write the line's result */
#define PG_LINE_OR 1    /* OR the result into output (accumulate, end/block_store.cc:173-226) */

typedef struct {
  uint64_t section;        /* section_t::sig() of the parent section */
  uint8_t dimension;       /* which way the line points (0..3) */
  uint8_t length;          /* length in blocks */
  uint8_t block_base[3];   /* block indices in the other three dimensions */
  uint8_t flags;           /* PG_LINE_STORE or PG_LINE_OR */
  uint8_t reserved[2];
  const uint64_t* input;   /* device: child line data (unused for 35-stone sections) */
  uint64_t* output;        /* device: parent line data */
  /* Node offset of child block k from `input`: input_block_offsets[k] if that
   * host array is given, else k * input_block_stride (0 = packed blocks).
   * The reference's own buffers use block_stride + 1 (end/compute.cc:135-138). */
  const int64_t* input_block_offsets;
  const int64_t* output_block_offsets;
  int64_t input_block_stride;
  int64_t output_block_stride;
} pg_line_t;

typedef struct {
  int64_t input_nodes;     /* nodes in the child line (0 for 35-stone sections) */
  int64_t output_nodes;    /* nodes in the output line */
  int32_t input_blocks;    /* child blocks along the line */
  int32_t block_stride;    /* nodes per full block of the line (end/compute.h:50) */
  uint64_t child_section;  /* sig of the standardized child section */
  int32_t child_dimension; /* dimension of the line inside the child section */
  int32_t input_shape[4];  /* unstandardized (end/compute.cc:27-37) */
  int32_t output_shape[4];
} pg_line_info_t;

/* Shapes of a line (line_data_t, pentago/end/compute.cc:24-46). */
int pg_line_info(const pg_line_t* line, pg_line_info_t* info);

/* Compute block lines: the GPU form of schedule_compute_line
 * (pentago/end/compute.h:122-123, compute.cc:394-404).  Lines whose outputs
 * overlap must not be passed in the same call. */
int pg_end_compute_lines(const pg_line_t* lines, int n, void* stream);

/* Prepared lines: plan once on the host (line_details_t's work,
 * compute.cc:55-123), run many times.  The plan keeps the lines' buffer
 * pointers; the buffers must outlive it.  A run launches one kernel per
 * dimension present.  When no line has PG_LINE_OR and no line's output can
 * touch a buffer range of a line of another dimension, those launches run on
 * streams of the plan's own, forked from and joined back into `stream`
 * (their last waves then overlap); otherwise one after another on `stream`.
 * A plan is run by one host thread at a time.  pg_end_plan_streams returns
 * how many streams a run uses (1 when the launches are serial). */
typedef struct pg_end_plan_s* pg_end_plan_t;
int pg_end_plan_create(const pg_line_t* lines, int n, pg_end_plan_t* plan);
int pg_end_plan_run(pg_end_plan_t plan, void* stream);
int pg_end_plan_streams(pg_end_plan_t plan);
int pg_end_plan_destroy(pg_end_plan_t plan);

/* Synchronize `stream` and report device-side bounds violations recorded by
 * the line kernel since the last call (PG_ERR_BOUNDS), clearing them. */
int pg_end_check(void* stream);

/* ---------------------------------------------------------------------------
 * Slice sweeps.  A slice tensor holds the sections of one slice (standardized,
 * sorted by sig) back to back, each in the block-major node order above.
 * ------------------------------------------------------------------------- */

/* offsets[i] = node offset of section i in the slice tensor; offsets[n] = total nodes. */
int pg_slice_layout(const uint64_t* sigs, int n, int64_t* offsets);

/* Standardized sections that `root` depends on at `slice`, sorted by sig
 * (descendent_sections, pentago/end/sections.cc:18-49).  Returns the count and
 * writes at most cap of them. */
int pg_descendent_sections(uint64_t root, int slice, uint64_t* sigs, int cap);

/* Compute every block line of every section of a slice: parent_slice (device)
 * receives the OR over the line dimensions (compute_lines + accumulate over a
 * slice).  child_slice is the slice above (ignored for slice 35). */
int pg_end_sweep_slice(const uint64_t* parent_sigs, int np, uint64_t* parent_slice,
                       const uint64_t* child_sigs, int nc, const uint64_t* child_slice, void* stream);
/* The lines of a slice that read one child section only, with that
 * section's nodes (block-major) at child_nodes: every such line ORs into
 * parent_slice, which must start zeroed.  Calling it for every child section
 * equals pg_end_sweep_slice, so a sweep can keep the child slice compressed
 * and decompress one section at a time. */
int pg_end_sweep_slice_child(const uint64_t* parent_sigs, int np, uint64_t* parent_slice, uint64_t child_section,
                             const uint64_t* child_nodes, void* stream);

/* Per-section (we-win, we-win-or-tie, total) counts over distinct positions
 * into device counts3[3 n] (count_block_wins, pentago/end/block_store.cc:330-352,
 * summed per section as in mpi/io.cc:553-594 before the black/white swap). */
int pg_section_counts(const uint64_t* sigs, int n, const uint64_t* slice, uint64_t* counts3, void* stream);

/* Shape of a section along its four quadrants (section_t::shape,
 * pentago/base/section.cc:38-43). */
int pg_section_shape(uint64_t section, int32_t* shape4);

/* Standardized section (section_t::standardize<8>, pentago/base/section.cc:88-101). */
int pg_section_standardize(uint64_t section, uint64_t* standard, int32_t* transform);

/* ---------------------------------------------------------------------------
 * Midsolve.
 *
 * pg_mid_values_t has the layout of the reference's wasm export
 * mid_values_t = pile<tuple<raw_t,int>, 1+18+8*18> (pentago/mid/midengine.h:34,
 * js_test.cc:9-20): an int count, then 163 16-byte (raw, value) records, in
 * midsolve_traverse order (midengine.cc:127-158).  raw_t is
 * board | middle << 63 (pentago/high/board.h:76).
 * ------------------------------------------------------------------------- */

typedef struct {
  uint64_t raw;
  int32_t value;  /* 1 win, 0 tie, -1 loss for the player to move at `raw` */
  int32_t pad;
} pg_mid_value_t;

typedef struct {
  int32_t size;
  int32_t pad;
  pg_mid_value_t entries[163];
} pg_mid_values_t;

/* Workspace entries midsolve needs for a board with `stones` stones
 * (midsolve_workspace_size, pentago/mid/midengine.cc:44-46). */
int pg_midsolve_workspace_size(int stones);

/* Device scratch bytes pg_midsolve_batch needs for these boards. */
int pg_midsolve_scratch_bytes(const uint64_t* raws, int n, int64_t* bytes);

/* Solve n boards (host array of raw_t, each with >= 18 stones), writing
 * device array out[n]: the GPU form of midsolve(board, workspace)
 * (pentago/mid/midengine.cc:161-169) and of the wasm export midsolve(raw,
 * results) (:171-178).  scratch: device buffer of pg_midsolve_scratch_bytes,
 * or NULL to allocate on the stream. */
int pg_midsolve_batch(const uint64_t* raws, int n, pg_mid_values_t* out, void* scratch,
                      int64_t scratch_bytes, void* stream);

/* Midsolve that allocates nothing (no counterpart in the reference).
 *
 * For callers that cannot allocate device memory when they need a solve: code
 * whose framework owns the device's memory pool, and latency-critical loops
 * that must not wait for or fail in an allocation.  It gives the same results
 * as pg_midsolve_batch but uses only fixed device arrays that are part of the
 * library image:
 * PG_NOALLOC_SCRATCH_BYTES of scratch (held on every GPU that loads the
 * library until the process exits) plus a fixed copy of the win-pattern
 * table.  The caller passes the inputs (host array of raw_t) and the outputs
 * (device array of n records), as for pg_midsolve_batch.
 *
 * Limits and rules:
 *   - the boards' job descriptors, per-level tables and (for boards with more
 *     than 10 empty spots) workspaces must fit in PG_NOALLOC_SCRATCH_BYTES
 *     together; otherwise the call returns PG_ERR_CAPACITY and does nothing.
 *     About 64 boards of 26+ stones, or one board of 22 stones, fit;
 *   - every board is solved by one CTA; pg_midsolve_batch spreads boards
 *     with more than 10 empty spots (25 stones or fewer) over many CTAs, so
 *     such boards take far longer here, and runs the two passes of a smaller
 *     board on two CTAs;
 *   - each call copies its boards' job descriptors from host memory to the
 *     fixed array with cudaMemcpyAsync on the given stream;
 *   - the first call on a device sets that device up (it resolves the arrays'
 *     device addresses and fills the pattern table; no allocation), once, with
 *     a lock, so threads may race to make it;
 *   - all calls share the one scratch array, which keeps the last call's
 *     contents; nothing in it needs to start at zero (every entry is written
 *     before it is read).  Calls whose kernels overlap on the GPU (for example
 *     on two streams without ordering) race on it and must not be made. */
#define PG_NOALLOC_SCRATCH_BYTES (16 << 20)
int pg_midsolve_batch_noalloc(const uint64_t* raws, int n, pg_mid_values_t* out, void* stream);

/* ---------------------------------------------------------------------------
 * Midsolve server: continuous batching on a persistent kernel (three worker
 * CTAs per SM; boards with many empty spots are solved by a gang of workers).
 * Requests are admitted while others run, as long as the request
 * ring has a free entry and the device scratch budget has room for the
 * board's tables and workspace; otherwise submit returns PG_ERR_CAPACITY and
 * the caller polls and retries.  Workers leave after ~2 s without work and
 * are relaunched by the next submit.
 * ------------------------------------------------------------------------- */

typedef struct pg_server_s* pg_server_t;
int pg_serve_open(int64_t budget_bytes, pg_server_t* server);
int64_t pg_serve_submit(pg_server_t server, uint64_t raw);          /* ticket >= 0 */
int pg_serve_poll(pg_server_t server, int64_t ticket, pg_mid_values_t* result); /* 1 done, 0 pending */
int pg_serve_close(pg_server_t server);
/* State of the server's workers: 1 running, 2 left after about 2 s without
 * requests (the next submit relaunches them), 3 closed, 0 never launched. */
int pg_serve_state(pg_server_t server);

/* ---------------------------------------------------------------------------
 * Static rANS coder for ternary win/tie/loss symbols, byte-identical to the
 * reference's serialized format version 2 (arithmetic_encode / _decode /
 * _serialize, pentago/shard/arithmetic.cc:366-495).  Many independent streams
 * per call; all arrays are device arrays.
 * ------------------------------------------------------------------------- */

/* Bytes a stream of n symbols may need. */
int64_t pg_rans_bound(int64_t n);

/* Stream s encodes symbols[offsets[s] .. offsets[s+1]) (values 0..2) into
 * out + out_offsets[s] (room for pg_rans_bound) and stores its size. */
int pg_rans_encode_batch(const uint8_t* symbols, const int64_t* offsets, int nstreams, uint8_t* out,
                         const int64_t* out_offsets, int64_t* sizes, void* stream);

/* Decode stream s (in + in_offsets[s], in_sizes[s] bytes) into symbols +
 * sym_offsets[s] (room for sym_caps[s]); status[s] = symbols decoded, or
 * PG_ERR_FORMAT for a malformed stream, PG_ERR_CAPACITY if it does not fit. */
int pg_rans_decode_batch(const uint8_t* in, const int64_t* in_offsets, const int64_t* in_sizes, int nstreams,
                         uint8_t* symbols, const int64_t* sym_offsets, const int64_t* sym_caps, int64_t* status,
                         void* stream);

/* Ternary symbols of n solved nodes, 256 per node (rotation-major within the
 * node): black wins + 2 white wins, the on-disk convention of
 * pentago/shard/shard.cc:448-449.  turn = 1 when white is to move. */
int pg_node_symbols(const uint64_t* nodes, int64_t n, int turn, uint8_t* symbols, void* stream);
/* The inverse: n nodes of the side to move from their 256 n symbols (device,
 * symbols 16-byte aligned). */
int pg_symbols_nodes(const uint8_t* symbols, int64_t n, int turn, uint64_t* nodes, void* stream);
/* Copy n coded streams (device bytes at in + in_offsets[s], sizes[s] long;
 * the three arrays on the device) back to back at out + out_offsets[s]. */
int pg_pack_streams(const uint8_t* in, const int64_t* in_offsets, const int64_t* sizes, int n, uint8_t* out,
                    const int64_t* out_offsets, void* stream);

/* ---------------------------------------------------------------------------
 * Store coder for solved blocks kept in device memory (deeper sweeps).  No
 * reference counterpart and no file format: an internal, lossless coding of
 * end-engine nodes (the sweep's [win, win or tie] form for side `turn`).
 * Symbols black wins + 2 white wins per rotation, static rANS over 1024
 * contexts (the four axis neighbours of the rotation in the node and the
 * same rotation of the previous node); one table of 1024 x 3 frequencies
 * (device uint16) per batch.  Block b = count[b] nodes (at most 4096) at
 * nodes + 8 first[b]; all arrays are device arrays.
 * ------------------------------------------------------------------------- */

/* Bytes a block of `nodes` nodes may need. */
int64_t pg_store_bound(int64_t nodes);
/* The frequency table of a batch of blocks, from the context counts of at
 * most 2048 of its blocks spread evenly over it. */
int pg_store_table(const uint64_t* nodes, const int64_t* first, const int32_t* count, int nblocks, int turn,
                   uint16_t* table, void* stream);
/* Block b into out + out_offsets[b] (room for pg_store_bound); sizes[b] = its bytes. */
int pg_store_encode(const uint64_t* nodes, const int64_t* first, const int32_t* count, int nblocks, int turn,
                    const uint16_t* table, uint8_t* out, const int64_t* out_offsets, int64_t* sizes, void* stream);
/* Stream b (in + in_offsets[b], in_sizes[b] bytes, count[b] nodes) back to
 * nodes + 8 dst[b]; status[b] = nodes decoded or PG_ERR_FORMAT. */
int pg_store_decode(const uint8_t* in, const int64_t* in_offsets, const int64_t* in_sizes, const int32_t* count,
                    const int64_t* dst, int nblocks, int turn, const uint16_t* table, uint64_t* nodes, int64_t* status,
                    void* stream);

/* ---------------------------------------------------------------------------
 * Learned-model rANS for solved blocks: stream format version 3.  No
 * reference counterpart; it replaces the per-block static table of format 2
 * (arithmetic_encode, pentago/shard/arithmetic.cc:366-401) by a 3-layer MLP
 * (hidden 64, bf16 weights, fp32 accumulation) that predicts each symbol from
 * the node's board, the rotation, the already coded neighbouring rotations
 * and the previous node's symbol.  Streams are blocks of a section; symbols
 * are pg_node_symbols' (256 per node, nodes in the block's C order).  The encoder keeps whichever
 * of format 3 and format 2 is smaller, and the decoder reads both.
 * ------------------------------------------------------------------------- */

typedef struct pg_block_ref_t {
  uint64_t section;   /* section signature (counts as in pg_line_t.section) */
  int32_t block[4];   /* block coordinates, 8 positions per block per quadrant */
} pg_block_ref_t;

/* Bytes of a serialized model: "PGLM", version 3, parameter count, bf16
 * parameters.  In a version-3 model every column of W1's rotation, neighbour
 * and previous-node rows (72..123) and of W2 lies on a grid (integers of magnitude at
 * most 127 times a power of two), which makes the coder's tensor-core sums
 * exact; pg_learned_export puts them there, and the coder refuses a model
 * whose weights are not. */
int64_t pg_learned_model_bytes(void);

/* Bytes a stream of a block with `nodes` nodes may need (either format). */
int64_t pg_rans_learned_bound(int64_t nodes);

/* Encode stream s: the symbols[offsets[s] .. offsets[s+1]) of block blocks[s]
 * (256 per node) into out + out_offsets[s] (room for pg_rans_learned_bound),
 * sizes[s] = its bytes or PG_ERR_ARG.  `model` and `blocks` are host arrays;
 * symbols, offsets, out, out_offsets and sizes are device arrays. */
int pg_rans_learned_encode(const uint8_t* model, const pg_block_ref_t* blocks, int nstreams, const uint8_t* symbols,
                           const int64_t* offsets, uint8_t* out, const int64_t* out_offsets, int64_t* sizes,
                           void* stream);

/* Decode stream s (either format) into symbols + sym_offsets[s] (room for
 * sym_caps[s]); status[s] = symbols decoded, PG_ERR_FORMAT (malformed, or
 * coded with another model or for another block) or PG_ERR_CAPACITY. */
int pg_rans_learned_decode(const uint8_t* model, const pg_block_ref_t* blocks, int nstreams, const uint8_t* in,
                           const int64_t* in_offsets, const int64_t* in_sizes, uint8_t* symbols,
                           const int64_t* sym_offsets, const int64_t* sym_caps, int64_t* status, void* stream);

/* The coder's integer frequencies (3 per sample) for samples (stream << 24 |
 * node << 8 | rotation), with the contexts taken from `symbols`. */
int pg_learned_freqs(const uint8_t* model, const pg_block_ref_t* blocks, int nstreams, const uint8_t* symbols,
                     const int64_t* offsets, const int64_t* samples, int64_t n, uint32_t* freqs, void* stream);

/* Training.  params/m/v/grad are device fp32 arrays of the model's parameter
 * count (pg_learned_model_bytes() - 12) / 2.  Samples are drawn from
 * candidates (stream << 16 | node) by a seeded hash of (seed, step, index). */
int pg_learned_samples(const int64_t* candidates, int64_t ncand, uint64_t seed, int64_t step, int64_t batch,
                       int64_t* samples, void* stream);
/* Gradient of the summed cross entropy of the samples with the parameters
 * rounded to bf16 (loss: device float, sum in bits; may be NULL). */
int pg_learned_grad(const float* params, const pg_block_ref_t* blocks, int nstreams, const uint8_t* symbols,
                    const int64_t* offsets, const int64_t* samples, int64_t n, float* grad, float* loss, void* stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on grad * scale; step counts from 1. */
int pg_learned_adam(float* params, float* m, float* v, const float* grad, int64_t step, float lr, float scale,
                    void* stream);
/* Serialize host fp32 parameters into a model (host, pg_learned_model_bytes). */
int pg_learned_export(const float* params, uint8_t* model);

/* ---------------------------------------------------------------------------
 * Slice files: the reference's .pentago supertensor format
 * (pentago/data/supertensor.h:1-232, supertensor.cc), single-section files
 * ("pentago supertensor\n") and multiple-section files ("pentago sections
 * \n", version 3).  Blocks are compressed independently with zlib (level
 * 1-9) or xz (level 20 + preset), as compress() does in
 * pentago/data/compress.cc:34-60; xz needs liblzma.so.5 at run time.  On disk
 * a node is the pair [black wins, white wins]; filter 1 interleaves the bits
 * of the two supers (interleave_super, pentago/data/filter.h:76-127).  The
 * filter and the conversion to and from the end engine's [we win, we win or
 * tie] nodes (pentago/mpi/io.cc:79-86, 476-481) run on the GPU; compression
 * runs on host threads.
 *
 * `turn` arguments: 0 = black to move (even slices), 1 = white to move, both
 * converting to/from the end engine's node form; PG_ST_RAW keeps the on-disk
 * pair.  Blocks are named by (section index in the file, 4 block coordinates);
 * their nodes are row-major in the block's own shape.
 * ------------------------------------------------------------------------- */

#define PG_ST_RAW 2

typedef struct {
  uint32_t version;     /* 2 or 3 */
  uint32_t valid;       /* 1 once the file was finalized */
  uint32_t stones;
  uint32_t block_size;  /* even, 2..26 */
  uint64_t section;     /* section signature (counts as in pg_line_t.section) */
  uint16_t shape[4];
  uint16_t blocks[4];   /* ceil(shape / block_size) */
  uint32_t filter;      /* 0 none, 1 interleave */
  uint32_t reserved;
  uint64_t index[3];    /* compressed block index: uncompressed size, compressed size, offset */
} pg_supertensor_header_t;

/* The 85-byte packed header (supertensor_header_t::pack / unpack,
 * pentago/data/supertensor.cc:95-129); unpack checks the magic string. */
int pg_supertensor_header_pack(const pg_supertensor_header_t* h, uint8_t* out85);
int pg_supertensor_header_unpack(const uint8_t* in85, pg_supertensor_header_t* h);

/* Filter n nodes (device) into their on-disk bytes (device, 64 per node), and back. */
int pg_supertensor_filter(const uint64_t* nodes, int64_t n, int turn, int filter, uint8_t* out, void* stream);
int pg_supertensor_unfilter(const uint8_t* in, int64_t n, int turn, int filter, uint64_t* nodes, void* stream);

/* Reading (supertensor_reader_t, open_supertensors).  pg_supertensor_open
 * returns the number of sections; every header is checked as the reference's
 * reader checks it (supertensor.cc:143-192), and the block indices are read. */
typedef struct pg_supertensor_reader_s* pg_supertensor_reader_t;
int pg_supertensor_open(const char* path, pg_supertensor_reader_t* reader);
int pg_supertensor_header(pg_supertensor_reader_t reader, int section, pg_supertensor_header_t* h);
/* blob3 = uncompressed size, compressed size, file offset of one block */
int pg_supertensor_block_blob(pg_supertensor_reader_t reader, int section, const uint8_t* block4, uint64_t* blob3);
/* Block i = (sections[i], blocks[4i .. 4i+3]): read and decompress its
 * on-disk bytes into host memory at out + out_offsets[i], on `threads` host
 * threads (0 = every core). */
int pg_supertensor_read_blocks_host(pg_supertensor_reader_t reader, int n, const int32_t* sections,
                                    const uint8_t* blocks, uint8_t* out, const int64_t* out_offsets, int threads);
/* The same blocks into device memory, unfiltered on the GPU: block i's nodes
 * go to nodes + 8 * node_offsets[i].  Decompression of one batch overlaps the
 * copy and unfilter of the previous one. */
int pg_supertensor_read_blocks(pg_supertensor_reader_t reader, int n, const int32_t* sections, const uint8_t* blocks,
                               uint64_t* nodes, const int64_t* node_offsets, int turn, int threads, void* stream);
int pg_supertensor_close(pg_supertensor_reader_t reader);

/* Writing (supertensor_writer_t, supertensor_writers).  A file of sections
 * sections[0..n); multiple = 0 writes a single-section file (n = 1).  Blocks
 * are placed in the order they are written; each may be written once. */
typedef struct pg_supertensor_writer_s* pg_supertensor_writer_t;
int pg_supertensor_create(const char* path, const uint64_t* sections, int n, int multiple, int block_size, int filter,
                          int level, pg_supertensor_writer_t* writer);
/* Blocks whose on-disk bytes (already filtered) are in host memory. */
int pg_supertensor_write_blocks_host(pg_supertensor_writer_t writer, int n, const int32_t* sections,
                                     const uint8_t* blocks, const uint8_t* data, const int64_t* data_offsets,
                                     int threads);
/* Blocks whose nodes are in device memory (block i at nodes + 8 *
 * node_offsets[i]): filtered on the GPU and compressed on host threads while
 * the GPU filters and copies the next batch. */
int pg_supertensor_write_blocks(pg_supertensor_writer_t writer, int n, const int32_t* sections, const uint8_t* blocks,
                                const uint64_t* nodes, const int64_t* node_offsets, int turn, int threads,
                                void* stream);
/* Write the block index and the header of one section (-1: every section);
 * fails if a block of it was never written. */
int pg_supertensor_finalize(pg_supertensor_writer_t writer, int section);
/* Close; a file with an unfinalized section is removed, as the reference's
 * writer removes it (supertensor.cc:281-289). */
int pg_supertensor_writer_close(pg_supertensor_writer_t writer);

/* ---------------------------------------------------------------------------
 * Shards of solved positions for training (pentago/shard/shard.h, shard.cc,
 * shard_permute.h), slices 0..18.  Entry (section, position, rotation) of a
 * slice has linear index offset[section] + 256 position + rotation, with the
 * sections of pg_shard_sections and positions row-major over the section's
 * shape; a fixed permutation shuffles it, and shard s of a power-of-two
 * count N holds the shuffled indices congruent to s mod N, at index >>
 * log2(N).  An entry's symbol is black wins + 2 white wins, as the reference
 * stores it (shard.cc:447-449); a shard's symbols of one slice are one
 * format-2 stream (pg_rans_encode_batch).
 * ------------------------------------------------------------------------- */

/* Sections of a slice in the mapping's order (all_boards_sections(slice, 8)). */
int pg_shard_sections(int slice, uint64_t* sigs, int cap);
/* Entries of a slice (256 x positions), and of one shard of it. */
int64_t pg_shard_total(int slice);
int64_t pg_shard_size(int slice, int total_shards, int shard);
/* The permutation (inverse = 1: its inverse) of n device indices. */
int pg_shard_permute(int slice, const uint64_t* in, int64_t n, int inverse, uint64_t* out, void* stream);
/* board_t of n shuffled indices (device arrays; shard_mapping_t::board). */
int pg_shard_boards(int slice, const uint64_t* shuffled, int64_t n, uint64_t* boards, void* stream);

typedef struct {
  int32_t section;     /* index into pg_shard_sections(slice) */
  uint8_t block[4];    /* block coordinates */
  int32_t block_size;  /* even, 2..26 (8 for the end engine's and the database's blocks) */
  int32_t reserved;
  int64_t node_offset; /* first node of the block in `nodes` (row-major in the block's shape) */
} pg_shard_block_t;

/* scatter_block (shard.cc:405-464) for a batch of blocks (host array): every
 * entry whose shard lies in [shard_lo, shard_hi) stores its symbol (one byte)
 * at symbols + shard_offsets[shard - shard_lo] + its position in the shard.
 * nodes (device) are on-disk pairs (turn = PG_ST_RAW) or end-engine nodes of
 * the side to move (turn 0 / 1).  shard_offsets is a host array (each shard
 * needs pg_shard_size bytes), or NULL for shards shard_lo .. shard_hi - 1
 * packed back to back from symbols, which is faster (no table lookups). */
int pg_shard_scatter(int slice, int total_shards, int shard_lo, int shard_hi, const pg_shard_block_t* blocks,
                     int nblocks, const uint64_t* nodes, int turn, uint8_t* symbols, const int64_t* shard_offsets,
                     void* stream);

/* ---------------------------------------------------------------------------
 * Board values from solved slice files (block_cache_t::lookup and value(),
 * pentago/data/block_cache.cc:27-58, pentago/high/check.cc:21-37), batched:
 * the boards are located on the GPU and their blocks found in a block cache
 * in device memory through a device hash table; only blocks not cached go
 * through the host, which reads them into free slots or slots no board of
 * the call uses (in clock order); the values are then read on the GPU.  Boards are absolute board_t (black moves first;
 * the side to move is the stone-count parity, not at a half move); a value
 * is 1 (the side to move wins), 0 (tie), -1 (loses) or PG_LOOKUP_MISSING
 * when no open file holds the board's section.
 * ------------------------------------------------------------------------- */

#define PG_LOOKUP_MISSING -2

typedef struct pg_lookup_s* pg_lookup_t;
/* Open slice files (block size 8) and a device cache of cache_bytes. */
int pg_lookup_open(const char* const* paths, int npaths, int64_t cache_bytes, pg_lookup_t* lookup);
/* boards and values are host arrays; one call may touch at most as many
 * distinct blocks as the cache has slots (else PG_ERR_CAPACITY). */
int pg_lookup_values(pg_lookup_t lookup, const uint64_t* boards, int64_t n, int32_t* values, void* stream);
int pg_lookup_close(pg_lookup_t lookup);
/* Boards served without reading a block, blocks read, and cache slots, so far. */
int pg_lookup_stats(pg_lookup_t lookup, int64_t* stats3);

/* ---------------------------------------------------------------------------
 * Unit-level device operations, used by tests to check the superscore
 * library against the reference (pentago/base/superscore.h, symmetry.h).
 *   op 0: out[i] = rmax(in[i])                         in: supers
 *   op 1: out[i] = super_wins(in[i])                   in: sides (1 uint64)
 *   op 2: out[i] = transform_super(sym[i], in[i])      sym = global << 8 | local
 *   op 3: out[i] = halfsuper_wins(in[i], sym[i] & 1)   in: sides; out: halfsupers
 *   op 4: out[i] = rmax(in[i])                         in, out: halfsupers
 * ------------------------------------------------------------------------- */
int pg_debug_super(int op, const uint64_t* in, const uint16_t* sym, uint64_t* out, int n, void* stream);

/* ---------------------------------------------------------------------------
 * Self-test entry points (CPU only).  They run the kernels' own arithmetic
 * (the same __host__ __device__ functions) sequentially on the host, so CPU
 * tests can check it against the oracle without a GPU.  They are not a
 * fallback: no entry point above ever calls them.
 * ------------------------------------------------------------------------- */
int pg_selftest_super_host(int op, const uint64_t* in, const uint16_t* sym, uint64_t* out, int n);
int pg_selftest_end_lines_host(const pg_line_t* lines, int n);  /* host buffers */
const void* pg_selftest_table(const char* name, int* bytes);
/* host out[n]; supers (optional, host): 19 x (win, notlose) halfsupers per board */
int pg_selftest_midsolve_host(const uint64_t* raws, int n, pg_mid_values_t* out, uint64_t* supers);
/* The same solve split into `groups` cooperating groups (one host thread
 * each, a shared barrier between levels), as the multi-CTA kernel splits it. */
int pg_selftest_midsolve_groups_host(const uint64_t* raws, int n, int groups, pg_mid_values_t* out);
/* A CTA waits at a two-CTA barrier that nobody else reaches, with a limit of
 * `polls` polls: the wait runs out and *fault_out = 1 (device check of the
 * bounded barrier the multi-CTA midsolve and the server use). */
int pg_debug_barrier_timeout(unsigned polls, int* fault_out);
/* The shard permutation (op 0 forward, 1 inverse) and boards (op 2) of n
 * host indices, with the kernels' own functions. */
int pg_selftest_shard_host(int op, int slice, const uint64_t* in, int64_t n, uint64_t* out);
/* The lookup's location of n boards on the host (the kernel's own code):
 * standardized section, rotation-minimal index per quadrant, symmetry, side to move. */
int pg_selftest_lookup_locate_host(const uint64_t* boards, int64_t n, uint64_t* sections, int32_t* index4,
                                   uint16_t* syms, int32_t* turns);

#ifdef __cplusplus
}
#endif
#endif
