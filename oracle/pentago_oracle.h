/* CPU oracle: a plain-C restatement of the reference's hot path, used only as
 * a checker by tests/, __graft_entry__.smoke() and bench.py's CPU baseline.
 * It is never linked or called by the product library.
 *
 * Parity pinning: the generated tables are checked in tests against the
 * SHA-1 hashes embedded in the reference's own table generator
 * (pentago/base/precompute.cc:169,194,293,617,929,1035-1038), and every
 * function is checked against the reference engine itself compiled in place
 * (oracle/_ref) and against the reference's golden vectors
 * (pentago/mid/benchmark_test.cc:42-58, pentago/high/high_test.cc:41-85,
 * data/counts-*.npy).
 *
 * Data formats are the reference's: a super is 4 little-endian uint64 words
 * (bit r = i0 + 4 i1 + 16 i2 + 64 i3, quadrant q rotated left i_q times); a
 * node is [win, notlost] = 8 uint64 (pentago/end/block_store.h:22-43); a
 * halfsuper is 2 uint64 (pentago/mid/halfsuper.h:4-60).
 */
#ifndef PENTAGO_ORACLE_H
#define PENTAGO_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

int or_init(void);
const void* or_table(const char* name, int* bytes);

void or_rmax(const uint64_t* in, uint64_t* out, int n);
void or_super_wins(const uint64_t* sides, uint64_t* out, int n);
void or_transform_super(const uint16_t* syms, const uint64_t* in, uint64_t* out, int n);
void or_symmetry_product(const uint16_t* a, const uint16_t* b, uint16_t* out, int n);
void or_halfsuper_wins(const uint64_t* sides, const uint8_t* parity, uint64_t* out, int n);
void or_halfsuper_rmax(const uint64_t* in, uint64_t* out, int n);

int or_line_sizes(uint64_t section_sig, int dim, int length, const uint8_t* block_base,
                  int64_t* input_nodes, int64_t* output_nodes);
int or_compute_line(uint64_t section_sig, int dim, int length, const uint8_t* block_base,
                    const uint64_t* input, uint64_t* output, int threads);
void or_count_block_wins(uint64_t section_sig, const uint8_t* block, const uint64_t* data,
                         uint64_t* counts3);
int or_section_shape(uint64_t section_sig, int* shape4);
uint64_t or_standardize_section(uint64_t section_sig, int* transform);
int or_descendent_sections(uint64_t root_sig, int slice, uint64_t* sigs, int cap);

int or_midsolve(uint64_t raw, uint64_t* out_raws, int32_t* out_values);
void or_midsolve_internal(uint64_t raw, uint64_t* out);
int or_midsolve_workspace_size(int stones);

/* Slice-file filter: the interleave of pentago/data/filter.h:76-127 (the
 * portable forms) with the node-form conversion of the slice writer and
 * reader, pentago/mpi/io.cc:79-86 and 476-481.  turn 0/1 converts from/to
 * [win, notlost] nodes of the side to move; turn 2 keeps the on-disk
 * [black wins, white wins] pair.  filter 0 leaves the bits in place. */
void or_st_filter(const uint64_t* nodes, int64_t n, int turn, int filter, uint64_t* out);
void or_st_unfilter(const uint64_t* in, int64_t n, int turn, int filter, uint64_t* nodes);

/* Shards (pentago/shard/shard.h, shard.cc, shard_permute.h): the sections of
 * a slice in all_boards_sections(slice, 8) order, the slice's entry count
 * (256 per position), the L/H window permutation, the board of a shuffled
 * index, a shard's size, and a shard's symbols (black wins + 2 white wins)
 * gathered from on-disk node pairs stored row-major per section at
 * nodes + 8 * (section_base[i] + position). */
int or_shard_sections(int slice, uint64_t* sigs, int cap);
uint64_t or_shard_total(int slice);
uint64_t or_shard_permute(int slice, uint64_t x, int inverse);
uint64_t or_shard_board(int slice, uint64_t shuffled);
uint64_t or_shard_size(int slice, int total_shards, int shard);
void or_shard_symbols(int slice, int total_shards, int shard, const uint64_t* nodes, const int64_t* section_base,
                      uint8_t* out);

/* Where a board's value lives in the solved database: block_cache_t::lookup
 * (pentago/data/block_cache.cc:27-58) for an absolute board (black moves
 * first; the side to move is the stone-count parity).  Outputs the
 * standardized section, the rotation-minimal index per quadrant, the
 * symmetry (global << 8 | local) that maps the stored super to the board's,
 * and the side to move.  The board's value is bit 0 of
 * transform_super(sym, extract(turn, aggressive, pair)) for aggressive 1
 * (win) and 0 (win or tie). */
void or_lookup_locate(uint64_t board, uint64_t* section, int32_t* index4, uint16_t* sym, int32_t* turn);
/* value() of n boards (1, 0, -1 for the side to move; -2 if the section is
 * absent) from slices held in host memory: sections secs[0..nsecs) sorted,
 * section i's on-disk pairs in 8^4-block-major order at data + 8 base[i]. */
void or_lookup_values(const uint64_t* boards, int64_t n, const uint64_t* secs, int nsecs, const int64_t* base,
                      const uint64_t* data, int32_t* values);

int64_t or_rans_encode(const uint8_t* symbols, int64_t n, uint8_t* out, int64_t cap);
int64_t or_rans_decode(const uint8_t* data, int64_t size, uint8_t* symbols, int64_t cap);

/* Learned coder, stream format version 3 (learned_oracle.c).  One block per
 * call: section signature and block coordinates; symbols 256 per node. */
int64_t or_lm_nodes(uint64_t section, const int* block);
int or_lm_freqs(const uint8_t* model, uint64_t section, const int* block, const uint8_t* symbols,
                const int64_t* samples, int64_t n, uint32_t* freqs);
int64_t or_lm_encode(const uint8_t* model, uint64_t section, const int* block, const uint8_t* symbols,
                     uint8_t* out, int64_t cap);
int64_t or_lm_decode(const uint8_t* model, uint64_t section, const int* block, const uint8_t* in, int64_t size,
                     uint8_t* symbols, int64_t cap);
double or_lm_grad(const float* params, uint64_t section, const int* block, const uint8_t* symbols,
                  const int64_t* samples, int64_t n, double* grad);

/* The library's store coder for slices kept in device memory (store_oracle.c):
 * the table of a batch of blocks, and one block's stream each way. */
int64_t or_store_bound(int64_t n);
void or_store_table(const uint64_t* nodes, const int64_t* first, const int32_t* count, int nblocks, int turn,
                    uint16_t* table);
int64_t or_store_encode_block(const uint64_t* nodes, int n, int turn, const uint16_t* table, uint8_t* out);
int64_t or_store_decode_block(const uint8_t* in, int64_t size, int n, int turn, const uint16_t* table,
                              uint64_t* nodes);

#ifdef __cplusplus
}
#endif
#endif
