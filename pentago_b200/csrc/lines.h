// Host planning for end-engine block lines: section algebra and the per-line
// descriptor the line kernel reads.  The index conventions restate
// line_data_t / line_details_t (pentago/end/compute.cc:24-123) and the
// per-microline setup of compute_microline (compute.cc:219-281).
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include "tables.h"

namespace pg {

struct section_t {
  uint8_t c[4][2];  // counts[quadrant][black, white]

  static section_t from_sig(uint64_t sig);
  uint64_t sig() const;
  int sum() const;
  bool valid() const;
  void shape(int* s) const;
  section_t transform(int global) const;               // section.cc:78-86
  section_t standardize(int* transform) const;          // section.cc:88-101
  section_t child(int q) const;                         // section.cc:51-57
};

// quadrant_permutation (section.cc:106-114): quadrant i maps to p[i]
void quadrant_permutation(int global, int* p);
inline int invert_global(int g) { return g ^ ((~g >> 2 & (g & 1)) << 1); }

// An axis permutation of the rotation index space Z_4^4, as where the
// content of axis q goes.
struct axis_perm { int to[4]; };
constexpr axis_perm perm_id() { return axis_perm{{0, 1, 2, 3}}; }
// p, then the contents of axes a and b exchanged.
constexpr axis_perm perm_swap(axis_perm p, int a, int b) {
  for (int q = 0; q < 4; q++) p.to[q] = p.to[q] == a ? b : p.to[q] == b ? a : p.to[q];
  return p;
}
// The axis permutation of a line's children's transform: that of phi_g (the
// conjugation by global symmetry g, without its negation of every axis when
// g reflects), then the exchange of the line's axis DIM with axis 3.
constexpr axis_perm line_sigma(int dim, int g) {
  axis_perm p = perm_id();
  if (g == 1) { p = perm_swap(p, 1, 3); p = perm_swap(p, 0, 3); p = perm_swap(p, 2, 3); }
  if (g == 2) { p = perm_swap(p, 0, 3); p = perm_swap(p, 1, 2); }
  if (g == 3) { p = perm_swap(p, 2, 3); p = perm_swap(p, 0, 3); p = perm_swap(p, 1, 3); }
  if (g == 4) { p = perm_swap(p, 0, 3); }
  if (g == 5) { p = perm_swap(p, 1, 3); p = perm_swap(p, 0, 2); }
  if (g == 6) { p = perm_swap(p, 1, 2); }
  if (g == 7) { p = perm_swap(p, 2, 3); p = perm_swap(p, 0, 1); }
  if (dim != 3) p = perm_swap(p, dim, 3);
  return p;
}
// A translation l (2 bits per axis) with its axes moved by p.
inline int sigma_apply(const axis_perm& p, int l) {
  int r = 0;
  for (int q = 0; q < 4; q++) r |= (l >> (2 * q) & 3) << (2 * p.to[q]);
  return r;
}

constexpr int kMaxBlocks = 64;   // 420 nodes / 8 per block < 64
constexpr int kMaxLine = 424;    // nodes along a quadrant axis, rounded up

// Per-parent facts that depend only on the parent's quadrant along the line
// (the same for every microline of every line of one section and
// dimension).  The kernel reads the first 16 bytes for every parent, the
// second only when the line quadrant has more than 6 empty cells, the third
// only on 35-stone sections.
struct alignas(16) parent_rec {
  uint8_t c0, c1;      // rotation classes (cls_rank) of the mover's / opponent's stone patterns
  uint8_t rot;         // bits 0-1 (2-3): the mover's (opponent's) pattern is its class rotated left this often
  uint8_t nmoves;
  uint16_t mv[14];     // per empty cell, increasing: the child quadrant as rotation r of rotation-minimal
                       // child j (rotation_minimal_quadrants_inverse = 4 j + r), stored as r * nchild + j
                       // (pair 0's slot of the child in the line kernel's shared memory, nchild the
                       // number of child quadrant states); at most 9 used, mv[0..5] in the first 16 bytes
  uint32_t usub[4];    // win terms (term_sub) the mover covers after a stone on some empty cell, per rotation
};
static_assert(sizeof(parent_rec) == 48, "parent_rec layout");

// Per child quadrant state j (index j of the rotation-minimal list of the
// line quadrant after the move): the win terms the mover's stones cover, per
// rotation of the quadrant.
struct alignas(16) child_rec {
  uint32_t csub[4];
};

// Per state of a cross quadrant (a quadrant other than the line's) and per
// side (the mover's, then the opponent's stones): the coverage of all 32 win
// patterns, 4 bits each (bit r: the side's stones, rotated left r times,
// cover the pattern's cells in that quadrant), pattern p at bits 4 (p % 8)
// of word p / 8.
struct alignas(16) cross_rec {
  uint32_t cov[4];
};

// Per rotation class of the line quadrant's stone patterns (the mover's
// classes, then the opponent's): the win terms its representative covers, per
// rotation.
struct alignas(16) class_rec {
  uint32_t sub[4];
};

// Everything a CTA needs to compute one microline of a line.  Plain data,
// copied to the device as is.
struct alignas(16) line_dev_t {
  int32_t dim, child_dim, turn, slice35, flags;
  int32_t g, inv_l;                 // base transform = (g, inv_l + reflection locals); inv_l and the
                                    // reflection locals below with their axes moved by line_sigma(dim, g)
  int32_t nparent, nchild, length, input_blocks, line_moves;
  int32_t odims[3], cross[3];       // the three cross dimensions and their extents
  int32_t perm[4], refl_moves[4], block0[4], first_child_block[4];
  int32_t out_shape[4];
  int32_t rmin_off[4];              // offsets of the parent quadrant lists in rmin_flat
  int32_t pat_off[2], npat[2];      // rotation classes of the line quadrant's stone patterns: mover, opponent
  uint32_t split_m[3];              // floor((2^32 - 1) / n) for n = nparent, nchild, npat[0] + npat[1]
  int32_t pad;
  const uint64_t* input;
  uint64_t* output;
  const parent_rec* recs;           // nparent records for this (section, dimension)
  const child_rec* crecs;           // nchild records for this (section, dimension)
  const cross_rec* xrecs;           // cross quadrant q's records start at xrecs + xoff[q], 2 per state
  const class_rec* precs;           // npat[0] + npat[1] records
  int32_t xoff[4];
  // The win patterns touching the line quadrant ("terms") with the one or two
  // other quadrants each touches, and the 15 that miss it with theirs (0xff: none).
  uint8_t term_pat[17], term_q[17][2];
  uint8_t miss_pat[15], miss_q[15][3];
  uint8_t pad2;
  int64_t in_off[kMaxBlocks], out_off[kMaxBlocks];
  uint8_t csym[kMaxLine];           // reflection rotations along the child dimension (0..3)
  uint8_t xsym[4][8];               // reflection locals of the cross dimensions (axes moved)
};

struct line_in_t {
  uint64_t section;
  int dim, length;
  uint8_t block_base[3];
  int flags;
  const uint64_t* input;
  uint64_t* output;
  const int64_t* input_offsets;
  const int64_t* output_offsets;
  int64_t input_stride, output_stride;
};

struct line_shapes_t {
  int in_shape[4], out_shape[4];
  int block_stride, input_blocks, child_dim, st;
  section_t child_std;
};

// Validate and compute shapes; returns false with a message on bad input.
bool line_shapes(const line_in_t& in, line_shapes_t& out, std::string& error);
// Fill the device descriptor (its record pointers are left null; see line_records).
bool plan_line(const line_in_t& in, line_dev_t& d, std::string& error);

// The records of a (section, dimension): nparent parent records, (below 35
// stones) nchild child records, the cross quadrants' records (quadrant q's at
// xoff[q]) and the pattern-class records.
struct line_rec_set {
  std::vector<parent_rec> recs;
  std::vector<child_rec> crecs;
  std::vector<cross_rec> xrecs;
  std::vector<class_rec> precs;
  int32_t xoff[4];
};
void line_records(uint64_t section, int dim, line_rec_set& out);

}  // namespace pg
