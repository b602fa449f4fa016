// Host-side lookup tables for the pentago hot path, generated from first
// principles at library load (no generated source is shipped).  The layouts of
// the tables that define storage order (rotation-minimal quadrant lists and
// their inverse) follow pentago/base/precompute.cc:967-1043 exactly, because
// they fix the order of nodes inside every section; the tests pin them with
// the SHA-1 hashes that generator embeds.
#pragma once
#include <cstdint>
#include <vector>

namespace pg {

struct tables_t {
  uint16_t pack[512];             // base-2 quadrant side -> base-3 digits (precompute.cc:158-172)
  uint16_t unpack[19683][2];      // base-3 quadrant -> (side0, side1)     (precompute.cc:174-197)
  uint16_t rot[512][2];           // [left, right] rotation of a quadrant (precompute.cc:278-296)
  uint16_t refl[512];             // reflection about x = y               (precompute.cc:606-620)
  uint64_t winpat[32];            // five-in-a-row masks                  (precompute.cc:198-253)
  uint16_t rmin_off[56];          // rotation_minimal_quadrants_offsets
  uint16_t rmin_flat[19683];      // rotation_minimal_quadrants_flat (first rmin_count used)
  int rmin_count;
  uint16_t rmin_inv[19683];       // rotation_minimal_quadrants_inverse: q -> 4*index + rotation
  uint16_t rmin_moved[55];        // rotation_minimal_quadrants_reflect_moved
  uint8_t commute[8][256];        // commute_global_local_symmetries: [g][l] = g' l g
  uint8_t gprod[8][8];            // product of global symmetries
  // Super-wins pattern factors, one 64-byte entry per (quadrant, 9-bit side),
  // laid out as described in superscore.cuh (win_factor_entry).
  uint32_t win_factors[4][512][16];
  // OR of win_factors[q][s0 | m] over the empty cells m of a quadrant whose
  // stones are s0 (mover) and s1, indexed by pack[s0] + 2 pack[s1]: the factor
  // of "the mover places one more stone in q", so that the union over all
  // such moves of super_wins costs one evaluation (4 x 19683 x 16 words).
  std::vector<uint32_t> win_union;
  // super_wins as 17 terms per quadrant D: the win patterns that touch D,
  // each with the one or two other quadrants it touches (0xff: none).
  // term_sub[D][v][r] has bit t set when side v of quadrant D, rotated left r
  // times, covers term t's cells in D; cov[p][q][v] bit r likewise for
  // pattern p in quadrant q.
  uint8_t term_pat[4][17];
  uint8_t term_other[4][17][2];
  // The 15 win patterns that miss quadrant D, with the quadrants they touch
  // (0xff pads to three).
  uint8_t miss_pat[4][15];
  uint8_t miss_quad[4][15][3];
  uint32_t term_sub[4][512][4];
  uint8_t cov[32][4][512];
  // 9-bit quadrant sides grouped by stone count: pop_masks[pop_off[k] + r] is
  // the r-th mask with k stones (increasing order) and rank9[mask] = r.
  uint16_t pop_off[11];
  uint16_t pop_masks[512];
  uint8_t rank9[512];
  // Rotation classes of 9-bit quadrant sides, grouped by stone count:
  // cls_masks[cls_off[k] + c] is the smallest mask of the c-th class with k
  // stones, and mask v = rotl^cls_rot[v](cls_masks[cls_off[k] + cls_rank[v]])
  // (rotl = rot[.][0], the least such count).
  uint16_t cls_off[11];
  uint16_t cls_masks[512];
  uint8_t cls_rank[512];
  uint8_t cls_rot[512];
};

// Built once on first use; thread safe.
const tables_t& tables();

// Rotation-minimal list for a (black, white) quadrant count.
inline int rmin_bucket(int b, int w) { return b * (21 - b) / 2 + w; }

}  // namespace pg
