/* CPU restatement of the library's store coder (test infrastructure only:
 * loaded by tests/, never linked by the product).
 *
 * The store coder is the library's own format for solved slices kept in
 * device memory during a sweep (the role of the reference's in-memory block
 * compression, pentago/end/fast_compress.cc, which it does not reproduce), so
 * there is no reference output to match; this file restates its specification
 * independently of the GPU code, rotation by rotation, so that tests can
 * compare the GPU's tables and stream bytes with it.
 *
 * Specification.
 *   Symbols: node = [win, win-or-tie] for the side to move (eight u64, the
 *   supers' bit r is rotation r).  With black = turn ? ~win-or-tie : win and
 *   white = turn ? win : ~win-or-tie, rotation r's symbol is black_r +
 *   2 white_r.
 *   Context of rotation r: c = 256 c0 + 64 c1 + 16 c2 + 4 c3 + cp, where
 *   c_q is the symbol of rotation r - 4^q when the base-4 digit q of r is
 *   non-zero (else 3) and cp is the same rotation's symbol in the previous
 *   node of the lane (3 for a lane's first node).
 *   Lanes: 32 per block; lane l takes nodes [l m, min(n, (l + 1) m)), m =
 *   ceil(n / 32).
 *   Table: counts of (context, symbol) over every stride-th block of the
 *   batch, stride = ceil(nblocks / 2048); per context f_s = floor(count_s
 *   2^14 / sum), at least 1, the difference to 2^14 added to the largest
 *   (the first of equal largest after rounding, in the order 1 over 0, 2 over
 *   1 and 0); a context never seen gets (5462, 5461, 5461).
 *   Coding: byte-wise rANS, state in [2^23, 2^31), 14-bit frequencies,
 *   cumulative frequencies in symbol order.  Each lane codes its nodes from
 *   the last to the first and each node's rotations from 255 to 0, starting
 *   from state 2^23, emitting the low byte while state >= 2^17 f; the lane's
 *   bytes are the emitted bytes in reverse order preceded by the final state
 *   (4 bytes, most significant first).  A lane's bytes may not exceed
 *   64 m + 64 minus 4 before the final state is written; if any lane would,
 *   the block is stored raw.
 *   Stream: 32 lane lengths (u32 little-endian), then the lanes' bytes in
 *   lane order; raw: 0xff x 4, 124 zero bytes, then the nodes as stored.
 */
#include <stdint.h>
#include <string.h>
#include <stdlib.h>

#define SO_LANES 32
#define SO_HEAD (4 * SO_LANES)
#define SO_CTX 1024
#define SO_TOT_BITS 14
#define SO_TOT (1u << SO_TOT_BITS)
#define SO_LOW (1u << 23)
#define SO_TABLE_BLOCKS 2048

static int so_sym(const uint64_t* node, int turn, int r) {
  const uint64_t win = node[r >> 6] >> (r & 63) & 1, nl = node[4 + (r >> 6)] >> (r & 63) & 1;
  const int black = (int)(turn ? !nl : win), white = (int)(turn ? win : !nl);
  return black + 2 * white;
}

static int so_context(const uint64_t* node, const uint64_t* prev, int turn, int r) {
  int c = 0;
  for (int q = 0; q < 4; q++) {
    const int digit = r >> (2 * q) & 3;
    c = 4 * c + (digit ? so_sym(node, turn, r - (1 << (2 * q))) : 3);
  }
  return 4 * c + (prev ? so_sym(prev, turn, r) : 3);
}

static int so_lane_nodes(int n) { return (n + SO_LANES - 1) / SO_LANES; }

int64_t or_store_bound(int64_t n) { return SO_HEAD + (int64_t)SO_LANES * ((int64_t)so_lane_nodes((int)n) * 64 + 64); }

void or_store_table(const uint64_t* nodes, const int64_t* first, const int32_t* count, int nblocks, int turn,
                    uint16_t* table) {
  uint64_t* hist = calloc(3 * SO_CTX, sizeof(uint64_t));
  const int stride = nblocks ? (nblocks + SO_TABLE_BLOCKS - 1) / SO_TABLE_BLOCKS : 1;
  for (int b = 0; b < nblocks; b += stride) {
    const int n = count[b], m = so_lane_nodes(n);
    const uint64_t* base = nodes + 8 * first[b];
    for (int k = 0; k < n; k++) {
      const uint64_t* prev = k % m ? base + 8 * (int64_t)(k - 1) : NULL;
      for (int r = 0; r < 256; r++)
        hist[3 * so_context(base + 8 * (int64_t)k, prev, turn, r) + so_sym(base + 8 * (int64_t)k, turn, r)]++;
    }
  }
  for (int c = 0; c < SO_CTX; c++) {
    const uint64_t* h = hist + 3 * c;
    const uint64_t sum = h[0] + h[1] + h[2];
    uint32_t f[3];
    if (!sum) {
      f[0] = SO_TOT - 2 * (SO_TOT / 3);
      f[1] = f[2] = SO_TOT / 3;
    } else {
      for (int i = 0; i < 3; i++) {
        f[i] = (uint32_t)(h[i] * SO_TOT / sum);
        if (!f[i]) f[i] = 1;
      }
      const int big = f[1] > f[0] ? (f[2] > f[1] ? 2 : 1) : (f[2] > f[0] ? 2 : 0);
      f[big] = (uint32_t)((int32_t)f[big] + (int32_t)SO_TOT - (int32_t)(f[0] + f[1] + f[2]));
    }
    for (int i = 0; i < 3; i++) table[3 * c + i] = (uint16_t)f[i];
  }
  free(hist);
}

/* One block of n nodes into out (room for or_store_bound(n)); returns its size. */
int64_t or_store_encode_block(const uint64_t* nodes, int n, int turn, const uint16_t* table, uint8_t* out) {
  const int m = so_lane_nodes(n);
  const int64_t cap = (int64_t)m * 64 + 64;
  uint8_t* lane_bytes = malloc((size_t)(SO_LANES * cap));
  uint32_t len[SO_LANES];
  int over = 0;
  for (int l = 0; l < SO_LANES && !over; l++) {
    uint8_t* slot = lane_bytes + l * cap;  /* bytes written from slot[cap - 1] downward */
    int64_t used = 0;
    uint32_t state = SO_LOW;
    const int k0 = l * m, k1 = k0 + m < n ? k0 + m : n;
    for (int k = k1 - 1; k >= k0 && !over; k--) {
      const uint64_t* node = nodes + 8 * (int64_t)k;
      const uint64_t* prev = k > k0 ? node - 8 : NULL;
      for (int r = 255; r >= 0 && !over; r--) {
        const int s = so_sym(node, turn, r);
        const int c = so_context(node, prev, turn, r);
        const uint32_t f = table[3 * c + s];
        uint32_t cum = 0;
        for (int i = 0; i < s; i++) cum += table[3 * c + i];
        while (state >= ((SO_LOW >> SO_TOT_BITS) << 8) * f) {
          if (cap - used <= 4) { over = 1; break; }
          slot[cap - 1 - used++] = (uint8_t)state;
          state >>= 8;
        }
        if (!over) state = ((state / f) << SO_TOT_BITS) + state % f + cum;
      }
    }
    if (over) break;
    for (int j = 0; j < 4; j++) slot[cap - 1 - used++] = (uint8_t)(state >> (8 * j));
    len[l] = (uint32_t)used;
  }
  int64_t size;
  if (over) {
    memset(out, 0, SO_HEAD);
    memset(out, 0xff, 4);
    memcpy(out + SO_HEAD, nodes, (size_t)n * 64);
    size = SO_HEAD + (int64_t)n * 64;
  } else {
    size = SO_HEAD;
    for (int l = 0; l < SO_LANES; l++) {
      for (int j = 0; j < 4; j++) out[4 * l + j] = (uint8_t)(len[l] >> (8 * j));
      memcpy(out + size, lane_bytes + l * cap + cap - len[l], len[l]);
      size += len[l];
    }
  }
  free(lane_bytes);
  return size;
}

/* Decode one block; returns n, or -1 for a stream that does not end exactly
 * where its lengths say with the initial state. */
int64_t or_store_decode_block(const uint8_t* in, int64_t size, int n, int turn, const uint16_t* table,
                              uint64_t* nodes) {
  if (size < SO_HEAD) return -1;
  if ((in[0] & in[1] & in[2] & in[3]) == 0xff) {
    if (size != SO_HEAD + (int64_t)n * 64) return -1;
    memcpy(nodes, in + SO_HEAD, (size_t)n * 64);
    return n;
  }
  uint32_t len[SO_LANES];
  int64_t total = 0;
  for (int l = 0; l < SO_LANES; l++) {
    len[l] = (uint32_t)in[4 * l] | (uint32_t)in[4 * l + 1] << 8 | (uint32_t)in[4 * l + 2] << 16 |
             (uint32_t)in[4 * l + 3] << 24;
    total += len[l];
  }
  if (total != size - SO_HEAD) return -1;
  const int m = so_lane_nodes(n);
  const uint8_t* p = in + SO_HEAD;
  for (int l = 0; l < SO_LANES; l++) {
    const uint8_t* end = p + len[l];
    uint32_t state = 0;
    for (int j = 0; j < 4 && p < end; j++) state = state << 8 | *p++;
    const int k0 = l * m, k1 = k0 + m < n ? k0 + m : n;
    /* the lane's nodes are built in the turn-0 form (win = black, win-or-tie
     * = ~white), in which so_sym reads the symbols decoded so far back, and
     * turned into the block's form once the lane is done */
    for (int k = k0; k < k1; k++) {
      uint64_t* node = nodes + 8 * (int64_t)k;
      const uint64_t* prev = k > k0 ? node - 8 : NULL;
      for (int w = 0; w < 4; w++) {
        node[w] = 0;
        node[4 + w] = ~(uint64_t)0;
      }
      for (int r = 0; r < 256; r++) {
        const int c = so_context(node, prev, 0, r);
        const uint32_t slot = state & (SO_TOT - 1);
        const uint32_t f0 = table[3 * c], f1 = table[3 * c + 1], f2 = table[3 * c + 2];
        const int s = slot < f0 ? 0 : slot < f0 + f1 ? 1 : 2;
        const uint32_t f = s == 0 ? f0 : s == 1 ? f1 : f2;
        const uint32_t cum = s == 0 ? 0 : s == 1 ? f0 : f0 + f1;
        state = f * (state >> SO_TOT_BITS) + slot - cum;
        while (state < SO_LOW && p < end) state = state << 8 | *p++;
        if (s & 1) node[r >> 6] |= (uint64_t)1 << (r & 63);
        if (s & 2) node[4 + (r >> 6)] &= ~((uint64_t)1 << (r & 63));
      }
    }
    if (p != end || state != SO_LOW) return -1;
    for (int k = k0; k < k1 && turn; k++) {
      uint64_t* node = nodes + 8 * (int64_t)k;
      for (int w = 0; w < 4; w++) {
        const uint64_t black = node[w], white = ~node[4 + w];
        node[w] = white;
        node[4 + w] = ~black;
      }
    }
  }
  return n;
}
