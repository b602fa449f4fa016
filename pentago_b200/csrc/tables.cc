// Host table generation.  See tables.h.
#include "tables.h"
#include <algorithm>
#include <array>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <vector>

namespace pg {
namespace {

uint16_t qbit(int x, int y) { return uint16_t(1u << (3 * x + y)); }

// A permutation of the 36 cells, composed as (g*h)[i] = g[h[i]].
using perm36 = std::array<uint8_t, 36>;
perm36 pid() { perm36 p; for (int i = 0; i < 36; i++) p[i] = uint8_t(i); return p; }
perm36 pmul(const perm36& g, const perm36& h) { perm36 r; for (int i = 0; i < 36; i++) r[i] = g[h[i]]; return r; }
perm36 pinv(const perm36& g) { perm36 r; for (int i = 0; i < 36; i++) r[g[i]] = uint8_t(i); return r; }

void build(tables_t& T) {
  // Radix-3 packing of one quadrant (two sides of 9 bits each)
  for (int v = 0; v < 512; v++) {
    int pv = 0;
    for (int i = 0, p3 = 1; i < 9; i++, p3 *= 3) if (v >> i & 1) pv += p3;
    T.pack[v] = uint16_t(pv);
  }
  for (int v = 0; v < 19683; v++) {
    uint16_t s[2] = {0, 0};
    for (int i = 0, vv = v; i < 9; i++, vv /= 3)
      if (vv % 3) s[vv % 3 - 1] |= uint16_t(1 << i);
    T.unpack[v][0] = s[0];
    T.unpack[v][1] = s[1];
  }
  // Quadrant rotations (left = counterclockwise) and the x = y reflection
  for (int v = 0; v < 512; v++) {
    uint16_t l = 0, r = 0, f = 0;
    for (int x = 0; x < 3; x++)
      for (int y = 0; y < 3; y++)
        if (v & qbit(x, y)) { l |= qbit(2 - y, x); r |= qbit(y, 2 - x); f |= qbit(2 - y, 2 - x); }
    T.rot[v][0] = l; T.rot[v][1] = r; T.refl[v] = f;
  }
  auto rotl = [&](uint16_t v, int n) { for (int i = 0; i < (n & 3); i++) v = T.rot[v][0]; return v; };
  auto rotr = [&](uint16_t v, int n) { for (int i = 0; i < (n & 3); i++) v = T.rot[v][1]; return v; };

  // The 32 ways to make five in a row, as side masks (order of precompute.cc:212-243)
  {
    auto bit = [](int x, int y, bool flip, bool rotate) {
      if (flip) std::swap(x, y);
      if (rotate) { const int t = 5 - y; y = x; x = t; }
      return uint64_t(1) << (16 * (2 * (x / 3) + y / 3) + 3 * (x % 3) + y % 3);
    };
    int n = 0;
    for (int x = 0; x < 2; x++)
      for (int y = 0; y < 2; y++) {
        uint64_t p = 0;
        for (int i = -2; i < 3; i++) p |= bit(2 + x + i, 2 + y + i * (x == y ? -1 : 1), false, false);
        T.winpat[n++] = p;
      }
    for (bool flip : {false, true})
      for (int x = 0; x < 2; x++)
        for (int y = 0; y < 6; y++) {
          uint64_t p = 0;
          for (int i = 0; i < 5; i++) p |= bit(x + i, y, flip, false);
          T.winpat[n++] = p;
        }
    for (bool rotate : {false, true})
      for (int x = 0; x < 2; x++) {
        uint64_t p = 0;
        for (int i = 0; i < 5; i++) p |= bit(i + x, i + x, false, rotate);
        T.winpat[n++] = p;
      }
  }

  // Rotation-minimal quadrants, ordered so reflected pairs are adjacent and
  // come first within each (black, white) bucket.
  {
    std::vector<uint16_t> minq(19683), all;
    for (int q = 0; q < 19683; q++) {
      uint16_t m = uint16_t(q);
      for (int r = 1; r < 4; r++)
        m = std::min<uint16_t>(m, uint16_t(T.pack[rotl(T.unpack[q][0], r)] + 2 * T.pack[rotl(T.unpack[q][1], r)]));
      minq[q] = m;
      if (m == q) all.push_back(uint16_t(q));
    }
    auto min_reflect = [&](uint16_t q) {
      return minq[T.pack[T.refl[T.unpack[q][0]]] + 2 * T.pack[T.refl[T.unpack[q][1]]]];
    };
    auto key = [&](uint16_t q) { const int r = min_reflect(q); return std::min<int>(q, r) + 19683 * (q == r); };
    std::stable_sort(all.begin(), all.end(), [&](uint16_t a, uint16_t b) { return key(a) < key(b); });
    std::vector<std::vector<uint16_t>> buckets(55);
    for (auto q : all)
      buckets[rmin_bucket(__builtin_popcount(T.unpack[q][0]), __builtin_popcount(T.unpack[q][1]))].push_back(q);
    T.rmin_off[0] = 0;
    int next = 0;
    for (int k = 0; k < 55; k++) {
      int moved = 0;
      for (auto q : buckets[k]) { T.rmin_flat[next++] = q; moved += min_reflect(q) != q; }
      T.rmin_off[k + 1] = uint16_t(next);
      T.rmin_moved[k] = uint16_t(moved);
    }
    T.rmin_count = next;
    std::vector<int> inv(19683, 1 << 20);
    for (int k = 0; k < 55; k++)
      for (int j = 0; j < int(buckets[k].size()); j++) {
        const uint16_t q0 = buckets[k][j];
        for (int r = 0; r < 4; r++) {
          const int q = T.pack[rotl(T.unpack[q0][0], r)] + 2 * T.pack[rotl(T.unpack[q0][1], r)];
          inv[q] = std::min(inv[q], 4 * j + r);
        }
      }
    for (int q = 0; q < 19683; q++) T.rmin_inv[q] = uint16_t(inv[q]);
  }

  // Global/local symmetry algebra as permutations of the 36 cells
  {
    perm36 reflect = pid(), gr = pid();
    for (int x = 0; x < 6; x++)
      for (int y = 0; y < 6; y++) {
        reflect[6 * x + y] = uint8_t(6 * (5 - y) + (5 - x));
        gr[6 * x + y] = uint8_t(6 * (5 - y) + x);
      }
    perm36 plr[4][4];
    for (int q = 0; q < 4; q++) {
      perm36 l = pid();
      const int d = 3 * (6 * (q / 2) + q % 2);
      for (int x = 0; x < 3; x++)
        for (int y = 0; y < 3; y++) l[d + 6 * x + y] = uint8_t(d + 6 * (2 - y) + x);
      plr[q][0] = pid();
      for (int i = 0; i < 3; i++) plr[q][i + 1] = pmul(l, plr[q][i]);
    }
    std::vector<perm36> local(256);
    for (int i = 0; i < 256; i++)
      local[i] = pmul(pmul(plr[0][i >> 6], plr[1][i >> 4 & 3]), pmul(plr[2][i >> 2 & 3], plr[3][i & 3]));
    perm36 global[8];
    global[0] = pid();
    for (int i = 0; i < 3; i++) global[i + 1] = pmul(gr, global[i]);
    for (int i = 0; i < 4; i++) global[4 + i] = pmul(reflect, global[i]);
    for (int g = 0; g < 8; g++)
      for (int l = 0; l < 256; l++) {
        const perm36 c = pmul(pmul(pinv(global[g]), local[l]), global[g]);
        const int k = int(std::find(local.begin(), local.end(), c) - local.begin());
        if (k >= 256) throw std::logic_error("commute table");
        T.commute[g][l] = uint8_t(k);
      }
    for (int a = 0; a < 8; a++)
      for (int b = 0; b < 8; b++) {
        const perm36 c = pmul(global[a], global[b]);
        for (int k = 0; k < 8; k++) if (global[k] == c) T.gprod[a][b] = uint8_t(k);
      }
  }

  // super_wins pattern factors (layout documented in superscore.cuh)
  {
    static const int pair_sets[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    static const int pair_count[6] = {6, 6, 2, 2, 6, 6};
    static const int triple_sets[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    std::vector<int> pats_pair[6], pats_triple[4];
    for (int p = 0; p < 32; p++) {
      int mask = 0;
      for (int q = 0; q < 4; q++) if (T.winpat[p] >> (16 * q) & 0x1ff) mask |= 1 << q;
      for (int s = 0; s < 6; s++)
        if (mask == (1 << pair_sets[s][0] | 1 << pair_sets[s][1])) pats_pair[s].push_back(p);
      for (int s = 0; s < 4; s++)
        if (mask == (1 << triple_sets[s][0] | 1 << triple_sets[s][1] | 1 << triple_sets[s][2])) pats_triple[s].push_back(p);
    }
    for (int s = 0; s < 6; s++)
      if (int(pats_pair[s].size()) != pair_count[s]) throw std::logic_error("win pattern pair sets");
    for (int s = 0; s < 4; s++)
      if (pats_triple[s].size() != 1) throw std::logic_error("win pattern triple sets");
    auto coverage = [&](int p, int q, int v) {
      const uint16_t piece = uint16_t(T.winpat[p] >> (16 * q) & 0x1ff);
      int c = 0;
      for (int r = 0; r < 4; r++) {
        const uint16_t need = rotr(piece, r);  // rotating q left r times covers piece
        if ((v & need) == need) c |= 1 << r;
      }
      return uint32_t(c);
    };
    auto spread = [](uint32_t c) {
      uint32_t s = 0;
      for (int k = 0; k < 4; k++) if (c >> k & 1) s |= 0xfu << (4 * k);
      return s;
    };
    memset(T.win_factors, 0, sizeof T.win_factors);
    for (int q = 0; q < 4; q++)
      for (int v = 0; v < 512; v++) {
        uint32_t* e = T.win_factors[q][v];
        int h = 0;
        for (int s = 0; s < 6; s++) {
          const int a = pair_sets[s][0], b = pair_sets[s][1];
          if (q != a && q != b) continue;
          for (int p : pats_pair[s]) {
            const uint32_t c = coverage(p, q, v);
            const uint32_t f = q == a ? c * 0x1111u : spread(c);
            e[h >> 1] |= f << (16 * (h & 1));
            h++;
          }
        }
        if (h != 14) throw std::logic_error("win factor halfwords");
        int w = 7;
        for (int s = 0; s < 4; s++) {
          const int* t = triple_sets[s];
          if (q != t[0] && q != t[1] && q != t[2]) continue;
          const uint32_t c = coverage(pats_triple[s][0], q, v);
          uint64_t f;
          if (q == t[0]) f = uint64_t(c) * 0x1111111111111111ull;
          else if (q == t[1]) f = uint64_t(spread(c)) * 0x0001000100010001ull;
          else {
            f = 0;
            for (int k = 0; k < 4; k++) if (c >> k & 1) f |= uint64_t(0xffff) << (16 * k);
          }
          e[w] = uint32_t(f);
          e[w + 1] = uint32_t(f >> 32);
          w += 2;
        }
      }
    // Terms per quadrant
    for (int p = 0; p < 32; p++)
      for (int q = 0; q < 4; q++)
        for (int v = 0; v < 512; v++) T.cov[p][q][v] = uint8_t(coverage(p, q, v));
    memset(T.term_sub, 0, sizeof T.term_sub);
    for (int d = 0; d < 4; d++) {
      int t = 0;
      for (int p = 0; p < 32; p++) {
        if (!(T.winpat[p] >> (16 * d) & 0x1ff)) continue;
        if (t >= 17) throw std::logic_error("win pattern terms");
        T.term_pat[d][t] = uint8_t(p);
        int k = 0;
        T.term_other[d][t][0] = T.term_other[d][t][1] = 0xff;
        for (int q = 0; q < 4; q++)
          if (q != d && (T.winpat[p] >> (16 * q) & 0x1ff)) T.term_other[d][t][k++] = uint8_t(q);
        for (int v = 0; v < 512; v++)
          for (int r = 0; r < 4; r++)
            if (T.cov[p][d][v] >> r & 1) T.term_sub[d][v][r] |= 1u << t;
        t++;
      }
      if (t != 17) throw std::logic_error("win pattern terms");
      int u = 0;
      for (int p = 0; p < 32; p++) {
        if (T.winpat[p] >> (16 * d) & 0x1ff) continue;
        if (u >= 15) throw std::logic_error("win patterns missing a quadrant");
        T.miss_pat[d][u] = uint8_t(p);
        int k = 0;
        for (int j = 0; j < 3; j++) T.miss_quad[d][u][j] = 0xff;
        for (int q = 0; q < 4; q++)
          if (T.winpat[p] >> (16 * q) & 0x1ff) T.miss_quad[d][u][k++] = uint8_t(q);
        u++;
      }
      if (u != 15) throw std::logic_error("win patterns missing a quadrant");
    }
  }
}

void build_pop(tables_t& T) {
  int next = 0;
  for (int k = 0; k <= 9; k++) {
    T.pop_off[k] = uint16_t(next);
    int r = 0;
    for (int m = 0; m < 512; m++)
      if (__builtin_popcount(m) == k) { T.pop_masks[next++] = uint16_t(m); T.rank9[m] = uint8_t(r++); }
  }
  T.pop_off[10] = uint16_t(next);
  // Rotation classes: each represented by its smallest mask
  auto rep_of = [&](int m) {
    int rep = m, v = m;
    for (int i = 1; i < 4; i++) { v = T.rot[v][0]; rep = std::min(rep, v); }
    return rep;
  };
  next = 0;
  for (int k = 0; k <= 9; k++) {
    T.cls_off[k] = uint16_t(next);
    int r = 0;
    for (int m = 0; m < 512; m++)
      if (__builtin_popcount(m) == k && rep_of(m) == m) { T.cls_masks[next++] = uint16_t(m); T.cls_rank[m] = uint8_t(r++); }
  }
  T.cls_off[10] = uint16_t(next);
  for (int m = 0; m < 512; m++) {
    const int rep = rep_of(m);
    int v = rep, rho = 0;
    while (v != m) { v = T.rot[v][0]; rho++; }
    T.cls_rank[m] = T.cls_rank[rep];
    T.cls_rot[m] = uint8_t(rho);
  }
}

void build_union(tables_t& T) {
  T.win_union.assign(size_t(4) * 19683 * 16, 0);
  for (int q = 0; q < 4; q++)
    for (int t = 0; t < 19683; t++) {
      const int s0 = T.unpack[t][0], s1 = T.unpack[t][1];
      uint32_t* e = &T.win_union[(size_t(q) * 19683 + t) * 16];
      for (int m = 0; m < 9; m++)
        if (!((s0 | s1) >> m & 1))
          for (int w = 0; w < 16; w++) e[w] |= T.win_factors[q][s0 | 1 << m][w];
    }
}

}  // namespace

const tables_t& tables() {
  static std::once_flag once;
  static std::unique_ptr<tables_t> t;
  std::call_once(once, [] {
    t.reset(new tables_t);
    build(*t);
    build_union(*t);
    build_pop(*t);
  });
  return *t;
}

}  // namespace pg
