/* CPU oracle for the pentago hot path.  TEST INFRASTRUCTURE ONLY: imported by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
 * checker; never linked or called by the product library.
 *
 * A plain-C restatement of the reference algorithms, written definitionally
 * where that is cheap (rmax, super_wins and transform_super loop over the 256
 * rotations instead of using the reference's bit tricks), and step by step
 * where the reference defines a storage convention (line layout, subset
 * indexing).  Each function cites the reference file:line it restates.
 * Parity is pinned in tests: table SHA-1s from pentago/base/precompute.cc,
 * the reference engine compiled in place (oracle/_ref), and the reference's
 * golden vectors.
 */
#include "pentago_oracle.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

typedef uint64_t u64;
typedef uint32_t u32;
typedef uint16_t u16;
typedef uint8_t u8;

/* ------------------------------------------------------------------------ */
/* Tables (pentago/base/precompute.cc)                                        */
/* ------------------------------------------------------------------------ */

static u16 T_pack[512];             /* precompute.cc:158-172 */
static u16 T_unpack[19683][2];      /* precompute.cc:174-197 */
static u16 T_rot[512][2];           /* precompute.cc:278-296: [left, right] */
static u16 T_refl[512];             /* precompute.cc:606-620 */
static u64 T_winpat[32];            /* precompute.cc:198-253 */
static u16 T_rmin_off[56];          /* precompute.cc:967-1043 */
static u16 T_rmin_flat[19683];
static int T_rmin_count;
static u16 T_rmin_inv[19683];
static u16 T_rmin_moved[55];
static u8 T_commute[8][256];        /* precompute.cc:883-931 */
static u8 T_gprod[8][8];            /* global part of symmetry_t product */
static int initialized = 0;

static u16 qbit(int x, int y) { return (u16)(1u << (3 * x + y)); }

static u16 rot_left_n(u16 v, int r) {
  for (int i = 0; i < (r & 3); i++) v = T_rot[v][0];
  return v;
}

static int popc64(u64 x) { return __builtin_popcountll(x); }

/* Sym: a permutation of the 36 board cells, (g*h).p[i] = g.p[h.p[i]]
 * (precompute.cc:822-881). */
typedef struct { u8 p[36]; } sym36;

static sym36 sym_id(void) { sym36 s; for (int i = 0; i < 36; i++) s.p[i] = (u8)i; return s; }
static sym36 sym_mul(sym36 g, sym36 h) { sym36 r; for (int i = 0; i < 36; i++) r.p[i] = g.p[h.p[i]]; return r; }
static sym36 sym_inv(sym36 g) { sym36 r; for (int i = 0; i < 36; i++) r.p[g.p[i]] = (u8)i; return r; }
static int sym_eq(sym36 a, sym36 b) { return !memcmp(a.p, b.p, 36); }

static void build_tables(void) {
  /* pack / unpack */
  for (int v = 0; v < 512; v++) {
    int pv = 0, p3 = 1;
    for (int i = 0; i < 9; i++, p3 *= 3) if (v >> i & 1) pv += p3;
    T_pack[v] = (u16)pv;
  }
  for (int v = 0; v < 19683; v++) {
    int vv = v; u16 p0 = 0, p1 = 0;
    for (int i = 0; i < 9; i++) {
      const int c = vv % 3; vv /= 3;
      if (c == 1) p0 |= (u16)(1 << i); else if (c == 2) p1 |= (u16)(1 << i);
    }
    T_unpack[v][0] = p0; T_unpack[v][1] = p1;
  }
  /* rotations and reflections of one 3x3 quadrant */
  for (int v = 0; v < 512; v++) {
    u16 left = 0, right = 0, refl = 0;
    for (int x = 0; x < 3; x++)
      for (int y = 0; y < 3; y++)
        if (v & qbit(x, y)) {
          left |= qbit(2 - y, x);
          right |= qbit(y, 2 - x);
          refl |= qbit(2 - y, 2 - x);
        }
    T_rot[v][0] = left; T_rot[v][1] = right; T_refl[v] = refl;
  }
  /* 32 five-in-a-row patterns as side_t masks */
  {
    int n = 0;
#define BIT(X, Y, FLIP, ROT) ({ int _x = (X), _y = (Y); if (FLIP) { int t = _x; _x = _y; _y = t; } \
      if (ROT) { int t = 5 - _y; _y = _x; _x = t; } (u64)1 << (16 * (2 * (_x / 3) + _y / 3) + 3 * (_x % 3) + _y % 3); })
    for (int x = 0; x < 2; x++)
      for (int y = 0; y < 2; y++) {
        u64 p = 0;
        for (int i = -2; i < 3; i++) p |= BIT(2 + x + i, 2 + y + i * (x == y ? -1 : 1), 0, 0);
        T_winpat[n++] = p;
      }
    for (int flip = 0; flip < 2; flip++)
      for (int x = 0; x < 2; x++)
        for (int y = 0; y < 6; y++) {
          u64 p = 0;
          for (int i = 0; i < 5; i++) p |= BIT(x + i, y, flip, 0);
          T_winpat[n++] = p;
        }
    for (int rot = 0; rot < 2; rot++)
      for (int x = 0; x < 2; x++) {
        u64 p = 0;
        for (int i = 0; i < 5; i++) p |= BIT(i + x, i + x, 0, rot);
        T_winpat[n++] = p;
      }
#undef BIT
  }
  /* rotation minimal quadrants (precompute.cc:967-1043) */
  {
    static u16 minq[19683], all[19683];
    int nall = 0;
    for (int q = 0; q < 19683; q++) {
      const u16 s0 = T_unpack[q][0], s1 = T_unpack[q][1];
      u16 m = (u16)q;
      for (int r = 1; r < 4; r++) {
        const u16 v = (u16)(T_pack[rot_left_n(s0, r)] + 2 * T_pack[rot_left_n(s1, r)]);
        if (v < m) m = v;
      }
      minq[q] = m;
      if (m == q) all[nall++] = (u16)q;
    }
#define MIN_REFLECT(q) (minq[T_pack[T_refl[T_unpack[q][0]]] + 2 * T_pack[T_refl[T_unpack[q][1]]]])
    /* stable sort by sig(q) = min(q, reflect(q)) + 3^9 * (q == reflect(q)) */
    static int key[19683];
    for (int i = 0; i < nall; i++) {
      const int q = all[i], r = MIN_REFLECT(q);
      key[i] = (q < r ? q : r) + 19683 * (q == r);
    }
    for (int i = 1; i < nall; i++) { /* insertion sort: stable */
      const u16 q = all[i]; const int k = key[i]; int j = i - 1;
      while (j >= 0 && key[j] > k) { all[j + 1] = all[j]; key[j + 1] = key[j]; j--; }
      all[j + 1] = q; key[j + 1] = k;
    }
    /* bucket by counts b*(21-b)/2 + w */
    int counts[55] = {0}, seen[55] = {0};
    for (int i = 0; i < nall; i++) {
      const int b = __builtin_popcount(T_unpack[all[i]][0]), w = __builtin_popcount(T_unpack[all[i]][1]);
      counts[b * (21 - b) / 2 + w]++;
    }
    T_rmin_off[0] = 0;
    for (int i = 0; i < 55; i++) T_rmin_off[i + 1] = (u16)(T_rmin_off[i] + counts[i]);
    for (int i = 0; i < nall; i++) {
      const int b = __builtin_popcount(T_unpack[all[i]][0]), w = __builtin_popcount(T_unpack[all[i]][1]);
      const int k = b * (21 - b) / 2 + w;
      T_rmin_flat[T_rmin_off[k] + seen[k]++] = all[i];
    }
    T_rmin_count = nall;
    for (int k = 0; k < 55; k++) {
      int m = 0;
      for (int j = T_rmin_off[k]; j < T_rmin_off[k + 1]; j++) m += MIN_REFLECT(T_rmin_flat[j]) != T_rmin_flat[j];
      T_rmin_moved[k] = (u16)m;
    }
    static int inv[19683];
    for (int q = 0; q < 19683; q++) inv[q] = 1 << 20;
    for (int k = 0; k < 55; k++)
      for (int j = 0; j < T_rmin_off[k + 1] - T_rmin_off[k]; j++) {
        const u16 q0 = T_rmin_flat[T_rmin_off[k] + j];
        for (int r = 0; r < 4; r++) {
          const int q = T_pack[rot_left_n(T_unpack[q0][0], r)] + 2 * T_pack[rot_left_n(T_unpack[q0][1], r)];
          if (4 * j + r < inv[q]) inv[q] = 4 * j + r;
        }
      }
    for (int q = 0; q < 19683; q++) T_rmin_inv[q] = (u16)inv[q];
#undef MIN_REFLECT
  }
  /* commute_global_local_symmetries: table[g][l] = local index of g' l g */
  {
    sym36 reflect = sym_id(), gr = sym_id(), lr[4], plr[4][4], global[8];
    for (int x = 0; x < 6; x++)
      for (int y = 0; y < 6; y++) {
        reflect.p[6 * x + y] = (u8)(6 * (5 - y) + (5 - x));
        gr.p[6 * x + y] = (u8)(6 * (5 - y) + x);
      }
    for (int q = 0; q < 4; q++) {
      lr[q] = sym_id();
      const int d = 3 * (6 * (q / 2) + q % 2);
      for (int x = 0; x < 3; x++)
        for (int y = 0; y < 3; y++) lr[q].p[d + 6 * x + y] = (u8)(d + 6 * (2 - y) + x);
      plr[q][0] = sym_id();
      for (int i = 0; i < 3; i++) plr[q][i + 1] = sym_mul(lr[q], plr[q][i]);
    }
    static sym36 local[256];
    for (int i0 = 0; i0 < 4; i0++)
      for (int i1 = 0; i1 < 4; i1++)
        for (int i2 = 0; i2 < 4; i2++)
          for (int i3 = 0; i3 < 4; i3++)
            local[((i0 * 4 + i1) * 4 + i2) * 4 + i3] =
                sym_mul(sym_mul(plr[0][i0], plr[1][i1]), sym_mul(plr[2][i2], plr[3][i3]));
    global[0] = sym_id();
    for (int i = 0; i < 3; i++) global[i + 1] = sym_mul(gr, global[i]);
    for (int i = 0; i < 4; i++) global[4 + i] = sym_mul(reflect, global[i]);
    for (int g = 0; g < 8; g++)
      for (int l = 0; l < 256; l++) {
        const sym36 c = sym_mul(sym_mul(sym_inv(global[g]), local[l]), global[g]);
        int found = -1;
        for (int k = 0; k < 256 && found < 0; k++) if (sym_eq(local[k], c)) found = k;
        T_commute[g][l] = (u8)found;
      }
    for (int a = 0; a < 8; a++)
      for (int b = 0; b < 8; b++) {
        const sym36 c = sym_mul(global[a], global[b]);
        for (int k = 0; k < 8; k++) if (sym_eq(global[k], c)) T_gprod[a][b] = (u8)k;
      }
  }
}

int or_init(void) {
  if (!initialized) { build_tables(); initialized = 1; }
  return 0;
}

const void* or_table(const char* name, int* bytes) {
  or_init();
#define T(n, x) if (!strcmp(name, n)) { *bytes = (int)sizeof(x); return (const void*)&x; }
  T("pack_table", T_pack) T("unpack_table", T_unpack) T("rotations", T_rot) T("reflections", T_refl)
  T("rotation_minimal_quadrants_offsets", T_rmin_off) T("rotation_minimal_quadrants_inverse", T_rmin_inv)
  T("rotation_minimal_quadrants_reflect_moved", T_rmin_moved) T("commute_global_local_symmetries", T_commute)
  T("win_patterns", T_winpat)
#undef T
  if (!strcmp(name, "rotation_minimal_quadrants_flat")) { *bytes = 2 * T_rmin_count; return T_rmin_flat; }
  *bytes = 0;
  return NULL;
}

/* ------------------------------------------------------------------------ */
/* Boards and supers (pentago/base/board.h, superscore.h, symmetry.h)        */
/* ------------------------------------------------------------------------ */

typedef struct { u64 w[4]; } super;

static int sget(const super* s, int r) { return (int)(s->w[r >> 6] >> (r & 63) & 1); }
static void sset(super* s, int r) { s->w[r >> 6] |= (u64)1 << (r & 63); }
static super szero(void) { super s; memset(&s, 0, sizeof s); return s; }
static super snot(super a) { for (int i = 0; i < 4; i++) a.w[i] = ~a.w[i]; return a; }
static super sor(super a, super b) { for (int i = 0; i < 4; i++) a.w[i] |= b.w[i]; return a; }
static super sand(super a, super b) { for (int i = 0; i < 4; i++) a.w[i] &= b.w[i]; return a; }

static u16 quadrant(u64 s, int q) { return (u16)(s >> (16 * q) & 0xffff); }

/* side with each quadrant q rotated left by (r >> 2q) & 3 */
static u64 rotate_side_local(u64 side, int r) {
  u64 out = 0;
  for (int q = 0; q < 4; q++) out |= (u64)rot_left_n(quadrant(side, q), r >> (2 * q) & 3) << (16 * q);
  return out;
}

/* five in a row: pentago/base/score.h:39-54 */
static int won(u64 side) {
  for (int i = 0; i < 32; i++) if ((side & T_winpat[i]) == T_winpat[i]) return 1;
  return 0;
}

/* super_wins (pentago/base/superscore.cc:38-96), by definition: the set of
 * local rotations after which `side` has five in a row. */
static super super_wins(u64 side) {
  super s = szero();
  for (int r = 0; r < 256; r++) if (won(rotate_side_local(side, r))) sset(&s, r);
  return s;
}

/* rmax(f)(a) = max over the 8 single rotations b of f(a+b)
 * (pentago/base/superscore.h:10-16, :264-306). */
static int radd(int a, int q, int d) { /* add d to coordinate q of index a, mod 4 */
  const int c = (a >> (2 * q) & 3);
  return (a & ~(3 << (2 * q))) | (((c + d) & 3) << (2 * q));
}
static super rmax(super f) {
  super s = szero();
  for (int a = 0; a < 256; a++)
    for (int q = 0; q < 4 && !sget(&s, a); q++)
      if (sget(&f, radd(a, q, 1)) || sget(&f, radd(a, q, 3))) sset(&s, a);
  return s;
}

/* symmetry_t = (global 3 bits, local 8 bits), product per
 * pentago/base/symmetry.h:83-100: (ag al)(bg bl) = ag bg (bg' al bg) bl. */
typedef struct { int g, l; } sym_t;
static int ladd(int a, int b) { /* componentwise add of two local fields mod 4 */
  return (((a & 0x33) + (b & 0x33)) & 0x33) + (((a & 0xcc) + (b & 0xcc)) & 0xcc);
}
static int lneg(int a) { int r = 0; for (int q = 0; q < 4; q++) r |= ((4 - (a >> 2 * q & 3)) & 3) << 2 * q; return r; }
static sym_t smul(sym_t a, sym_t b) {
  sym_t r;
  r.g = T_gprod[a.g][b.g];
  r.l = ladd(T_commute[b.g][a.l], b.l);
  return r;
}
static int ginv(int g) { for (int h = 0; h < 8; h++) if (T_gprod[g][h] == 0) return h; return -1; }

/* transform_super (pentago/base/symmetry.h:103-112): for s = g y,
 * s(C) = { g z y' g' : z in C }, and g w g' = commute[g^-1][w]. */
static super transform_super(sym_t s, super c) {
  super out = szero();
  const int gi = ginv(s.g);
  for (int z = 0; z < 256; z++)
    if (sget(&c, z)) sset(&out, T_commute[gi][ladd(z, lneg(s.l))]);
  return out;
}

/* halfsuper split by parity (pentago/mid/halfsuper.h:4-60):
 * h(p)(a,b,c,d) = s(2a + (b+c+d+p)%2, b, c, d), h index a + 2b + 8c + 32d. */
typedef struct { u64 w[2]; } half;
static half split(super s, int p) {
  half h = {{0, 0}};
  for (int i = 0; i < 128; i++) {
    const int a = i & 1, b = i >> 1 & 3, c = i >> 3 & 3, d = i >> 5 & 3;
    const int r = (2 * a + ((b + c + d + p) & 1)) + 4 * b + 16 * c + 64 * d;
    if (sget(&s, r)) h.w[i >> 6] |= (u64)1 << (i & 63);
  }
  return h;
}
static super merge(half h, int p) { /* inverse of split on parity-p support */
  super s = szero();
  for (int i = 0; i < 128; i++)
    if (h.w[i >> 6] >> (i & 63) & 1) {
      const int a = i & 1, b = i >> 1 & 3, c = i >> 3 & 3, d = i >> 5 & 3;
      sset(&s, (2 * a + ((b + c + d + p) & 1)) + 4 * b + 16 * c + 64 * d);
    }
  return s;
}
static half hnot(half a) { a.w[0] = ~a.w[0]; a.w[1] = ~a.w[1]; return a; }
static half hor(half a, half b) { a.w[0] |= b.w[0]; a.w[1] |= b.w[1]; return a; }
static half hand(half a, half b) { a.w[0] &= b.w[0]; a.w[1] &= b.w[1]; return a; }
static half hwins(u64 side, int parity) { return split(super_wins(side), parity); }
/* halfsuper rmax flips parity (pentago/mid/halfsuper.h:150-203) */
static half hrmax(half h) { return split(rmax(merge(h, 0)), 1); }

void or_rmax(const u64* in, u64* out, int n) {
  or_init();
  for (int i = 0; i < n; i++) { super s; memcpy(&s, in + 4 * i, 32); s = rmax(s); memcpy(out + 4 * i, &s, 32); }
}
void or_super_wins(const u64* sides, u64* out, int n) {
  or_init();
  for (int i = 0; i < n; i++) { super s = super_wins(sides[i]); memcpy(out + 4 * i, &s, 32); }
}
void or_transform_super(const u16* syms, const u64* in, u64* out, int n) {
  or_init();
  for (int i = 0; i < n; i++) {
    super s; memcpy(&s, in + 4 * i, 32);
    const sym_t t = {syms[i] >> 8, syms[i] & 255};
    s = transform_super(t, s);
    memcpy(out + 4 * i, &s, 32);
  }
}
void or_symmetry_product(const u16* a, const u16* b, u16* out, int n) {
  or_init();
  for (int i = 0; i < n; i++) {
    const sym_t x = {a[i] >> 8, a[i] & 255}, y = {b[i] >> 8, b[i] & 255};
    const sym_t p = smul(x, y);
    out[i] = (u16)(p.g << 8 | p.l);
  }
}
void or_halfsuper_wins(const u64* sides, const u8* parity, u64* out, int n) {
  or_init();
  for (int i = 0; i < n; i++) { half h = hwins(sides[i], parity[i]); memcpy(out + 2 * i, &h, 16); }
}
void or_halfsuper_rmax(const u64* in, u64* out, int n) {
  or_init();
  for (int i = 0; i < n; i++) { half h; memcpy(&h, in + 2 * i, 16); h = hrmax(h); memcpy(out + 2 * i, &h, 16); }
}

/* ------------------------------------------------------------------------ */
/* Sections (pentago/base/section.h, section.cc)                            */
/* ------------------------------------------------------------------------ */

typedef struct { u8 c[4][2]; } section;

static section sec_from_sig(u64 sig) {
  section s;
  for (int q = 0; q < 4; q++) for (int k = 0; k < 2; k++) s.c[q][k] = (u8)(sig >> (16 * q + 8 * k));
  return s;
}
static u64 sec_sig(section s) {
  u64 r = 0;
  for (int q = 0; q < 4; q++) for (int k = 0; k < 2; k++) r |= (u64)s.c[q][k] << (16 * q + 8 * k);
  return r;
}
static int sec_sum(section s) { int t = 0; for (int q = 0; q < 4; q++) t += s.c[q][0] + s.c[q][1]; return t; }
static int rmin_bucket(int b, int w) { return b * (21 - b) / 2 + w; }
static int rmin_size(int b, int w) { const int k = rmin_bucket(b, w); return T_rmin_off[k + 1] - T_rmin_off[k]; }
static const u16* rmin_list(int b, int w) { return T_rmin_flat + T_rmin_off[rmin_bucket(b, w)]; }
static int rmin_moved(int b, int w) { return T_rmin_moved[rmin_bucket(b, w)]; }
static void sec_shape(section s, int* shape) { for (int q = 0; q < 4; q++) shape[q] = rmin_size(s.c[q][0], s.c[q][1]); }

/* section_t::transform (section.cc:78-86) */
static section sec_transform(section s, int g) {
  static const int source[4][4] = {{0, 1, 2, 3}, {1, 3, 0, 2}, {3, 2, 1, 0}, {2, 0, 3, 1}};
  section t;
  const int r = g & 3;
  for (int i = 0; i < 4; i++) for (int k = 0; k < 2; k++) t.c[i][k] = s.c[source[r][i]][k];
  if (g & 4) for (int k = 0; k < 2; k++) { u8 x = t.c[0][k]; t.c[0][k] = t.c[3][k]; t.c[3][k] = x; }
  return t;
}
/* section_t::standardize<8> (section.cc:88-101) */
static section sec_standardize(section s, int* best_g) {
  section best = s; int bg = 0;
  for (int g = 1; g < 8; g++) {
    const section t = sec_transform(s, g);
    if (sec_sig(best) > sec_sig(t)) { best = t; bg = g; }
  }
  if (best_g) *best_g = bg;
  return best;
}
static section sec_child(section s, int q) { s.c[q][sec_sum(s) & 1]++; return s; }
/* section_t::quadrant_permutation (section.cc:106-114): quadrant i maps to p[i] */
static void quadrant_permutation(int g, int* p) {
  section s; memset(&s, 0, sizeof s);
  for (int i = 0; i < 4; i++) s.c[i][0] = (u8)i;
  const section t = sec_transform(s, g);
  for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) if (t.c[j][0] == i && t.c[j][1] == 0) p[i] = j;
}
static int invert_global(int g) { return g ^ ((~g >> 2 & (g & 1)) << 1); }  /* symmetry.h:53-55 */

int or_section_shape(u64 sig, int* shape4) { or_init(); sec_shape(sec_from_sig(sig), shape4); return 0; }
u64 or_standardize_section(u64 sig, int* transform) { or_init(); return sec_sig(sec_standardize(sec_from_sig(sig), transform)); }

/* ------------------------------------------------------------------------ */
/* End engine line compute (pentago/end/compute.cc)                          */
/* ------------------------------------------------------------------------ */

static int imin(int a, int b) { return a < b ? a : b; }
static int bshape(int shape, int block) { return imin(shape, 8 * (block + 1)) - 8 * block; }  /* end/blocks.h:15-18 */

typedef struct {
  section sec; int dim, length; int block0[4];
  int in_shape[4], out_shape[4];
  int block_stride;
  section child_std; int st; int perm[4]; int child_dim; int input_blocks;
  int first_child_block[4];
  sym_t inverse_transform;
  const u16* rmin[4];
  int refl_moves[4];
  int rs_off[5]; int* rsyms;
} line_info;

/* line_data_t (compute.cc:24-46) and line_details_t (compute.cc:55-123) */
static void line_setup(line_info* L, u64 sig, int dim, int length, const u8* block_base) {
  memset(L, 0, sizeof *L);
  L->sec = sec_from_sig(sig); L->dim = dim; L->length = length;
  for (int i = 0, k = 0; i < 4; i++) L->block0[i] = i == dim ? 0 : block_base[k++];
  int shape[4], cshape[4];
  sec_shape(L->sec, shape);
  const section child = sec_child(L->sec, dim);
  sec_shape(child, cshape);
  for (int i = 0; i < 4; i++) L->out_shape[i] = i == dim ? shape[i] : bshape(shape[i], L->block0[i]);
  for (int i = 0; i < 4; i++) L->in_shape[i] = i == dim ? cshape[i] : L->out_shape[i];
  if (sec_sum(L->sec) == 35) for (int i = 0; i < 4; i++) L->in_shape[i] = 0;
  L->block_stride = 8;
  for (int i = 0; i < 4; i++) if (i != dim) L->block_stride *= bshape(shape[i], L->block0[i]);
  L->child_std = sec_standardize(child, &L->st);
  quadrant_permutation(invert_global(L->st), L->perm);
  for (int i = 0; i < 4; i++) if (L->perm[i] == dim) L->child_dim = i;
  L->input_blocks = (L->in_shape[dim] + 7) / 8;
  for (int i = 0; i < 4; i++) L->first_child_block[i] = L->block0[L->perm[i]];
  {
    const int st = L->st;
    const sym_t a = {(4 - (st & 3)) & 3, 0x55 * (st & 3)}, b = {st & 4, 0};
    L->inverse_transform = smul(a, b);
  }
  for (int q = 0; q < 4; q++) L->rmin[q] = rmin_list(L->sec.c[q][0], L->sec.c[q][1]);
  if (L->st & 4)
    for (int i = 0; i < 4; i++) L->refl_moves[i] = rmin_moved(L->child_std.c[i][0], L->child_std.c[i][1]);
  int sis[4], total = 0;
  for (int i = 0; i < 4; i++) { sis[i] = L->in_shape[L->perm[i]]; total += sis[i]; }
  L->rsyms = (int*)calloc(total + 1, sizeof(int));
  L->rs_off[0] = 0;
  for (int i = 0; i < 4; i++) {
    L->rs_off[i + 1] = L->rs_off[i] + sis[i];
    if (L->st & 4) {
      const u16* crmin = rmin_list(L->child_std.c[i][0], L->child_std.c[i][1]);
      for (int j = 0; j < sis[i]; j++) {
        const u16 q = crmin[8 * L->first_child_block[i] + j];
        const int rq = T_pack[T_refl[T_unpack[q][0]]] + 2 * T_pack[T_refl[T_unpack[q][1]]];
        L->rsyms[L->rs_off[i] + j] = (T_rmin_inv[rq] & 3) << (2 * i);
      }
    }
  }
}

static void strides4(const int* shape, int* st) {
  st[3] = 1;
  for (int i = 2; i >= 0; i--) st[i] = st[i + 1] * shape[i + 1];
}

/* compute_microline (compute.cc:219-371); input/output packed (block step =
 * block_stride, the reference uses block_stride + 1 for compressed receives). */
static void compute_microline(const line_info* L, const int* base3, const u64* input, u64* output) {
  const int dim = L->dim, child_dim = L->child_dim;
  const int slice35 = sec_sum(L->sec) == 35;
  int full_base[4];
  for (int i = 0, k = 0; i < 4; i++) full_base[i] = i == dim ? 0 : base3[k++];
  int first_node[4];
  for (int i = 0; i < 4; i++) first_node[i] = 8 * L->block0[i] + full_base[i];
  u16 bq[4];
  for (int q = 0; q < 4; q++) bq[q] = q == dim ? 0 : L->rmin[q][first_node[q]];
  const int turn = sec_sum(L->sec) & 1;
  u64 base_side0 = 0, base_side1 = 0;
  for (int q = 0; q < 4; q++) {
    base_side0 |= (u64)T_unpack[bq[q]][turn] << (16 * q);
    base_side1 |= (u64)T_unpack[bq[q]][1 - turn] << (16 * q);
  }
  const int nrmin = L->out_shape[dim];
  const int shift = 16 * dim;

  int obs[4], obst[4];
  for (int i = 0; i < 4; i++) obs[i] = L->out_shape[i];
  obs[dim] = 8;
  strides4(obs, obst);
  const int output_stride = obst[dim];
  int output_base = 0;
  for (int i = 0; i < 4; i++) output_base += obst[i] * full_base[i];

  int ibs[4], ibst[4], fcb[4], fcn[4], rcb[4];
  for (int i = 0; i < 4; i++) ibs[i] = obs[L->perm[i]];
  strides4(ibs, ibst);
  const int input_stride = ibst[child_dim];
  for (int i = 0; i < 4; i++) fcb[i] = full_base[L->perm[i]];
  for (int i = 0; i < 4; i++) fcn[i] = 8 * L->first_child_block[i] + fcb[i];
  for (int i = 0; i < 4; i++) rcb[i] = fcb[i] ^ (child_dim != i && fcn[i] < L->refl_moves[i]);
  int input_base = 0;
  for (int i = 0; i < 4; i++) input_base += ibst[i] * rcb[i];
  const int line_moves = L->refl_moves[child_dim];

  obs[dim] = (nrmin & 7) ? (nrmin & 7) : 8;
  strides4(obs, obst);
  int last_output_base = 0;
  for (int i = 0; i < 4; i++) last_output_base += obst[i] * full_base[i];
  ibs[child_dim] = (L->in_shape[dim] & 7) ? (L->in_shape[dim] & 7) : 8;
  strides4(ibs, ibst);
  int last_input_base = 0;
  for (int i = 0; i < 4; i++) last_input_base += ibst[i] * rcb[i];

  int local = 0;
  if (L->rs_off[4])
    for (int i = 0; i < 4; i++) if (i != child_dim) local += L->rsyms[L->rs_off[i] + fcb[i]];
  const sym_t lsym = {0, local};
  const sym_t base_transform = smul(L->inverse_transform, lsym);
  const int* syms = L->rsyms + L->rs_off[child_dim];

  for (int i = 0; i < nrmin; i++) {
    const u16 q = L->rmin[dim][i];
    const u16 sq0 = T_unpack[q][turn], sq1 = T_unpack[q][1 - turn];
    const u64 side0 = base_side0 | (u64)sq0 << shift, side1 = base_side1 | (u64)sq1 << shift;
    const super wins0 = super_wins(side0), wins1 = super_wins(side1);
    const super immediate = sor(wins0, wins1);
    super wins = szero(), not_loss = szero();
    for (int b = 0; b < 9; b++) {
      if ((sq0 | sq1) >> b & 1) continue;
      const u16 move = (u16)(1 << b);
      const super new_wins = super_wins(side0 | (u64)move << shift);
      wins = sor(wins, new_wins);
      if (slice35) {
        wins = sor(wins, rmax(sand(new_wins, snot(wins1))));
        not_loss = sor(not_loss, rmax(sor(new_wins, snot(wins1))));
      } else {
        const int new_q = q + (1 + turn) * T_pack[move];
        const int ir = T_rmin_inv[new_q];
        const int j = ir / 4;
        const sym_t lr = {0, (ir & 3) << (2 * dim)}, lj = {0, syms[j]};
        const sym_t s = smul(smul(lr, base_transform), lj);
        const int jj = j ^ (j < line_moves);
        const int blk = j >> 3;
        const long idx = (long)((blk == L->input_blocks - 1) ? last_input_base : input_base) +
                         (long)L->block_stride * blk + (long)input_stride * (jj & 7);
        super c0, c1;
        memcpy(&c0, input + 8 * idx, 32);
        memcpy(&c1, input + 8 * idx + 4, 32);
        wins = sor(wins, rmax(transform_super(s, snot(c1))));
        not_loss = sor(not_loss, rmax(transform_super(s, snot(c0))));
      }
    }
    const int blk = i >> 3;
    const long oidx = (long)((blk == L->length - 1) ? last_output_base : output_base) +
                      (long)L->block_stride * blk + (long)output_stride * (i & 7);
    const super r0 = sor(sand(wins, snot(immediate)), sand(wins0, snot(wins1)));
    const super r1 = sor(sand(not_loss, snot(immediate)), wins0);
    memcpy(output + 8 * oidx, &r0, 32);
    memcpy(output + 8 * oidx + 4, &r1, 32);
  }
}

int or_line_sizes(u64 sig, int dim, int length, const u8* block_base, int64_t* in_nodes, int64_t* out_nodes) {
  or_init();
  line_info L;
  line_setup(&L, sig, dim, length, block_base);
  *in_nodes = (int64_t)L.in_shape[0] * L.in_shape[1] * L.in_shape[2] * L.in_shape[3];
  *out_nodes = (int64_t)L.out_shape[0] * L.out_shape[1] * L.out_shape[2] * L.out_shape[3];
  free(L.rsyms);
  return 0;
}

typedef struct {
  const line_info* L; const u64* input; u64* output;
  int cross[3]; int next; int stride; int tid;
} line_job;

static void* line_worker(void* arg) {
  line_job* J = (line_job*)arg;
  const int total = J->cross[0] * J->cross[1] * J->cross[2];
  for (int m = J->tid; m < total; m += J->stride) {
    const int base3[3] = {m / (J->cross[1] * J->cross[2]), m / J->cross[2] % J->cross[1], m % J->cross[2]};
    compute_microline(J->L, base3, J->input, J->output);
  }
  return NULL;
}

/* schedule_compute_line (compute.cc:394-404): one job per microline, here
 * spread over `threads` pthreads. */
int or_compute_line(u64 sig, int dim, int length, const u8* block_base, const u64* input, u64* output,
                    int threads) {
  or_init();
  line_info L;
  line_setup(&L, sig, dim, length, block_base);
  int cross[3], k = 0;
  for (int i = 0; i < 4; i++) if (i != dim) cross[k++] = L.out_shape[i];
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  pthread_t tids[256];
  line_job jobs[256];
  for (int t = 0; t < threads; t++) {
    jobs[t].L = &L; jobs[t].input = input; jobs[t].output = output;
    memcpy(jobs[t].cross, cross, sizeof cross);
    jobs[t].stride = threads; jobs[t].tid = t;
    if (threads > 1) pthread_create(&tids[t], NULL, line_worker, &jobs[t]);
  }
  if (threads == 1) line_worker(&jobs[0]);
  else for (int t = 0; t < threads; t++) pthread_join(tids[t], NULL);
  free(L.rsyms);
  return 0;
}

/* count_block_wins (end/block_store.cc:330-352) over popcounts_over_stabilizers
 * (base/count.cc:235-261) */
static int log_stabilizers(u16 q) {
  const u16 s0 = T_unpack[q][0], s1 = T_unpack[q][1];
  const u16 s0r = T_rot[s0][0], s1r = T_rot[s1][0];
  if (s0 == s0r && s1 == s1r) return 2;
  return s0 == T_rot[s0r][0] && s1 == T_rot[s1r][0] ? 1 : 0;
}
void or_count_block_wins(u64 sig, const u8* block, const u64* data, u64* counts3) {
  or_init();
  const section s = sec_from_sig(sig);
  int shape[4], bs[4];
  sec_shape(s, shape);
  for (int i = 0; i < 4; i++) bs[i] = bshape(shape[i], block[i]);
  counts3[0] = counts3[1] = counts3[2] = 0;
  long n = 0;
  for (int i0 = 0; i0 < bs[0]; i0++)
    for (int i1 = 0; i1 < bs[1]; i1++)
      for (int i2 = 0; i2 < bs[2]; i2++)
        for (int i3 = 0; i3 < bs[3]; i3++, n++) {
          const int idx[4] = {i0, i1, i2, i3};
          int sh = 0;
          for (int q = 0; q < 4; q++) sh += log_stabilizers(rmin_list(s.c[q][0], s.c[q][1])[8 * block[q] + idx[q]]);
          const u64* node = data + 8 * n;
          const int w0 = popc64(node[0]) + popc64(node[1]) + popc64(node[2]) + popc64(node[3]);
          const int w1 = popc64(node[4]) + popc64(node[5]) + popc64(node[6]) + popc64(node[7]);
          counts3[0] += (u64)(w0 >> sh);
          counts3[1] += (u64)(w1 >> sh);
          counts3[2] += (u64)(256 >> sh);
        }
}

/* descendent_sections (end/sections.cc:18-49) */
static int cmp_u64(const void* a, const void* b) {
  const u64 x = *(const u64*)a, y = *(const u64*)b;
  return x < y ? -1 : x > y;
}
int or_descendent_sections(u64 root_sig, int slice, u64* sigs, int cap) {
  or_init();
  enum { MAXS = 1 << 16 };
  u64* seen = (u64*)malloc(sizeof(u64) * MAXS);
  u64* stack = (u64*)malloc(sizeof(u64) * MAXS);
  int nseen = 0, nstack = 0, nout = 0;
  stack[nstack++] = root_sig;
  while (nstack) {
    const section s = sec_standardize(sec_from_sig(stack[--nstack]), NULL);
    const u64 sig = sec_sig(s);
    int found = 0;
    for (int i = 0; i < nseen && !found; i++) found = seen[i] == sig;
    if (found) continue;
    seen[nseen++] = sig;
    const int n = sec_sum(s);
    if (n == slice) { if (nout < cap) sigs[nout] = sig; nout++; }
    if (n < slice && n < 35)
      for (int q = 0; q < 4; q++)
        if (s.c[q][0] + s.c[q][1] < 9) stack[nstack++] = sec_sig(sec_child(s, q));
  }
  if (nout <= cap) qsort(sigs, nout, sizeof(u64), cmp_u64);
  free(seen);
  free(stack);
  return nout;
}

/* ------------------------------------------------------------------------ */
/* Midsolve (pentago/mid)                                                     */
/* ------------------------------------------------------------------------ */

static int choose(int n, int k) {  /* mid/subsets.h:23-32 */
  if (n < 0 || k < 0 || k > n) return 0;
  long r = 1;
  for (int i = 0; i < k; i++) r = r * (n - i) / (i + 1);
  return (int)r;
}

typedef u64 set_t;
typedef struct { int n, k, size; } sets_t;
static sets_t make_sets(int n, int k) { sets_t s = {n, k, choose(n, k)}; return s; }

/* subset(n,k,index): the index-th k-subset of [0,n) in large-entry-major
 * order, packed 5 bits per entry (mid/subsets.h:34-52) */
static set_t subset(int n, int k, int index) {
  set_t set = 0;
  for (int i = k - 1; i >= 0; i--) {
    int j = i, base = 0;
    for (; j < n; j++) {
      const int next = base + choose(j, i);
      if (index < next) break;
      base = next;
    }
    set |= (set_t)j << (5 * i);
    index -= base;
  }
  return set;
}

typedef struct { u64 side[2]; u32 ply; } hboard;  /* high/board_c.h */
static int hcount(hboard b) { return (int)((b.ply + 1) >> 1); }
static int hturn(hboard b) { return (int)((b.ply >> 1) & 1); }
static int hmiddle(hboard b) { return (int)(b.ply & 1); }
static const u64 side_mask = 0x01ff01ff01ff01ffull;
static u64 hempty(hboard b) { return side_mask ^ b.side[0] ^ b.side[1]; }

/* high_board_t raw conversion (high/board.cc:84-111) */
static u64 hboard_board(hboard b) {
  u64 board = 0;
  for (int q = 0; q < 4; q++) {
    u16 quad = 0;
    for (int i = 8; i >= 0; i--) {
      const int j = 16 * q + i;
      quad = (u16)(3 * quad + (b.side[0] >> j & 1) + 2 * (b.side[1] >> j & 1));
    }
    board |= (u64)quad << (16 * q);
  }
  return board;
}
static u64 hraw(hboard b) { return hboard_board(b) | (u64)hmiddle(b) << 63; }
static hboard from_board(u64 board, int middle) {
  hboard h = {{0, 0}, 0};
  for (int q = 0; q < 4; q++) {
    u16 quad = (u16)(board >> 16 * q);
    for (int i = 0; i < 9; i++) {
      const int s = quad % 3;
      quad /= 3;
      const int j = 16 * q + i;
      h.side[0] |= (u64)(s == 1) << j;
      h.side[1] |= (u64)(s == 2) << j;
    }
  }
  h.ply = (u32)(2 * popc64(h.side[0] | h.side[1]) - middle);
  return h;
}
static hboard from_raw(u64 raw) { return from_board(raw << 1 >> 1, (int)(raw >> 63)); }
static hboard hplace(hboard b, int bit) {
  b.side[hturn(b)] |= (u64)1 << bit;
  b.ply++;
  return b;
}
static hboard hrotate(hboard b, int q, int d) {  /* high/board.cc:66-82 */
  for (int s = 0; s < 2; s++) {
    const u16 old = quadrant(b.side[s], q);
    u16 quad = 0;
    for (int i = 0; i < 9; i++)
      if (old >> i & 1) {
        const int x = i / 3, y = i % 3;
        quad |= (u16)(1 << (4 - d * (3 * y - x - 2)));
      }
    b.side[s] ^= (u64)(old ^ quad) << (16 * q);
  }
  b.ply++;
  return b;
}
static int slow_won(u64 side) { return won(side); }
static void done_and_value(hboard b, int* done, int* value) {  /* high/board.cc:20-29 */
  const int bw = slow_won(b.side[0]), ww = slow_won(b.side[1]);
  if (bw || ww) { *done = 1; *value = (bw && ww) ? 0 : (bw == !hturn(b) ? 1 : -1); return; }
  if (b.ply == 72) { *done = 1; *value = 0; return; }
  *done = 0; *value = 0;
}

typedef struct { int ny, lo, size; } grab_t;
typedef struct {
  hboard root; int spots; u8 empty[18];
  grab_t spaces[20];
  int sets0_off[20], sets1p_off[20], cs1ps_off[20], wins1_off[20];
} info_t;

static int bottleneck(int spots) {  /* mid/internal.h:37-47 */
  int worst = 0, prev = 1;
  for (int n = 0; n <= spots; n++) {
    int next = choose(spots, n + 1);
    if (next) next *= choose(n + 1, (n + 1) / 2);
    if (prev + next > worst) worst = prev + next;
    prev = next;
  }
  return worst;
}

/* helper_t (mid/internal.h:10-26) */
#define K0 (n >> 1)
#define K1 (n - (n >> 1))
static int hparity(const info_t* I, int n) { return (int)((n + I->root.ply) & 1); }
static u64 hroot0(const info_t* I, int n) { return I->root.side[(I->spots + n) & 1]; }
static u64 hroot1(const info_t* I, int n) { return I->root.side[(I->spots + n + 1) & 1]; }

static u64 side_of(const info_t* I, sets_t sets, set_t set) {  /* mid/subsets.h:90-95 */
  u64 s = 0;
  for (int i = 0; i < sets.k; i++) s |= (u64)1 << I->empty[set >> 5 * i & 0x1f];
  return s;
}

static info_t make_info(hboard root) {  /* mid/internal.h:49-69 */
  info_t I;
  memset(&I, 0, sizeof I);
  I.root = root;
  I.spots = 36 - hcount(root);
  {
    const u64 free_ = hempty(root);
    int next = 0;
    for (int i = 0; i < 64; i++) if (free_ >> i & 1) I.empty[next++] = (u8)i;
  }
  const int ws = bottleneck(I.spots);
  for (int n = 0; n <= I.spots; n++) {
    const sets_t s0 = make_sets(I.spots, K0), s1 = make_sets(I.spots, K1);
    const sets_t s0p = make_sets(I.spots - K1, K0), s1p = make_sets(I.spots - K0, K1);
    I.sets0_off[n + 1] = I.sets0_off[n] + s0.size;
    I.sets1p_off[n + 1] = I.sets1p_off[n] + s1p.size;
    I.cs1ps_off[n + 1] = I.cs1ps_off[n] + s1p.size * (I.spots - K0);
    I.wins1_off[n + 1] = I.wins1_off[n] + s1.size;
    I.spaces[n].ny = s0p.size;
    I.spaces[n].lo = (n & 1) ? ws - s1.size * s0p.size : 0;
    I.spaces[n].size = s1.size * s0p.size;
  }
  I.spaces[I.spots + 1].ny = I.spaces[I.spots + 1].lo = I.spaces[I.spots + 1].size = 0;
  return I;
}

typedef struct { half after, before; } wins1_t;
typedef struct { half wins0; u16 child_s0s[18]; u16 offset0[90]; u8 empty1[18]; } set0_info_t;

/* make_cs1ps (mid/internal.h:135-150) */
static u16 make_cs1ps(const info_t* I, const set_t* sets1p, int n, int index) {
  const int k0 = K0, k1 = K1;
  const int s1p = index / (I->spots - k0);
  const int j = index - s1p * (I->spots - k0);
  u16 c = (u16)s1p;
  for (int a = 0; a < k1; a++) {
    const int v = (int)(sets1p[s1p] >> 5 * a & 0x1f);
    if (j < v) c = (u16)(c - choose(v - 1, a));
  }
  return c;
}

/* make_set0_info (mid/internal.h:174-259) */
static set0_info_t make_set0_info(const info_t* I, int n, int s0) {
  set0_info_t I0;
  memset(&I0, 0, sizeof I0);
  const int k0 = K0, k1 = K1;
  const sets_t sets0 = make_sets(I->spots, k0);
  const set_t set0 = subset(sets0.n, sets0.k, s0);
  const u64 side0 = hroot0(I, n) | side_of(I, sets0, set0);
  I0.wins0 = hwins(side0, hparity(I, n));
  {
    const u64 free_ = side_mask & ~side0;
    int next = 0;
    for (int i = 0; i < I->spots; i++) if (free_ >> I->empty[i] & 1) I0.empty1[next++] = (u8)i;
  }
  for (int i = 0; i < I->spots - k0; i++) {
    const int j = I0.empty1[i] - i;
    int v = choose(I0.empty1[i], j + 1);
    for (int a = 0; a < k0; a++) v += choose((int)(set0 >> 5 * a & 0x1f), a + (a >= j) + 1);
    I0.child_s0s[i] = (u16)v;
  }
  for (int a = 0; a < k1; a++)
    for (int q = 0; q < I->spots - k0; q++) {
      u16 offset = (u16)(a ? 0 : s0);
      for (int i = I0.empty1[q] - q; i < k0; i++) {
        const int v = (int)(set0 >> 5 * i & 0x1f);
        if (v > a) offset = (u16)(offset - choose(v - a - 1, i));
      }
      I0.offset0[a * (I->spots - k0) + q] = offset;
    }
  return I0;
}

/* inner (mid/internal.h:358-408) */
static void inner(const info_t* I, int n, const u16* cs1ps, const set_t* sets1p, const wins1_t* wins1s,
                  half* results, half* ws, const set0_info_t* I0, int s1p, int aggressive) {
  const set_t set1p = sets1p[s1p];
  const grab_t in = I->spaces[n + 1], out = I->spaces[n];
  const int spots = I->spots, done = spots == n, k0 = K0, k1 = K1;
  const int turn_aggressive = aggressive ^ (n & 1);
  u32 filled1p = 0;
  u16 s1 = 0, s0p = 0;
  for (int i = 0; i < k1; i++) {
    const int q = (int)(set1p >> 5 * i & 0x1f);
    filled1p |= 1u << q;
    s1 = (u16)(s1 + choose(I0->empty1[q], i + 1));
    s0p = (u16)(s0p + I0->offset0[i * (spots - k0) + q]);
  }
  half us = {{0, 0}};
  if (done && !turn_aggressive) us = hnot(us);
  for (int i = 0, m = 0; i < 32 && m < spots - n; i++) {
    if (filled1p >> i & 1) continue;
    m++;
    const half c = ws[in.lo + (long)I0->child_s0s[i] * in.ny + cs1ps[s1p * (spots - k0) + i]];
    us = hor(us, c);
  }
  const wins1_t w1 = wins1s[s1];
  const half inplay = hnot(hor(I0->wins0, w1.after));
  const half mask = turn_aggressive ? hnot(w1.after) : hnot((half){{0, 0}});
  us = hor(hand(inplay, us), hand(I0->wins0, mask));
  if (n <= 1) results[n + s1p] = us;
  ws[out.lo + (long)s1 * out.ny + s0p] = hor(hrmax(hnot(us)), w1.before);
}

/* midsolve_internal (mid/midengine.cc:93-125); out = 19 x [win, notlose] */
static void midsolve_internal(hboard root, half* out) {
  const info_t I = make_info(root);
  half* ws = (half*)calloc((size_t)bottleneck(I.spots), sizeof(half));
  set_t* sets1p = (set_t*)malloc(sizeof(set_t) * (I.sets1p_off[I.spots + 1] + 1));
  wins1_t* wins1 = (wins1_t*)malloc(sizeof(wins1_t) * (I.wins1_off[I.spots + 1] + 1));
  u16* cs1ps = (u16*)malloc(sizeof(u16) * (I.cs1ps_off[I.spots + 1] + 1));
  for (int n = I.spots; n >= 0; n--) {  /* midsolve_precompute (midengine.cc:57-76) */
    const sets_t s1p = make_sets(I.spots - K0, K1), s1 = make_sets(I.spots, K1);
    set_t* sp = sets1p + I.sets1p_off[n];
    for (int i = 0; i < s1p.size; i++) sp[i] = subset(s1p.n, s1p.k, i);
    for (int s = 0; s < s1.size; s++) {
      const u64 side1 = hroot1(&I, n) | side_of(&I, s1, subset(s1.n, s1.k, s));
      wins1[I.wins1_off[n] + s].after = hwins(side1, hparity(&I, n));
      wins1[I.wins1_off[n] + s].before = hwins(side1, !hparity(&I, n));
    }
    for (int i = 0; i < s1p.size * (I.spots - K0); i++) cs1ps[I.cs1ps_off[n] + i] = make_cs1ps(&I, sp, n, i);
  }
  half raw[2][19];
  memset(raw, 0, sizeof raw);
  for (int aggressive = 0; aggressive < 2; aggressive++)
    for (int n = I.spots; n >= 0; n--) {  /* midsolve_loop (midengine.cc:78-91) */
      const sets_t s0 = make_sets(I.spots, K0), s1p = make_sets(I.spots - K0, K1);
      for (int a = 0; a < s0.size; a++) {
        const set0_info_t I0 = make_set0_info(&I, n, a);
        for (int b = 0; b < s1p.size; b++)
          inner(&I, n, cs1ps + I.cs1ps_off[n], sets1p + I.sets1p_off[n], wins1 + I.wins1_off[n], raw[aggressive],
                ws, &I0, b, aggressive);
      }
    }
  for (int i = 0; i < 19; i++)
    for (int j = 0; j < 2; j++) out[2 * i + j] = raw[j ^ (i == 0)][i];
  free(ws); free(sets1p); free(wins1); free(cs1ps);
}

static int hbit(half h, int i) { return (int)(h.w[(i >> 6) & 1] >> (i & 63) & 1); }
static int mid_value(const half* r, int s) {  /* mid/midengine.h:29-31 */
  return hbit(r[0], s >> 1) + hbit(r[1], s >> 1) - 1;
}

/* midsolve_traverse (mid/midengine.cc:127-158) */
static int traverse(hboard b, const half* supers, u64* raws, int32_t* values, int* count) {
  int value, done, iv;
  done_and_value(b, &done, &iv);
  if (done) value = iv;
  else if (!hmiddle(b)) {
    value = -1;
    const u64 e = hempty(b);
    int s = 0;
    for (int bit = 0; bit < 64; bit++)
      if (e >> bit & 1) {
        s++;
        const int v = traverse(hplace(b, bit), supers + 2 * s, raws, values, count);
        if (v > value) value = v;
      }
  } else {
    value = -1;
    for (int s = 0; s < 8; s++) {
      const int q = s >> 1, d = (s & 1) ? -1 : 1;
      const int v = mid_value(supers, (d & 3) << 2 * q);
      raws[*count] = hraw(hrotate(b, q, d));
      values[*count] = v;
      (*count)++;
      if (-v > value) value = -v;
    }
  }
  raws[*count] = hraw(b);
  values[*count] = value;
  (*count)++;
  return value;
}

int or_midsolve(u64 raw, u64* out_raws, int32_t* out_values) {
  or_init();
  const hboard b = from_raw(raw);
  half supers[38];
  midsolve_internal(b, supers);
  int count = 0;
  traverse(b, supers, out_raws, out_values, &count);
  return count;
}

void or_midsolve_internal(u64 raw, u64* out) {
  or_init();
  half supers[38];
  midsolve_internal(from_raw(raw), supers);
  memcpy(out, supers, sizeof supers);
}

int or_midsolve_workspace_size(int stones) { return bottleneck(36 - stones); }

/* ------------------------------------------------------------------------ */
/* Static rANS, format version 2 (pentago/shard/arithmetic.cc)              */
/* ------------------------------------------------------------------------ */

enum { LANES = 8, TOTAL_BITS = 14 };
static const u32 RANS_TOTAL = 1u << 14, RANS_LOWER = 1u << 23;
typedef struct { u32 freq[3], cum[3], xmax[3]; } freq_t;

static freq_t make_freq(const u64* counts) {  /* arithmetic.cc:48-77 */
  freq_t t;
  const u64 sum = counts[0] + counts[1] + counts[2];
  u32 f[3];
  if (sum) {
    for (int i = 0; i < 3; i++) f[i] = (u32)(counts[i] * RANS_TOTAL / sum);
    for (int i = 0; i < 3; i++) if (!f[i]) f[i] = 1;
    const int32_t adjust = (int32_t)RANS_TOTAL - (int32_t)(f[0] + f[1] + f[2]);
    int largest = 0;
    if (f[1] > f[largest]) largest = 1;
    if (f[2] > f[largest]) largest = 2;
    f[largest] = (u32)((int32_t)f[largest] + adjust);
  } else {
    f[0] = f[1] = f[2] = RANS_TOTAL / 3;
    f[0] += RANS_TOTAL - 3 * (RANS_TOTAL / 3);
  }
  const u32 xm = (RANS_LOWER >> TOTAL_BITS) << 8;
  for (int i = 0; i < 3; i++) { t.freq[i] = f[i]; t.xmax[i] = xm * f[i]; }
  t.cum[0] = 0; t.cum[1] = f[0]; t.cum[2] = f[0] + f[1];
  return t;
}

int64_t or_rans_encode(const u8* sym, int64_t n, u8* out, int64_t cap) {  /* arithmetic.cc:366-401,456-472 */
  u64 counts[3] = {0, 0, 0};
  for (int64_t i = 0; i < n; i++) counts[sym[i]]++;
  const freq_t t = make_freq(counts);
  const int64_t bufcap = n / LANES * 2 + 64;
  u8* bufs = (u8*)malloc((size_t)(bufcap * LANES));
  u8* cur[LANES];
  u32 st[LANES];
  for (int l = 0; l < LANES; l++) { st[l] = RANS_LOWER; cur[l] = bufs + bufcap * (l + 1); }
  for (int64_t i = n - 1; i >= 0; i--) {
    const int l = (int)(i % LANES), s = sym[i];
    while (st[l] >= t.xmax[s]) { *--cur[l] = (u8)(st[l] & 0xff); st[l] >>= 8; }
    st[l] = ((st[l] / t.freq[s]) << TOTAL_BITS) + (st[l] % t.freq[s]) + t.cum[s];
  }
  for (int l = 0; l < LANES; l++)
    for (int j = 0; j < 4; j++) *--cur[l] = (u8)(st[l] >> (8 * j) & 0xff);
  int64_t total = 60;
  u32 len[LANES];
  for (int l = 0; l < LANES; l++) { len[l] = (u32)(bufs + bufcap * (l + 1) - cur[l]); total += len[l]; }
  if (total > cap) { free(bufs); return -1; }
  u8* p = out;
  const u32 version = 2;
  memcpy(p, &version, 4); p += 4;
  memcpy(p, counts, 24); p += 24;
  memcpy(p, len, 32); p += 32;
  for (int l = 0; l < LANES; l++) { memcpy(p, cur[l], len[l]); p += len[l]; }
  free(bufs);
  return total;
}

int64_t or_rans_decode(const u8* data, int64_t size, u8* sym, int64_t cap) {  /* arithmetic.cc:403-452,474-495 */
  if (size < 60) return -2;
  u32 version, len[LANES];
  u64 counts[3];
  memcpy(&version, data, 4);
  memcpy(counts, data + 4, 24);
  memcpy(len, data + 28, 32);
  if (version != 2) return -2;
  u64 sum = 0;
  for (int l = 0; l < LANES; l++) sum += len[l];
  if (sum != (u64)(size - 60)) return -2;
  const u64 n = counts[0] + counts[1] + counts[2];
  if (counts[0] > n || counts[1] > n || counts[2] > n || n > ~(u64)0 / 0x3fff) return -2;
  if ((int64_t)n > cap) return -1;
  const freq_t t = make_freq(counts);
  const u8 *ptr[LANES], *end[LANES];
  u32 st[LANES];
  const u8* base = data + 60;
  for (int l = 0; l < LANES; l++) {
    const u8* p = base;
    const u8* e = base + len[l];
    base = e;
    st[l] = 0;
    for (int j = 0; j < 4 && p < e; j++) st[l] = (st[l] << 8) | *p++;
    ptr[l] = p; end[l] = e;
  }
  for (u64 i = 0; i < n; i++) {
    const int l = (int)(i % LANES);
    const u32 slot = st[l] & (RANS_TOTAL - 1);
    const int s = slot < t.cum[1] ? 0 : slot < t.cum[2] ? 1 : 2;
    st[l] = t.freq[s] * (st[l] >> TOTAL_BITS) + slot - t.cum[s];
    while (st[l] < RANS_LOWER && ptr[l] < end[l]) st[l] = (st[l] << 8) | *ptr[l]++;
    sym[i] = (u8)s;
  }
  return (int64_t)n;
}

/* ------------------------------------------------------------------------
 * Slice-file filter (pentago/data/filter.h:76-127, portable forms) and the
 * conversion between [win, notlost] nodes and the on-disk [black wins,
 * white wins] pair (pentago/mpi/io.cc:79-86 writing, 476-481 reading).
 * ------------------------------------------------------------------------ */
static u64 st_expand(u64 a) { /* low 32 bits to the even bits */
  a &= 0x00000000ffffffffull;
  a = (a | a << 16) & 0x0000ffff0000ffffull;
  a = (a | a << 8) & 0x00ff00ff00ff00ffull;
  a = (a | a << 4) & 0x0f0f0f0f0f0f0f0full;
  a = (a | a << 2) & 0x3333333333333333ull;
  a = (a | a << 1) & 0x5555555555555555ull;
  return a;
}
static u64 st_contract(u64 a) { /* even bits to the low 32 bits */
  a &= 0x5555555555555555ull;
  a = (a | a >> 1) & 0x3333333333333333ull;
  a = (a | a >> 2) & 0x0f0f0f0f0f0f0f0full;
  a = (a | a >> 4) & 0x00ff00ff00ff00ffull;
  a = (a | a >> 8) & 0x0000ffff0000ffffull;
  a = (a | a >> 16) & 0x00000000ffffffffull;
  return a;
}

void or_st_filter(const u64* nodes, int64_t n, int turn, int filter, u64* out) {
  for (int64_t i = 0; i < n; i++) {
    const u64* x = nodes + 8 * i;
    u64 s0[4], s1[4], *o = out + 8 * i;
    for (int k = 0; k < 4; k++) {
      if (turn == 0) { s0[k] = x[k]; s1[k] = ~x[4 + k]; }
      else if (turn == 1) { s0[k] = ~x[4 + k]; s1[k] = x[k]; }
      else { s0[k] = x[k]; s1[k] = x[4 + k]; }
    }
    if (!filter) {
      for (int k = 0; k < 4; k++) { o[k] = s0[k]; o[4 + k] = s1[k]; }
      continue;
    }
    /* super h of the output interleaves words 2h, 2h+1 of both supers:
       LO(a)|LO(a')<<1, HI(a)|HI(a')<<1, LO(b)|LO(b')<<1, HI(b)|HI(b')<<1 */
    for (int h = 0; h < 2; h++)
      for (int j = 0; j < 2; j++) {
        const u64 a = s0[2 * h + j], b = s1[2 * h + j];
        o[4 * h + 2 * j] = st_expand(a) | st_expand(b) << 1;
        o[4 * h + 2 * j + 1] = st_expand(a >> 32) | st_expand(b >> 32) << 1;
      }
  }
}

void or_st_unfilter(const u64* in, int64_t n, int turn, int filter, u64* nodes) {
  for (int64_t i = 0; i < n; i++) {
    const u64* x = in + 8 * i;
    u64 s0[4], s1[4], *o = nodes + 8 * i;
    for (int m = 0; m < 4; m++) {
      if (filter) {
        s0[m] = st_contract(x[2 * m]) | st_contract(x[2 * m + 1]) << 32;
        s1[m] = st_contract(x[2 * m] >> 1) | st_contract(x[2 * m + 1] >> 1) << 32;
      } else {
        s0[m] = x[m];
        s1[m] = x[4 + m];
      }
    }
    for (int k = 0; k < 4; k++) {
      if (turn == 0) { o[k] = s0[k]; o[4 + k] = ~s1[k]; }
      else if (turn == 1) { o[k] = s1[k]; o[4 + k] = ~s0[k]; }
      else { o[k] = s0[k]; o[4 + k] = s1[k]; }
    }
  }
}

/* ------------------------------------------------------------------------
 * Shards.  The shuffled index of (section, position, rotation) is
 * permute(offset[section] + 256 position + rotation), positions row-major
 * over the section's shape (pentago/shard/shard.cc:44-135); a shard of a
 * power-of-two count takes the indices congruent to it (shard.h:87-115).
 * ------------------------------------------------------------------------ */

/* Shift amounts of the permutation per slice (pentago/shard/shard_permute.h:40-60;
 * the entry counts there equal or_shard_total). */
static const u8 perm_shifts[19][8] = {
  {3,2,1,5,2,2,3,6}, {6,6,4,1,3,2,6,4}, {4,6,4,8,7,6,6,3}, {14,6,13,12,9,7,10,3},
  {6,13,8,10,6,15,4,1}, {15,17,6,16,15,13,5,18}, {19,21,17,16,23,16,11,20},
  {15,26,10,16,13,16,9,22}, {22,23,17,24,16,19,25,21}, {11,24,29,23,16,21,23,1},
  {24,27,3,24,7,29,25,30}, {27,30,7,27,1,28,9,31}, {29,33,10,34,7,29,1,31},
  {18,7,4,31,34,26,18,2}, {24,29,14,35,15,22,10,18}, {4,9,23,41,10,37,32,35},
  {8,35,33,34,14,38,7,5}, {4,42,19,41,5,39,17,37}, {33,40,33,39,5,42,34,37}};

typedef struct {
  int nsec;
  u64* sigs;
  u64* offsets;  /* nsec + 1 */
} shard_map;
static shard_map shard_maps[19];

/* all_boards_sections(n, 8) (pentago/base/all_boards.cc:160-203): counts of
 * quadrants 3, 2, 1 in nested loops, quadrant 0 determined, standardized
 * sections only, sorted by signature */
int or_shard_sections(int n, u64* out, int cap) {
  or_init();
  const int white = n / 2, black = n - white;
  int count = 0;
  enum { MAXSEC = 16384 };
  u64* sigs = (u64*)malloc(sizeof(u64) * MAXSEC);
  for (int b3 = 0; b3 <= (black < 9 ? black : 9); b3++)
    for (int w3 = 0; w3 <= (white < 9 - b3 ? white : 9 - b3); w3++) {
      const int lb = black - b3, lw = white - w3;
      for (int b2 = 0; b2 <= (lb < 9 ? lb : 9); b2++) {
        const int w2lo = lw - (18 - (lb - b2)) > 0 ? lw - (18 - (lb - b2)) : 0, w2hi = lw < 9 - b2 ? lw : 9 - b2;
        for (int w2 = w2lo; w2 <= w2hi; w2++) {
          const int lb2 = lb - b2, lw2 = lw - w2;
          const int b1lo = lb2 - 9 > 0 ? lb2 - 9 : 0, b1hi = lb2 < 9 ? lb2 : 9;
          for (int b1 = b1lo; b1 <= b1hi; b1++) {
            const int w1lo = lw2 - (9 - lb2 + b1) > 0 ? lw2 - (9 - lb2 + b1) : 0, w1hi = lw2 < 9 - b1 ? lw2 : 9 - b1;
            for (int w1 = w1lo; w1 <= w1hi; w1++) {
              section s;
              s.c[0][0] = (u8)(lb2 - b1); s.c[0][1] = (u8)(lw2 - w1);
              s.c[1][0] = (u8)b1; s.c[1][1] = (u8)w1;
              s.c[2][0] = (u8)b2; s.c[2][1] = (u8)w2;
              s.c[3][0] = (u8)b3; s.c[3][1] = (u8)w3;
              if (sec_sig(sec_standardize(s, NULL)) != sec_sig(s)) continue;
              if (count < MAXSEC) sigs[count] = sec_sig(s);
              count++;
            }
          }
        }
      }
    }
  if (count <= MAXSEC) {
    qsort(sigs, (size_t)count, sizeof(u64), cmp_u64);
    for (int i = 0; i < count && i < cap; i++) out[i] = sigs[i];
  } else
    count = -1;
  free(sigs);
  return count;
}

static const shard_map* shard_map_of(int slice) {
  shard_map* m = &shard_maps[slice];
  if (m->sigs) return m;
  const int n = or_shard_sections(slice, NULL, 0);
  u64* sigs = (u64*)malloc(sizeof(u64) * (n ? n : 1));
  u64* off = (u64*)malloc(sizeof(u64) * (n + 1));
  or_shard_sections(slice, sigs, n);
  off[0] = 0;
  for (int i = 0; i < n; i++) {
    int sh[4];
    sec_shape(sec_from_sig(sigs[i]), sh);
    off[i + 1] = off[i] + 256ull * sh[0] * sh[1] * sh[2] * sh[3];
  }
  m->nsec = n;
  m->offsets = off;
  m->sigs = sigs;
  return m;
}

uint64_t or_shard_total(int slice) { or_init(); const shard_map* m = shard_map_of(slice); return m->offsets[m->nsec]; }

/* The permutation: two overlapping power-of-two windows L = [0, 2^k) and
 * H = [n - 2^k, n), with k = floor(log2 n); steps in pairs on L, H, L, H,
 * each pair x ^= x >> s then x += x << s (mod 2^k) (shard_permute.h:62-170). */
uint64_t or_shard_permute(int slice, u64 x, int inverse) {
  const u64 n = or_shard_total(slice);
  const int k = 63 - __builtin_clzll(n);
  const u64 pow2k = 1ull << k, mask = pow2k - 1, offset = n - pow2k;
  const u8* s = perm_shifts[slice];
  for (int j = 0; j < 4; j++) {
    const int pair = inverse ? 3 - j : j, i = 2 * pair;
    const int high = pair & 1;
    if (high ? x < offset : x >= pow2k) continue;
    u64 t = high ? x - offset : x;
    if (!inverse) {
      t ^= t >> s[i];
      t = (t + (t << s[i + 1])) & mask;
    } else {
      /* (1 + 2^s)^-1 = (1 - 2^s)(1 + 2^2s)(1 + 2^4s)..., (I + R^s)^-1 = (I + R^s)(I + R^2s)... */
      t = (t - (t << s[i + 1])) & mask;
      for (int s2 = 2 * s[i + 1]; s2 < k; s2 *= 2) t = (t + (t << s2)) & mask;
      for (int s2 = s[i]; s2 < k; s2 *= 2) t ^= t >> s2;
    }
    x = high ? t + offset : t;
  }
  return x;
}

uint64_t or_shard_board(int slice, u64 shuffled) {
  const shard_map* m = shard_map_of(slice);
  const u64 linear = or_shard_permute(slice, shuffled, 1);
  int si = 0;
  while (m->offsets[si + 1] <= linear) si++;
  const u64 within = linear - m->offsets[si];
  u64 pos = within >> 8;
  const int rot = (int)(within & 255);
  const section s = sec_from_sig(m->sigs[si]);
  int sh[4], idx[4];
  sec_shape(s, sh);
  for (int q = 3; q >= 0; q--) { idx[q] = (int)(pos % (u64)sh[q]); pos /= (u64)sh[q]; }
  u64 board = 0;
  for (int q = 0; q < 4; q++) {
    const u16 v = rmin_list(s.c[q][0], s.c[q][1])[idx[q]];
    const int r = rot >> (2 * q) & 3;
    const u16 w = (u16)(T_pack[rot_left_n(T_unpack[v][0], r)] + 2 * T_pack[rot_left_n(T_unpack[v][1], r)]);
    board |= (u64)w << (16 * q);
  }
  return board;
}

uint64_t or_shard_size(int slice, int total_shards, int shard) {
  const int shift = __builtin_ctz((unsigned)total_shards);
  return (or_shard_total(slice) + (u64)(total_shards - 1) - (u64)shard) >> shift;
}

void or_shard_symbols(int slice, int total_shards, int shard, const u64* nodes, const int64_t* section_base, u8* out) {
  const shard_map* m = shard_map_of(slice);
  const int shift = __builtin_ctz((unsigned)total_shards);
  const u64 size = or_shard_size(slice, total_shards, shard);
  for (u64 i = 0; i < size; i++) {
    const u64 linear = or_shard_permute(slice, (i << shift) | (u64)shard, 1);
    int si = 0;
    while (m->offsets[si + 1] <= linear) si++;
    const u64 within = linear - m->offsets[si];
    const u64* node = nodes + 8 * (section_base[si] + (int64_t)(within >> 8));
    const int r = (int)(within & 255);
    out[i] = (u8)((node[r >> 6] >> (r & 63) & 1) + 2 * (node[4 + (r >> 6)] >> (r & 63) & 1));
  }
}

/* ------------------------------------------------------------------------
 * Board lookup in the solved database (pentago/data/block_cache.cc:27-58,
 * with transform_board of pentago/base/symmetry.cc:46-78).
 * ------------------------------------------------------------------------ */
static u64 or_transform_board_global(int g, u64 board) {
  static const int rotate_quadrants[4][4] = {{0, 1, 2, 3}, {1, 3, 0, 2}, {3, 2, 1, 0}, {2, 0, 3, 1}};
  u16 q[4][2], r[4][2];
  for (int i = 0; i < 4; i++) {
    const u16 v = quadrant(board, i);
    q[i][0] = rot_left_n(T_unpack[v][0], g & 3);
    q[i][1] = rot_left_n(T_unpack[v][1], g & 3);
  }
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 2; k++) r[i][k] = q[rotate_quadrants[g & 3][i]][k];
  if (g & 4) {
    for (int k = 0; k < 2; k++) { const u16 t = r[0][k]; r[0][k] = r[3][k]; r[3][k] = t; }
    for (int i = 0; i < 4; i++)
      for (int k = 0; k < 2; k++) r[i][k] = T_refl[r[i][k]];
  }
  u64 out = 0;
  for (int i = 0; i < 4; i++) out |= (u64)(T_pack[r[i][0]] + 2 * T_pack[r[i][1]]) << (16 * i);
  return out;
}

void or_lookup_locate(u64 board, u64* section_out, int32_t* index4, u16* sym, int32_t* turn) {
  or_init();
  section s;
  int stones = 0;
  for (int q = 0; q < 4; q++) {
    const u16 v = quadrant(board, q);
    s.c[q][0] = (u8)popc64(T_unpack[v][0]);
    s.c[q][1] = (u8)popc64(T_unpack[v][1]);
    stones += s.c[q][0] + s.c[q][1];
  }
  int g = 0;
  const section std = sec_standardize(s, &g);
  const u64 b1 = or_transform_board_global(g, board);
  int local = 0;
  for (int q = 0; q < 4; q++) {
    const int ir = T_rmin_inv[quadrant(b1, q)];
    index4[q] = ir >> 2;
    local |= (ir & 3) << (2 * q);
  }
  /* symmetry1.inverse() * local: the inverse of a pure global symmetry is
     global, and a local factor on the right only sets the local part */
  *sym = (u16)(invert_global(g) << 8 | local);
  *section_out = sec_sig(std);
  *turn = stones & 1;
}

void or_lookup_values(const u64* boards, int64_t n, const u64* secs, int nsecs, const int64_t* base, const u64* data,
                      int32_t* values) {
  or_init();
  for (int64_t i = 0; i < n; i++) {
    u64 sec;
    int32_t idx[4], turn;
    u16 sym;
    or_lookup_locate(boards[i], &sec, idx, &sym, &turn);
    int lo = 0, hi = nsecs;
    while (lo < hi) { const int mid = (lo + hi) / 2; if (secs[mid] < sec) lo = mid + 1; else hi = mid; }
    if (lo == nsecs || secs[lo] != sec) { values[i] = -2; continue; }
    /* the node's offset in the block-major layout: blocks row-major, each row-major in its shape */
    int shape[4], b[4], bs[4];
    sec_shape(sec_from_sig(sec), shape);
    for (int q = 0; q < 4; q++) { b[q] = idx[q] / 8; bs[q] = shape[q] - 8 * b[q] < 8 ? shape[q] - 8 * b[q] : 8; }
    int64_t off = 0, before = 1;
    for (int q = 0; q < 4; q++) {
      int64_t after = 1;
      for (int r = q + 1; r < 4; r++) after *= shape[r];
      off += before * 8 * b[q] * after;
      before *= bs[q];
    }
    const int64_t in = (((int64_t)(idx[0] % 8) * bs[1] + idx[1] % 8) * bs[2] + idx[2] % 8) * bs[3] + idx[3] % 8;
    const u64* node = data + 8 * (base[lo] + off + in);
    int v = -1;
    for (int aggressive = 1; aggressive >= 0; aggressive--) {
      super s;
      u64 w[4];
      for (int k = 0; k < 4; k++) {
        const u64 black = node[k], white = node[4 + k];
        w[k] = aggressive ? (turn ? white : black) : ~(turn ? black : white);
      }
      memcpy(&s, w, 32);
      const sym_t t = {sym >> 8, sym & 255};
      s = transform_super(t, s);
      memcpy(w, &s, 32);
      v += (int)(w[0] & 1);
    }
    values[i] = v;
  }
}
