/* CPU oracle for the learned-model rANS coder (stream format version 3) and
 * its training gradient: test infrastructure only, never linked by the
 * product.  The format has no counterpart in the reference (whose coder is
 * format 2, pentago/shard/arithmetic.cc:366-495); this file restates the
 * format's own specification independently of the GPU code, so that a stream
 * written on the GPU decodes here and the bytes written here equal the GPU's:
 *
 *   coding order of a node: 128 steps, step s codes rotation s then s + 128;
 *   features of symbol r of node i of a block (124 binary inputs):
 *     18 q + 2 c + colour    stone of colour (0 black, 1 white) on cell c of quadrant q
 *     72 + 4 q + i_q         rotation r = i0 + 4 i1 + 16 i2 + 64 i3
 *     88 + 4 n + v           neighbour n = 2 q + e (quadrant q turned +1 for e = 0,
 *                            +3 for e = 1): its symbol if its step is earlier, else v = 3
 *     120 + v                the previous node of the lane's run: its symbol r, 3 for
 *                            a run's first node
 *   network: W1 (124 x 64), b1, W2 (64 x 64), b2, W3 (64 x 3), b3 as bf16 (model
 *     version 3: every column of W1 rows 72..123 and of W2 is integers of magnitude
 *     at most 127 times 2^-e, e = 7 - x for the column's largest magnitude f 2^x,
 *     f in [0.5, 1)); a1 = node + S1 with node = b1 + stone rows ascending and S1 the
 *     exact sum of the rows of the 4 rotation, 8 neighbour and 1 previous-node features;
 *     hq = rint(min(max(a1 * 16, 0), 255)); a2 = fma(C, 1/16, b2) with C = the exact
 *     sum over k of W2[k][j] hq[k]; relu(a) = a > 0 ? a : 0; z = b3 + ((P_0 + P_1) +
 *     (P_2 + P_3)) where P_t is the fma chain from 0 over the columns j with
 *     (j >> 1) & 3 = t ascending of W3[j][c] relu(a2[j])
 *   frequencies (15 bits): e_c = 2^((z_c - max) * 1.44269504f) by floor/Taylor
 *     degree 7, f_c = 1 + trunc(e_c / (e0 + e1 + e2) * 32765), remainder to the
 *     first largest
 *   stream: version 3 | FNV-1a-64 of the model | nodes | words | 32 lane states |
 *     16-bit words; lane l codes the run of nodes l R .. l R + R - 1 (R = ceil(n / 32)),
 *     node l R + k in round k; the encoder runs the decoder's sequence (round,
 *     step, rotation s then s + 128) backward, and renormalizing lanes append
 *     x & 0xffff in lane order when x >= f << 17.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "pentago_oracle.h"

#define NIN 124
#define NH 64
#define NP (NIN * NH + NH + NH * NH + NH + NH * 3 + 3)
#define OFF_W1 0
#define OFF_B1 (NIN * NH)
#define OFF_W2 (OFF_B1 + NH)
#define OFF_B2 (OFF_W2 + NH * NH)
#define OFF_W3 (OFF_B2 + NH)
#define OFF_B3 (OFF_W3 + NH * 3)
#define MODEL_BYTES (12 + 2 * NP)
#define HEADER (20 + 4 * 32)

static float bits_float(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static uint32_t float_bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static float bf16(uint16_t h) { return bits_float((uint32_t)h << 16); }
static float round_bf16(float f) {
  const uint32_t u = float_bits(f);
  return bits_float(((u + 0x7fffu + ((u >> 16) & 1u)) >> 16) << 16);
}
static float relu(float a) { return a > 0.f ? a : 0.f; }

typedef struct {
  int64_t nodes;
  int qbase[4], shape[4];
} geom;

static const uint16_t* rmin_flat;
static const uint16_t (*unpack)[2];
static const uint16_t* rmin_off;

static int block_geom(uint64_t section, const int* block, geom* g) {
  int bytes;
  rmin_flat = (const uint16_t*)or_table("rotation_minimal_quadrants_flat", &bytes);
  unpack = (const uint16_t(*)[2])or_table("unpack_table", &bytes);
  rmin_off = (const uint16_t*)or_table("rotation_minimal_quadrants_offsets", &bytes);
  g->nodes = 1;
  for (int q = 0; q < 4; q++) {
    const int b = (section >> (16 * q)) & 255, w = (section >> (16 * q + 8)) & 255;
    if (b + w > 9) return -1;
    const int k = b * (21 - b) / 2 + w;
    const int size = rmin_off[k + 1] - rmin_off[k];
    if (block[q] < 0 || 8 * block[q] >= size) return -1;
    g->qbase[q] = rmin_off[k] + 8 * block[q];
    g->shape[q] = size - 8 * block[q] < 8 ? size - 8 * block[q] : 8;
    g->nodes *= g->shape[q];
  }
  return 0;
}

int64_t or_lm_nodes(uint64_t section, const int* block) {
  geom g;
  return block_geom(section, block, &g) ? -1 : g.nodes;
}

/* Stone features of node i, ascending; returns the count. */
static int stones(const geom* g, int64_t i, int* f) {
  int idx[4], n = 0;
  for (int q = 3; q >= 0; q--) { idx[q] = (int)(i % g->shape[q]); i /= g->shape[q]; }
  for (int q = 0; q < 4; q++) {
    const uint16_t id = rmin_flat[g->qbase[q] + idx[q]];
    for (int c = 0; c < 9; c++) {
      if (unpack[id][0] >> c & 1) f[n++] = 18 * q + 2 * c;
      if (unpack[id][1] >> c & 1) f[n++] = 18 * q + 2 * c + 1;
    }
  }
  return n;
}

static int neighbour(int r, int n) {
  const int q = n >> 1, i = (r >> (2 * q)) & 3, j = (i + ((n & 1) ? 3 : 1)) & 3;
  return r + ((j - i) << (2 * q));
}

static int context(const uint8_t* sym, int r, int nb) {
  const int a = neighbour(r, nb);
  return (a & 127) < (r & 127) ? (sym[a] & 3) : 3;
}

typedef struct { float p[NP]; } model;

/* The grid of a column of n weights w[0], w[stride], ...: each to the nearest
 * multiple of 2^-e (ties to even), clamped to +-127 2^-e, e = 7 - x for the
 * largest magnitude f 2^x. */
static void grid_column(float* w, int n, int stride) {
  float mx = 0.f;
  for (int k = 0; k < n; k++) mx = fmaxf(mx, fabsf(w[stride * k]));
  if (!(mx > 0.f)) {
    for (int k = 0; k < n; k++) w[stride * k] = 0.f;
    return;
  }
  int x;
  frexpf(mx, &x);
  const int e = 7 - x;
  for (int k = 0; k < n; k++) {
    float q = nearbyintf(ldexpf(w[stride * k], e));
    q = q > 127.f ? 127.f : q < -127.f ? -127.f : q;
    w[stride * k] = ldexpf(q, -e);
  }
}
/* Every grid column: W1 rows 72..119 per hidden unit, W2 per output. */
static void grid_params(float* p) {
  for (int k = 0; k < NH; k++) grid_column(p + OFF_W1 + 72 * NH + k, NIN - 72, NH);
  for (int j = 0; j < NH; j++) grid_column(p + OFF_W2 + j, NH, NH);
}

static int load_model(const uint8_t* bytes, model* m) {
  uint32_t h[3];
  memcpy(h, bytes, 12);
  if (h[0] != 0x4d4c4750u || h[1] != 3 || h[2] != NP) return -1;
  for (int i = 0; i < NP; i++) m->p[i] = bf16((uint16_t)(bytes[12 + 2 * i] | bytes[13 + 2 * i] << 8));
  float* q = malloc(sizeof(float) * NP);
  memcpy(q, m->p, sizeof(float) * NP);
  grid_params(q);
  const int same = !memcmp(q, m->p, sizeof(float) * NP);
  free(q);
  return same ? 0 : -1;
}

#define W1(f, k) m->p[OFF_W1 + (f) * NH + (k)]

static float act_q(float a) {
  float v = a * 16.f;
  v = v > 0.f ? v : 0.f;
  v = v < 255.f ? v : 255.f;
  return (v + 8388608.f) - 8388608.f;
}

/* The 13 rotation, neighbour and previous-node features of symbol r (rows of
 * W1); prev is the previous node's symbols, or null for a run's first node. */
static void ctx_features(int r, const uint8_t* sym, const uint8_t* prev, int* f) {
  for (int q = 0; q < 4; q++) f[q] = 72 + 4 * q + ((r >> (2 * q)) & 3);
  for (int nb = 0; nb < 8; nb++) f[4 + nb] = 88 + 4 * nb + context(sym, r, nb);
  f[12] = 120 + (prev ? (prev[r] & 3) : 3);
}

/* The run length of a block of n nodes (lane l codes nodes l R .. l R + R - 1),
 * and node i's previous node's symbols (null for a run's first node). */
static int64_t run_length(int64_t n) { return (n + 31) / 32; }
static const uint8_t* prev_of(const uint8_t* symbols, int64_t n, int64_t i) {
  return i % run_length(n) ? symbols + 256 * (i - 1) : NULL;
}

static void logits(const model* m, const float* node, int r, const uint8_t* sym, const uint8_t* prev, float* z) {
  float hq[NH], part[4][3];
  int f[13];
  ctx_features(r, sym, prev, f);
  for (int k = 0; k < NH; k++) {
    double s1 = 0;   /* exact: at most 13 x 127 units of 2^-e_k */
    for (int i = 0; i < 13; i++) s1 += W1(f[i], k);
    hq[k] = act_q(node[k] + (float)s1);
  }
  memset(part, 0, sizeof part);
  for (int j = 0; j < NH; j++) {
    double c = 0;   /* exact: at most 64 x 127 x 255 units of 2^-e_j */
    for (int k = 0; k < NH; k++) c += (double)m->p[OFF_W2 + k * NH + j] * hq[k];
    const float h = relu(fmaf((float)c, 0.0625f, m->p[OFF_B2 + j]));
    const int t = (j >> 1) & 3;
    for (int cc = 0; cc < 3; cc++) part[t][cc] = fmaf(m->p[OFF_W3 + 3 * j + cc], h, part[t][cc]);
  }
  for (int cc = 0; cc < 3; cc++)
    z[cc] = m->p[OFF_B3 + cc] + ((part[0][cc] + part[1][cc]) + (part[2][cc] + part[3][cc]));
}

static float exp2_spec(float d) {
  if (!(d >= -24.f)) return 0.f;
  const float n = floorf(d), t = d - n;
  static const float C[8] = {1.0f, 6.9314718e-01f, 2.4022651e-01f, 5.5504109e-02f,
                             9.6181291e-03f, 1.3333558e-03f, 1.5403530e-04f, 1.5252734e-05f};
  float p = C[7];
  for (int i = 6; i >= 0; i--) p = fmaf(p, t, C[i]);
  return p * bits_float((uint32_t)(127 + (int)n) << 23);
}

static void freqs(const float* z, uint32_t* f) {
  float m = z[0];
  if (z[1] > m) m = z[1];
  if (z[2] > m) m = z[2];
  float e[3];
  for (int c = 0; c < 3; c++) e[c] = exp2_spec((z[c] - m) * 1.44269504f);
  const float s = (e[0] + e[1]) + e[2];
  for (int c = 0; c < 3; c++) {
    const float q = e[c] / s * 32765.0f;
    f[c] = 1 + (q >= 1.f ? (uint32_t)q : 0u);
  }
  int big = 0;
  if (f[1] > f[big]) big = 1;
  if (f[2] > f[big]) big = 2;
  f[big] += 32768u - (f[0] + f[1] + f[2]);
}

static void node_sum(const model* m, const geom* g, int64_t i, float* node) {
  int f[36];
  const int nf = stones(g, i, f);
  for (int k = 0; k < NH; k++) {
    float a = m->p[OFF_B1 + k];
    for (int t = 0; t < nf; t++) a = a + W1(f[t], k);
    node[k] = a;
  }
}

int or_lm_freqs(const uint8_t* model_bytes, uint64_t section, const int* block, const uint8_t* symbols,
                const int64_t* samples, int64_t n, uint32_t* out) {
  geom g;
  model* m = malloc(sizeof(model));
  if (block_geom(section, block, &g) || load_model(model_bytes, m)) { free(m); return -1; }
  for (int64_t t = 0; t < n; t++) {
    const int64_t i = samples[t] >> 8;
    const int r = (int)(samples[t] & 255);
    float node[NH], z[3];
    node_sum(m, &g, i, node);
    logits(m, node, r, symbols + 256 * i, prev_of(symbols, g.nodes, i), z);
    freqs(z, out + 3 * t);
  }
  free(m);
  return 0;
}

static uint64_t fnv1a(const uint8_t* p, int64_t n) {
  uint64_t h = 0xcbf29ce484222325ull;
  for (int64_t i = 0; i < n; i++) h = (h ^ p[i]) * 0x100000001b3ull;
  return h;
}

static void put32(uint8_t* p, uint32_t v) { for (int i = 0; i < 4; i++) p[i] = (uint8_t)(v >> (8 * i)); }
static uint32_t get32(const uint8_t* p) {
  return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24;
}

/* Learned stream of one block (no format-2 fallback); returns its size, or -1. */
int64_t or_lm_encode(const uint8_t* model_bytes, uint64_t section, const int* block, const uint8_t* symbols,
                     uint8_t* out, int64_t cap) {
  geom g;
  model* m = malloc(sizeof(model));
  if (block_geom(section, block, &g) || load_model(model_bytes, m)) { free(m); return -1; }
  const int64_t n = g.nodes, rounds = run_length(n);
  if (cap < HEADER + 2 * 256 * n) { free(m); return -1; }
  uint32_t x[32];
  for (int l = 0; l < 32; l++) x[l] = 1u << 16;
  int64_t len = 0;
  float (*node)[NH] = malloc(sizeof(float) * NH * 32);
  for (int64_t round = rounds - 1; round >= 0; round--) {
    for (int l = 0; l < 32; l++)
      if (rounds * l + round < n) node_sum(m, &g, rounds * l + round, node[l]);
    for (int t = 255; t >= 0; t--)
      for (int l = 0; l < 32; l++) {
        const int r = (t >> 1) + 128 * (t & 1);  /* decoder sequence t: step t / 2, half t % 2 */
        const int64_t i = rounds * l + round;
        if (i >= n) continue;
        const uint8_t* sym = symbols + 256 * i;
        if (sym[r] > 2) { free(node); free(m); return -1; }
        float z[3];
        uint32_t f[3];
        logits(m, node[l], r, sym, prev_of(symbols, n, i), z);
        freqs(z, f);
        const int v = sym[r];
        const uint32_t cum = v == 0 ? 0 : v == 1 ? f[0] : f[0] + f[1];
        if (x[l] >= f[v] << 17) {
          out[HEADER + 2 * len] = (uint8_t)x[l];
          out[HEADER + 2 * len + 1] = (uint8_t)(x[l] >> 8);
          len++;
          x[l] >>= 16;
        }
        x[l] = ((x[l] / f[v]) << 15) + x[l] % f[v] + cum;
      }
  }
  const uint64_t h = fnv1a(model_bytes, MODEL_BYTES);
  put32(out, 3);
  put32(out + 4, (uint32_t)h);
  put32(out + 8, (uint32_t)(h >> 32));
  put32(out + 12, (uint32_t)n);
  put32(out + 16, (uint32_t)len);
  for (int l = 0; l < 32; l++) put32(out + 20 + 4 * l, x[l]);
  free(node);
  free(m);
  return HEADER + 2 * len;
}

/* Decode a learned stream of one block; returns the symbols written or -1. */
int64_t or_lm_decode(const uint8_t* model_bytes, uint64_t section, const int* block, const uint8_t* in, int64_t size,
                     uint8_t* symbols, int64_t cap) {
  geom g;
  model* m = malloc(sizeof(model));
  if (block_geom(section, block, &g) || load_model(model_bytes, m)) { free(m); return -1; }
  const int64_t n = g.nodes, rounds = run_length(n);
  const uint64_t h = fnv1a(model_bytes, MODEL_BYTES);
  if (size < HEADER || get32(in) != 3 || get32(in + 4) != (uint32_t)h || get32(in + 8) != (uint32_t)(h >> 32) ||
      get32(in + 12) != (uint32_t)n || HEADER + 2 * (int64_t)get32(in + 16) != size || cap < 256 * n) {
    free(m);
    return -1;
  }
  int64_t ptr = get32(in + 16);
  uint32_t x[32];
  for (int l = 0; l < 32; l++) x[l] = get32(in + 20 + 4 * l);
  float (*node)[NH] = malloc(sizeof(float) * NH * 32);
  int bad = 0;
  for (int64_t round = 0; round < rounds; round++) {
    for (int l = 0; l < 32; l++)
      if (rounds * l + round < n) node_sum(m, &g, rounds * l + round, node[l]);
    for (int t = 0; t < 256; t++) {
      const int r = (t >> 1) + 128 * (t & 1);
      int need[32], k = 0;
      for (int l = 0; l < 32; l++) {
        const int64_t i = rounds * l + round;
        need[l] = 0;
        if (i >= n) continue;
        uint8_t* sym = symbols + 256 * i;
        float z[3];
        uint32_t f[3];
        logits(m, node[l], r, sym, prev_of(symbols, n, i), z);
        freqs(z, f);
        const uint32_t slot = x[l] & 32767u;
        const int v = slot < f[0] ? 0 : slot < f[0] + f[1] ? 1 : 2;
        const uint32_t cum = v == 0 ? 0 : v == 1 ? f[0] : f[0] + f[1];
        x[l] = f[v] * (x[l] >> 15) + slot - cum;
        sym[r] = (uint8_t)v;
        if (x[l] < (1u << 16)) { need[l] = 1; k++; }
      }
      for (int l = 0, rank = 0; l < 32; l++) {
        if (!need[l]) continue;
        const int64_t at = ptr - k + rank++;
        if (at < 0) { bad = 1; continue; }
        x[l] = (x[l] << 16) | (uint32_t)(in[HEADER + 2 * at] | in[HEADER + 2 * at + 1] << 8);
      }
      ptr -= k;
    }
  }
  for (int l = 0; l < 32; l++) bad |= x[l] != (1u << 16);
  free(node);
  free(m);
  return bad || ptr != 0 ? -1 : 256 * n;
}

/* Gradient of the summed cross entropy (natural log) over samples (node << 8 |
 * rotation) of one block, with the parameters rounded to bf16; forward in the
 * training kernel's float order, backward in double.  Returns the loss in bits. */
double or_lm_grad(const float* params, uint64_t section, const int* block, const uint8_t* symbols,
                  const int64_t* samples, int64_t n, double* grad) {
  geom g;
  if (block_geom(section, block, &g)) return -1;
  model* m = malloc(sizeof(model));
  for (int i = 0; i < NP; i++) m->p[i] = round_bf16(params[i]);
  {   /* the grid columns from the fp32 parameters */
    float* q = malloc(sizeof(float) * NP);
    memcpy(q, params, sizeof(float) * NP);
    grid_params(q);
    for (int i = OFF_W1 + 72 * NH; i < OFF_B1; i++) m->p[i] = q[i];
    for (int i = OFF_W2; i < OFF_B2; i++) m->p[i] = q[i];
    free(q);
  }
  memset(grad, 0, sizeof(double) * NP);
  double loss = 0;
  for (int64_t t = 0; t < n; t++) {
    const int64_t i = samples[t] >> 8;
    const int r = (int)(samples[t] & 255);
    const uint8_t* sym = symbols + 256 * i;
    if (i >= g.nodes || sym[r] > 2) continue;
    const int y = sym[r];
    int f[49];
    int nf = stones(&g, i, f);
    for (int q = 0; q < 4; q++) f[nf++] = 72 + 4 * q + ((r >> (2 * q)) & 3);
    for (int nb = 0; nb < 8; nb++) f[nf++] = 88 + 4 * nb + context(sym, r, nb);
    const uint8_t* prev = prev_of(symbols, g.nodes, i);
    f[nf++] = 120 + (prev ? (prev[r] & 3) : 3);
    float h1[NH], a2[NH], h2[NH], z[3];
    for (int k = 0; k < NH; k++) {   /* h1 = hq / 16; the last 13 rows summed exactly */
      float a = m->p[OFF_B1 + k];
      double s1 = 0;
      for (int q = 0; q < nf - 13; q++) a = a + W1(f[q], k);
      for (int q = nf - 13; q < nf; q++) s1 += W1(f[q], k);
      h1[k] = act_q(a + (float)s1) * 0.0625f;
    }
    for (int j = 0; j < NH; j++) {
      double c = 0;
      for (int k = 0; k < NH; k++) c += (double)m->p[OFF_W2 + k * NH + j] * h1[k];
      a2[j] = m->p[OFF_B2 + j] + (float)c;
    }
    for (int c = 0; c < 3; c++) z[c] = m->p[OFF_B3 + c];
    for (int j = 0; j < NH; j++) {
      h2[j] = relu(a2[j]);
      for (int c = 0; c < 3; c++) z[c] = fmaf(m->p[OFF_W3 + 3 * j + c], h2[j], z[c]);
    }
    const double zm = fmax(z[0], fmax(z[1], z[2]));
    double e[3], es = 0;
    for (int c = 0; c < 3; c++) { e[c] = exp(z[c] - zm); es += e[c]; }
    loss += (log(es) - (z[y] - zm)) / log(2.0);
    double dz[3], d2[NH], d1[NH];
    for (int c = 0; c < 3; c++) dz[c] = e[c] / es - (c == y);
    for (int j = 0; j < NH; j++) {
      d2[j] = 0;
      if (a2[j] > 0)
        for (int c = 0; c < 3; c++) d2[j] += m->p[OFF_W3 + 3 * j + c] * dz[c];
      for (int c = 0; c < 3; c++) grad[OFF_W3 + 3 * j + c] += h2[j] * dz[c];
    }
    for (int c = 0; c < 3; c++) grad[OFF_B3 + c] += dz[c];
    for (int k = 0; k < NH; k++) {   /* straight through the quantizer below the clamp */
      d1[k] = 0;
      if (h1[k] > 0 && h1[k] < 255.f * 0.0625f)
        for (int j = 0; j < NH; j++) d1[k] += m->p[OFF_W2 + k * NH + j] * d2[j];
      for (int j = 0; j < NH; j++) grad[OFF_W2 + k * NH + j] += h1[k] * d2[j];
    }
    for (int j = 0; j < NH; j++) grad[OFF_B2 + j] += d2[j];
    for (int k = 0; k < NH; k++) {
      grad[OFF_B1 + k] += d1[k];
      for (int q = 0; q < nf; q++) grad[OFF_W1 + f[q] * NH + k] += d1[k];
    }
  }
  free(m);
  return loss;
}
