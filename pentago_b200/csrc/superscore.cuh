// Device-side operations on 256-bit rotation sets ("supers").
//
// A super is the reference's super_t (pentago/base/superscore.h:29-44): bit
// r = i0 + 4 i1 + 16 i2 + 64 i3 is set when the position rotated left i_q
// times in quadrant q has the property.  On the device it lives in eight
// 32-bit registers, word k = bits 32k..32k+31 (the little-endian u64 layout of
// the reference read as u32).  Within a word, index bits 0-1 (axis 0) select
// the bit in a nibble, bits 2-3 (axis 1) the nibble in a 16-bit chunk, bit 4
// (low bit of axis 2) the half word; the word number carries the high bit of
// axis 2 and axis 3.  Every operation below is written for that split.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

// Every operation is usable on the host too, so CPU tests can check the exact
// arithmetic the kernels run.
#define PG_HD __host__ __device__ __forceinline__

namespace pg {

PG_HD uint32_t funnel_r(uint32_t lo, uint32_t hi, int s) {
#ifdef __CUDA_ARCH__
  return __funnelshift_r(lo, hi, s);
#else
  return uint32_t(((uint64_t(hi) << 32) | lo) >> (s & 31));
#endif
}

template<class T> PG_HD T ldg(const T* p) {
#ifdef __CUDA_ARCH__
  return __ldg(p);
#else
  return *p;
#endif
}

PG_HD int ctz32(uint32_t x) {
#ifdef __CUDA_ARCH__
  return __ffs(x) - 1;
#else
  return __builtin_ctz(x);
#endif
}

struct super8 {
  uint32_t w[8];
};

PG_HD super8 s_zero() { super8 s; for (int i = 0; i < 8; i++) s.w[i] = 0; return s; }
PG_HD super8 s_not(const super8& a) { super8 s; for (int i = 0; i < 8; i++) s.w[i] = ~a.w[i]; return s; }
PG_HD super8 s_or(const super8& a, const super8& b) { super8 s; for (int i = 0; i < 8; i++) s.w[i] = a.w[i] | b.w[i]; return s; }
PG_HD super8 s_and(const super8& a, const super8& b) { super8 s; for (int i = 0; i < 8; i++) s.w[i] = a.w[i] & b.w[i]; return s; }
PG_HD super8 s_andnot(const super8& a, const super8& b) { super8 s; for (int i = 0; i < 8; i++) s.w[i] = a.w[i] & ~b.w[i]; return s; }

PG_HD super8 s_load(const uint64_t* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  const uint4 a = q[0], b = q[1];
  return super8{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w}};
}
PG_HD super8 s_load_ldg(const uint64_t* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  const uint4 a = ldg(q), b = ldg(q + 1);
  return super8{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w}};
}
PG_HD void s_store(uint64_t* p, const super8& s) {
  uint4* q = reinterpret_cast<uint4*>(p);
  q[0] = make_uint4(s.w[0], s.w[1], s.w[2], s.w[3]);
  q[1] = make_uint4(s.w[4], s.w[5], s.w[6], s.w[7]);
}

// A super in one 256-bit global access (sm_100): p must be 32-byte aligned,
// which callers check before choosing these over the 128-bit forms above.
// Each writes or reads a whole 32-byte sector in one instruction.
PG_HD super8 s_load_nc32(const uint64_t* p) {
#ifdef __CUDA_ARCH__
  super8 s;
  asm("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(s.w[0]), "=r"(s.w[1]), "=r"(s.w[2]), "=r"(s.w[3]), "=r"(s.w[4]), "=r"(s.w[5]), "=r"(s.w[6]),
        "=r"(s.w[7])
      : "l"(p));
  return s;
#else
  return s_load(p);
#endif
}
// (Not ordered against other memory operations by the compiler: callers
// read memory that no other access of theirs writes before this load.)
PG_HD super8 s_load32(const uint64_t* p) {
#ifdef __CUDA_ARCH__
  super8 s;
  asm("ld.global.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(s.w[0]), "=r"(s.w[1]), "=r"(s.w[2]), "=r"(s.w[3]), "=r"(s.w[4]), "=r"(s.w[5]), "=r"(s.w[6]),
        "=r"(s.w[7])
      : "l"(p));
  return s;
#else
  return s_load(p);
#endif
}
PG_HD void s_store32(uint64_t* p, const super8& s) {
#ifdef __CUDA_ARCH__
  asm volatile("st.global.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "r"(s.w[0]), "r"(s.w[1]), "r"(s.w[2]),
               "r"(s.w[3]), "r"(s.w[4]), "r"(s.w[5]), "r"(s.w[6]), "r"(s.w[7])
               : "memory");
#else
  s_store(p, s);
#endif
}

// rmax(f)(a) = max over the 8 single rotations b of f(a + b)
// (pentago/base/superscore.h:10-16): the OR of f shifted by +-1 along each axis.
PG_HD super8 s_rmax(const super8& f) {
  super8 r;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const uint32_t x = f.w[i];
    const uint32_t a0 = ((x >> 1) & 0x77777777u) | ((x << 3) & 0x88888888u) |
                        ((x << 1) & 0xeeeeeeeeu) | ((x >> 3) & 0x11111111u);
    const uint32_t a1 = ((x >> 4) & 0x0fff0fffu) | ((x << 12) & 0xf000f000u) |
                        ((x << 4) & 0xfff0fff0u) | ((x >> 12) & 0x000f000fu);
    r.w[i] = a0 | a1;
  }
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t lo = f.w[2 * k], hi = f.w[2 * k + 1];
    const uint32_t a2 = funnel_r(lo, hi, 16) | funnel_r(hi, lo, 16);
    r.w[2 * k] |= a2;
    r.w[2 * k + 1] |= a2;
  }
  const uint32_t e0 = f.w[2] | f.w[6], e1 = f.w[3] | f.w[7], o0 = f.w[0] | f.w[4], o1 = f.w[1] | f.w[5];
  r.w[0] |= e0; r.w[1] |= e1; r.w[4] |= e0; r.w[5] |= e1;
  r.w[2] |= o0; r.w[3] |= o1; r.w[6] |= o0; r.w[7] |= o1;
  return r;
}

// Translation along one axis: out[x] = in[x + k e_axis] (k in 0..3).  This is
// transform_super by a purely local symmetry on one quadrant.
PG_HD super8 s_translate0(const super8& c, int k) {
  const uint32_t lo = (0xfu >> k) * 0x11111111u;
  super8 r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.w[i] = ((c.w[i] >> k) & lo) | ((c.w[i] << (4 - k)) & ~lo);
  return r;
}
PG_HD super8 s_translate1(const super8& c, int k) {
  const uint32_t lo = (0xffffu >> (4 * k)) * 0x10001u;
  super8 r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.w[i] = ((c.w[i] >> (4 * k)) & lo) | ((c.w[i] << (16 - 4 * k)) & ~lo);
  return r;
}
PG_HD super8 s_translate2(const super8& c, int k) {
  super8 r;
#pragma unroll
  for (int p = 0; p < 4; p++) {
    uint32_t lo = c.w[2 * p], hi = c.w[2 * p + 1];
    if (k & 2) { const uint32_t t = lo; lo = hi; hi = t; }
    if (k & 1) {
      const uint32_t nl = funnel_r(lo, hi, 16), nh = funnel_r(hi, lo, 16);
      lo = nl; hi = nh;
    }
    r.w[2 * p] = lo; r.w[2 * p + 1] = hi;
  }
  return r;
}
PG_HD super8 s_translate3(const super8& c, int k) {
  super8 r;
#pragma unroll
  for (int p = 0; p < 4; p++) {
    const int s0 = (p + k) & 3;
    // runtime pair select written as a small switch the compiler turns into selects
    uint32_t lo = c.w[0], hi = c.w[1];
    lo = s0 == 1 ? c.w[2] : lo; hi = s0 == 1 ? c.w[3] : hi;
    lo = s0 == 2 ? c.w[4] : lo; hi = s0 == 2 ? c.w[5] : hi;
    lo = s0 == 3 ? c.w[6] : lo; hi = s0 == 3 ? c.w[7] : hi;
    r.w[2 * p] = lo; r.w[2 * p + 1] = hi;
  }
  return r;
}
// Translation by a full local symmetry l (2 bits per quadrant): out = in - l
// read as a set, i.e. out[x] = in[x + l].
PG_HD super8 s_translate(const super8& c, int l) {
  super8 r = c;
  if (l & 3) r = s_translate0(r, l & 3);
  if (l >> 2 & 3) r = s_translate1(r, l >> 2 & 3);
  if (l >> 4 & 3) r = s_translate2(r, l >> 4 & 3);
  if (l >> 6 & 3) r = s_translate3(r, l >> 6 & 3);
  return r;
}
template<int AXIS> PG_HD super8 s_translate_axis(const super8& c, int k) {
  if (AXIS == 0) return s_translate0(c, k);
  if (AXIS == 1) return s_translate1(c, k);
  if (AXIS == 2) return s_translate2(c, k);
  return s_translate3(c, k);
}

// Exchange index bits I < J of the 256-entry tensor (a delta swap).
template<int I, int J> PG_HD void s_swap_bits(super8& s) {
  static_assert(I < J && J < 8, "");
  if constexpr (J < 5) {
    constexpr int d = (1 << J) - (1 << I);
    uint32_t m = 0;
#pragma unroll
    for (int b = 0; b < 32; b++) if ((b >> I & 1) && !(b >> J & 1)) m |= 1u << b;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const uint32_t x = s.w[i];
      const uint32_t t = ((x >> d) ^ x) & m;
      s.w[i] = x ^ t ^ (t << d);
    }
  } else if constexpr (I < 5) {
    constexpr int wb = J - 5, sh = 1 << I;
    uint32_t m = 0;
#pragma unroll
    for (int b = 0; b < 32; b++) if (!(b >> I & 1)) m |= 1u << b;
#pragma unroll
    for (int w = 0; w < 8; w++) {
      if (w >> wb & 1) continue;
      const uint32_t lo = s.w[w], hi = s.w[w | (1 << wb)];
      const uint32_t t = ((lo >> sh) ^ hi) & m;
      s.w[w | (1 << wb)] = hi ^ t;
      s.w[w] = lo ^ (t << sh);
    }
  } else {
    constexpr int a = I - 5, b = J - 5;
#pragma unroll
    for (int w = 0; w < 8; w++) {
      if ((w >> a & 1) && !(w >> b & 1)) {
        const int v = w - (1 << a) + (1 << b);
        const uint32_t t = s.w[w]; s.w[w] = s.w[v]; s.w[v] = t;
      }
    }
  }
}
template<int A, int B> PG_HD void s_swap_axes(super8& s) {
  s_swap_bits<2 * A, 2 * B>(s);
  s_swap_bits<2 * A + 1, 2 * B + 1>(s);
}
// x -> -x on every axis (the quadrant-local reflection part of a global reflection).
PG_HD void s_negate(super8& s) {
#pragma unroll
  for (int i = 0; i < 8; i++) {
    uint32_t x = s.w[i];
    uint32_t t = ((x >> 2) ^ x) & 0x22222222u;
    x ^= t ^ (t << 2);
    t = ((x >> 8) ^ x) & 0x00f000f0u;
    x ^= t ^ (t << 8);
    s.w[i] = x;
  }
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t t = (s.w[2 * k] ^ s.w[2 * k + 1]) & 0xffff0000u;
    s.w[2 * k] ^= t;
    s.w[2 * k + 1] ^= t;
  }
  uint32_t t = s.w[2]; s.w[2] = s.w[6]; s.w[6] = t;
  t = s.w[3]; s.w[3] = s.w[7]; s.w[7] = t;
}

// phi_g(w) = g w g^-1 acting on Z_4^4: moves axis q to axis pi_g(q) and
// negates every axis when g contains the reflection.  out[phi(z)] = in[z].
// (Conjugation in the semidirect product of pentago/base/symmetry.h:15-20;
// the axis maps follow from commute_global_local_symmetries.)
template<int G> PG_HD void s_phi(super8& s) {
  if constexpr (G == 1) { s_swap_axes<1, 3>(s); s_swap_axes<0, 3>(s); s_swap_axes<2, 3>(s); }
  if constexpr (G == 2) { s_swap_axes<0, 3>(s); s_swap_axes<1, 2>(s); }
  if constexpr (G == 3) { s_swap_axes<2, 3>(s); s_swap_axes<0, 3>(s); s_swap_axes<1, 3>(s); }
  if constexpr (G == 4) { s_swap_axes<0, 3>(s); }
  if constexpr (G == 5) { s_swap_axes<1, 3>(s); s_swap_axes<0, 2>(s); }
  if constexpr (G == 6) { s_swap_axes<1, 2>(s); }
  if constexpr (G == 7) { s_swap_axes<2, 3>(s); s_swap_axes<0, 1>(s); }
  if constexpr (G >= 4) s_negate(s);
}
PG_HD void s_phi_runtime(super8& s, int g) {
  switch (g) {
    case 1: s_phi<1>(s); break;
    case 2: s_phi<2>(s); break;
    case 3: s_phi<3>(s); break;
    case 4: s_phi<4>(s); break;
    case 5: s_phi<5>(s); break;
    case 6: s_phi<6>(s); break;
    case 7: s_phi<7>(s); break;
    default: break;
  }
}
// transform_super (pentago/base/symmetry.cc:146-307) for s = (g, l):
// s(C) = phi_g(C - l).
PG_HD super8 s_transform(const super8& c, int g, int l) {
  super8 r = s_translate(c, l);
  s_phi_runtime(r, g);
  return r;
}

// ---------------------------------------------------------------------------
// super_wins: the set of local rotations after which a side has five in a row.
//
// Each of the 32 win patterns touches 2 or 3 quadrants.  For pattern p and
// quadrant q, the rotations r_q of q that cover p's cells in q form a 4-bit
// coverage vector c.  The pattern wins exactly on the product set of its
// quadrants' coverage vectors, so the answer is an OR over patterns of outer
// products.  Patterns are grouped by quadrant set: six pairs {01,02,03,12,13,
// 23} (with 6,6,2,2,6,6 patterns) and four triples {012,013,023,123} (one
// each).  A pair set's OR of outer products is a 16-bit 4x4 matrix W indexed
// r_a + 4 r_b; a triple's is a 64-bit cube indexed r_a + 4 r_b + 16 r_c.
//
// win_factor_entry(q, side_q) holds, for every set containing q, quadrant q's
// pre-spread factor so that a pair's W is an AND of two halfwords and a
// triple's an AND of three 64-bit words:
//   pair (a,b):   quadrant a stores c * 0x1111 (c replicated over r_b),
//                 quadrant b stores spread(c) (bit k -> nibble k all ones)
//   triple (a,b,c): a: c replicated 16x; b: spread(c) replicated 4x;
//                 c: 16-bit chunk k all ones iff bit k
// Halfwords 0..13 (words 0..6) hold the three pair sets containing q in the
// order of the list above, 14 halfwords in all and always word aligned with
// the partner quadrant; words 7..12 hold the three triple sets containing q.
// ---------------------------------------------------------------------------

PG_HD uint32_t spread4(uint32_t n) {
  const uint32_t x = n | (n << 3) | (n << 6) | (n << 9);
  return (x & 0x1111u) * 0xfu;
}

struct win_sets {
  uint32_t p01, p02, p03, p12, p13, p23;  // 16-bit matrices
  uint64_t t012, t013, t023, t123;        // 64-bit cubes
};

PG_HD uint32_t fold16(uint32_t x) { return (x | (x >> 16)) & 0xffffu; }
PG_HD uint64_t u64of(uint32_t lo, uint32_t hi) { return (uint64_t)hi << 32 | lo; }

// Combine four quadrant factor entries (16 words each) into the set matrices.
PG_HD win_sets win_combine(const uint32_t* e0, const uint32_t* e1, const uint32_t* e2,
                                                const uint32_t* e3) {
  win_sets s;
  s.p01 = fold16((e0[0] & e1[0]) | (e0[1] & e1[1]) | (e0[2] & e1[2]));
  s.p02 = fold16((e0[3] & e2[0]) | (e0[4] & e2[1]) | (e0[5] & e2[2]));
  s.p03 = fold16(e0[6] & e3[0]);
  s.p12 = fold16(e1[3] & e2[3]);
  s.p13 = fold16((e1[4] & e3[1]) | (e1[5] & e3[2]) | (e1[6] & e3[3]));
  s.p23 = fold16((e2[4] & e3[4]) | (e2[5] & e3[5]) | (e2[6] & e3[6]));
  s.t012 = u64of(e0[7] & e1[7] & e2[7], e0[8] & e1[8] & e2[8]);
  s.t013 = u64of(e0[9] & e1[9] & e3[7], e0[10] & e1[10] & e3[8]);
  s.t023 = u64of(e0[11] & e2[9] & e3[9], e0[12] & e2[10] & e3[10]);
  s.t123 = u64of(e1[11] & e2[11] & e3[11], e1[12] & e2[12] & e3[12]);
  return s;
}

// Set bits of win_sets, in the order of the struct.
enum : int {
  kP01 = 1, kP02 = 2, kP03 = 4, kP12 = 8, kP13 = 16, kP23 = 32,
  kT012 = 64, kT013 = 128, kT023 = 256, kT123 = 512, kAllSets = 1023
};
// The pattern sets touching quadrant D.
template<int D> constexpr int sets_with() {
  return D == 0 ? kP01 | kP02 | kP03 | kT012 | kT013 | kT023
       : D == 1 ? kP01 | kP12 | kP13 | kT012 | kT013 | kT123
       : D == 2 ? kP02 | kP12 | kP23 | kT012 | kT023 | kT123
                : kP03 | kP13 | kP23 | kT013 | kT023 | kT123;
}

// Only the sets in MASK, from four quadrant entries.
template<int MASK>
PG_HD win_sets win_combine_sets(const uint32_t* e0, const uint32_t* e1, const uint32_t* e2, const uint32_t* e3) {
  win_sets s = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (MASK & kP01) s.p01 = fold16((e0[0] & e1[0]) | (e0[1] & e1[1]) | (e0[2] & e1[2]));
  if (MASK & kP02) s.p02 = fold16((e0[3] & e2[0]) | (e0[4] & e2[1]) | (e0[5] & e2[2]));
  if (MASK & kP03) s.p03 = fold16(e0[6] & e3[0]);
  if (MASK & kP12) s.p12 = fold16(e1[3] & e2[3]);
  if (MASK & kP13) s.p13 = fold16((e1[4] & e3[1]) | (e1[5] & e3[2]) | (e1[6] & e3[3]));
  if (MASK & kP23) s.p23 = fold16((e2[4] & e3[4]) | (e2[5] & e3[5]) | (e2[6] & e3[6]));
  if (MASK & kT012) s.t012 = u64of(e0[7] & e1[7] & e2[7], e0[8] & e1[8] & e2[8]);
  if (MASK & kT013) s.t013 = u64of(e0[9] & e1[9] & e3[7], e0[10] & e1[10] & e3[8]);
  if (MASK & kT023) s.t023 = u64of(e0[11] & e2[9] & e3[9], e0[12] & e2[10] & e3[10]);
  if (MASK & kT123) s.t123 = u64of(e1[11] & e2[11] & e3[11], e1[12] & e2[12] & e3[12]);
  return s;
}

// Broadcast the set matrices in MASK into the 256-bit layout and OR them together.
template<int MASK>
PG_HD super8 win_assemble_sets(const win_sets& s) {
  super8 r;
  const uint32_t p01 = (MASK & kP01) ? s.p01 | (s.p01 << 16) : 0;
  uint32_t p02[2] = {0, 0}, p12[2] = {0, 0}, t012[2] = {0, 0};
  if (MASK & kP02) {
    p02[0] = ((s.p02 & 15) | (s.p02 >> 4 & 15) << 16) * 0x1111u;
    p02[1] = ((s.p02 >> 8 & 15) | (s.p02 >> 12 & 15) << 16) * 0x1111u;
  }
  if (MASK & kP12) {
    p12[0] = spread4(s.p12 & 15) | spread4(s.p12 >> 4 & 15) << 16;
    p12[1] = spread4(s.p12 >> 8 & 15) | spread4(s.p12 >> 12 & 15) << 16;
  }
  if (MASK & kT012) { t012[0] = (uint32_t)s.t012; t012[1] = (uint32_t)(s.t012 >> 32); }
#pragma unroll
  for (int r3 = 0; r3 < 4; r3++) {
    const uint32_t p03 = (MASK & kP03) ? (s.p03 >> (4 * r3) & 15) * 0x11111111u : 0;
    const uint32_t p13 = (MASK & kP13) ? spread4(s.p13 >> (4 * r3) & 15) * 0x10001u : 0;
    const uint32_t t013 = (MASK & kT013) ? (uint32_t)(s.t013 >> (16 * r3) & 0xffff) * 0x10001u : 0;
    const uint32_t m023 = (uint32_t)(s.t023 >> (16 * r3) & 0xffff);
    const uint32_t m123 = (uint32_t)(s.t123 >> (16 * r3) & 0xffff);
#pragma unroll
    for (int par = 0; par < 2; par++) {
      const int w = 2 * r3 + par;
      uint32_t v = p01 | p02[par] | p03 | p12[par] | p13 | t012[par] | t013;
      if (MASK & kP23)
        v |= ((s.p23 >> (2 * w) & 1) ? 0x0000ffffu : 0u) | ((s.p23 >> (2 * w + 1) & 1) ? 0xffff0000u : 0u);
      if (MASK & kT023) v |= ((m023 >> (8 * par) & 15) | (m023 >> (8 * par + 4) & 15) << 16) * 0x1111u;
      if (MASK & kT123) v |= spread4(m123 >> (8 * par) & 15) | spread4(m123 >> (8 * par + 4) & 15) << 16;
      r.w[w] = v;
    }
  }
  return r;
}

PG_HD super8 win_assemble(const win_sets& s) { return win_assemble_sets<kAllSets>(s); }

PG_HD void load_entry(const uint32_t* __restrict__ table, int q, int side_q, uint32_t* e) {
  const uint4* p = reinterpret_cast<const uint4*>(table + ((q * 512 + side_q) << 4));
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const uint4 v = ldg(p + i);
    e[4 * i] = v.x; e[4 * i + 1] = v.y; e[4 * i + 2] = v.z; e[4 * i + 3] = v.w;
  }
}

// super_wins of a side whose quadrants other than D are fixed: `fixed` holds
// the four quadrant entries (slot D unused) and c0 the part of the answer that
// comes from pattern sets not touching D.  `ed` is quadrant D's entry.
template<int D>
PG_HD super8 win_eval(const uint32_t* ed, const uint32_t* fixed, const super8& c0) {
  const uint32_t* e0 = D == 0 ? ed : fixed;
  const uint32_t* e1 = D == 1 ? ed : fixed + 16;
  const uint32_t* e2 = D == 2 ? ed : fixed + 32;
  const uint32_t* e3 = D == 3 ? ed : fixed + 48;
  constexpr int M = sets_with<D>();
  return s_or(win_assemble_sets<M>(win_combine_sets<M>(e0, e1, e2, e3)), c0);
}
// The part of super_wins that does not depend on quadrant D.
template<int D>
PG_HD super8 win_const(const uint32_t* fixed) {
  constexpr int M = kAllSets & ~sets_with<D>();
  return win_assemble_sets<M>(win_combine_sets<M>(fixed, fixed + 16, fixed + 32, fixed + 48));
}

// super_wins (pentago/base/superscore.cc:38-96) for a whole side.
PG_HD super8 s_super_wins(const uint32_t* __restrict__ table, uint64_t side) {
  uint32_t e0[16], e1[16], e2[16], e3[16];
  load_entry(table, 0, (int)(side & 511), e0);
  load_entry(table, 1, (int)(side >> 16 & 511), e1);
  load_entry(table, 2, (int)(side >> 32 & 511), e2);
  load_entry(table, 3, (int)(side >> 48 & 511), e3);
  return win_assemble(win_combine(e0, e1, e2, e3));
}

// ---------------------------------------------------------------------------
// Halfsupers (pentago/mid/halfsuper.h:4-60): the half of a super with one
// rotation parity.  h(p)(a,b,c,d) = s(2a + (b+c+d+p)%2, b, c, d), stored at
// bit a + 2b + 8c + 32d of four 32-bit words; within a word a, b and c sit in
// bits 0-4 and the word number is d.
// ---------------------------------------------------------------------------

struct half4 {
  uint32_t w[4];
};

PG_HD half4 h_zero() { return half4{{0, 0, 0, 0}}; }
PG_HD half4 h_not(const half4& a) { return half4{{~a.w[0], ~a.w[1], ~a.w[2], ~a.w[3]}}; }
PG_HD half4 h_or(const half4& a, const half4& b) {
  return half4{{a.w[0] | b.w[0], a.w[1] | b.w[1], a.w[2] | b.w[2], a.w[3] | b.w[3]}};
}
PG_HD half4 h_and(const half4& a, const half4& b) {
  return half4{{a.w[0] & b.w[0], a.w[1] & b.w[1], a.w[2] & b.w[2], a.w[3] & b.w[3]}};
}
PG_HD half4 h_from(const uint4 v) { return half4{{v.x, v.y, v.z, v.w}}; }
PG_HD uint4 h_to(const half4& h) { return make_uint4(h.w[0], h.w[1], h.w[2], h.w[3]); }

// rmax on a halfsuper, which flips its parity: an OR over the parity pair
// (axis 0), and +-1 shifts along b (bits 1-2 of each byte), c (byte within a
// word) and d (word).
PG_HD half4 h_rmax(const half4& x) {
  half4 r;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const uint32_t v = x.w[i];
    const uint32_t t = (v | (v >> 1)) & 0x55555555u;
    const uint32_t a = t | (t << 1);
    const uint32_t b = ((v >> 2) & 0x3f3f3f3fu) | ((v << 6) & 0xc0c0c0c0u) |
                       ((v << 2) & 0xfcfcfcfcu) | ((v >> 6) & 0x03030303u);
    const uint32_t c = funnel_r(v, v, 8) | funnel_r(v, v, 24);
    r.w[i] = a | b | c;
  }
  const uint32_t d0 = x.w[1] | x.w[3], d1 = x.w[0] | x.w[2];
  r.w[0] |= d0; r.w[2] |= d0;
  r.w[1] |= d1; r.w[3] |= d1;
  return r;
}

// The parity-p half of a super: from nibble j = b + 4c + 16d of s keep bits
// q and q + 2, q = (b + c + d + p) % 2.
PG_HD half4 s_split(const super8& s, int p) {
  half4 h = h_zero();
#pragma unroll
  for (int w = 0; w < 8; w++) {
    const uint32_t M = ((w >> 1) ^ p) & 1 ? 0xf0f00f0fu : 0x0f0ff0f0u;  // nibbles with q = 1
    uint32_t z = ((s.w[w] & ~M) | ((s.w[w] >> 1) & M)) & 0x55555555u;
    z = (z | (z >> 1)) & 0x33333333u;
    z = (z | (z >> 2)) & 0x0f0f0f0fu;
    z = (z | (z >> 4)) & 0x00ff00ffu;
    z = (z | (z >> 8)) & 0x0000ffffu;
    h.w[w >> 1] |= z << (16 * (w & 1));
  }
  return h;
}

}  // namespace pg
