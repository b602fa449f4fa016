// Host planning for end-engine block lines.  See lines.h.
#include "lines.h"
#include <algorithm>
#include <cstring>

namespace pg {

section_t section_t::from_sig(uint64_t sig) {
  section_t s;
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 2; k++) s.c[q][k] = uint8_t(sig >> (16 * q + 8 * k));
  return s;
}

uint64_t section_t::sig() const {
  uint64_t r = 0;
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 2; k++) r |= uint64_t(c[q][k]) << (16 * q + 8 * k);
  return r;
}

int section_t::sum() const {
  int t = 0;
  for (int q = 0; q < 4; q++) t += c[q][0] + c[q][1];
  return t;
}

bool section_t::valid() const {  // section.cc:116-126
  int b = 0, w = 0;
  for (int q = 0; q < 4; q++) {
    if (c[q][0] + c[q][1] > 9) return false;
    b += c[q][0];
    w += c[q][1];
  }
  return w <= b && b <= w + 1;
}

void section_t::shape(int* s) const {
  const auto& T = tables();
  for (int q = 0; q < 4; q++) {
    const int k = rmin_bucket(c[q][0], c[q][1]);
    s[q] = T.rmin_off[k + 1] - T.rmin_off[k];
  }
}

section_t section_t::transform(int g) const {
  static const int source[4][4] = {{0, 1, 2, 3}, {1, 3, 0, 2}, {3, 2, 1, 0}, {2, 0, 3, 1}};
  section_t t;
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 2; k++) t.c[i][k] = c[source[g & 3][i]][k];
  if (g & 4)
    for (int k = 0; k < 2; k++) std::swap(t.c[0][k], t.c[3][k]);
  return t;
}

section_t section_t::standardize(int* transform_out) const {
  section_t best = *this;
  int bg = 0;
  for (int g = 1; g < 8; g++) {
    const section_t t = transform(g);
    if (best.sig() > t.sig()) { best = t; bg = g; }
  }
  if (transform_out) *transform_out = bg;
  return best;
}

section_t section_t::child(int q) const {
  section_t s = *this;
  s.c[q][sum() & 1]++;
  return s;
}

void quadrant_permutation(int g, int* p) {
  section_t s;
  memset(&s, 0, sizeof s);
  for (int i = 0; i < 4; i++) s.c[i][0] = uint8_t(i);
  const section_t t = s.transform(g);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      if (t.c[j][0] == i) p[i] = j;
}

static int bshape(int shape, int block) { return std::min(shape, 8 * (block + 1)) - 8 * block; }

bool line_shapes(const line_in_t& in, line_shapes_t& o, std::string& error) {
  const section_t sec = section_t::from_sig(in.section);
  if (!sec.valid() || sec.sum() > 35) { error = "invalid section"; return false; }
  if (in.dim < 0 || in.dim > 3) { error = "invalid dimension"; return false; }
  if (sec.c[in.dim][0] + sec.c[in.dim][1] >= 9) { error = "line along a full quadrant"; return false; }
  int shape[4], cshape[4], block0[4];
  sec.shape(shape);
  const section_t child = sec.child(in.dim);
  child.shape(cshape);
  for (int i = 0, k = 0; i < 4; i++) block0[i] = i == in.dim ? 0 : in.block_base[k++];
  for (int i = 0; i < 4; i++)
    if (i != in.dim && 8 * block0[i] >= shape[i]) { error = "block_base out of range"; return false; }
  if (in.length != (shape[in.dim] + 7) / 8) { error = "line length does not match the section"; return false; }
  o.block_stride = 8;
  for (int i = 0; i < 4; i++) {
    o.out_shape[i] = i == in.dim ? shape[i] : bshape(shape[i], block0[i]);
    o.in_shape[i] = i == in.dim ? cshape[i] : o.out_shape[i];
    if (i != in.dim) o.block_stride *= o.out_shape[i];
  }
  if (sec.sum() == 35)
    for (int i = 0; i < 4; i++) o.in_shape[i] = 0;
  o.child_std = child.standardize(&o.st);
  int perm[4];
  quadrant_permutation(invert_global(o.st), perm);
  for (int i = 0; i < 4; i++) if (perm[i] == in.dim) o.child_dim = i;
  o.input_blocks = (o.in_shape[in.dim] + 7) / 8;
  return true;
}

bool plan_line(const line_in_t& in, line_dev_t& d, std::string& error) {
  const auto& T = tables();
  line_shapes_t s;
  if (!line_shapes(in, s, error)) return false;
  memset(&d, 0, sizeof d);
  const section_t sec = section_t::from_sig(in.section);
  const int dim = in.dim;
  d.dim = dim;
  d.turn = sec.sum() & 1;
  d.slice35 = sec.sum() == 35;
  d.flags = in.flags;
  d.nparent = s.out_shape[dim];
  d.nchild = s.in_shape[dim];
  d.length = in.length;
  d.input_blocks = s.input_blocks;
  d.child_dim = s.child_dim;
  quadrant_permutation(invert_global(s.st), d.perm);
  for (int i = 0, k = 0; i < 4; i++) {
    d.block0[i] = i == dim ? 0 : in.block_base[k];
    if (i != dim) { d.odims[k] = i; d.cross[k] = s.out_shape[i]; k++; }
    d.out_shape[i] = s.out_shape[i];
    d.rmin_off[i] = T.rmin_off[rmin_bucket(sec.c[i][0], sec.c[i][1])];
  }
  for (int i = 0; i < 4; i++) d.first_child_block[i] = d.block0[d.perm[i]];
  // inverse_transform = (-(st&3), 0x55 (st&3)) * (st&4, 0)  (compute.cc:76-77)
  {
    const int st = s.st;
    const int ag = (4 - (st & 3)) & 3, al = 0x55 * (st & 3), bg = st & 4;
    d.g = T.gprod[ag][bg];
    d.inv_l = sigma_apply(line_sigma(dim, d.g), T.commute[bg][al]);
  }
  const axis_perm sg = line_sigma(dim, d.g);
  if (sg.to[s.child_dim] != 3) { error = "child dimension does not map to the line axis"; return false; }
  // Reflection bookkeeping (compute.cc:96-122)
  if (s.st & 4) {
    for (int i = 0; i < 4; i++) {
      const int k = rmin_bucket(s.child_std.c[i][0], s.child_std.c[i][1]);
      d.refl_moves[i] = T.rmin_moved[k];
      const int n = s.in_shape[d.perm[i]];
      const uint16_t* crmin = T.rmin_flat + T.rmin_off[k];
      for (int j = 0; j < n; j++) {
        const uint16_t q = crmin[8 * d.first_child_block[i] + j];
        const int rq = T.pack[T.refl[T.unpack[q][0]]] + 2 * T.pack[T.refl[T.unpack[q][1]]];
        const int rot = T.rmin_inv[rq] & 3;
        if (i == s.child_dim) { if (j < kMaxLine) d.csym[j] = uint8_t(rot); }
        else if (j < 8) d.xsym[i][j] = uint8_t(sigma_apply(sg, rot << (2 * i)));
      }
    }
  }
  d.line_moves = d.refl_moves[d.child_dim];
  for (int side = 0; side < 2; side++) {  // stones of mover (side 0) and opponent in the line quadrant
    const int k = sec.c[dim][side ? 1 - d.turn : d.turn];
    d.pat_off[side] = T.cls_off[k];
    d.npat[side] = T.cls_off[k + 1] - T.cls_off[k];
  }
  for (int t = 0; t < 17; t++) {
    d.term_pat[t] = T.term_pat[dim][t];
    for (int k = 0; k < 2; k++) d.term_q[t][k] = T.term_other[dim][t][k];
  }
  for (int u = 0; u < 15; u++) {
    d.miss_pat[u] = T.miss_pat[dim][u];
    for (int k = 0; k < 3; k++) d.miss_q[u][k] = T.miss_quad[dim][u][k];
  }
  const int counts[3] = {d.nparent, d.nchild, d.npat[0] + d.npat[1]};
  for (int i = 0; i < 3; i++) d.split_m[i] = counts[i] > 0 ? 0xffffffffu / uint32_t(counts[i]) : 0u;
  d.input = in.input;
  d.output = in.output;
  if (s.input_blocks > kMaxBlocks || in.length > kMaxBlocks || d.nchild > kMaxLine) {
    error = "line too long";
    return false;
  }
  for (int k = 0; k < s.input_blocks; k++)
    d.in_off[k] = in.input_offsets ? in.input_offsets[k] : k * (in.input_stride ? in.input_stride : s.block_stride);
  for (int k = 0; k < in.length; k++)
    d.out_off[k] = in.output_offsets ? in.output_offsets[k] : k * (in.output_stride ? in.output_stride : s.block_stride);
  return true;
}

void line_records(uint64_t section, int dim, line_rec_set& out) {
  std::vector<parent_rec>& recs = out.recs;
  std::vector<child_rec>& crecs = out.crecs;
  const auto& T = tables();
  const section_t sec = section_t::from_sig(section);
  const int turn = sec.sum() & 1;
  const int k = rmin_bucket(sec.c[dim][0], sec.c[dim][1]);
  const int n = T.rmin_off[k + 1] - T.rmin_off[k];
  int nchild = 0;
  if (sec.sum() < 35) {
    const section_t child = sec.child(dim);
    const int kc = rmin_bucket(child.c[dim][0], child.c[dim][1]);
    nchild = T.rmin_off[kc + 1] - T.rmin_off[kc];
  }
  recs.assign(n, parent_rec{});
  for (int i = 0; i < n; i++) {
    const uint16_t q = T.rmin_flat[T.rmin_off[k] + i];
    const uint16_t s0 = T.unpack[q][turn], s1 = T.unpack[q][1 - turn];
    parent_rec& r = recs[i];
    r.c0 = T.cls_rank[s0];
    r.c1 = T.cls_rank[s1];
    r.rot = uint8_t(T.cls_rot[s0] | T.cls_rot[s1] << 2);
    int m = 0;
    for (int b = 0, p3 = 1; b < 9; b++, p3 *= 3)
      if (!((s0 | s1) >> b & 1)) {
        const int ir = T.rmin_inv[q + (1 + turn) * p3];
        r.mv[m++] = uint16_t((ir & 3) * nchild + (ir >> 2));
        for (int k = 0; k < 4; k++) r.usub[k] |= T.term_sub[dim][s0 | 1 << b][k];
      }
    r.nmoves = uint8_t(m);
  }
  crecs.clear();
  if (sec.sum() < 35) {
    const section_t child = sec.child(dim);
    const int kc = rmin_bucket(child.c[dim][0], child.c[dim][1]);
    const int nc = T.rmin_off[kc + 1] - T.rmin_off[kc];
    crecs.assign(nc, child_rec{});
    for (int j = 0; j < nc; j++) {
      const uint16_t mover = T.unpack[T.rmin_flat[T.rmin_off[kc] + j]][turn];
      for (int r = 0; r < 4; r++) crecs[j].csub[r] = T.term_sub[dim][mover][r];
    }
  }
  // Cross quadrants: the coverage of every win pattern by each side's stones
  out.xrecs.clear();
  for (int q = 0; q < 4; q++) {
    out.xoff[q] = int32_t(out.xrecs.size());
    if (q == dim) continue;
    const int kq = rmin_bucket(sec.c[q][0], sec.c[q][1]);
    for (int f = T.rmin_off[kq]; f < T.rmin_off[kq + 1]; f++)
      for (int side = 0; side < 2; side++) {
        const uint16_t stones = T.unpack[T.rmin_flat[f]][side ? 1 - turn : turn];
        cross_rec e{};
        for (int p = 0; p < 32; p++) e.cov[p >> 3] |= uint32_t(T.cov[p][q][stones]) << (4 * (p & 7));
        out.xrecs.push_back(e);
      }
  }
  // Stone-pattern classes of the line quadrant: the terms they cover
  out.precs.clear();
  for (int side = 0; side < 2; side++) {
    const int kc = sec.c[dim][side ? 1 - turn : turn];
    for (int r = T.cls_off[kc]; r < T.cls_off[kc + 1]; r++) {
      class_rec e{};
      for (int k = 0; k < 4; k++) e.sub[k] = T.term_sub[dim][T.cls_masks[r]][k];
      out.precs.push_back(e);
    }
  }
}

}  // namespace pg
