// ORACLE — test infrastructure, not product code.
//
// A CPU restatement of the rivet-h26x encoders' motion-estimation path,
// written from the reference's Rust sources (cited per function, paths
// relative to the rivet-h26x crate). It is the parity checker for the CUDA
// library and, built with its AVX2 distortion kernels, the timed host
// baseline. Only tests/, __graft_entry__.smoke() and bench.py's CPU legs
// load it; the product library (librivet_me.so) never links or calls it.
//
// Parity pins: the reference ships no golden motion vectors (its tests are
// property tests), so this restatement is pinned by re-running those
// property tests against it — distortion closed forms and the direct
// Hadamard product (dsp/distortion.rs:465-576), plane equality against a
// direct evaluation of 8.4.2.2.1 and 8.5.3.3.3.1 (h264_hpel.rs:1033-1075,
// h265_search.rs:289-353), and the translation-found searches
// (h264_me.rs:3937-4118, h265_me.rs:5222-5369) — plus golden fixtures
// committed under tests/golden/ that freeze its outputs. The Rust crate
// cannot be built in this environment (no Rust toolchain), so MV-for-MV
// parity with a reference run is not pinned beyond those tests.
//
// Floating point: the reference computes its Lagrangians and its H.264
// rate table in f32 (h264_hpel.rs:407-469, h265_intra.rs:1141-2013). This
// file is compiled with -ffp-contract=off so every f32 expression rounds
// exactly as Rust's does (Rust never fuses a multiply-add).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/rivet_me.h"

namespace orc {

struct Mv {
  int16_t x = 0, y = 0;
  Mv() = default;
  Mv(int x_, int y_) : x((int16_t)x_), y((int16_t)y_) {}
  bool operator==(const Mv& o) const { return x == o.x && y == o.y; }
  bool operator!=(const Mv& o) const { return !(*this == o); }
};

// ---------------------------------------------------------------------------
// Planes: padded, edge-replicated, row-major (hevc/frame.rs:135-200,
// h264/frame.rs PaddedPlane — the same layout).
// ---------------------------------------------------------------------------
template <class S>
struct Plane {
  std::vector<S> data;
  int width = 0, height = 0, pad = 0, stride = 0;
  Plane() = default;
  Plane(int w, int h, int p)
      : data((size_t)(w + 2 * p) * (h + 2 * p)), width(w), height(h), pad(p), stride(w + 2 * p) {}
  ptrdiff_t origin() const { return (ptrdiff_t)pad * stride + pad; }
  ptrdiff_t offset(int x, int y) const { return origin() + (ptrdiff_t)y * stride + x; }
  int rows() const { return height + 2 * pad; }
  // hevc/frame.rs:171-176: coordinates clamped to the visible picture.
  S at_clamped(int x, int y) const {
    int xx = std::clamp(x, 0, width - 1), yy = std::clamp(y, 0, height - 1);
    return data[offset(xx, yy)];
  }
  // The visible picture from `src` (stride `ss`), then the border replicated
  // (extend_rows over all rows, extend_top, extend_bottom: frame.rs:178-214).
  void load(const S* src, ptrdiff_t ss) {
    for (int y = 0; y < height; ++y)
      std::memcpy(&data[offset(0, y)], src + (ptrdiff_t)y * ss, sizeof(S) * width);
    for (int y = 0; y < height; ++y) {
      ptrdiff_t row = offset(0, y);
      S l = data[row], r = data[row + width - 1];
      for (int i = 1; i <= pad; ++i) data[row - i] = l;
      for (int i = 0; i < pad; ++i) data[row + width + i] = r;
    }
    ptrdiff_t first = origin() - pad;
    for (int i = 1; i <= pad; ++i)
      std::memcpy(&data[first - (ptrdiff_t)i * stride], &data[first], sizeof(S) * stride);
    ptrdiff_t last = origin() + (ptrdiff_t)(height - 1) * stride - pad;
    for (int i = 1; i <= pad; ++i)
      std::memcpy(&data[last + (ptrdiff_t)i * stride], &data[last], sizeof(S) * stride);
  }
};

// ---------------------------------------------------------------------------
// Distortion (dsp/distortion.rs)
// ---------------------------------------------------------------------------
// dsp/distortion.rs:254-270
template <class S>
uint32_t sad_scalar(const S* a, ptrdiff_t as, const S* b, ptrdiff_t bs, int w, int h) {
  uint32_t sum = 0;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      int d = (int)a[y * as + x] - (int)b[y * bs + x];
      sum += (uint32_t)(d < 0 ? -d : d);
    }
  return sum;
}

// dsp/distortion.rs:326-343 (rows, then columns).
inline void hadamard4x4(int32_t d[16]) {
  for (int i = 0; i < 4; ++i) {
    int32_t a = d[i * 4], b = d[i * 4 + 1], c = d[i * 4 + 2], e = d[i * 4 + 3];
    int32_t s0 = a + e, s1 = b + c, s2 = b - c, s3 = a - e;
    d[i * 4] = s0 + s1;
    d[i * 4 + 1] = s3 + s2;
    d[i * 4 + 2] = s0 - s1;
    d[i * 4 + 3] = s3 - s2;
  }
  for (int j = 0; j < 4; ++j) {
    int32_t a = d[j], b = d[4 + j], c = d[8 + j], e = d[12 + j];
    int32_t s0 = a + e, s1 = b + c, s2 = b - c, s3 = a - e;
    d[j] = s0 + s1;
    d[4 + j] = s3 + s2;
    d[8 + j] = s0 - s1;
    d[12 + j] = s3 - s2;
  }
}

// dsp/distortion.rs:350-381: per 4x4 tile (sum + 1) >> 1.
template <class S>
uint32_t satd_scalar(const S* a, ptrdiff_t as, const S* b, ptrdiff_t bs, int w, int h) {
  uint32_t total = 0;
  for (int by = 0; by < h; by += 4)
    for (int bx = 0; bx < w; bx += 4) {
      int32_t d[16];
      for (int y = 0; y < 4; ++y)
        for (int x = 0; x < 4; ++x)
          d[y * 4 + x] = (int)a[(by + y) * as + bx + x] - (int)b[(by + y) * bs + bx + x];
      hadamard4x4(d);
      uint32_t sum = 0;
      for (int k = 0; k < 16; ++k) sum += (uint32_t)(d[k] < 0 ? -d[k] : d[k]);
      total += (sum + 1) >> 1;
    }
  return total;
}

template <class S>
struct Dist {
  uint32_t (*sad)(const S*, ptrdiff_t, const S*, ptrdiff_t, int, int);
  uint32_t (*satd)(const S*, ptrdiff_t, const S*, ptrdiff_t, int, int);
};
template <class S>
Dist<S> dist_scalar() { return Dist<S>{&sad_scalar<S>, &satd_scalar<S>}; }
// AVX2 rungs (me_oracle_avx2.cpp), following distortion_x86*.rs's designs.
Dist<uint8_t> dist_avx2_u8();
Dist<uint16_t> dist_avx2_u16();

// ---------------------------------------------------------------------------
// H.264 (encode/h264_hpel.rs)
// ---------------------------------------------------------------------------
inline int tap6(int a, int b, int c, int d, int e, int f) { return a + f - 5 * (b + e) + 20 * (c + d); }

// h264_hpel.rs:129-189: the three half-sample planes of the padded plane d.
// Positions whose six-tap window would leave the plane hold the integer
// sample.
template <class S>
void hpel_planes(const S* d, size_t len, int stride, int maxv, S* h, S* v, S* c) {
  int rows = (int)(len / stride);
  std::memcpy(h, d, len * sizeof(S));
  std::memcpy(v, d, len * sizeof(S));
  std::memcpy(c, d, len * sizeof(S));
  for (int y = 0; y < rows; ++y) {
    const S* row = d + (size_t)y * stride;
    S* out = h + (size_t)y * stride;
    for (int x = 2; x < stride - 3; ++x) {
      int t = tap6(row[x - 2], row[x - 1], row[x], row[x + 1], row[x + 2], row[x + 3]);
      out[x] = (S)std::clamp((t + 16) >> 5, 0, maxv);
    }
  }
  std::vector<int> inter(stride);
  for (int y = 2; y < std::max(rows - 3, 0); ++y) {
    for (int x = 0; x < stride; ++x) {
      inter[x] = tap6(d[(size_t)(y - 2) * stride + x], d[(size_t)(y - 1) * stride + x],
                      d[(size_t)y * stride + x], d[(size_t)(y + 1) * stride + x],
                      d[(size_t)(y + 2) * stride + x], d[(size_t)(y + 3) * stride + x]);
    }
    S* vo = v + (size_t)y * stride;
    for (int x = 0; x < stride; ++x) vo[x] = (S)std::clamp((inter[x] + 16) >> 5, 0, maxv);
    S* co = c + (size_t)y * stride;
    for (int x = 2; x < stride - 3; ++x) {
      int t = tap6(inter[x - 2], inter[x - 1], inter[x], inter[x + 1], inter[x + 2], inter[x + 3]);
      co[x] = (S)std::clamp((t + 512) >> 10, 0, maxv);
    }
  }
}

// The integer plane and its b, h, j half planes (h264_hpel.rs:38, 193-202).
template <class S>
struct Hpel {
  std::vector<S> p[3];
  void build(const Plane<S>& g, int maxv) {  // build_hpel, h264_hpel.rs:95-124
    for (auto& q : p) q.assign(g.data.size(), S(0));
    hpel_planes(g.data.data(), g.data.size(), g.stride, maxv, p[0].data(), p[1].data(), p[2].data());
  }
};

// h264_hpel.rs:205-222: per quarter fraction (fy*4+fx) the one or two
// (plane, dx, dy) views whose rounded average is the sample.
static const int8_t H264_QPEL[16][6] = {
    {0, 0, 0, -1, 0, 0}, {0, 0, 0, 1, 0, 0}, {1, 0, 0, -1, 0, 0}, {1, 0, 0, 0, 1, 0},
    {0, 0, 0, 2, 0, 0},  {1, 0, 0, 2, 0, 0}, {1, 0, 0, 3, 0, 0},  {1, 0, 0, 2, 1, 0},
    {2, 0, 0, -1, 0, 0}, {2, 0, 0, 3, 0, 0}, {3, 0, 0, -1, 0, 0}, {3, 0, 0, 2, 1, 0},
    {2, 0, 0, 0, 0, 1},  {2, 0, 0, 1, 0, 1}, {3, 0, 0, 1, 0, 1},  {2, 1, 0, 1, 0, 1},
};

template <class S>
struct MeRef {
  const Plane<S>* g = nullptr;
  const S* planes[4] = {nullptr, nullptr, nullptr, nullptr};
  MeRef() = default;
  MeRef(const Plane<S>* g_, const Hpel<S>* h) : g(g_) {
    planes[0] = g->data.data();
    for (int k = 0; k < 3; ++k) planes[k + 1] = h->p[k].data();
  }
  const S* at(int plane, int x, int y) const { return planes[plane] + g->offset(x, y); }
  // MeRef::pred (h264_hpel.rs:258-281) + avg_into (353-399): a view into a
  // plane, or the rounded average of two views into buf (stride 16... or w).
  const S* pred(int x, int y, Mv mv, int w, int h, S* buf, int* stride) const {
    int xi = x + (mv.x >> 2), yi = y + (mv.y >> 2);
    const int8_t* q = H264_QPEL[(mv.y & 3) * 4 + (mv.x & 3)];
    const S* a = at(q[0], xi + q[1], yi + q[2]);
    if (q[3] < 0) {
      *stride = g->stride;
      return a;
    }
    const S* b = at(q[3], xi + q[4], yi + q[5]);
    int gs = g->stride;
    for (int yy = 0; yy < h; ++yy)
      for (int xx = 0; xx < w; ++xx)
        buf[yy * w + xx] = (S)(((int)a[yy * gs + xx] + (int)b[yy * gs + xx] + 1) >> 1);
    *stride = w;
    return buf;
  }
};

// h264_hpel.rs:407-429 (f32 arithmetic, as the reference's).
inline float h264_mvd_bits(int d) {
  uint32_t a = (uint32_t)(d < 0 ? -(int64_t)d : d);
  if (a == 0) return 1.0f;
  float prefix = (float)std::min(a, 9u);
  float bits = 1.0f + 0.85f * prefix;
  if (a < 9) {
    bits += 0.85f;
  } else {
    uint32_t v = a - 9, k = 3;
    while (v >= (1u << k)) {
      v -= 1u << k;
      k += 1;
    }
    bits += (float)(k - 3 + 1 + k);
  }
  return bits + 1.0f;
}

constexpr int MV_SPAN = 4096;  // h264_hpel.rs:432
constexpr int MV_TAB = 2 * MV_SPAN + 1;

// MvCostTable::new (h264_hpel.rs:453-459).
inline void h264_cost_table(float lambda, uint16_t* tab) {
  for (int d = -MV_SPAN; d <= MV_SPAN; ++d) {
    float t = std::min(lambda * h264_mvd_bits(d) + 0.5f, 65535.0f);
    tab[d + MV_SPAN] = (uint16_t)t;
  }
}
inline uint32_t h264_mv_comp(const uint16_t* tab, int d) {
  return tab[std::clamp(d, -MV_SPAN, MV_SPAN) + MV_SPAN];
}

// lambda_satd (h264_analyse.rs:402-404).
inline float h264_lambda_satd(int qp) {
  return std::sqrt(0.85f * std::exp2((float)(qp - 12) / 3.0f));
}

// search_bounds (h264_hpel.rs:476-488): (lo_x, hi_x, lo_y, hi_y).
inline void h264_search_bounds(int width, int height, int pad, int x, int y, int w, int h,
                               int vr, int b[4]) {
  b[0] = 4 - pad - x;
  b[1] = width + pad - (w + 4) - x;
  b[2] = std::max(4 - pad - y, -vr);
  b[3] = std::min(height + pad - (h + 4) - y, vr);
}

struct MeCfg {  // h264_hpel.rs:492-519
  int range = 0, hpel_iters = 0, qpel_iters = 0;
  bool umh = false, qpel_diamond = false, dia = false;
  static MeCfg score() { return MeCfg{}; }
};

// One block's search (Search, h264_hpel.rs:522-1021).
template <class S>
struct H264Search {
  const Dist<S>* dist;
  const MeRef<S>* r;
  const S* src;
  ptrdiff_t src_stride;
  int x, y, w, h;
  Mv pred;
  const uint16_t* tab;
  int bounds[4];
  uint32_t n_sad = 0, n_satd = 0;

  const S* hot_at(int plane, int dx, int dy) const { return r->at(plane, x + dx, y + dy); }
  uint32_t rate(int qx, int qy) const {
    return h264_mv_comp(tab, qx - pred.x) + h264_mv_comp(tab, qy - pred.y);
  }
  // sad_full (h264_hpel.rs:624-634)
  uint32_t sad_full(int fx, int fy) {
    ++n_sad;
    return dist->sad(src, src_stride, hot_at(0, fx, fy), r->g->stride, w, h) + rate(fx * 4, fy * 4);
  }
  // satd (h264_hpel.rs:682-705): SATD of the prediction at mv, no rate.
  uint32_t satd(Mv mv) {
    ++n_satd;
    S buf[64 * 64];
    int ps;
    const S* p = r->pred(x, y, mv, w, h, buf, &ps);
    return dist->satd(src, src_stride, p, ps, w, h);
  }

  // int_search (h264_hpel.rs:789-952). Returns the whole-sample winner (in
  // quarter samples) and its SAD + rate.
  Mv int_search(const Mv* cands, int nc, const MeCfg& cfg, uint32_t* cost_out) {
    int lx = bounds[0], hx = bounds[1], ly = bounds[2], hy = bounds[3];
    auto clampf = [&](Mv m, int* fx, int* fy) {
      *fx = std::clamp((m.x + 2) >> 2, lx, hx);
      *fy = std::clamp((m.y + 2) >> 2, ly, hy);
    };
    int bx, by;
    clampf(pred, &bx, &by);
    // The predictor and the distinct candidates, scored in order.
    int px[16], py[16], np = 0;
    px[np] = bx;
    py[np] = by;
    ++np;
    int tx[12], ty[12], nt = 0;
    for (int i = 0; i < nc; ++i) {
      int fx, fy;
      clampf(cands[i], &fx, &fy);
      bool seen = (fx == bx && fy == by);
      for (int k = 0; k < nt && !seen; ++k) seen = (tx[k] == fx && ty[k] == fy);
      if (seen) continue;
      if (nt < 12) {
        tx[nt] = fx;
        ty[nt] = fy;
        ++nt;
      }
      px[np] = fx;
      py[np] = fy;
      ++np;
    }
    uint32_t sc[16] = {};
    for (int k = 0; k < np; ++k) sc[k] = sad_full(px[k], py[k]);
    uint32_t bcost = sc[0];
    for (int k = 1; k < np; ++k)
      if (sc[k] < bcost) {
        bcost = sc[k];
        bx = px[k];
        by = py[k];
      }
    int sx = bx, sy = by;
    int bx0 = std::max(sx - cfg.range, lx), bx1 = std::min(sx + cfg.range, hx);
    int by0 = std::max(sy - cfg.range, ly), by1 = std::min(sy + cfg.range, hy);
    auto ok = [&](int fx, int fy) { return fx >= bx0 && fx <= bx1 && fy >= by0 && fy <= by1; };
    // ring: points around a fixed centre, scored together, accepted in order
    // where strictly cheaper; returns the offset index of the last taken.
    auto ring = [&](int cx, int cy, const int (*offs)[2], int n) -> int {
      int qx[16], qy[16], idx[16], nq = 0;
      for (int k = 0; k < n; ++k) {
        int fx = cx + offs[k][0], fy = cy + offs[k][1];
        if (ok(fx, fy) && !(fx == cx && fy == cy)) {
          idx[nq] = k;
          qx[nq] = fx;
          qy[nq] = fy;
          ++nq;
        }
      }
      uint32_t s[16];
      for (int k = 0; k < nq; ++k) s[k] = sad_full(qx[k], qy[k]);
      int moved = -1;
      for (int k = 0; k < nq; ++k)
        if (s[k] < bcost) {
          bcost = s[k];
          bx = qx[k];
          by = qy[k];
          moved = idx[k];
        }
      return moved;
    };
    auto try_at = [&](int fx, int fy) {
      if (ok(fx, fy) && !(fx == bx && fy == by)) {
        uint32_t s = sad_full(fx, fy);
        if (s < bcost) {
          bcost = s;
          bx = fx;
          by = fy;
        }
      }
    };
    if (cfg.umh) {
      int cx = bx, cy = by;
      for (int rr = 2; rr <= cfg.range; rr += 2) {
        const int cross[4][2] = {{-rr, 0}, {rr, 0}, {0, -rr}, {0, rr}};
        for (auto& o : cross) try_at(cx + o[0], cy + o[1]);
      }
      static const int HEX12[12][2] = {{-2, 1}, {-2, -1}, {2, 1},  {2, -1}, {-1, 2},  {1, 2},
                                       {-1, -2}, {1, -2}, {-2, 2}, {2, 2},  {-2, -2}, {2, -2}};
      for (int rr = 4; rr <= cfg.range; rr += 4)
        for (auto& o : HEX12) try_at(cx + o[0] * rr / 2, cy + o[1] * rr / 2);
    }
    if (cfg.dia) {
      static const int DIA[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
      for (int it = 0; it < cfg.range; ++it) {
        int cx = bx, cy = by;
        ring(cx, cy, DIA, 4);
        if (bx == cx && by == cy) break;
      }
      *cost_out = bcost;
      return Mv(bx * 4, by * 4);
    }
    static const int HEX[6][2] = {{-2, 0}, {-1, -2}, {1, -2}, {2, 0}, {1, 2}, {-1, 2}};
    int dir = ring(bx, by, HEX, 6);
    int it = 1;
    while (dir != -1 && it < cfg.range) {
      int ks[3] = {(dir + 5) % 6, dir, (dir + 1) % 6};
      int offs[3][2];
      for (int k = 0; k < 3; ++k) {
        offs[k][0] = HEX[ks[k]][0];
        offs[k][1] = HEX[ks[k]][1];
      }
      int moved = ring(bx, by, offs, 3);
      dir = moved == -1 ? -1 : ks[moved];
      ++it;
    }
    static const int SQ[8][2] = {{-1, -1}, {0, -1}, {1, -1}, {-1, 0},
                                 {1, 0},   {-1, 1}, {0, 1},  {1, 1}};
    ring(bx, by, SQ, 8);
    *cost_out = bcost;
    return Mv(bx * 4, by * 4);
  }

  // refine (h264_hpel.rs:956-1021): returns (mv, satd, cost).
  Mv refine(Mv mv, const MeCfg& cfg, uint32_t* satd_out, uint32_t* cost_out) {
    int lx = bounds[0] * 4, hx = bounds[1] * 4, ly = bounds[2] * 4, hy = bounds[3] * 4;
    Mv best = mv;
    uint32_t bsatd = satd(best);
    uint32_t bcost = bsatd + rate(best.x, best.y);
    static const int RING[8][2] = {{0, -1}, {-1, 0}, {1, 0}, {0, 1},
                                   {-1, -1}, {1, -1}, {-1, 1}, {1, 1}};
    const int steps[2] = {2, 1};
    const int iters[2] = {cfg.hpel_iters, cfg.qpel_iters};
    for (int s = 0; s < 2; ++s) {
      int step = steps[s];
      int pts = (step == 1 && cfg.qpel_diamond) ? 4 : 8;
      bool has_prev = false;
      Mv prev;
      for (int it = 0; it < iters[s]; ++it) {
        Mv c = best;
        Mv ms[8];
        int n = 0;
        for (int k = 0; k < pts; ++k) {
          Mv m((int16_t)(c.x + RING[k][0] * step), (int16_t)(c.y + RING[k][1] * step));
          int qx = m.x, qy = m.y;
          bool inb = qx >= lx && qx <= hx && qy >= ly && qy <= hy;
          bool near_prev = has_prev && std::abs(m.x - prev.x) <= step && std::abs(m.y - prev.y) <= step;
          if (!inb || near_prev) continue;
          ms[n++] = m;
        }
        uint32_t ss[8];
        for (int k = 0; k < n; ++k) ss[k] = satd(ms[k]);
        for (int k = 0; k < n; ++k) {
          uint32_t rc = rate(ms[k].x, ms[k].y);
          if (ss[k] + rc < bcost) {
            bcost = ss[k] + rc;
            bsatd = ss[k];
            best = ms[k];
          }
        }
        if (best == c) break;
        prev = c;
        has_prev = true;
      }
    }
    *satd_out = bsatd;
    *cost_out = bcost;
    return best;
  }
};

// H.264 qpel[16] (dsp/h264.rs:436-495): the decoder's direct evaluation of
// 8.4.2.2.1, src at the window origin (two left of and two above the block).
template <class S>
void h264_qpel_direct(S* dst, int ds, const S* src, ptrdiff_t stride, int w, int h, int xf, int yf,
                      int maxv) {
  auto g = [&](int x, int y) { return (int)src[(y + 2) * stride + x + 2]; };
  auto b1 = [&](int x, int yy) {
    const S* r = src + yy * stride + x;
    return tap6(r[0], r[1], r[2], r[3], r[4], r[5]);
  };
  auto h1 = [&](int xx, int y) {
    const S* c = src + y * stride + xx;
    return tap6(c[0], c[stride], c[2 * stride], c[3 * stride], c[4 * stride], c[5 * stride]);
  };
  auto b = [&](int x, int y) { return std::clamp((b1(x, y + 2) + 16) >> 5, 0, maxv); };
  auto hh = [&](int x, int y) { return std::clamp((h1(x + 2, y) + 16) >> 5, 0, maxv); };
  auto j = [&](int x, int y) {
    int j1 = tap6(b1(x, y), b1(x, y + 1), b1(x, y + 2), b1(x, y + 3), b1(x, y + 4), b1(x, y + 5));
    return std::clamp((j1 + 512) >> 10, 0, maxv);
  };
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      int v = 0;
      switch (yf * 4 + xf) {
        case 0: v = g(x, y); break;
        case 1: v = (g(x, y) + b(x, y) + 1) >> 1; break;
        case 2: v = b(x, y); break;
        case 3: v = (g(x + 1, y) + b(x, y) + 1) >> 1; break;
        case 4: v = (g(x, y) + hh(x, y) + 1) >> 1; break;
        case 8: v = hh(x, y); break;
        case 12: v = (g(x, y + 1) + hh(x, y) + 1) >> 1; break;
        case 10: v = j(x, y); break;
        case 5: v = (b(x, y) + hh(x, y) + 1) >> 1; break;
        case 7: v = (b(x, y) + hh(x + 1, y) + 1) >> 1; break;
        case 13: v = (hh(x, y) + b(x, y + 1) + 1) >> 1; break;
        case 15: v = (hh(x + 1, y) + b(x, y + 1) + 1) >> 1; break;
        case 6: v = (b(x, y) + j(x, y) + 1) >> 1; break;
        case 14: v = (j(x, y) + b(x, y + 1) + 1) >> 1; break;
        case 9: v = (hh(x, y) + j(x, y) + 1) >> 1; break;
        case 11: v = (j(x, y) + hh(x + 1, y) + 1) >> 1; break;
      }
      dst[y * ds + x] = (S)v;
    }
}

// ---------------------------------------------------------------------------
// HEVC (dsp/hevc.rs, hevc/tables_gen.rs, encode/h265_search.rs, h265_me.rs)
// ---------------------------------------------------------------------------
// hevc/tables_gen.rs:186-191 (8 taps of each fraction) and 172-181.
static const int8_t QPEL_FILTERS[4][8] = {{0, 0, 0, 0, 0, 0, 0, 0},
                                          {-1, 4, -10, 58, 17, -5, 1, 0},
                                          {-1, 4, -11, 40, 40, -11, 4, -1},
                                          {0, 1, -5, 17, 58, -10, 4, -1}};
static const int8_t EPEL_FILTERS[8][4] = {{0, 0, 0, 0},     {-2, 58, 10, -2}, {-4, 54, 16, -2},
                                          {-6, 46, 28, -4}, {-4, 36, 36, -4}, {-4, 28, 46, -6},
                                          {-2, 16, 54, -4}, {-2, 10, 58, -2}};

// dsp/hevc.rs:677-756 (luma) and 757-821 (chroma): the filters of
// 8.5.3.3.3, taps taken from `taps` starting at src.
template <class S, int T>
void filt_h(int16_t* dst, const S* src, ptrdiff_t ss, int w, int h, const int8_t* f, int shift) {
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      int acc = 0;
      for (int k = 0; k < T; ++k) acc += f[k] * (int)src[y * ss + x + k];
      dst[y * w + x] = (int16_t)(acc >> shift);
    }
}
template <class S, int T>
void filt_v(int16_t* dst, const S* src, ptrdiff_t ss, int w, int h, const int8_t* f, int shift) {
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      int acc = 0;
      for (int k = 0; k < T; ++k) acc += f[k] * (int)src[(y + k) * ss + x];
      dst[y * w + x] = (int16_t)(acc >> shift);
    }
}
template <int T>
void filt_v2(int16_t* dst, const int16_t* src, int sstride, int w, int h, const int8_t* f) {
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      int acc = 0;
      for (int k = 0; k < T; ++k) acc += f[k] * (int)src[(y + k) * sstride + x];
      dst[y * w + x] = (int16_t)(acc >> 6);
    }
}
template <class S>
void hevc_copy(int16_t* dst, const S* src, ptrdiff_t ss, int w, int h, int shift) {
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) dst[y * w + x] = (int16_t)((int)src[y * ss + x] << shift);
}
// dsp/hevc.rs:997-1013
template <class S>
void hevc_uni(S* dst, ptrdiff_t ds, const int16_t* src, int w, int h, int shift, int maxv) {
  int round = shift > 0 ? 1 << (shift - 1) : 0;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) dst[y * ds + x] = (S)std::clamp(((int)src[y * w + x] + round) >> shift, 0, maxv);
}

// The luma interpolation passes HalfPlanes::build runs, as a table: the
// scalar forms above, or the AVX2 rungs (me_oracle_avx2.cpp, following the
// pairwise-multiply-add design of dsp/hevc_avx2.rs / hevc_avx2_u8.rs), which
// must give the same numbers (tests/test_oracle.py compares the planes).
template <class S>
struct Interp {
  void (*h8)(int16_t*, const S*, ptrdiff_t, int, int, const int8_t*, int);
  void (*v8)(int16_t*, const S*, ptrdiff_t, int, int, const int8_t*, int);
  void (*v2_8)(int16_t*, const int16_t*, int, int, int, const int8_t*);
  void (*uni)(S*, ptrdiff_t, const int16_t*, int, int, int, int);
};
template <class S>
Interp<S> interp_scalar() {
  return Interp<S>{&filt_h<S, 8>, &filt_v<S, 8>, &filt_v2<8>, &hevc_uni<S>};
}
Interp<uint8_t> interp_avx2_u8();
Interp<uint16_t> interp_avx2_u16();

// One component's 14-bit prediction of a w x h block at integer position
// (xi, yi) with fractions (xf, yf): hevc/inter.rs:92-124 `source` (window
// gathered with at_clamped when it leaves the padded plane) and 130-196
// `interp`. taps 8 (luma, quarter fractions) or 4 (chroma, eighths).
template <class S>
void hevc_interp(const Plane<S>& pl, int xi, int yi, int xf, int yf, int w, int h, bool luma, int bd,
                 int16_t* out) {
  int reach = luma ? 3 : 1, taps = luma ? 8 : 4;
  int shift1 = std::min(bd, 12) - 8, shift3 = 14 - bd;
  int x0 = xi - reach, y0 = yi - reach, ww = w + taps - 1, hh = h + taps - 1;
  int pad = pl.pad;
  bool inside = x0 >= -pad && y0 >= -pad && x0 + ww <= pl.width + pad && y0 + hh <= pl.height + pad;
  std::vector<S> window;
  const S* src;
  ptrdiff_t stride;
  if (inside) {
    src = pl.data.data() + pl.offset(x0, y0);
    stride = pl.stride;
  } else {
    window.resize((size_t)ww * hh);
    for (int yy = 0; yy < hh; ++yy)
      for (int xx = 0; xx < ww; ++xx) window[yy * ww + xx] = pl.at_clamped(x0 + xx, y0 + yy);
    src = window.data();
    stride = ww;
  }
  if (xf == 0 && yf == 0) {
    hevc_copy(out, src + reach * stride + reach, stride, w, h, shift3);
  } else if (yf == 0) {
    if (luma) filt_h<S, 8>(out, src + reach * stride, stride, w, h, QPEL_FILTERS[xf], shift1);
    else filt_h<S, 4>(out, src + reach * stride, stride, w, h, EPEL_FILTERS[xf], shift1);
  } else if (xf == 0) {
    if (luma) filt_v<S, 8>(out, src + reach, stride, w, h, QPEL_FILTERS[yf], shift1);
    else filt_v<S, 4>(out, src + reach, stride, w, h, EPEL_FILTERS[yf], shift1);
  } else {
    std::vector<int16_t> tmp((size_t)w * hh);
    if (luma) {
      filt_h<S, 8>(tmp.data(), src, stride, w, hh, QPEL_FILTERS[xf], shift1);
      filt_v2<8>(out, tmp.data(), w, w, h, QPEL_FILTERS[yf]);
    } else {
      filt_h<S, 4>(tmp.data(), src, stride, w, hh, EPEL_FILTERS[xf], shift1);
      filt_v2<4>(out, tmp.data(), w, w, h, EPEL_FILTERS[yf]);
    }
  }
}

constexpr size_t QUARTER_LIMIT = 2200000;  // h265_search.rs:35
constexpr int HP_MARGIN = 4;               // h265_search.rs:64
constexpr int HP_REACH = 16;               // h265_search.rs:71

// HalfPlanes (h265_search.rs:42-202): exact uni-predicted fractional phases
// of a reference luma plane, same layout as the plane.
template <class S>
struct HalfPlanes {
  std::vector<S> planes[15];
  int stride = 0, pad = 0, ext = 0, width = 0, height = 0;

  // HalfPlanes::new (h265_search.rs:79-170), 64x64 tiles over the plane
  // less MARGIN, REACH samples outside the picture.
  void build(const Plane<S>& p, int bd, bool force_quarter = false, const Interp<S>* rung = nullptr) {
    const Interp<S> I = rung ? *rung : interp_scalar<S>();
    const int T = 64;
    stride = p.stride;
    int rows = p.rows();
    bool quarter = force_quarter || (size_t)p.width * p.height <= QUARTER_LIMIT;
    int shift1 = std::min(bd, 12) - 8, shift3 = 14 - bd, maxv = (1 << bd) - 1;
    auto wanted = [&](int fx, int fy) { return quarter || (fx % 2 == 0 && fy % 2 == 0); };
    const S* d = p.data.data();
    for (int ph = 1; ph < 16; ++ph) {
      if (wanted(ph % 4, ph / 4)) planes[ph - 1].assign(p.data.size(), S(0));
      else planes[ph - 1].clear();
    }
    std::vector<int16_t> tmp((size_t)T * (T + 7)), out14((size_t)T * T);
    ext = std::min(HP_REACH, p.pad - HP_MARGIN);
    int lo = p.pad - ext, hi_x = p.pad + p.width + ext, hi_y = std::min(p.pad + p.height + ext, rows - HP_MARGIN);
    for (int y0 = lo; y0 < hi_y;) {
      int th = std::min(T, hi_y - y0);
      for (int x0 = lo; x0 < hi_x;) {
        int tw = std::min(T, hi_x - x0);
        ptrdiff_t at = (ptrdiff_t)y0 * stride + x0;
        for (int fx = 0; fx < 4; ++fx) {
          bool any = false;
          for (int fy = 1; fy < 4; ++fy) any = any || wanted(fx, fy);
          if (fx != 0 && any)
            I.h8(tmp.data(), d + at - 3 * stride - 3, stride, tw, th + 7, QPEL_FILTERS[fx], shift1);
          for (int fy = 0; fy < 4; ++fy) {
            if ((fx == 0 && fy == 0) || !wanted(fx, fy)) continue;
            if (fy == 0) I.h8(out14.data(), d + at - 3, stride, tw, th, QPEL_FILTERS[fx], shift1);
            else if (fx == 0) I.v8(out14.data(), d + at - 3 * stride, stride, tw, th, QPEL_FILTERS[fy], shift1);
            else I.v2_8(out14.data(), tmp.data(), tw, tw, th, QPEL_FILTERS[fy]);
            I.uni(planes[fy * 4 + fx - 1].data() + at, stride, out14.data(), tw, th, shift3, maxv);
          }
        }
        x0 += tw;
      }
      y0 += th;
    }
    pad = p.pad;
    width = p.width;
    height = p.height;
  }

  // HalfPlanes::at (h265_search.rs:177-202).
  const S* at(int x, int y, int w, int h, int mvx, int mvy) const {
    int phase = (mvy & 3) * 4 + (mvx & 3);
    if (phase == 0 || planes[phase - 1].empty()) return nullptr;
    int xi = x + (mvx >> 2), yi = y + (mvy >> 2), lim = ext;
    if (xi < -lim || yi < -lim || xi + w > width + lim || yi + h > height + lim) return nullptr;
    size_t off = (size_t)(pad + yi) * stride + (size_t)(pad + xi);
    return planes[phase - 1].data() + off;
  }
};

// mvd_bits_of / mvd_component_bits / mv_bits (h265_search.rs:212-255).
inline uint32_t hevc_mvd_bits_of(uint32_t a) {
  if (a == 0) return 1;
  if (a == 1) return 3;
  uint32_t v = a - 2, k = 1, bits = 0;
  while (v >= (1u << k)) {
    bits += 1;
    v -= 1u << k;
    k += 1;
  }
  return 3 + bits + 1 + k;
}
inline uint32_t hevc_mvd_component_bits(int d) {
  uint32_t a = (uint32_t)(d < 0 ? -(int64_t)d : d);
  return hevc_mvd_bits_of(a);  // the 2048-entry table holds the same values
}
inline uint32_t hevc_mv_bits(int mvx, int mvy, const int pq[2][2]) {
  uint32_t b0 = hevc_mvd_component_bits(mvx - pq[0][0]) + hevc_mvd_component_bits(mvy - pq[0][1]);
  uint32_t b1 = hevc_mvd_component_bits(mvx - pq[1][0]) + hevc_mvd_component_bits(mvy - pq[1][1]);
  return std::min(b0, b1) + 1;
}

// base_lambda / satd_lambda / satd_lambda_scale (h265_intra.rs:1141-1143,
// 1973-1975, 2011-2013) and lambda (h265_me.rs:4421): the SATD Lagrangian
// of a P picture at qp, bit depth bd, Tune multiplier `scale`.
inline float hevc_lambda(int qp, int bd, float scale) {
  float base = 0.85f * std::exp2((float)(qp - 12) / 3.0f) * scale;
  return std::sqrt(base) * (float)(1u << (bd - 8));
}
inline uint32_t hevc_rate(float lam, uint32_t bits) { return (uint32_t)(lam * (float)bits); }

template <class S>
struct HevcSearch {
  const Dist<S>* dist;
  const Plane<S>* refp;
  const HalfPlanes<S>* half;  // may be null
  int bd;
  const S* src;
  ptrdiff_t src_stride;
  int x, y, w, h;
  float lam;
  int pq[2][2];
  int search_range = 48, search_rings = 0;
  bool quarter_cross = false;
  uint32_t n_sad = 0, n_satd = 0;

  // read_at + satd_at_weighted under default weighting
  // (h265_me.rs:3630-3655, 4039-4074).
  // Explicit weighting of a weighted list (satd_at_weighted's Explicit arm,
  // h265_me.rs:4057-4073): every candidate, whole samples included, is the
  // 14-bit prediction through weighted_uni (dsp/hevc.rs:1036-1062).
  bool wp = false;
  int wp_log2 = 0, wp_w = 1, wp_o = 0;

  uint32_t satd_at(Mv mv) {
    if (wp) return satd_weighted(mv);
    ++n_satd;
    int mvx = mv.x, mvy = mv.y;
    if ((mvx & 3) == 0 && (mvy & 3) == 0) {
      int xi = x + (mvx >> 2), yi = y + (mvy >> 2), lim = refp->pad;
      if (!(xi < -lim || yi < -lim || xi + w > refp->width + lim || yi + h > refp->height + lim))
        return dist->satd(src, src_stride, refp->data.data() + refp->offset(xi, yi), refp->stride, w, h);
    } else if (half) {
      const S* p = half->at(x, y, w, h, mvx, mvy);
      if (p) return dist->satd(src, src_stride, p, half->stride, w, h);
    }
    // predict14 (h265_me.rs:4366-4415) + uni (dsp/hevc.rs:997).
    std::vector<int16_t> p14((size_t)w * h);
    std::vector<S> pred((size_t)w * h);
    hevc_interp(*refp, x + (mvx >> 2), y + (mvy >> 2), mvx & 3, mvy & 3, w, h, true, bd, p14.data());
    hevc_uni(pred.data(), w, p14.data(), w, h, 14 - bd, (1 << bd) - 1);
    return dist->satd(src, src_stride, pred.data(), w, w, h);
  }

  uint32_t satd_weighted(Mv mv) {
    ++n_satd;
    const int maxv = (1 << bd) - 1;
    std::vector<int16_t> p14((size_t)w * h);
    std::vector<S> pred((size_t)w * h);
    hevc_interp(*refp, x + (mv.x >> 2), y + (mv.y >> 2), mv.x & 3, mv.y & 3, w, h, true, bd, p14.data());
    for (size_t i = 0; i < pred.size(); ++i) {
      const int v = wp_log2 >= 1 ? (((int)p14[i] * wp_w + (1 << (wp_log2 - 1))) >> wp_log2) + wp_o
                                 : (int)p14[i] * wp_w + wp_o;
      pred[i] = (S)std::clamp(v, 0, maxv);
    }
    return dist->satd(src, src_stride, pred.data(), w, w, h);
  }

  uint32_t cost_of(int fx, int fy) {
    ++n_sad;
    const S* rp = refp->data.data() + refp->offset(x + fx, y + fy);
    uint32_t sad = dist->sad(src, src_stride, rp, refp->stride, w, h);
    return sad + hevc_rate(lam, hevc_mv_bits(fx * 4, fy * 4, pq));
  }

  // search_full (h265_me.rs:3749-3858). Returns the best whole-sample
  // vector in quarter units and its SAD + rate.
  Mv search_full(const Mv* seeds, int ns, uint32_t* cost_out) {
    int pad = refp->pad - HP_MARGIN;
    auto clamp_pos = [&](int fx, int fy, int* ox, int* oy) {
      int xi = std::clamp(x + fx, -pad, refp->width + pad - w);
      int yi = std::clamp(y + fy, -pad, refp->height + pad - h);
      *ox = xi - x;
      *oy = yi - y;
    };
    int bx = 0, by = 0;
    uint32_t best_cost = UINT32_MAX;
    int tx[16], ty[16];
    bool tset[16] = {false};
    for (int i = 0; i < 16; ++i) {
      tx[i] = INT32_MIN;
      ty[i] = 0;
    }
    for (int i = 0; i < ns; ++i) {
      int cx, cy;
      clamp_pos(seeds[i].x >> 2, seeds[i].y >> 2, &cx, &cy);
      bool seen = false;
      for (int k = 0; k < 16 && !seen; ++k) seen = (tx[k] == cx && ty[k] == cy);
      if (seen) continue;
      if (i < 16) {
        tx[i] = cx;
        ty[i] = cy;
        tset[i] = true;
      }
      uint32_t c = cost_of(cx, cy);
      if (c < best_cost) {
        best_cost = c;
        bx = cx;
        by = cy;
      }
    }
    (void)tset;
    int ox = bx, oy = by;  // centre
    auto inside = [&](int cx, int cy) {
      int qx, qy;
      clamp_pos(cx, cy, &qx, &qy);
      return std::abs(cx - ox) <= search_range && std::abs(cy - oy) <= search_range && qx == cx && qy == cy;
    };
    int rings = 0;
    for (;;) {
      for (int it = 0; it < 2 * search_range; ++it) {
        bool improved = false;
        int fx0 = bx, fy0 = by;
        static const int D[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};
        for (auto& d : D) {
          int cx = fx0 + d[0], cy = fy0 + d[1];
          if (!inside(cx, cy)) continue;
          uint32_t c = cost_of(cx, cy);
          if (c < best_cost) {
            best_cost = c;
            bx = cx;
            by = cy;
            improved = true;
          }
        }
        if (!improved) break;
      }
      if (rings >= search_rings) break;
      ++rings;
      int fx0 = bx, fy0 = by;
      bool moved = false;
      for (int r : {4, 8, 16}) {
        const int R[8][2] = {{r, 0}, {-r, 0}, {0, r}, {0, -r}, {r, r}, {-r, r}, {r, -r}, {-r, -r}};
        for (auto& d : R) {
          int cx = fx0 + d[0], cy = fy0 + d[1];
          if (!inside(cx, cy)) continue;
          uint32_t c = cost_of(cx, cy);
          if (c < best_cost) {
            best_cost = c;
            bx = cx;
            by = cy;
            moved = true;
          }
        }
      }
      if (!moved) break;
    }
    *cost_out = best_cost;
    return Mv(bx * 4, by * 4);
  }

  // refine_subpel (h265_me.rs:3868-3922), default weighting.
  Mv refine_subpel(Mv start, uint32_t* satd_out, uint32_t* cost_out) {
    auto rate = [&](Mv mv) { return hevc_rate(lam, hevc_mv_bits(mv.x, mv.y, pq)); };
    Mv best = start;
    uint32_t best_satd = satd_at(start);
    uint32_t best_cost = best_satd + rate(start);
    for (int step : {2, 1}) {
      Mv centre = best;
      bool cross = step == 1 && quarter_cross;
      for (int dy : {-step, 0, step})
        for (int dx : {-step, 0, step}) {
          if ((dx == 0 && dy == 0) || (cross && dx != 0 && dy != 0)) continue;
          Mv mv((int16_t)(centre.x + dx), (int16_t)(centre.y + dy));
          uint32_t s = satd_at(mv);
          uint32_t c = s + rate(mv);
          if (c < best_cost) {
            best_cost = c;
            best_satd = s;
            best = mv;
          }
        }
    }
    *satd_out = best_satd;
    *cost_out = best_cost;
    return best;
  }
};

}  // namespace orc
