// ORACLE — test infrastructure, not product code.
//
// Frame-level drivers of the oracle and its C entry points (orc_*), loaded
// by tests/ and bench.py through ctypes. The search arithmetic lives in
// me_oracle.hpp; this file restates how the encoders drive it
// (h264_analyse.rs p_mb's search section, h265_me.rs pick_pu's seed
// assembly) in the two modes of include/rivet_me.h:
//   GIVEN       one search per caller job, exactly as the encoder calls it;
//   STANDALONE  the frame's own results feed the predictors, in the
//               wavefront rule below (the same rule the CUDA library runs).
#include <atomic>
#include <functional>
#include <chrono>
#include <cstdio>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "me_oracle.hpp"

using namespace orc;

namespace {

int level_sizes(const rme_params* p, int* sizes) {  // largest first
  int n = 0;
  for (int k = 3; k >= 0; --k)
    if (p->hevc_pu_mask & (1 << k)) sizes[n++] = 8 << k;
  return n;
}

// The two PUs of an asymmetric partition of the N x N CU at (x, y): mode
// bit 0 2NxnU, 1 2NxnD, 2 nLx2N, 3 nRx2N (H.265 Table 7-10), part 0 the
// top/left unit.
void amp_pu(int mode, int part, int x, int y, int N, int32_t* b) {
  const int q = N / 4;
  b[0] = x;
  b[1] = y;
  b[2] = N;
  b[3] = N;
  switch (mode) {
    case 0: b[3] = part ? 3 * q : q; b[1] = part ? y + q : y; break;
    case 1: b[3] = part ? q : 3 * q; b[1] = part ? y + 3 * q : y; break;
    case 2: b[2] = part ? 3 * q : q; b[0] = part ? x + q : x; break;
    default: b[2] = part ? q : 3 * q; b[0] = part ? x + 3 * q : x; break;
  }
}

// HEVC STANDALONE blocks: per size level (largest first), the 2Nx2N PUs
// that lie wholly inside the picture, raster order; then, where asked
// (hevc_amp), per level of 16 or more, per such CU in raster order, per
// enabled AMP mode (bit order), its two PUs.
int hevc_blocks(int W, int H, const rme_params* p, int32_t* blocks) {
  int sizes[4], nl = level_sizes(p, sizes), n = 0;
  for (int l = 0; l < nl; ++l) {
    int N = sizes[l];
    for (int by = 0; by + N <= H; by += N)
      for (int bx = 0; bx + N <= W; bx += N) {
        if (blocks) {
          blocks[4 * n] = bx;
          blocks[4 * n + 1] = by;
          blocks[4 * n + 2] = N;
          blocks[4 * n + 3] = N;
        }
        ++n;
      }
  }
  for (int l = 0; l < nl && sizes[l] >= 16; ++l) {
    int N = sizes[l];
    for (int by = 0; by + N <= H; by += N)
      for (int bx = 0; bx + N <= W; bx += N)
        for (int m = 0; m < 4; ++m)
          if ((p->hevc_amp >> m) & 1)
            for (int k = 0; k < 2; ++k, ++n)
              if (blocks) amp_pu(m, k, bx, by, N, blocks + 4 * n);
  }
  return n;
}

int h264_blocks(int W, int H, int32_t* blocks) {
  int mbw = (W + 15) / 16, mbh = (H + 15) / 16, n = 0;
  for (int my = 0; my < mbh; ++my)
    for (int mx = 0; mx < mbw; ++mx) {
      if (blocks) {
        blocks[4 * n] = mx * 16;
        blocks[4 * n + 1] = my * 16;
        blocks[4 * n + 2] = 16;
        blocks[4 * n + 3] = 16;
      }
      ++n;
    }
  return n;
}

// An H.264 picture is searched at its coded size (whole macroblocks,
// h264_syntax.rs:349-358), the picture extended to it by edge replication.
template <class S>
std::vector<S> coded_h264(const S* src, int W, int H, ptrdiff_t ss, int CW, int CH) {
  std::vector<S> out((size_t)CW * CH);
  for (int y = 0; y < CH; ++y)
    for (int x = 0; x < CW; ++x) out[(size_t)y * CW + x] = src[(ptrdiff_t)std::min(y, H - 1) * ss + std::min(x, W - 1)];
  return out;
}

struct NbMotion {  // h264/mb.rs:913-929
  bool avail = false;
  int ref = -1;
  Mv mv;
};

// median_mvp (h264/mb.rs:1170-1189).
Mv median_mvp(NbMotion a, NbMotion b, NbMotion c, int ref) {
  if (!b.avail && !c.avail && a.avail) {
    b = a;
    c = a;
  }
  bool ma = a.ref == ref, mb = b.ref == ref, mc = c.ref == ref;
  if (ma && !mb && !mc) return a.mv;
  if (!ma && mb && !mc) return b.mv;
  if (!ma && !mb && mc) return c.mv;
  auto med = [](int x, int y, int z) { return std::min(std::max(x, y), std::max(std::min(x, y), z)); };
  return Mv(med(a.mv.x, b.mv.x, c.mv.x), med(a.mv.y, b.mv.y, c.mv.y));
}

uint32_t h264_ref_bits_cost(float lam1, int r, int nref) {  // h264_analyse.rs:1934-1942
  float bits;
  if (nref == 1) bits = 0.0f;
  else if (nref == 2) bits = 1.0f;
  else bits = (float)(2 * (32 - __builtin_clz((unsigned)(r + 1))) - 1);
  return (uint32_t)(lam1 * bits);
}

MeCfg h264_cfg(const rme_params* p) {
  MeCfg c;
  c.range = p->h264_range;
  c.hpel_iters = p->h264_hpel_iters;
  c.qpel_iters = p->h264_qpel_iters;
  c.umh = p->h264_umh != 0;
  c.qpel_diamond = p->h264_qpel_diamond != 0;
  c.dia = p->h264_dia != 0;
  return c;
}

template <class S>
struct H264Ref {
  Plane<S> g;
  Hpel<S> hp;
  MeRef<S> me;
};

template <class S>
void h264_prepare_ref(H264Ref<S>& r, const S* luma, int W, int H, ptrdiff_t ss, int pad, int bd) {
  int CW = (W + 15) / 16 * 16, CH = (H + 15) / 16 * 16;
  auto coded = coded_h264(luma, W, H, ss, CW, CH);
  r.g = Plane<S>(CW, CH, pad);
  r.g.load(coded.data(), CW);
  r.hp.build(r.g, (1 << bd) - 1);
  r.me = MeRef<S>(&r.g, &r.hp);
}

template <class S>
void h264_frame(const Dist<S>& dist, const S* src_luma, int W, int H, ptrdiff_t ss, int nref,
                H264Ref<S>* const* refs, const rme_params* p, const rme_job* jobs, int njobs, rme_result* out) {
  int CW = (W + 15) / 16 * 16, CH = (H + 15) / 16 * 16;
  auto src = coded_h264(src_luma, W, H, ss, CW, CH);
  float lam1 = h264_lambda_satd(p->qp);
  std::vector<uint16_t> tab(MV_TAB);
  h264_cost_table(lam1, tab.data());
  MeCfg me = h264_cfg(p);
  int pad = p->h264_pad, vr = p->h264_vertical_range;
  if (p->predictor_mode == RME_PRED_GIVEN) {
    for (int j = 0; j < njobs; ++j) {
      const rme_job& jb = jobs[j];
      H264Search<S> s{&dist, &refs[jb.ref]->me, src.data() + (size_t)jb.y * CW + jb.x, CW, jb.x, jb.y, jb.w, jb.h,
                      Mv(jb.mvp[0].x, jb.mvp[0].y), tab.data(), {0, 0, 0, 0}};
      h264_search_bounds(CW, CH, pad, jb.x, jb.y, jb.w, jb.h, vr, s.bounds);
      Mv cands[RME_MAX_SEEDS];
      for (int k = 0; k < jb.nseeds; ++k) cands[k] = Mv(jb.seeds[k].x, jb.seeds[k].y);
      uint32_t ci, sat, c;
      Mv mi = s.int_search(cands, jb.nseeds, me, &ci);
      Mv m = s.refine(mi, (jb.flags & RME_JOB_SCORE_ONLY) ? MeCfg::score() : me, &sat, &c);
      rme_result& o = out[j];
      o.mv = {m.x, m.y};
      o.ref = jb.ref;
      o.cost = c;
      o.satd = sat;
      o.int_mv = {mi.x, mi.y};
      o.int_cost = ci;
      o.n_sad = s.n_sad;
      o.n_satd = s.n_satd;
    }
    return;
  }
  // STANDALONE: p_mb's search section (h264_analyse.rs:1884-1975) per
  // macroblock in raster order, its predictors derived from the frame's own
  // results: every coded macroblock is a 16x16 inter one at its best
  // reference, so A, B, C (or D) are available exactly where they exist.
  int mbw = CW / 16, mbh = CH / 16;
  std::vector<uint32_t> rb(nref);
  for (int r = 0; r < nref; ++r) rb[r] = h264_ref_bits_cost(lam1, r, nref);
  for (int my = 0; my < mbh; ++my)
    for (int mx = 0; mx < mbw; ++mx) {
      auto nb = [&](int x, int y) {
        NbMotion m;
        if (x < 0 || y < 0 || x >= mbw) return m;
        const rme_result& q = out[y * mbw + x];
        m.avail = true;
        m.ref = q.ref;
        m.mv = Mv(q.mv.x, q.mv.y);
        return m;
      };
      NbMotion A = nb(mx - 1, my), B = nb(mx, my - 1), C = nb(mx + 1, my - 1), D = nb(mx - 1, my - 1);
      NbMotion Cc = C.avail ? C : D;  // prediction_neighbours: C, else D
      auto pmv = [&](int r) { return median_mvp(A, B, Cc, r); };
      // p_skip_mv (h264/mb.rs:1235-1246)
      Mv skip;
      if (!(!A.avail || !B.avail || (A.ref == 0 && A.mv == Mv()) || (B.ref == 0 && B.mv == Mv()))) skip = pmv(0);
      // cands = [skip_mv, 0, neighbour vectors] (h264_pic.rs:713-751, p_mb 1889-1899)
      Mv cands[8];
      int nc = 0;
      cands[nc++] = skip;
      cands[nc++] = Mv();
      Mv nbv[4];
      int nn = 0;
      for (const NbMotion* q : {&A, &B, &C}) {
        if (!q->avail || q->ref < 0 || nn >= 4) continue;
        bool dup = false;
        for (int k = 0; k < nn; ++k) dup = dup || nbv[k] == q->mv;
        if (!dup) nbv[nn++] = q->mv;
      }
      for (int k = 0; k < nn && nc < 8; ++k) cands[nc++] = nbv[k];
      int x = mx * 16, y = my * 16;
      Mv mv16;
      uint32_t c16 = UINT32_MAX, s16 = 0, int16 = UINT32_MAX, ci16 = 0, nsad = 0, nsatd = 0;
      Mv mi16;
      int r16 = 0;
      for (int r = 0; r < nref; ++r) {
        Mv pr = pmv(r);
        if (r > 0 && nc < 8) cands[nc] = pr;
        int k = r > 0 ? std::min(nc + 1, 8) : nc;
        H264Search<S> s{&dist, &refs[r]->me, src.data() + (size_t)y * CW + x, CW, x, y, 16, 16, pr,
                        tab.data(), {0, 0, 0, 0}};
        h264_search_bounds(CW, CH, pad, x, y, 16, 16, vr, s.bounds);
        uint32_t ci, sat, c;
        Mv mi = s.int_search(cands, k, me, &ci);
        ci += rb[r];
        bool gate = r > 0 && p->h264_refine_ratio > 0.0f && (float)ci >= p->h264_refine_ratio * (float)int16;
        Mv m = s.refine(mi, gate ? MeCfg::score() : me, &sat, &c);
        int16 = std::min(int16, ci);
        c += rb[r];
        nsad += s.n_sad;
        nsatd += s.n_satd;
        if (c < c16) {
          mv16 = m;
          c16 = c;
          s16 = sat;
          r16 = r;
          mi16 = mi;
          ci16 = ci;
        }
      }
      rme_result& o = out[my * mbw + mx];
      o.mv = {mv16.x, mv16.y};
      o.ref = r16;
      o.cost = c16;
      o.satd = s16;
      o.int_mv = {mi16.x, mi16.y};
      o.int_cost = ci16;
      o.n_sad = nsad;
      o.n_satd = nsatd;
    }
}

template <class S>
struct HevcRef {
  Plane<S> g;
  HalfPlanes<S> hp;
};

template <class S>
Interp<S> pick_interp(int simd);

// `simd`: the phase planes through the AVX2 interpolation rung where the
// CPU has it (the same planes).
template <class S>
void hevc_prepare_ref(HevcRef<S>& r, const S* luma, int W, int H, ptrdiff_t ss, int pad, int bd, int simd = 0) {
  r.g = Plane<S>(W, H, pad);
  r.g.load(luma, ss);
  const Interp<S> I = pick_interp<S>(simd);
  r.hp.build(r.g, bd, false, &I);
}

template <class S>
void hevc_one(const Dist<S>& dist, const HevcRef<S>& ref, int bd, const S* src, ptrdiff_t ss, int x, int y,
              int w, int h, float lam, const rme_params* p, const Mv mvp[2], const Mv* seeds, int ns, int r,
              rme_result& o) {
  HevcSearch<S> s{&dist, &ref.g, &ref.hp, bd, src + (ptrdiff_t)y * ss + x, ss, x, y, w, h, lam, {{0, 0}, {0, 0}}};
  s.pq[0][0] = mvp[0].x;
  s.pq[0][1] = mvp[0].y;
  s.pq[1][0] = mvp[1].x;
  s.pq[1][1] = mvp[1].y;
  s.search_range = p->hevc_search_range;
  s.search_rings = p->hevc_search_rings;
  s.quarter_cross = p->hevc_quarter_cross != 0;
  uint32_t fc, sat, c;
  Mv full = s.search_full(seeds, ns, &fc);
  Mv m = s.refine_subpel(full, &sat, &c);
  o.mv = {m.x, m.y};
  o.ref = r;
  o.cost = c;
  o.satd = sat;
  o.int_mv = {full.x, full.y};
  o.int_cost = fc;
  o.n_sad = s.n_sad;
  o.n_satd = s.n_satd;
}

template <class S>
void hevc_frame(const Dist<S>& dist, const S* src, int W, int H, ptrdiff_t ss, int bd, int nref,
                HevcRef<S>* const* refs, const rme_params* p, const rme_job* jobs, int njobs, rme_result* out) {
  float lam = hevc_lambda(p->qp, bd, p->hevc_lambda_scale);
  if (p->predictor_mode == RME_PRED_GIVEN) {
    for (int j = 0; j < njobs; ++j) {
      const rme_job& jb = jobs[j];
      Mv mvp[2] = {Mv(jb.mvp[0].x, jb.mvp[0].y), Mv(jb.mvp[1].x, jb.mvp[1].y)};
      Mv seeds[RME_MAX_SEEDS];
      for (int k = 0; k < jb.nseeds; ++k) seeds[k] = Mv(jb.seeds[k].x, jb.seeds[k].y);
      hevc_one(dist, *refs[jb.ref], bd, src, ss, jb.x, jb.y, jb.w, jb.h, lam, p, mvp, seeds, jb.nseeds, jb.ref,
               out[j]);
    }
    return;
  }
  // STANDALONE: per size level (largest first), raster order, every
  // reference: seeds = [zero, mvp0, mvp1, parent] as pick_pu orders them
  // (h265_me.rs:1327-1348), where the AMVP pair is the spatial part of
  // 8.5.3.2.7 over this level's results (left A, above B; a duplicate B
  // dropped; zero-filled) and the parent seed is the result of the
  // enclosing PU one evaluated size up (parent_seed, h265_me.rs:3709).
  int sizes[4], nl = level_sizes(p, sizes);
  int base[5] = {0}, nbx[4], nby[4];
  for (int l = 0; l < nl; ++l) {
    nbx[l] = W / sizes[l];
    nby[l] = H / sizes[l];
    base[l + 1] = base[l] + nbx[l] * nby[l];
  }
  auto at = [&](int l, int bx, int by, int r) -> rme_result& {
    return out[(size_t)(base[l] + by * nbx[l] + bx) * nref + r];
  };
  for (int l = 0; l < nl; ++l) {
    int N = sizes[l];
    for (int by = 0; by < nby[l]; ++by)
      for (int bx = 0; bx < nbx[l]; ++bx)
        for (int r = 0; r < nref; ++r) {
          Mv cand[2];
          int na = 0;
          if (bx > 0) cand[na++] = Mv(at(l, bx - 1, by, r).mv.x, at(l, bx - 1, by, r).mv.y);
          if (by > 0) {
            Mv b(at(l, bx, by - 1, r).mv.x, at(l, bx, by - 1, r).mv.y);
            if (na == 0 || cand[0] != b) cand[na++] = b;
          }
          Mv mvp[2] = {na > 0 ? cand[0] : Mv(), na > 1 ? cand[1] : Mv()};
          Mv seeds[4] = {Mv(), mvp[0], mvp[1], Mv()};
          int ns = 3;
          if (l > 0) {
            int Np = sizes[l - 1], px = bx * N / Np, py = by * N / Np;
            if (px < nbx[l - 1] && py < nby[l - 1]) {
              const rme_result& q = at(l - 1, px, py, r);
              seeds[ns++] = Mv(q.mv.x, q.mv.y);
            }
          }
          hevc_one(dist, *refs[r], bd, src, ss, bx * N, by * N, N, N, lam, p, mvp, seeds, ns, r, at(l, bx, by, r));
        }
  }
  // AMP (hevc_amp): each CU's two units per enabled mode, searched from the
  // CU's own 2Nx2N result `own` — the parts search's own seed first
  // (pick_pu under part_seeded, h265_me.rs:1327-1348) — with the AMVP pair
  // [own, 0] (two zeros when own is zero): seeds [own, mvp0, mvp1].
  size_t k = base[nl];
  for (int l = 0; l < nl && sizes[l] >= 16; ++l) {
    int N = sizes[l];
    for (int by = 0; by < nby[l]; ++by)
      for (int bx = 0; bx < nbx[l]; ++bx)
        for (int m = 0; m < 4; ++m)
          if ((p->hevc_amp >> m) & 1)
            for (int part = 0; part < 2; ++part, ++k) {
              int32_t b[4];
              amp_pu(m, part, bx * N, by * N, N, b);
              for (int r = 0; r < nref; ++r) {
                Mv own(at(l, bx, by, r).mv.x, at(l, bx, by, r).mv.y);
                Mv mvp[2] = {own, Mv()};
                Mv seeds[3] = {own, mvp[0], mvp[1]};
                hevc_one(dist, *refs[r], bd, src, ss, b[0], b[1], b[2], b[3], lam, p, mvp, seeds, 3, r,
                         out[k * nref + r]);
              }
            }
  }
}

template <class S>
Dist<S> pick_dist(int simd);
bool have_avx2() { return __builtin_cpu_supports("avx2"); }
template <>
Dist<uint8_t> pick_dist<uint8_t>(int simd) { return simd && have_avx2() ? dist_avx2_u8() : dist_scalar<uint8_t>(); }
template <>
Dist<uint16_t> pick_dist<uint16_t>(int simd) {
  return simd && have_avx2() ? dist_avx2_u16() : dist_scalar<uint16_t>();
}
template <>
Interp<uint8_t> pick_interp<uint8_t>(int simd) {
  return simd && have_avx2() ? interp_avx2_u8() : interp_scalar<uint8_t>();
}
template <>
Interp<uint16_t> pick_interp<uint16_t>(int simd) {
  return simd && have_avx2() ? interp_avx2_u16() : interp_scalar<uint16_t>();
}

bool valid_desc(const rme_picture_desc* d) {
  return d && (d->codec == RME_CODEC_H264 || d->codec == RME_CODEC_HEVC) && d->bit_depth >= 8 &&
         d->bit_depth <= 12 && d->width >= 16 && d->height >= 16 && d->stride >= d->width;
}

// Run frames[i] (src pointer + nref reference pointers); references that
// appear in several frames (a sequence: frame t searches t-1 and t-2) are
// prepared once, as the encoders cache them (hpel_for, retain_reference).
template <class S>
int run_frames(const rme_picture_desc* d, int nframes, const void* const* srcs, int nref, const void* const* refs,
               const rme_params* p, int simd, int threads, rme_result* out, const int64_t* offsets,
               double* seconds, double* plane_seconds) {
  Dist<S> dist = pick_dist<S>(simd);
  int W = d->width, H = d->height, bd = d->bit_depth;
  ptrdiff_t ss = d->stride;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<const void*> uniq;
  std::unordered_map<const void*, int> index;
  for (int i = 0; i < nframes * nref; ++i)
    if (!index.count(refs[i])) {
      index[refs[i]] = (int)uniq.size();
      uniq.push_back(refs[i]);
    }
  bool h264 = d->codec == RME_CODEC_H264;
  std::vector<H264Ref<S>> r264(h264 ? uniq.size() : 0);
  std::vector<HevcRef<S>> r265(h264 ? 0 : uniq.size());
  threads = std::max(1, threads);
  auto parallel = [&](int n, auto&& fn) {
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < std::min(threads, std::max(n, 1)); ++t)
      pool.emplace_back([&] {
        for (int i; (i = next.fetch_add(1)) < n;) fn(i);
      });
    for (auto& th : pool) th.join();
  };
  parallel((int)uniq.size(), [&](int i) {
    if (h264) h264_prepare_ref(r264[i], (const S*)uniq[i], W, H, ss, p->h264_pad, bd);
    else hevc_prepare_ref(r265[i], (const S*)uniq[i], W, H, ss, p->hevc_pad, bd, simd);
  });
  auto t1 = std::chrono::steady_clock::now();
  parallel(nframes, [&](int f) {
    rme_result* o = out + (offsets ? offsets[f] : 0);
    if (h264) {
      std::vector<H264Ref<S>*> rr(nref);
      for (int r = 0; r < nref; ++r) rr[r] = &r264[index[refs[f * nref + r]]];
      h264_frame<S>(dist, (const S*)srcs[f], W, H, ss, nref, rr.data(), p, nullptr, 0, o);
    } else {
      std::vector<HevcRef<S>*> rr(nref);
      for (int r = 0; r < nref; ++r) rr[r] = &r265[index[refs[f * nref + r]]];
      hevc_frame<S>(dist, (const S*)srcs[f], W, H, ss, bd, nref, rr.data(), p, nullptr, 0, o);
    }
  });
  auto t2 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t2 - t0).count();
  if (plane_seconds) *plane_seconds = std::chrono::duration<double>(t1 - t0).count();
  return 0;
}

// ---- B pictures: bi-prediction (HEVC) ----------------------------------------

// read_at (h265_me.rs:3630-3655): a whole-sample vector's block read from
// the reference itself while it stays within the plane's border, a
// fractional one's from HalfPlanes; null where neither can be read.
template <class S>
const S* hevc_read_at(const HevcRef<S>& r, int x, int y, int w, int h, Mv mv, ptrdiff_t* stride) {
  const int mvx = mv.x, mvy = mv.y;
  if ((mvx & 3) == 0 && (mvy & 3) == 0) {
    const int xi = x + (mvx >> 2), yi = y + (mvy >> 2), lim = r.g.pad;
    if (xi < -lim || yi < -lim || xi + w > r.g.width + lim || yi + h > r.g.height + lim) return nullptr;
    *stride = r.g.stride;
    return r.g.data.data() + r.g.offset(xi, yi);
  }
  *stride = r.hp.stride;
  return r.hp.at(x, y, w, h, mvx, mvy);
}

// The 14-bit prediction of a block (predict14, h265_me.rs:4366-4415).
template <class S>
void hevc_pred14(const HevcRef<S>& r, int x, int y, int w, int h, Mv mv, int bd, int16_t* out) {
  hevc_interp(r.g, x + (mv.x >> 2), y + (mv.y >> 2), mv.x & 3, mv.y & 3, w, h, true, bd, out);
}

// satd_bi_at (h265_me.rs:4209-4264) under default weighting: both blocks
// readable, their samples averaged (a + b + 1) >> 1; otherwise both 14-bit
// predictions through bi at 15 - bd (dsp/hevc.rs:1015-1031).
template <class S>
uint32_t hevc_satd_bi(const Dist<S>& dist, const HevcRef<S>& r0, const HevcRef<S>& r1, int bd, const S* src,
                      ptrdiff_t ss, int x, int y, int w, int h, Mv mv0, Mv mv1) {
  const int maxv = (1 << bd) - 1;
  std::vector<S> pred((size_t)w * h);
  ptrdiff_t s0 = 0, s1 = 0;
  const S* p0 = hevc_read_at(r0, x, y, w, h, mv0, &s0);
  const S* p1 = hevc_read_at(r1, x, y, w, h, mv1, &s1);
  if (p0 && p1) {
    for (int yy = 0; yy < h; ++yy)
      for (int xx = 0; xx < w; ++xx)
        pred[(size_t)yy * w + xx] = (S)(((int)p0[yy * s0 + xx] + p1[yy * s1 + xx] + 1) >> 1);
  } else {
    std::vector<int16_t> a((size_t)w * h), b((size_t)w * h);
    hevc_pred14(r0, x, y, w, h, mv0, bd, a.data());
    hevc_pred14(r1, x, y, w, h, mv1, bd, b.data());
    const int shift = 15 - bd, round = 1 << (shift - 1);
    for (size_t i = 0; i < pred.size(); ++i) pred[i] = (S)std::clamp((a[i] + b[i] + round) >> shift, 0, maxv);
  }
  return dist.satd(src + (ptrdiff_t)y * ss + x, ss, pred.data(), w, w, h);
}

// satd_bi_at's explicit arm (h265_me.rs:4247-4261): both lists' 14-bit
// predictions through weighted_bi (dsp/hevc.rs:1064-1086).
template <class S>
uint32_t hevc_satd_bi_weighted(const Dist<S>& dist, const HevcRef<S>& r0, const HevcRef<S>& r1, int bd, const S* src,
                               ptrdiff_t ss, int x, int y, int w, int h, Mv mv0, Mv mv1, const int wt[5]) {
  const int maxv = (1 << bd) - 1, log2_wd = wt[0], w0 = wt[1], w1 = wt[2], o0 = wt[3], o1 = wt[4];
  std::vector<int16_t> a((size_t)w * h), b((size_t)w * h);
  std::vector<S> pred((size_t)w * h);
  hevc_pred14(r0, x, y, w, h, mv0, bd, a.data());
  hevc_pred14(r1, x, y, w, h, mv1, bd, b.data());
  const int round = (o0 + o1 + 1) << log2_wd;
  for (size_t i = 0; i < pred.size(); ++i)
    pred[i] = (S)std::clamp(((int)a[i] * w0 + (int)b[i] * w1 + round) >> (log2_wd + 1), 0, maxv);
  return dist.satd(src + (ptrdiff_t)y * ss + x, ss, pred.data(), w, w, h);
}

// refine_bi (h265_me.rs:3933-4014): the other list's prediction at its
// vector (read_at, else predict14 + uni) held fixed, the target
// clip(2 * src - it); search_full from the list's own vector, then
// refine_subpel, against the target at 2 * lam with the job's AMVP pair.
template <class S>
void hevc_refine_bi(const Dist<S>& dist, HevcRef<S>* const* refs, int bd, const S* src, ptrdiff_t ss, float lam,
                    const rme_params* p, const rme_bi_job& j, rme_result& o) {
  const int list = j.list, other = 1 - list, x = j.x, y = j.y, w = j.w, h = j.h, maxv = (1 << bd) - 1;
  const HevcRef<S>& ro = *refs[j.ref[other]];
  const Mv mo(j.mv[other].x, j.mv[other].y);
  std::vector<S> pred((size_t)w * h), t((size_t)w * h);
  ptrdiff_t ps = 0;
  const S* pp = hevc_read_at(ro, x, y, w, h, mo, &ps);
  if (!pp) {
    std::vector<int16_t> p14((size_t)w * h);
    hevc_pred14(ro, x, y, w, h, mo, bd, p14.data());
    hevc_uni(pred.data(), w, p14.data(), w, h, 14 - bd, maxv);
    pp = pred.data();
    ps = w;
  }
  for (int yy = 0; yy < h; ++yy)
    for (int xx = 0; xx < w; ++xx)
      t[(size_t)yy * w + xx] = (S)std::clamp(2 * (int)src[(yy + y) * ss + x + xx] - (int)pp[yy * ps + xx], 0, maxv);
  const HevcRef<S>& rl = *refs[j.ref[list]];
  HevcSearch<S> sr{&dist, &rl.g, &rl.hp, bd, t.data(), w, x, y, w, h, 2.0f * lam, {{0, 0}, {0, 0}}};
  sr.pq[0][0] = j.mvp[0].x;
  sr.pq[0][1] = j.mvp[0].y;
  sr.pq[1][0] = j.mvp[1].x;
  sr.pq[1][1] = j.mvp[1].y;
  sr.search_range = p->hevc_search_range;
  sr.search_rings = p->hevc_search_rings;
  sr.quarter_cross = p->hevc_quarter_cross != 0;
  const Mv seed(j.mv[list].x, j.mv[list].y);
  uint32_t fc, sat, c;
  Mv full = sr.search_full(&seed, 1, &fc);
  Mv m = sr.refine_subpel(full, &sat, &c);
  o.mv = {m.x, m.y};
  o.ref = j.ref[list];
  o.cost = c;
  o.satd = sat;
  o.int_mv = {full.x, full.y};
  o.int_cost = fc;
  o.n_sad = sr.n_sad;
  o.n_satd = sr.n_satd;
}

template <class S>
int bi_frame(const rme_picture_desc* d, const void* src, int nref, const void* const* refs, const rme_params* p,
             const rme_bi_job* jobs, int n, int refine, uint32_t* satd, rme_result* out, const int* wt = nullptr) {
  Dist<S> dist = dist_scalar<S>();
  const int W = d->width, H = d->height, bd = d->bit_depth;
  std::vector<HevcRef<S>> rr(nref);
  std::vector<HevcRef<S>*> rp(nref);
  for (int r = 0; r < nref; ++r) {
    hevc_prepare_ref(rr[r], (const S*)refs[r], W, H, d->stride, p->hevc_pad, bd);
    rp[r] = &rr[r];
  }
  const float lam = hevc_lambda(p->qp, bd, p->hevc_lambda_scale);
  for (int i = 0; i < n; ++i) {
    const rme_bi_job& j = jobs[i];
    if (refine)
      hevc_refine_bi<S>(dist, rp.data(), bd, (const S*)src, d->stride, lam, p, j, out[i]);
    else if (wt)
      satd[i] = hevc_satd_bi_weighted<S>(dist, *rp[j.ref[0]], *rp[j.ref[1]], bd, (const S*)src, d->stride, j.x, j.y,
                                         j.w, j.h, Mv(j.mv[0].x, j.mv[0].y), Mv(j.mv[1].x, j.mv[1].y), wt);
    else
      satd[i] = hevc_satd_bi<S>(dist, *rp[j.ref[0]], *rp[j.ref[1]], bd, (const S*)src, d->stride, j.x, j.y, j.w, j.h,
                                Mv(j.mv[0].x, j.mv[0].y), Mv(j.mv[1].x, j.mv[1].y));
  }
  return 0;
}

template <class S>
int given_frame(const rme_picture_desc* d, const void* src, int nref, const void* const* refs, const rme_params* p,
                const rme_job* jobs, int njobs, int simd, rme_result* out) {
  Dist<S> dist = pick_dist<S>(simd);
  int W = d->width, H = d->height, bd = d->bit_depth;
  for (int j = 0; j < njobs; ++j)
    if (jobs[j].ref < 0 || jobs[j].ref >= nref || jobs[j].nseeds < 0 || jobs[j].nseeds > RME_MAX_SEEDS)
      return RME_EINVAL;
  if (d->codec == RME_CODEC_H264) {
    std::vector<H264Ref<S>> rr(nref);
    std::vector<H264Ref<S>*> rp(nref);
    for (int r = 0; r < nref; ++r) {
      h264_prepare_ref(rr[r], (const S*)refs[r], W, H, d->stride, p->h264_pad, bd);
      rp[r] = &rr[r];
    }
    h264_frame<S>(dist, (const S*)src, W, H, d->stride, nref, rp.data(), p, jobs, njobs, out);
  } else {
    std::vector<HevcRef<S>> rr(nref);
    std::vector<HevcRef<S>*> rp(nref);
    for (int r = 0; r < nref; ++r) {
      hevc_prepare_ref(rr[r], (const S*)refs[r], W, H, d->stride, p->hevc_pad, bd);
      rp[r] = &rr[r];
    }
    hevc_frame<S>(dist, (const S*)src, W, H, d->stride, bd, nref, rp.data(), p, jobs, njobs, out);
  }
  return 0;
}

uint32_t hevc_ref_idx_bits(int r, int nref) {  // ref_idx_lX, truncated unary, cMax nref-1
  if (nref <= 1) return 0;
  return r < nref - 1 ? (uint32_t)(r + 1) : (uint32_t)r;
}

}  // namespace

namespace {

// ---- lookahead (HEVC cutree) at half resolution -------------------------------
// encode/h265_cutree.rs: B = 8, PAD = 24, RANGE = 16.
constexpr int LA_B = 8, LA_PAD = 24, LA_RANGE = 16;

struct LowRes {
  std::vector<uint8_t> luma;
  int stride = 0, w = 0, h = 0, bw = 0, bh = 0;
  std::vector<uint32_t> intra;
  ptrdiff_t off(int x, int y) const { return (ptrdiff_t)(y + LA_PAD) * stride + x + LA_PAD; }
};

// LowRes::new (h265_cutree.rs:61-110): each sample the mean of a 2x2
// square of the picture (clamped at its edges), shifted to 8 bits, over
// whole 8x8 blocks; the padding edge-replicated.
template <class S>
LowRes lowres_new(const S* y, int w, int h, ptrdiff_t ys, int bd) {
  LowRes L;
  const int lw = (w + 1) / 2, lh = (h + 1) / 2;
  L.bw = (lw + LA_B - 1) / LA_B;
  L.bh = (lh + LA_B - 1) / LA_B;
  const int pw = L.bw * LA_B, ph = L.bh * LA_B;
  L.w = pw;
  L.h = ph;
  L.stride = pw + 2 * LA_PAD;
  L.luma.assign((size_t)L.stride * (ph + 2 * LA_PAD), 0);
  const int shift = bd - 8;
  auto at = [&](int x, int y0) { return (int)y[(ptrdiff_t)std::min(y0, h - 1) * ys + std::min(x, w - 1)]; };
  for (int yy = 0; yy < ph; ++yy)
    for (int xx = 0; xx < pw; ++xx) {
      const int x2 = 2 * std::min(xx, lw - 1), y2 = 2 * std::min(yy, lh - 1);
      const int sum = at(x2, y2) + at(x2 + 1, y2) + at(x2, y2 + 1) + at(x2 + 1, y2 + 1);
      L.luma[(size_t)(yy + LA_PAD) * L.stride + xx + LA_PAD] = (uint8_t)std::min(((sum + 2) >> 2) >> shift, 255);
    }
  for (int yy = LA_PAD; yy < LA_PAD + ph; ++yy) {
    uint8_t* row = &L.luma[(size_t)yy * L.stride];
    std::fill(row, row + LA_PAD, row[LA_PAD]);
    std::fill(row + LA_PAD + pw, row + L.stride, row[LA_PAD + pw - 1]);
  }
  for (int yy = 0; yy < LA_PAD; ++yy) {
    std::memcpy(&L.luma[(size_t)yy * L.stride], &L.luma[(size_t)LA_PAD * L.stride], L.stride);
    std::memcpy(&L.luma[(size_t)(LA_PAD + ph + yy) * L.stride], &L.luma[(size_t)(LA_PAD + ph - 1) * L.stride],
                L.stride);
  }
  // intra_cost (h265_cutree.rs:118-140): the least SATD of a flat (DC of
  // the 8 samples above and 8 left), a horizontal and a vertical
  // prediction; floored at 2 * B.
  L.intra.resize((size_t)L.bw * L.bh);
  for (int b = 0; b < L.bw * L.bh; ++b) {
    const int x = (b % L.bw) * LA_B, yb = (b / L.bw) * LA_B;
    const ptrdiff_t o = L.off(x, yb);
    const uint8_t* src = &L.luma[o];
    int top[LA_B], left[LA_B], st = 0;
    for (int i = 0; i < LA_B; ++i) {
      top[i] = L.luma[o - L.stride + i];
      left[i] = L.luma[o + (ptrdiff_t)i * L.stride - 1];
      st += top[i] + left[i];
    }
    uint8_t pred[LA_B * LA_B];
    std::fill(pred, pred + LA_B * LA_B, (uint8_t)((st + LA_B) / (2 * LA_B)));
    uint32_t best = satd_scalar<uint8_t>(src, L.stride, pred, LA_B, LA_B, LA_B);
    for (int i = 0; i < LA_B * LA_B; ++i) pred[i] = (uint8_t)left[i / LA_B];
    best = std::min(best, satd_scalar<uint8_t>(src, L.stride, pred, LA_B, LA_B, LA_B));
    for (int i = 0; i < LA_B * LA_B; ++i) pred[i] = (uint8_t)top[i % LA_B];
    best = std::min(best, satd_scalar<uint8_t>(src, L.stride, pred, LA_B, LA_B, LA_B));
    L.intra[b] = std::max(best, (uint32_t)(LA_B * 2));
  }
  return L;
}

// search (h265_cutree.rs:152-216): per block in raster order, seeds zero,
// left and above vectors (scored in order, strict <, within the padded
// plane); a cross descent at steps 4, 2, 1 from a fixed `from` per round,
// confined to +-RANGE around the best seed; SAD + 2 * min(|dx| + |dy|, 32);
// the winner's SATD as the cost.
void lowres_search(const LowRes& cur, const LowRes& refp, uint32_t* cost, rme_mv* mv, uint32_t* nsad) {
  const int n = cur.bw * cur.bh, lim = LA_PAD - 1;
  for (int b = 0; b < n; ++b) {
    const int bx = b % cur.bw, by = b / cur.bw, x = bx * LA_B, y = by * LA_B;
    const uint8_t* src = &cur.luma[cur.off(x, y)];
    uint32_t count = 0;
    auto ok = [&](int dx, int dy) {
      return x + dx >= -lim && y + dy >= -lim && x + dx + LA_B <= refp.w + lim && y + dy + LA_B <= refp.h + lim;
    };
    auto sad = [&](int dx, int dy) {
      ++count;
      return sad_scalar<uint8_t>(src, cur.stride, &refp.luma[refp.off(x + dx, y + dy)], refp.stride, LA_B, LA_B) +
             2u * (uint32_t)std::min(std::abs(dx) + std::abs(dy), 32);
    };
    int sx[3] = {0, 0, 0}, sy[3] = {0, 0, 0}, ns = 1;
    if (bx > 0) {
      sx[ns] = mv[b - 1].x;
      sy[ns++] = mv[b - 1].y;
    }
    if (by > 0) {
      sx[ns] = mv[b - cur.bw].x;
      sy[ns++] = mv[b - cur.bw].y;
    }
    int bxm = 0, bym = 0;
    uint32_t bc = UINT32_MAX;
    for (int k = 0; k < ns; ++k)
      if (ok(sx[k], sy[k])) {
        const uint32_t c = sad(sx[k], sy[k]);
        if (c < bc) {
          bc = c;
          bxm = sx[k];
          bym = sy[k];
        }
      }
    const int cx = bxm, cy = bym;
    for (int step : {4, 2, 1}) {
      for (;;) {
        const int fx = bxm, fy = bym;
        const int dirs[4][2] = {{step, 0}, {-step, 0}, {0, step}, {0, -step}};
        for (auto& d : dirs) {
          const int dx = fx + d[0], dy = fy + d[1];
          if (std::abs(dx - cx) > LA_RANGE || std::abs(dy - cy) > LA_RANGE || !ok(dx, dy)) continue;
          const uint32_t c = sad(dx, dy);
          if (c < bc) {
            bc = c;
            bxm = dx;
            bym = dy;
          }
        }
        if (bxm == fx && bym == fy) break;
      }
    }
    cost[b] = satd_scalar<uint8_t>(src, cur.stride, &refp.luma[refp.off(x + bxm, y + bym)], refp.stride, LA_B, LA_B);
    mv[b].x = (int16_t)bxm;
    mv[b].y = (int16_t)bym;
    if (nsad) nsad[b] = count;
  }
}

// bi_cost (h265_cutree.rs:222-243): SATD against the rounded average of
// the two displaced blocks.
uint32_t lowres_bi_cost(const LowRes& cur, const LowRes& r0, rme_mv m0, const LowRes& r1, rme_mv m1, int b) {
  const int x = (b % cur.bw) * LA_B, y = (b / cur.bw) * LA_B;
  const ptrdiff_t o0 = r0.off(x + m0.x, y + m0.y), o1 = r1.off(x + m1.x, y + m1.y);
  uint8_t pred[LA_B * LA_B];
  for (int yy = 0; yy < LA_B; ++yy)
    for (int xx = 0; xx < LA_B; ++xx)
      pred[yy * LA_B + xx] =
          (uint8_t)((r0.luma[o0 + (ptrdiff_t)yy * r0.stride + xx] + r1.luma[o1 + (ptrdiff_t)yy * r1.stride + xx] + 1) >> 1);
  return satd_scalar<uint8_t>(&cur.luma[cur.off(x, y)], cur.stride, pred, LA_B, LA_B, LA_B);
}

// ---- lookahead (H.264) at half resolution -----------------------------------
// encode/h264_lookahead.rs: PAD = 24, RANGE = 16; the plane keeps the
// stream's sample type.
template <class S>
struct LowResS {
  Plane<S> low;
  int bw = 0, bh = 0;
  std::vector<uint32_t> intra;
};

// Lookahead::add (h264_lookahead.rs:87-117): each sample the rounded mean
// of the 2x2 square of the picture at (2x, 2y), clamped to the picture,
// over the macroblock grid (8 samples per macroblock); the border
// replicated (extend_edges).
template <class S>
LowResS<S> lowres_h264(const S* y, int w, int h, ptrdiff_t ys) {
  LowResS<S> L;
  L.bw = (w + 15) / 16;
  L.bh = (h + 15) / 16;
  const int lw = L.bw * 8, lh = L.bh * 8;
  std::vector<S> flat((size_t)lw * lh);
  for (int yy = 0; yy < lh; ++yy) {
    const int y0 = std::min(2 * yy, h - 1), y1 = std::min(2 * yy + 1, h - 1);
    for (int xx = 0; xx < lw; ++xx) {
      const int x0 = std::min(2 * xx, w - 1), x1 = std::min(2 * xx + 1, w - 1);
      const int s = (int)y[y0 * ys + x0] + y[y0 * ys + x1] + y[y1 * ys + x0] + y[y1 * ys + x1];
      flat[(size_t)yy * lw + xx] = (S)((s + 2) >> 2);
    }
  }
  L.low = Plane<S>(lw, lh, LA_PAD);
  L.low.load(flat.data(), lw);
  // intra_costs (h264_lookahead.rs:146-222): DC from the neighbours there
  // are (the block's own mean with none), the vertical and horizontal
  // predictions where their edge exists, the bilinear blend of both edges;
  // the least SATD, plus 12.
  L.intra.resize((size_t)L.bw * L.bh);
  for (int by = 0; by < L.bh; ++by)
    for (int bx = 0; bx < L.bw; ++bx) {
      const int x = bx * 8, yb = by * 8;
      const S* src = &L.low.data[L.low.offset(x, yb)];
      const ptrdiff_t st = L.low.stride;
      int t[8], l[8];
      for (int i = 0; i < 8; ++i) {
        t[i] = L.low.data[L.low.offset(x + i, yb - 1)];
        l[i] = L.low.data[L.low.offset(x - 1, yb + i)];
      }
      const bool ht = by > 0, hl = bx > 0;
      int dc;
      if (ht && hl) {
        int sum = 8;
        for (int i = 0; i < 8; ++i) sum += t[i] + l[i];
        dc = sum >> 4;
      } else if (ht || hl) {
        int sum = 4;
        for (int i = 0; i < 8; ++i) sum += ht ? t[i] : l[i];
        dc = sum >> 3;
      } else {
        int sum = 32;
        for (int yy = 0; yy < 8; ++yy)
          for (int xx = 0; xx < 8; ++xx) sum += src[yy * st + xx];
        dc = sum >> 6;
      }
      S pred[64];
      std::fill(pred, pred + 64, (S)dc);
      uint32_t best = satd_scalar<S>(src, st, pred, 8, 8, 8);
      if (ht) {
        for (int i = 0; i < 64; ++i) pred[i] = (S)t[i % 8];
        best = std::min(best, satd_scalar<S>(src, st, pred, 8, 8, 8));
      }
      if (hl) {
        for (int i = 0; i < 64; ++i) pred[i] = (S)l[i / 8];
        best = std::min(best, satd_scalar<S>(src, st, pred, 8, 8, 8));
      }
      if (ht && hl) {
        for (int yy = 0; yy < 8; ++yy)
          for (int xx = 0; xx < 8; ++xx)
            pred[yy * 8 + xx] = (S)((t[xx] * (8 - yy) + l[yy] * (8 - xx) + t[7] * yy + l[7] * xx + 8) >> 4);
        best = std::min(best, satd_scalar<S>(src, st, pred, 8, 8, 8));
      }
      L.intra[(size_t)by * L.bw + bx] = best + 12;
    }
  return L;
}

// Lookahead::search (h264_lookahead.rs:227-376) for every block in raster
// order, the candidates being the left and above blocks' vectors (zero where
// there is no such block): SAD + 2 * min(|mx| + |my|, 64) from the zero
// vector; each candidate clamped to the window and scored unless it is the
// best's point; the hexagon with its three-new-points continuation, at
// most RANGE rounds; the square; the winner's SATD.
template <class S>
void lowres_search_h264(const LowResS<S>& cur, const LowResS<S>& refp, uint32_t* cost, rme_mv* mv, uint32_t* nsad) {
  static const int HEX[6][2] = {{-2, 0}, {-1, -2}, {1, -2}, {2, 0}, {1, 2}, {-1, 2}};
  static const int SQ[8][2] = {{-1, -1}, {0, -1}, {1, -1}, {-1, 0}, {1, 0}, {-1, 1}, {0, 1}, {1, 1}};
  const int lim = LA_PAD - 8, n = cur.bw * cur.bh;
  for (int b = 0; b < n; ++b) {
    const int bx = b % cur.bw, by = b / cur.bw, x = bx * 8, y = by * 8;
    const S* src = &cur.low.data[cur.low.offset(x, y)];
    const ptrdiff_t cs = cur.low.stride, rs = refp.low.stride;
    const int lx = std::max(-x - lim, -LA_RANGE * 2), hx = std::min(cur.low.width - 8 - x + lim, LA_RANGE * 2);
    const int ly = std::max(-y - lim, -LA_RANGE * 2), hy = std::min(cur.low.height - 8 - y + lim, LA_RANGE * 2);
    uint32_t count = 0;
    auto sad = [&](int mx, int my) {
      ++count;
      return sad_scalar<S>(src, cs, &refp.low.data[refp.low.offset(x + mx, y + my)], rs, 8, 8) +
             2u * (uint32_t)std::min(std::abs(mx) + std::abs(my), 64);
    };
    int bmx = 0, bmy = 0;
    uint32_t bc = sad(0, 0);
    const int cand[2][2] = {{bx > 0 ? mv[b - 1].x : 0, bx > 0 ? mv[b - 1].y : 0},
                            {by > 0 ? mv[b - cur.bw].x : 0, by > 0 ? mv[b - cur.bw].y : 0}};
    for (auto& c : cand) {
      const int cx = std::clamp(c[0], lx, hx), cy = std::clamp(c[1], ly, hy);
      if (cx != bmx || cy != bmy) {
        const uint32_t v = sad(cx, cy);
        if (v < bc) {
          bc = v;
          bmx = cx;
          bmy = cy;
        }
      }
    }
    int from = -1;
    for (int it = 0; it < LA_RANGE; ++it) {
      const int cx = bmx, cy = bmy;
      int step = -1;
      uint32_t live = 0x3f;
      if (from >= 0) {
        const uint32_t r = 7u << (from + 5);
        live = (r | r >> 6 | r >> 12) & 0x3f;
      }
      for (int k = 0; k < 6; ++k) {
        const int mx = cx + HEX[k][0], my = cy + HEX[k][1];
        if (!((live >> k) & 1) || mx < lx || mx > hx || my < ly || my > hy) continue;
        const uint32_t v = sad(mx, my);
        if (v < bc) {
          bc = v;
          bmx = mx;
          bmy = my;
          step = k;
        }
      }
      if (bmx == cx && bmy == cy) break;
      from = step;
    }
    const int cx = bmx, cy = bmy;
    for (auto& q : SQ) {
      const int mx = cx + q[0], my = cy + q[1];
      if (mx < lx || mx > hx || my < ly || my > hy) continue;
      const uint32_t v = sad(mx, my);
      if (v < bc) {
        bc = v;
        bmx = mx;
        bmy = my;
      }
    }
    cost[b] = satd_scalar<S>(src, cs, &refp.low.data[refp.low.offset(x + bmx, y + bmy)], rs, 8, 8);
    mv[b].x = (int16_t)bmx;
    mv[b].y = (int16_t)bmy;
    if (nsad) nsad[b] = count;
  }
}

// The average-of-two cost of estimate() (h264_lookahead.rs:417-432).
template <class S>
uint32_t lowres_bi_h264(const LowResS<S>& cur, const LowResS<S>& r0, rme_mv m0, const LowResS<S>& r1, rme_mv m1,
                        int b) {
  const int x = (b % cur.bw) * 8, y = (b / cur.bw) * 8;
  const S* a = &r0.low.data[r0.low.offset(x + m0.x, y + m0.y)];
  const S* c = &r1.low.data[r1.low.offset(x + m1.x, y + m1.y)];
  S avg[64];
  for (int yy = 0; yy < 8; ++yy)
    for (int xx = 0; xx < 8; ++xx)
      avg[yy * 8 + xx] = (S)(((int)a[yy * r0.low.stride + xx] + c[yy * r1.low.stride + xx] + 1) >> 1);
  return satd_scalar<S>(&cur.low.data[cur.low.offset(x, y)], cur.low.stride, avg, 8, 8, 8);
}

template <class S>
LowRes lowres_of(const rme_picture_desc* d, const void* luma) {
  return lowres_new<S>((const S*)luma, d->width, d->height, d->stride, d->bit_depth);
}
LowRes lowres_any(const rme_picture_desc* d, const void* luma) {
  return d->bit_depth == 8 ? lowres_of<uint8_t>(d, luma) : lowres_of<uint16_t>(d, luma);
}

template <class S>
LowResS<S> lowres_h264_of(const rme_picture_desc* d, const void* luma) {
  return lowres_h264<S>((const S*)luma, d->width, d->height, d->stride);
}

// ---- H.264 B macroblocks: the joint bi refinement ----------------------------

// bi_refine (h264_analyse.rs:2793-2900) under default weighting, on the
// source `src` (coded size, stride ss) and the pair's references.
template <class S>
void h264_bi_refine(const Dist<S>& dist, const S* src, ptrdiff_t ss, const H264Ref<S>* const R[2],
                    const uint16_t* tab, const rme_h264_bi_job& j, int rounds, bool diamond, rme_mv* mv_out,
                    uint32_t* cost_out) {
  static const int RING[8][2] = {{0, -1}, {-1, 0}, {1, 0}, {0, 1}, {-1, -1}, {1, -1}, {-1, 1}, {1, 1}};
  const int x = j.x, y = j.y, w = j.w, h = j.h;
  const Mv p[2] = {Mv(j.mvp[0].x, j.mvp[0].y), Mv(j.mvp[1].x, j.mvp[1].y)};
  // satd(r, PRED_BI, ...): each list's MeRef::pred, averaged (avg_into).
  auto satd_bi = [&](const Mv m[2]) -> uint32_t {
    S b0[256], b1[256], avg[256];
    int s0 = 0, s1 = 0;
    const S* p0 = R[0]->me.pred(x, y, m[0], w, h, b0, &s0);
    const S* p1 = R[1]->me.pred(x, y, m[1], w, h, b1, &s1);
    for (int yy = 0; yy < h; ++yy)
      for (int xx = 0; xx < w; ++xx)
        avg[yy * w + xx] = (S)(((int)p0[yy * s0 + xx] + (int)p1[yy * s1 + xx] + 1) >> 1);
    return dist.satd(src + (ptrdiff_t)y * ss + x, ss, avg, w, w, h);
  };
  auto rate = [&](const Mv m[2]) -> uint32_t {
    return h264_mv_comp(tab, m[0].x - p[0].x) + h264_mv_comp(tab, m[0].y - p[0].y) +
           h264_mv_comp(tab, m[1].x - p[1].x) + h264_mv_comp(tab, m[1].y - p[1].y);
  };
  Mv mbi[2] = {Mv(j.mv[0].x, j.mv[0].y), Mv(j.mv[1].x, j.mv[1].y)};
  uint32_t bi_cost = satd_bi(mbi) + rate(mbi);
  const int nr = bi_cost > j.limit ? 0 : rounds, npts = diamond ? 4 : 8;
  for (int it = 0; it < nr; ++it) {
    const Mv before[2] = {mbi[0], mbi[1]};
    for (int l = 0; l < 2; ++l) {
      const Mv c = mbi[l];
      Mv ms[8][2];
      uint32_t sc[8];
      for (int k = 0; k < npts; ++k) {
        ms[k][0] = mbi[0];
        ms[k][1] = mbi[1];
        ms[k][l] = Mv(c.x + RING[k][0], c.y + RING[k][1]);
        sc[k] = satd_bi(ms[k]);
      }
      for (int k = 0; k < npts; ++k) {
        const uint32_t rc = rate(ms[k]);
        if (rc >= bi_cost) continue;
        if (sc[k] + rc < bi_cost) {
          bi_cost = sc[k] + rc;
          mbi[0] = ms[k][0];
          mbi[1] = ms[k][1];
        }
      }
    }
    if (mbi[0] == before[0] && mbi[1] == before[1]) break;
  }
  mv_out[0] = {mbi[0].x, mbi[0].y};
  mv_out[1] = {mbi[1].x, mbi[1].y};
  *cost_out = bi_cost;
}

template <class S>
int h264_bi_frame(const rme_picture_desc* d, const void* src_luma, int nref, const void* const* refs,
                  const rme_params* p, const rme_h264_bi_job* jobs, int n, int rounds, int diamond, rme_mv* mv_out,
                  uint32_t* cost_out) {
  const int W = d->width, H = d->height, bd = d->bit_depth, CW = (W + 15) / 16 * 16, CH = (H + 15) / 16 * 16;
  Dist<S> dist = dist_scalar<S>();
  std::vector<H264Ref<S>> rr(nref);
  for (int r = 0; r < nref; ++r) h264_prepare_ref(rr[r], (const S*)refs[r], W, H, d->stride, p->h264_pad, bd);
  auto src = coded_h264((const S*)src_luma, W, H, d->stride, CW, CH);
  std::vector<uint16_t> tab(MV_TAB);
  h264_cost_table(h264_lambda_satd(p->qp), tab.data());
  for (int i = 0; i < n; ++i) {
    const rme_h264_bi_job& j = jobs[i];
    // Every vector the job can reach reads inside its search planes.
    for (int l = 0; l < 2; ++l) {
      int b[4];
      h264_search_bounds(CW, CH, p->h264_pad, j.x, j.y, j.w, j.h, INT32_MAX, b);
      const int lo_x = (j.mv[l].x - rounds) >> 2, hi_x = (j.mv[l].x + rounds) >> 2;
      const int lo_y = (j.mv[l].y - rounds) >> 2, hi_y = (j.mv[l].y + rounds) >> 2;
      if (lo_x < b[0] || hi_x >= b[1] || lo_y < b[2] || hi_y >= b[3]) return RME_EINVAL;
    }
    const H264Ref<S>* R[2] = {&rr[j.ref[0]], &rr[j.ref[1]]};
    h264_bi_refine<S>(dist, src.data(), CW, R, tab.data(), j, rounds, diamond != 0, mv_out + 2 * i, cost_out + i);
  }
  return 0;
}

// ---- weighted prediction: search planes and fit moments ---------------------

// wp_moments (dsp/distortion.rs:206-226) over the w x h display area: the
// sums of r, c, r*r, r*c and |c - r| (out[0..4]).
template <class S>
void wp_moments(const S* cur, ptrdiff_t cs, const S* ref, ptrdiff_t rs, int w, int h, uint64_t* out) {
  uint64_t sr = 0, sc = 0, srr = 0, src = 0, sad = 0;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const uint64_t r = ref[y * rs + x], c = cur[y * cs + x];
      sr += r;
      sc += c;
      srr += r * r;
      src += r * c;
      sad += r > c ? r - c : c - r;
    }
  out[0] = sr;
  out[1] = sc;
  out[2] = srr;
  out[3] = src;
  out[4] = sad;
}

// weighted_sad (dsp/distortion.rs:228-252): sum of |clip(((r * weight +
// round) >> shift) + offset) - c|, round = 2^(shift-1) (none at shift 0).
template <class S>
uint64_t weighted_sad(const S* cur, ptrdiff_t cs, const S* ref, ptrdiff_t rs, int w, int h, int weight, int shift,
                      int offset, int maxv) {
  const int round = shift >= 1 ? 1 << (shift - 1) : 0;
  uint64_t sad = 0;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const int p = (((int)ref[y * rs + x] * weight + round) >> shift) + offset;
      sad += (uint64_t)std::abs(std::clamp(p, 0, maxv) - (int)cur[y * cs + x]);
    }
  return sad;
}

// The weighted search plane's per-sample formula: H.264
// weighted_search_plane (h264_me.rs:653-672), ((v * w + 2^(log_wd-1)) >>
// log_wd) + o, no rounding at log_wd 0; HEVC weighted_search_plane
// (h265_me.rs:4275-4293), (((v << (14 - bd)) * w + 2^(log_wd-1)) >> log_wd)
// + o; clipped to the sample range.
inline int weighted_sample(int codec, int bd, int v, int log_wd, int w, int o) {
  const int maxv = (1 << bd) - 1;
  int p;
  if (codec == RME_CODEC_H264) {
    const int x = v * w;
    p = log_wd >= 1 ? ((x + (1 << (log_wd - 1))) >> log_wd) + o : x + o;
  } else {
    p = (((v << (14 - bd)) * w + (1 << (log_wd - 1))) >> log_wd) + o;
  }
  return std::clamp(p, 0, maxv);
}

}  // namespace

extern "C" {

void orc_params_default(rme_params* p, int32_t codec, int32_t qp) {
  std::memset(p, 0, sizeof(*p));
  p->codec = codec;
  p->qp = qp;
  p->predictor_mode = RME_PRED_STANDALONE;
  p->h264_range = 16;  // AnalysisCfg::MEDIUM.me (h264_analyse.rs:193-240)
  p->h264_hpel_iters = 2;
  p->h264_qpel_iters = 2;
  p->h264_refine_ratio = 1.5f;
  p->h264_vertical_range = 0x7ffffffe;  // MotionLimits::NONE.vertical_search
  p->h264_pad = 32;                     // h264/frame.rs LUMA_PAD
  p->hevc_search_range = 48;            // h265_me.rs SEARCH_RANGE
  p->hevc_search_rings = 0;             // Tune medium
  p->hevc_quarter_cross = 0;
  p->hevc_lambda_scale = 0.85f;  // h265_tune.rs:411
  p->hevc_pad = 80;              // hevc/frame.rs LUMA_PAD
  p->hevc_pu_mask = 0xF;
  p->hevc_amp = 0;
}

int orc_standalone_blocks(const rme_picture_desc* d, const rme_params* p, int32_t* blocks, int32_t* count) {
  if (!valid_desc(d) || !p || !count) return RME_EINVAL;
  *count = d->codec == RME_CODEC_H264 ? h264_blocks(d->width, d->height, blocks)
                                      : hevc_blocks(d->width, d->height, p, blocks);
  return 0;
}

int orc_frame_result_count(const rme_picture_desc* d, const rme_params* p, int32_t nref, int32_t njobs,
                           int32_t* count) {
  if (!valid_desc(d) || !p || !count) return RME_EINVAL;
  if (p->predictor_mode == RME_PRED_GIVEN) *count = njobs;
  else if (d->codec == RME_CODEC_H264) *count = h264_blocks(d->width, d->height, nullptr);
  else *count = hevc_blocks(d->width, d->height, p, nullptr) * nref;
  return 0;
}

// One frame: src and the nref references are unpadded pictures of `d`.
int orc_frame_search(const rme_picture_desc* d, const void* src, int32_t nref, const void* const* refs,
                     const rme_params* p, const rme_job* jobs, int32_t njobs, int32_t simd, rme_result* out) {
  if (!valid_desc(d) || !p || !src || !out || nref < 1 || nref > RME_MAX_REFS) return RME_EINVAL;
  if (p->predictor_mode == RME_PRED_GIVEN) {
    if (!jobs && njobs > 0) return RME_EINVAL;
    return d->bit_depth == 8 ? given_frame<uint8_t>(d, src, nref, refs, p, jobs, njobs, simd, out)
                             : given_frame<uint16_t>(d, src, nref, refs, p, jobs, njobs, simd, out);
  }
  return d->bit_depth == 8
             ? run_frames<uint8_t>(d, 1, &src, nref, refs, p, simd, 1, out, nullptr, nullptr, nullptr)
             : run_frames<uint16_t>(d, 1, &src, nref, refs, p, simd, 1, out, nullptr, nullptr, nullptr);
}

// A weighted list's sub-sample refinement (refine_subpel under Explicit
// weighting, h265_me.rs:3868-3922 with satd_at_weighted): per GIVEN job,
// from its first seed (a whole-sample vector) with its AMVP pair.
int orc_hevc_weighted_refine(const rme_picture_desc* d, const void* src, int32_t nref, const void* const* refs,
                             const rme_params* p, const rme_job* jobs, int32_t n, int32_t log2_wd, int32_t weight,
                             int32_t offset, rme_result* out) {
  if (!valid_desc(d) || d->codec != RME_CODEC_HEVC || !p || nref < 1 || nref > RME_MAX_REFS || n < 0 ||
      (n > 0 && (!jobs || !out)))
    return RME_EINVAL;
  auto run = [&](auto tag) {
    using S = decltype(tag);
    const int W = d->width, H = d->height, bd = d->bit_depth;
    Dist<S> dist = dist_scalar<S>();
    std::vector<HevcRef<S>> rr(nref);
    for (int r = 0; r < nref; ++r) hevc_prepare_ref(rr[r], (const S*)refs[r], W, H, d->stride, p->hevc_pad, bd);
    const float lam = hevc_lambda(p->qp, bd, p->hevc_lambda_scale);
    for (int i = 0; i < n; ++i) {
      const rme_job& j = jobs[i];
      HevcSearch<S> sr{&dist, &rr[j.ref].g, nullptr, bd, (const S*)src + (ptrdiff_t)j.y * d->stride + j.x,
                       d->stride, j.x, j.y, j.w, j.h, lam, {{0, 0}, {0, 0}}};
      sr.pq[0][0] = j.mvp[0].x;
      sr.pq[0][1] = j.mvp[0].y;
      sr.pq[1][0] = j.mvp[1].x;
      sr.pq[1][1] = j.mvp[1].y;
      sr.quarter_cross = p->hevc_quarter_cross != 0;
      sr.wp = true;
      sr.wp_log2 = log2_wd;
      sr.wp_w = weight;
      sr.wp_o = offset;
      const Mv start(j.seeds[0].x, j.seeds[0].y);
      uint32_t sat = 0, c = 0;
      const Mv m = sr.refine_subpel(start, &sat, &c);
      rme_result& o = out[i];
      o.mv = {m.x, m.y};
      o.ref = j.ref;
      o.cost = c;
      o.satd = sat;
      o.int_mv = {start.x, start.y};
      o.int_cost = 0;
      o.n_sad = 0;
      o.n_satd = sr.n_satd;
    }
  };
  for (int i = 0; i < n; ++i)
    if (jobs[i].ref < 0 || jobs[i].ref >= nref || jobs[i].w < 4 || jobs[i].h < 4 || jobs[i].w > 64 || jobs[i].h > 64 ||
        (jobs[i].w & 3) || (jobs[i].h & 3) || jobs[i].x < 0 || jobs[i].y < 0 || jobs[i].x + jobs[i].w > d->width ||
        jobs[i].y + jobs[i].h > d->height || jobs[i].nseeds < 1)
      return RME_EINVAL;
  if (d->bit_depth == 8) run(uint8_t{});
  else run(uint16_t{});
  return 0;
}

// HEVC bi-prediction jobs: satd_bi_at per job (refine == 0, into `satd`)
// or refine_bi per job (refine == 1, into `out`).
int orc_hevc_bi(const rme_picture_desc* d, const void* src, int32_t nref, const void* const* refs, const rme_params* p,
                const rme_bi_job* jobs, int32_t n, int32_t refine, uint32_t* satd, rme_result* out) {
  if (!valid_desc(d) || d->codec != RME_CODEC_HEVC || !p || nref < 1 || nref > RME_MAX_REFS || n < 0) return RME_EINVAL;
  for (int i = 0; i < n; ++i) {
    const rme_bi_job& j = jobs[i];
    if (j.ref[0] < 0 || j.ref[0] >= nref || j.ref[1] < 0 || j.ref[1] >= nref || j.list < 0 || j.list > 1 ||
        j.w < 4 || j.h < 4 || j.w > 64 || j.h > 64 || (j.w & 3) || (j.h & 3) || j.x < 0 || j.y < 0 ||
        j.x + j.w > d->width || j.y + j.h > d->height)
      return RME_EINVAL;
  }
  if (refine ? !out : !satd) return RME_EINVAL;
  return d->bit_depth == 8 ? bi_frame<uint8_t>(d, src, nref, refs, p, jobs, n, refine, satd, out)
                           : bi_frame<uint16_t>(d, src, nref, refs, p, jobs, n, refine, satd, out);
}

// H.264 B pairs: bi_refine per job (mv_out 2 per job, cost_out 1).
int orc_h264_bi_refine(const rme_picture_desc* d, const void* src, int32_t nref, const void* const* refs,
                       const rme_params* p, const rme_h264_bi_job* jobs, int32_t n, int32_t rounds, int32_t diamond,
                       rme_mv* mv_out, uint32_t* cost_out) {
  if (!valid_desc(d) || d->codec != RME_CODEC_H264 || !p || nref < 1 || nref > RME_MAX_REFS || n < 0 ||
      rounds < 0 || rounds > 16 || (n > 0 && (!jobs || !mv_out || !cost_out)))
    return RME_EINVAL;
  const int CW = (d->width + 15) / 16 * 16, CH = (d->height + 15) / 16 * 16;
  for (int i = 0; i < n; ++i) {
    const rme_h264_bi_job& j = jobs[i];
    if (j.ref[0] < 0 || j.ref[0] >= nref || j.ref[1] < 0 || j.ref[1] >= nref || j.w < 4 || j.h < 4 || j.w > 16 ||
        j.h > 16 || (j.w & 3) || (j.h & 3) || j.x < 0 || j.y < 0 || j.x + j.w > CW || j.y + j.h > CH)
      return RME_EINVAL;
  }
  return d->bit_depth == 8
             ? h264_bi_frame<uint8_t>(d, src, nref, refs, p, jobs, n, rounds, diamond, mv_out, cost_out)
             : h264_bi_frame<uint16_t>(d, src, nref, refs, p, jobs, n, rounds, diamond, mv_out, cost_out);
}

// Weighted prediction: the fit moments of `cur` against `ref` (out[5]).
int orc_wp_moments(const rme_picture_desc* d, const void* cur, const void* ref, uint64_t* out) {
  if (!valid_desc(d) || !cur || !ref || !out) return RME_EINVAL;
  if (d->bit_depth == 8)
    wp_moments<uint8_t>((const uint8_t*)cur, d->stride, (const uint8_t*)ref, d->stride, d->width, d->height, out);
  else
    wp_moments<uint16_t>((const uint16_t*)cur, d->stride, (const uint16_t*)ref, d->stride, d->width, d->height, out);
  return 0;
}

int orc_weighted_sad(const rme_picture_desc* d, const void* cur, const void* ref, int32_t weight, int32_t shift,
                     int32_t offset, uint64_t* out) {
  if (!valid_desc(d) || !cur || !ref || !out || shift < 0 || shift > 14) return RME_EINVAL;
  const int maxv = (1 << d->bit_depth) - 1;
  *out = d->bit_depth == 8 ? weighted_sad<uint8_t>((const uint8_t*)cur, d->stride, (const uint8_t*)ref, d->stride,
                                                   d->width, d->height, weight, shift, offset, maxv)
                           : weighted_sad<uint16_t>((const uint16_t*)cur, d->stride, (const uint16_t*)ref, d->stride,
                                                    d->width, d->height, weight, shift, offset, maxv);
  return 0;
}

// The weighted search plane's formula over `n` samples (any layout: the
// weighting is per sample, so it commutes with the border replication).
int orc_weighted_samples(int32_t codec, int32_t bit_depth, const void* in, int64_t n, int32_t log_wd, int32_t weight,
                         int32_t offset, void* out) {
  if (bit_depth < 8 || bit_depth > 12 || !in || !out || n < 0) return RME_EINVAL;
  if (codec == RME_CODEC_HEVC && log_wd < 1) return RME_EINVAL;
  for (int64_t i = 0; i < n; ++i) {
    const int v = bit_depth == 8 ? ((const uint8_t*)in)[i] : ((const uint16_t*)in)[i];
    const int q = weighted_sample(codec, bit_depth, v, log_wd, weight, offset);
    if (bit_depth == 8) ((uint8_t*)out)[i] = (uint8_t)q;
    else ((uint16_t*)out)[i] = (uint16_t)q;
  }
  return 0;
}

// satd_bi_at under explicit weighting per job (weights: log2_wd, w0, w1,
// o0, o1; offsets at the sample depth).
int orc_hevc_bi_weighted(const rme_picture_desc* d, const void* src, int32_t nref, const void* const* refs,
                         const rme_params* p, const rme_bi_job* jobs, int32_t n, const int32_t* weights,
                         uint32_t* satd) {
  if (!weights || weights[0] < 0 || weights[0] > 14 || weights[1] < -128 || weights[1] > 255 || weights[2] < -128 ||
      weights[2] > 255 || std::abs(weights[3]) > 4096 || std::abs(weights[4]) > 4096)
    return RME_EINVAL;
  if (!valid_desc(d) || d->codec != RME_CODEC_HEVC || !p || nref < 1 || nref > RME_MAX_REFS || n < 0 || !satd)
    return RME_EINVAL;
  for (int i = 0; i < n; ++i) {
    const rme_bi_job& j = jobs[i];
    if (j.ref[0] < 0 || j.ref[0] >= nref || j.ref[1] < 0 || j.ref[1] >= nref || j.w < 4 || j.h < 4 || j.w > 64 ||
        j.h > 64 || (j.w & 3) || (j.h & 3) || j.x < 0 || j.y < 0 || j.x + j.w > d->width || j.y + j.h > d->height)
      return RME_EINVAL;
  }
  int wt[5];
  for (int k = 0; k < 5; ++k) wt[k] = weights[k];
  return d->bit_depth == 8 ? bi_frame<uint8_t>(d, src, nref, refs, p, jobs, n, 0, satd, nullptr, wt)
                           : bi_frame<uint16_t>(d, src, nref, refs, p, jobs, n, 0, satd, nullptr, wt);
}

// Many STANDALONE frames on `threads` host threads (the timed CPU
// baseline): frame f reads srcs[f] and refs[f*nref .. f*nref+nref), writes
// out + offsets[f]. `seconds` = wall time including the plane builds.
int orc_frames_search_mt(const rme_picture_desc* d, int32_t nframes, const void* const* srcs, int32_t nref,
                         const void* const* refs, const rme_params* p, int32_t simd, int32_t threads,
                         rme_result* out, const int64_t* offsets, double* seconds, double* plane_seconds) {
  if (!valid_desc(d) || !p || nframes < 0 || nref < 1 || nref > RME_MAX_REFS) return RME_EINVAL;
  if (p->predictor_mode != RME_PRED_STANDALONE) return RME_EINVAL;
  return d->bit_depth == 8 ? run_frames<uint8_t>(d, nframes, srcs, nref, refs, p, simd, threads, out, offsets,
                                                 seconds, plane_seconds)
                           : run_frames<uint16_t>(d, nframes, srcs, nref, refs, p, simd, threads, out, offsets,
                                                  seconds, plane_seconds);
}

// The STANDALONE decision (chosen reference per block and the 2Nx2N
// quadtree), the rule rme_hevc_decide documents.
int orc_hevc_decide(const rme_picture_desc* d, const rme_params* p, int32_t nref, const rme_result* res,
                    int32_t* best, uint8_t* part) {
  if (!valid_desc(d) || !p || !res || nref < 1) return RME_EINVAL;
  int W = d->width, H = d->height;
  float lam = hevc_lambda(p->qp, d->bit_depth, p->hevc_lambda_scale);
  int sizes[4], nl = level_sizes(p, sizes);
  int base[5] = {0}, nbx[4], nby[4];
  for (int l = 0; l < nl; ++l) {
    nbx[l] = W / sizes[l];
    nby[l] = H / sizes[l];
    base[l + 1] = base[l] + nbx[l] * nby[l];
  }
  const int nb_all = hevc_blocks(W, H, p, nullptr);
  std::vector<uint64_t> cost(nb_all);
  for (int b = 0; b < nb_all; ++b) {
    int br = 0;
    uint64_t bc = UINT64_MAX;
    for (int r = 0; r < nref; ++r) {
      uint64_t c = (uint64_t)res[(size_t)b * nref + r].cost + hevc_rate(lam, hevc_ref_idx_bits(r, nref));
      if (c < bc) {
        bc = c;
        br = r;
      }
    }
    cost[b] = bc;
    if (best) best[b] = br;
  }
  if (!part) return 0;
  int cw = W / 8, ch = H / 8;
  std::memset(part, 0, (size_t)cw * ch);
  // decide(l, x, y): least summed cost over the area of a level-l block at
  // (x, y): its own PU (when it exists) against its children's decisions;
  // a tie keeps the larger PU. Returns UINT64_MAX where nothing covers it.
  auto log2i = [](int v) { return 31 - __builtin_clz((unsigned)v); };
  std::function<uint64_t(int, int, int, bool)> decide = [&](int l, int x, int y, bool mark) -> uint64_t {
    int N = sizes[l];
    if (x >= W || y >= H) return 0;
    bool exists = x + N <= W && y + N <= H;
    uint64_t own = exists ? cost[base[l] + (y / N) * nbx[l] + x / N] : UINT64_MAX;
    uint64_t split = UINT64_MAX;
    if (l + 1 < nl) {
      int M = sizes[l + 1];
      split = 0;
      for (int yy = y; yy < y + N; yy += M)
        for (int xx = x; xx < x + N; xx += M) {
          uint64_t c = decide(l + 1, xx, yy, false);
          if (c == UINT64_MAX) {
            split = UINT64_MAX;
            yy = y + N;
            break;
          }
          split += c;
        }
    }
    bool take_split = split < own;
    if (mark) {
      if (take_split) {
        int M = sizes[l + 1];
        for (int yy = y; yy < y + N; yy += M)
          for (int xx = x; xx < x + N; xx += M) decide(l + 1, xx, yy, true);
      } else if (exists) {
        for (int yy = y / 8; yy < (y + N) / 8 && yy < ch; ++yy)
          for (int xx = x / 8; xx < (x + N) / 8 && xx < cw; ++xx) part[yy * cw + xx] = (uint8_t)log2i(N);
      }
    }
    return take_split ? split : own;
  };
  int N0 = sizes[0];
  for (int y = 0; y < H; y += N0)
    for (int x = 0; x < W; x += N0) decide(0, x, y, true);
  return 0;
}

// ---- kernels and planes, for the property tests ----------------------------

uint32_t orc_sad(int32_t bd, const void* a, int64_t as, const void* b, int64_t bs, int32_t w, int32_t h,
                 int32_t simd) {
  if (bd == 8) return pick_dist<uint8_t>(simd).sad((const uint8_t*)a, as, (const uint8_t*)b, bs, w, h);
  return pick_dist<uint16_t>(simd).sad((const uint16_t*)a, as, (const uint16_t*)b, bs, w, h);
}
uint32_t orc_satd(int32_t bd, const void* a, int64_t as, const void* b, int64_t bs, int32_t w, int32_t h,
                  int32_t simd) {
  if (bd == 8) return pick_dist<uint8_t>(simd).satd((const uint8_t*)a, as, (const uint8_t*)b, bs, w, h);
  return pick_dist<uint16_t>(simd).satd((const uint16_t*)a, as, (const uint16_t*)b, bs, w, h);
}

float orc_h264_lambda(int32_t qp) { return h264_lambda_satd(qp); }
float orc_hevc_lambda(int32_t qp, int32_t bd, float scale) { return hevc_lambda(qp, bd, scale); }
void orc_h264_cost_table(float lambda, uint16_t* tab) { h264_cost_table(lambda, tab); }
uint32_t orc_hevc_mv_bits(int32_t mvx, int32_t mvy, const int32_t* pq4) {
  int pq[2][2] = {{pq4[0], pq4[1]}, {pq4[2], pq4[3]}};
  return hevc_mv_bits(mvx, mvy, pq);
}

// H.264: the padded plane (pad `pad`, coded size) and its b, h, j planes,
// 4 planes of (CW+2pad)*(CH+2pad) samples into out.
int orc_h264_planes(const rme_picture_desc* d, const void* luma, int32_t pad, void* out) {
  if (!valid_desc(d)) return RME_EINVAL;
  auto run = [&](auto tag) {
    using S = decltype(tag);
    H264Ref<S> r;
    h264_prepare_ref(r, (const S*)luma, d->width, d->height, d->stride, pad, d->bit_depth);
    size_t n = r.g.data.size();
    std::memcpy((S*)out, r.g.data.data(), n * sizeof(S));
    for (int k = 0; k < 3; ++k) std::memcpy((S*)out + (k + 1) * n, r.hp.p[k].data(), n * sizeof(S));
  };
  if (d->bit_depth == 8) run(uint8_t{});
  else run(uint16_t{});
  return 0;
}

// HEVC: the padded plane and its fifteen fractional phases (16 planes;
// phases HalfPlanes left unbuilt are zero), and HalfPlanes::ext. `flags`:
// bit 0 builds the quarter phases at any size, bit 1 interpolates with the
// AVX2 rung.
int orc_hevc_planes(const rme_picture_desc* d, const void* luma, int32_t pad, int32_t flags, void* out,
                    int32_t* ext) {
  if (!valid_desc(d)) return RME_EINVAL;
  auto run = [&](auto tag) {
    using S = decltype(tag);
    HevcRef<S> r;
    r.g = Plane<S>(d->width, d->height, pad);
    r.g.load((const S*)luma, d->stride);
    const Interp<S> I = pick_interp<S>((flags >> 1) & 1);
    r.hp.build(r.g, d->bit_depth, (flags & 1) != 0, &I);
    size_t n = r.g.data.size();
    std::memcpy((S*)out, r.g.data.data(), n * sizeof(S));
    for (int k = 0; k < 15; ++k) {
      if (r.hp.planes[k].empty()) std::memset((S*)out + (k + 1) * n, 0, n * sizeof(S));
      else std::memcpy((S*)out + (k + 1) * n, r.hp.planes[k].data(), n * sizeof(S));
    }
    if (ext) *ext = r.hp.ext;
  };
  if (d->bit_depth == 8) run(uint8_t{});
  else run(uint16_t{});
  return 0;
}

// The decoders' direct predictions, for plane-equality tests: H.264 qpel[]
// (dsp/h264.rs:436-495) of a w x h block at integer (xi, yi) and fraction
// (xf, yf); HEVC predict14 + uni (8.5.3.3.3.1). `luma` unpadded.
int orc_h264_qpel_direct(const rme_picture_desc* d, const void* luma, int32_t pad, int32_t xi, int32_t yi,
                         int32_t xf, int32_t yf, int32_t w, int32_t h, void* out) {
  if (!valid_desc(d)) return RME_EINVAL;
  auto run = [&](auto tag) {
    using S = decltype(tag);
    H264Ref<S> r;
    h264_prepare_ref(r, (const S*)luma, d->width, d->height, d->stride, pad, d->bit_depth);
    h264_qpel_direct<S>((S*)out, w, r.g.data.data() + r.g.offset(xi - 2, yi - 2), r.g.stride, w, h, xf, yf,
                        (1 << d->bit_depth) - 1);
  };
  if (d->bit_depth == 8) run(uint8_t{});
  else run(uint16_t{});
  return 0;
}

int orc_hevc_predict(const rme_picture_desc* d, const void* luma, int32_t pad, int32_t x, int32_t y, int32_t mvx,
                     int32_t mvy, int32_t w, int32_t h, void* out) {
  if (!valid_desc(d)) return RME_EINVAL;
  auto run = [&](auto tag) {
    using S = decltype(tag);
    Plane<S> g(d->width, d->height, pad);
    g.load((const S*)luma, d->stride);
    std::vector<int16_t> p14((size_t)w * h);
    hevc_interp(g, x + (mvx >> 2), y + (mvy >> 2), mvx & 3, mvy & 3, w, h, true, d->bit_depth, p14.data());
    hevc_uni((S*)out, w, p14.data(), w, h, 14 - d->bit_depth, (1 << d->bit_depth) - 1);
  };
  if (d->bit_depth == 8) run(uint8_t{});
  else run(uint16_t{});
  return 0;
}

// Chroma of chosen vectors (4:2:0). cb/cr unpadded (W/2 x H/2, cstride).
// HEVC: predict_block's chroma arm (hevc/inter.rs:555-660), CHROMA_PAD 40.
// H.264: chroma_pred_into (h264_me.rs:812-837) + chroma_scalar
// (dsp/h264.rs:499-520), CHROMA_PAD 16 (the window clamped outside it).
int orc_chroma_predict(const rme_picture_desc* d, const void* cb, const void* cr, int32_t cstride, int32_t nblocks,
                       const int32_t* blocks, const rme_mv* mvs, void* out) {
  if (!valid_desc(d)) return RME_EINVAL;
  int cw0 = d->width / 2, ch0 = d->height / 2;
  auto run = [&](auto tag) {
    using S = decltype(tag);
    int pad = d->codec == RME_CODEC_HEVC ? 40 : 16;
    Plane<S> pl[2] = {Plane<S>(cw0, ch0, pad), Plane<S>(cw0, ch0, pad)};
    pl[0].load((const S*)cb, cstride);
    pl[1].load((const S*)cr, cstride);
    S* o = (S*)out;
    int bd = d->bit_depth, maxv = (1 << bd) - 1;
    for (int i = 0; i < nblocks; ++i) {
      int x = blocks[4 * i], y = blocks[4 * i + 1], w = blocks[4 * i + 2] / 2, h = blocks[4 * i + 3] / 2;
      int mx = mvs[i].x, my = mvs[i].y;
      for (int c = 0; c < 2; ++c) {
        if (d->codec == RME_CODEC_HEVC) {
          std::vector<int16_t> p14((size_t)w * h);
          hevc_interp(pl[c], x / 2 + (mx >> 3), y / 2 + (my >> 3), mx & 7, my & 7, w, h, false, bd, p14.data());
          hevc_uni(o, w, p14.data(), w, h, 14 - bd, maxv);
        } else {
          int xci = x / 2 + (mx >> 3), yci = y / 2 + (my >> 3), xf = mx & 7, yf = my & 7;
          int A = (8 - xf) * (8 - yf), B = xf * (8 - yf), C = (8 - xf) * yf, D = xf * yf;
          for (int yy = 0; yy < h; ++yy)
            for (int xx = 0; xx < w; ++xx) {
              int v = A * pl[c].at_clamped(xci + xx, yci + yy) + B * pl[c].at_clamped(xci + xx + 1, yci + yy) +
                      C * pl[c].at_clamped(xci + xx, yci + yy + 1) + D * pl[c].at_clamped(xci + xx + 1, yci + yy + 1);
              o[yy * w + xx] = (S)((v + 32) >> 6);
            }
        }
        o += (size_t)w * h;
      }
    }
    (void)maxv;
  };
  if (d->bit_depth == 8) run(uint8_t{});
  else run(uint16_t{});
  return 0;
}

// The lookahead's half-resolution plane (padded, stride returned) and
// per-block intra costs of one picture.
int orc_lowres(const rme_picture_desc* d, const void* luma, uint8_t* plane, int32_t* stride, int32_t* rows,
               uint32_t* intra, int32_t* nblocks) {
  if (!valid_desc(d) || !luma) return RME_EINVAL;
  if (d->codec == RME_CODEC_H264) {
    auto run = [&](auto tag) {
      using S = decltype(tag);
      LowResS<S> L = lowres_h264_of<S>(d, luma);
      if (stride) *stride = L.low.stride;
      if (rows) *rows = L.low.rows();
      if (nblocks) *nblocks = L.bw * L.bh;
      if (plane) std::memcpy(plane, L.low.data.data(), L.low.data.size() * sizeof(S));
      if (intra) std::memcpy(intra, L.intra.data(), L.intra.size() * sizeof(uint32_t));
    };
    if (d->bit_depth == 8) run(uint8_t{});
    else run(uint16_t{});
    return 0;
  }
  LowRes L = lowres_any(d, luma);
  if (stride) *stride = L.stride;
  if (rows) *rows = L.h + 2 * LA_PAD;
  if (nblocks) *nblocks = L.bw * L.bh;
  if (plane) std::memcpy(plane, L.luma.data(), L.luma.size());
  if (intra) std::memcpy(intra, L.intra.data(), L.intra.size() * sizeof(uint32_t));
  return 0;
}

// The lookahead's search of `cur` against `ref` (both full-resolution
// pictures of one format), and optionally the bi cost against a second
// reference with vectors mv1.
int orc_lowres_search(const rme_picture_desc* d, const void* cur, const void* ref, uint32_t* cost, rme_mv* mv,
                      uint32_t* nsad) {
  if (!valid_desc(d) || !cur || !ref) return RME_EINVAL;
  if (d->codec == RME_CODEC_H264) {
    auto run = [&](auto tag) {
      using S = decltype(tag);
      lowres_search_h264<S>(lowres_h264_of<S>(d, cur), lowres_h264_of<S>(d, ref), cost, mv, nsad);
    };
    if (d->bit_depth == 8) run(uint8_t{});
    else run(uint16_t{});
    return 0;
  }
  LowRes C = lowres_any(d, cur), R = lowres_any(d, ref);
  lowres_search(C, R, cost, mv, nsad);
  return 0;
}

int orc_lowres_bi_cost(const rme_picture_desc* d, const void* cur, const void* r0, const rme_mv* mv0, const void* r1,
                       const rme_mv* mv1, uint32_t* cost) {
  if (!valid_desc(d) || !cur || !r0 || !r1) return RME_EINVAL;
  if (d->codec == RME_CODEC_H264) {
    auto run = [&](auto tag) {
      using S = decltype(tag);
      auto C = lowres_h264_of<S>(d, cur), A = lowres_h264_of<S>(d, r0), B = lowres_h264_of<S>(d, r1);
      for (int b = 0; b < C.bw * C.bh; ++b) cost[b] = lowres_bi_h264<S>(C, A, mv0[b], B, mv1[b], b);
    };
    if (d->bit_depth == 8) run(uint8_t{});
    else run(uint16_t{});
    return 0;
  }
  LowRes C = lowres_any(d, cur), A = lowres_any(d, r0), B = lowres_any(d, r1);
  for (int b = 0; b < C.bw * C.bh; ++b) cost[b] = lowres_bi_cost(C, A, mv0[b], B, mv1[b], b);
  return 0;
}

}  // extern "C"
