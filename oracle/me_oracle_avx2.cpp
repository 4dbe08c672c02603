// ORACLE — test infrastructure, not product code.
//
// AVX2 rungs of the oracle's SAD and SATD (this file is compiled with
// -mavx2; me_oracle.cpp uses them only where the CPU reports AVX2), for the timed host baseline. They
// follow the reference's x86 designs (dsp/distortion_x86.rs: psadbw for
// 8-bit SAD; 16-bit lanes, a butterfly Hadamard and pmaddwd sums for SATD;
// distortion_x86_u16.rs for 16-bit samples) and are checked against the
// scalar restatement in tests/test_oracle.py before anything is timed.
#include <immintrin.h>

#include "me_oracle.hpp"

namespace orc {
namespace {

uint32_t sad_u8_avx2(const uint8_t* a, ptrdiff_t as, const uint8_t* b,
                                                     ptrdiff_t bs, int w, int h) {
  __m256i acc = _mm256_setzero_si256();
  uint32_t tail = 0;
  for (int y = 0; y < h; ++y) {
    const uint8_t* ra = a + y * as;
    const uint8_t* rb = b + y * bs;
    int x = 0;
    for (; x + 32 <= w; x += 32)
      acc = _mm256_add_epi64(acc, _mm256_sad_epu8(_mm256_loadu_si256((const __m256i*)(ra + x)),
                                                  _mm256_loadu_si256((const __m256i*)(rb + x))));
    for (; x + 16 <= w; x += 16)
      acc = _mm256_add_epi64(
          acc, _mm256_castsi128_si256(_mm_sad_epu8(_mm_loadu_si128((const __m128i*)(ra + x)),
                                                   _mm_loadu_si128((const __m128i*)(rb + x)))));
    for (; x + 8 <= w; x += 8)
      acc = _mm256_add_epi64(
          acc, _mm256_castsi128_si256(_mm_sad_epu8(_mm_loadl_epi64((const __m128i*)(ra + x)),
                                                   _mm_loadl_epi64((const __m128i*)(rb + x)))));
    for (; x < w; ++x) tail += (uint32_t)std::abs((int)ra[x] - (int)rb[x]);
  }
  __m128i s = _mm_add_epi64(_mm256_castsi256_si128(acc), _mm256_extracti128_si256(acc, 1));
  s = _mm_add_epi64(s, _mm_unpackhi_epi64(s, s));
  return (uint32_t)_mm_cvtsi128_si64(s) + tail;
}

uint32_t sad_u16_avx2(const uint16_t* a, ptrdiff_t as, const uint16_t* b,
                                                      ptrdiff_t bs, int w, int h) {
  __m256i acc = _mm256_setzero_si256();
  const __m256i ones = _mm256_set1_epi16(1);
  uint32_t tail = 0;
  for (int y = 0; y < h; ++y) {
    const uint16_t* ra = a + y * as;
    const uint16_t* rb = b + y * bs;
    int x = 0;
    for (; x + 16 <= w; x += 16) {
      __m256i va = _mm256_loadu_si256((const __m256i*)(ra + x));
      __m256i vb = _mm256_loadu_si256((const __m256i*)(rb + x));
      __m256i d = _mm256_or_si256(_mm256_subs_epu16(va, vb), _mm256_subs_epu16(vb, va));
      // |d| <= 65535 per lane: widen by halves, then add as 32-bit.
      __m256i lo = _mm256_unpacklo_epi16(d, _mm256_setzero_si256());
      __m256i hi = _mm256_unpackhi_epi16(d, _mm256_setzero_si256());
      acc = _mm256_add_epi32(acc, _mm256_add_epi32(lo, hi));
    }
    (void)ones;
    for (; x < w; ++x) tail += (uint32_t)std::abs((int)ra[x] - (int)rb[x]);
  }
  __m128i s = _mm_add_epi32(_mm256_castsi256_si128(acc), _mm256_extracti128_si256(acc, 1));
  s = _mm_add_epi32(s, _mm_unpackhi_epi64(s, s));
  s = _mm_add_epi32(s, _mm_shuffle_epi32(s, 0x55));
  return (uint32_t)_mm_cvtsi128_si32(s) + tail;
}

// Four rows of 16-bit differences, two 4x4 tiles per 128-bit lane (four
// tiles per register set): the column butterfly across the rows, a 4x4
// transpose per tile, the row butterfly, |.|, and a per-tile sum. Exact for
// |differences| <= 1023 (every intermediate fits 16 bits).
inline uint32_t satd_4tiles(__m256i r0, __m256i r1, __m256i r2, __m256i r3) {
  __m256i s0 = _mm256_add_epi16(r0, r3), s3 = _mm256_sub_epi16(r0, r3);
  __m256i s1 = _mm256_add_epi16(r1, r2), s2 = _mm256_sub_epi16(r1, r2);
  __m256i c0 = _mm256_add_epi16(s0, s1), c2 = _mm256_sub_epi16(s0, s1);
  __m256i c1 = _mm256_add_epi16(s3, s2), c3 = _mm256_sub_epi16(s3, s2);
  // Transpose: element k of every row into one half register per tile.
  __m256i u0 = _mm256_unpacklo_epi16(c0, c1), u1 = _mm256_unpacklo_epi16(c2, c3);
  __m256i u2 = _mm256_unpackhi_epi16(c0, c1), u3 = _mm256_unpackhi_epi16(c2, c3);
  // Tile A (elements 0..3 of each lane) and tile B (elements 4..7).
  __m256i A01 = _mm256_unpacklo_epi32(u0, u1), A23 = _mm256_unpackhi_epi32(u0, u1);
  __m256i B01 = _mm256_unpacklo_epi32(u2, u3), B23 = _mm256_unpackhi_epi32(u2, u3);
  const __m256i ones = _mm256_set1_epi16(1);
  auto tile = [&](__m256i e01, __m256i e23) {
    // halves: e01 = [e0 | e1], e23 = [e2 | e3] (rows of one tile per half)
    __m256i e32 = _mm256_shuffle_epi32(e23, 0x4E);  // [e3 | e2]
    __m256i P = _mm256_add_epi16(e01, e32);         // [s0 | s1]
    __m256i M = _mm256_sub_epi16(e01, e32);         // [s3 | s2]
    __m256i Ps = _mm256_shuffle_epi32(P, 0x4E), Ms = _mm256_shuffle_epi32(M, 0x4E);
    __m256i t = _mm256_madd_epi16(_mm256_abs_epi16(_mm256_add_epi16(P, Ps)), ones);
    t = _mm256_add_epi32(t, _mm256_madd_epi16(_mm256_abs_epi16(_mm256_sub_epi16(P, Ps)), ones));
    t = _mm256_add_epi32(t, _mm256_madd_epi16(_mm256_abs_epi16(_mm256_add_epi16(M, Ms)), ones));
    t = _mm256_add_epi32(t, _mm256_madd_epi16(_mm256_abs_epi16(_mm256_sub_epi16(M, Ms)), ones));
    // Each 128-bit lane holds one tile twice: its sum is half the lane's.
    __m256i h1 = _mm256_add_epi32(t, _mm256_shuffle_epi32(t, 0x4E));
    h1 = _mm256_add_epi32(h1, _mm256_shuffle_epi32(h1, 0xB1));
    uint32_t lo = (uint32_t)_mm256_cvtsi256_si32(h1) >> 1;
    uint32_t hi = (uint32_t)_mm_cvtsi128_si32(_mm256_extracti128_si256(h1, 1)) >> 1;
    return ((lo + 1) >> 1) + ((hi + 1) >> 1);
  };
  return tile(A01, A23) + tile(B01, B23);
}

// An 8-wide column of 4x4 tiles, eight rows at a time: row y of the upper
// tile pair and row y + 4 of the lower pair share a register, so the four
// tiles run through the same 16-lane transform as a 16-wide strip.
template <class S>
uint32_t satd_w8(const S* a, ptrdiff_t as, const S* b, ptrdiff_t bs, int h) {
  uint32_t total = 0;
  for (int by = 0; by < h; by += 8) {
    __m256i r[4];
    for (int y = 0; y < 4; ++y) {
      const S* ra = a + (by + y) * as;
      const S* rb = b + (by + y) * bs;
      __m256i va, vb;
      if constexpr (sizeof(S) == 1) {
        va = _mm256_cvtepu8_epi16(_mm_unpacklo_epi64(_mm_loadl_epi64((const __m128i*)ra),
                                                     _mm_loadl_epi64((const __m128i*)(ra + 4 * as))));
        vb = _mm256_cvtepu8_epi16(_mm_unpacklo_epi64(_mm_loadl_epi64((const __m128i*)rb),
                                                     _mm_loadl_epi64((const __m128i*)(rb + 4 * bs))));
      } else {
        va = _mm256_set_m128i(_mm_loadu_si128((const __m128i*)(ra + 4 * as)), _mm_loadu_si128((const __m128i*)ra));
        vb = _mm256_set_m128i(_mm_loadu_si128((const __m128i*)(rb + 4 * bs)), _mm_loadu_si128((const __m128i*)rb));
      }
      r[y] = _mm256_sub_epi16(va, vb);
    }
    total += satd_4tiles(r[0], r[1], r[2], r[3]);
  }
  return total;
}

uint32_t satd_u8_avx2(const uint8_t* a, ptrdiff_t as, const uint8_t* b,
                                                      ptrdiff_t bs, int w, int h) {
  if (w % 16 != 0) {
    if (w % 8 != 0 || h % 8 != 0) return satd_scalar<uint8_t>(a, as, b, bs, w, h);
    uint32_t t = 0;
    for (int bx = 0; bx < w; bx += 8) t += satd_w8<uint8_t>(a + bx, as, b + bx, bs, h);
    return t;
  }
  uint32_t total = 0;
  for (int by = 0; by < h; by += 4)
    for (int bx = 0; bx < w; bx += 16) {
      __m256i r[4];
      for (int y = 0; y < 4; ++y) {
        __m256i va = _mm256_cvtepu8_epi16(_mm_loadu_si128((const __m128i*)(a + (by + y) * as + bx)));
        __m256i vb = _mm256_cvtepu8_epi16(_mm_loadu_si128((const __m128i*)(b + (by + y) * bs + bx)));
        r[y] = _mm256_sub_epi16(va, vb);
      }
      total += satd_4tiles(r[0], r[1], r[2], r[3]);
    }
  return total;
}

uint32_t satd_u16_avx2(const uint16_t* a, ptrdiff_t as, const uint16_t* b,
                                                       ptrdiff_t bs, int w, int h) {
  // 16-bit lanes are exact up to 10-bit samples; deeper ones take the
  // scalar path (checked per block: cheap next to the transform).
  const __m256i lim = _mm256_set1_epi16(1023);
  if (w % 16 != 0) {
    if (w % 8 != 0 || h % 8 != 0) return satd_scalar<uint16_t>(a, as, b, bs, w, h);
    uint32_t t = 0;
    for (int by = 0; by < h; by += 8)
      for (int bx = 0; bx < w; bx += 8) {
        __m256i over = _mm256_setzero_si256();
        for (int y = 0; y < 8; ++y) {
          over = _mm256_or_si256(over, _mm256_subs_epu16(_mm256_castsi128_si256(_mm_loadu_si128(
                                                             (const __m128i*)(a + (by + y) * as + bx))), lim));
          over = _mm256_or_si256(over, _mm256_subs_epu16(_mm256_castsi128_si256(_mm_loadu_si128(
                                                             (const __m128i*)(b + (by + y) * bs + bx))), lim));
        }
        over = _mm256_castsi128_si256(_mm256_castsi256_si128(over));
        t += _mm256_testz_si256(over, over) ? satd_w8<uint16_t>(a + by * as + bx, as, b + by * bs + bx, bs, 8)
                                            : satd_scalar<uint16_t>(a + by * as + bx, as, b + by * bs + bx, bs, 8, 8);
      }
    return t;
  }
  uint32_t total = 0;
  for (int by = 0; by < h; by += 4)
    for (int bx = 0; bx < w; bx += 16) {
      __m256i r[4];
      __m256i over = _mm256_setzero_si256();
      for (int y = 0; y < 4; ++y) {
        __m256i va = _mm256_loadu_si256((const __m256i*)(a + (by + y) * as + bx));
        __m256i vb = _mm256_loadu_si256((const __m256i*)(b + (by + y) * bs + bx));
        over = _mm256_or_si256(over, _mm256_subs_epu16(va, lim));
        over = _mm256_or_si256(over, _mm256_subs_epu16(vb, lim));
        r[y] = _mm256_sub_epi16(va, vb);
      }
      if (!_mm256_testz_si256(over, over))
        total += satd_scalar<uint16_t>(a + by * as + bx, as, b + by * bs + bx, bs, 16, 4);
      else
        total += satd_4tiles(r[0], r[1], r[2], r[3]);
    }
  return total;
}

// ---- HEVC luma interpolation (dsp/hevc.rs qpel_h / qpel_v / qpel_v2 /
// uni at 8.5.3.3.3.1), 16 outputs at a time: taps taken in pairs, each pair
// of rows (or columns) interleaved and multiplied-and-added in 32 bits
// (pmaddwd), shifted, packed back to 16 bits with saturation (the scalar
// forms' int16 store; the sums fit). Columns past the last 16-multiple go
// through the scalar form.
inline __m256i tap_pair(const int8_t* f, int k) {
  return _mm256_set1_epi32((int)(uint16_t)(int16_t)f[k] | ((int)(int16_t)f[k + 1] << 16));
}
template <class S>
inline __m256i load16(const S* p) {
  if constexpr (sizeof(S) == 1) return _mm256_cvtepu8_epi16(_mm_loadu_si128((const __m128i*)p));
  else return _mm256_loadu_si256((const __m256i*)p);
}
// Sum over k of f[k] * v[k] for eight 16-lane vectors, shifted right.
inline __m256i fir8(const __m256i v[8], const __m256i c[4], __m128i sh) {
  __m256i lo = _mm256_setzero_si256(), hi = _mm256_setzero_si256();
  for (int k = 0; k < 4; ++k) {
    lo = _mm256_add_epi32(lo, _mm256_madd_epi16(_mm256_unpacklo_epi16(v[2 * k], v[2 * k + 1]), c[k]));
    hi = _mm256_add_epi32(hi, _mm256_madd_epi16(_mm256_unpackhi_epi16(v[2 * k], v[2 * k + 1]), c[k]));
  }
  return _mm256_packs_epi32(_mm256_sra_epi32(lo, sh), _mm256_sra_epi32(hi, sh));
}

template <class S>
void h8_avx2(int16_t* dst, const S* src, ptrdiff_t ss, int w, int h, const int8_t* f, int shift) {
  const int wv = w & ~15;
  const __m256i c[4] = {tap_pair(f, 0), tap_pair(f, 2), tap_pair(f, 4), tap_pair(f, 6)};
  const __m128i sh = _mm_cvtsi32_si128(shift);
  for (int y = 0; y < h; ++y) {
    const S* s = src + y * ss;
    for (int x = 0; x < wv; x += 16) {
      __m256i v[8];
      for (int k = 0; k < 8; ++k) v[k] = load16<S>(s + x + k);
      _mm256_storeu_si256((__m256i*)(dst + y * w + x), fir8(v, c, sh));
    }
  }
  if (wv < w)
    for (int y = 0; y < h; ++y)
      for (int x = wv; x < w; ++x) {
        int acc = 0;
        for (int k = 0; k < 8; ++k) acc += f[k] * (int)src[y * ss + x + k];
        dst[y * w + x] = (int16_t)(acc >> shift);
      }
}

template <class S>
void v8_avx2(int16_t* dst, const S* src, ptrdiff_t ss, int w, int h, const int8_t* f, int shift) {
  const int wv = w & ~15;
  const __m256i c[4] = {tap_pair(f, 0), tap_pair(f, 2), tap_pair(f, 4), tap_pair(f, 6)};
  const __m128i sh = _mm_cvtsi32_si128(shift);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < wv; x += 16) {
      __m256i v[8];
      for (int k = 0; k < 8; ++k) v[k] = load16<S>(src + (y + k) * ss + x);
      _mm256_storeu_si256((__m256i*)(dst + y * w + x), fir8(v, c, sh));
    }
  if (wv < w)
    for (int y = 0; y < h; ++y)
      for (int x = wv; x < w; ++x) {
        int acc = 0;
        for (int k = 0; k < 8; ++k) acc += f[k] * (int)src[(y + k) * ss + x];
        dst[y * w + x] = (int16_t)(acc >> shift);
      }
}

void v2_8_avx2(int16_t* dst, const int16_t* src, int sstride, int w, int h, const int8_t* f) {
  const int wv = w & ~15;
  const __m256i c[4] = {tap_pair(f, 0), tap_pair(f, 2), tap_pair(f, 4), tap_pair(f, 6)};
  const __m128i sh = _mm_cvtsi32_si128(6);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < wv; x += 16) {
      __m256i v[8];
      for (int k = 0; k < 8; ++k) v[k] = _mm256_loadu_si256((const __m256i*)(src + (y + k) * sstride + x));
      _mm256_storeu_si256((__m256i*)(dst + y * w + x), fir8(v, c, sh));
    }
  if (wv < w)
    for (int y = 0; y < h; ++y)
      for (int x = wv; x < w; ++x) {
        int acc = 0;
        for (int k = 0; k < 8; ++k) acc += f[k] * (int)src[(y + k) * sstride + x];
        dst[y * w + x] = (int16_t)(acc >> 6);
      }
}

// uni: clip((x + 2^(shift-1)) >> shift) in 32-bit lanes (no 16-bit overflow
// whatever the intermediate), packed to the sample width.
template <class S>
void uni_avx2(S* dst, ptrdiff_t ds, const int16_t* src, int w, int h, int shift, int maxv) {
  const int wv = w & ~15;
  const __m256i rnd = _mm256_set1_epi32(shift > 0 ? 1 << (shift - 1) : 0), mx = _mm256_set1_epi32(maxv);
  const __m128i sh = _mm_cvtsi32_si128(shift);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < wv; x += 16) {
      const __m256i v = _mm256_loadu_si256((const __m256i*)(src + y * w + x));
      __m256i lo = _mm256_cvtepi16_epi32(_mm256_castsi256_si128(v));
      __m256i hi = _mm256_cvtepi16_epi32(_mm256_extracti128_si256(v, 1));
      lo = _mm256_min_epi32(_mm256_max_epi32(_mm256_sra_epi32(_mm256_add_epi32(lo, rnd), sh), _mm256_setzero_si256()), mx);
      hi = _mm256_min_epi32(_mm256_max_epi32(_mm256_sra_epi32(_mm256_add_epi32(hi, rnd), sh), _mm256_setzero_si256()), mx);
      // packus keeps 128-bit lanes apart: lo's lanes then hi's, reordered.
      const __m256i p16 = _mm256_permute4x64_epi64(_mm256_packus_epi32(lo, hi), 0xD8);
      if constexpr (sizeof(S) == 1) {
        const __m128i p8 = _mm_packus_epi16(_mm256_castsi256_si128(p16), _mm256_extracti128_si256(p16, 1));
        _mm_storeu_si128((__m128i*)(dst + y * ds + x), p8);
      } else {
        _mm256_storeu_si256((__m256i*)(dst + y * ds + x), p16);
      }
    }
  if (wv < w) {
    const int round = shift > 0 ? 1 << (shift - 1) : 0;
    for (int y = 0; y < h; ++y)
      for (int x = wv; x < w; ++x) dst[y * ds + x] = (S)std::clamp(((int)src[y * w + x] + round) >> shift, 0, maxv);
  }
}

}  // namespace

Interp<uint8_t> interp_avx2_u8() {
  return Interp<uint8_t>{&h8_avx2<uint8_t>, &v8_avx2<uint8_t>, &v2_8_avx2, &uni_avx2<uint8_t>};
}
Interp<uint16_t> interp_avx2_u16() {
  return Interp<uint16_t>{&h8_avx2<uint16_t>, &v8_avx2<uint16_t>, &v2_8_avx2, &uni_avx2<uint16_t>};
}

Dist<uint8_t> dist_avx2_u8() { return Dist<uint8_t>{&sad_u8_avx2, &satd_u8_avx2}; }
Dist<uint16_t> dist_avx2_u16() { return Dist<uint16_t>{&sad_u16_avx2, &satd_u16_avx2}; }

}  // namespace orc
