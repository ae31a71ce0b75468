// leco_decode.cuh -- per-block decode / random-access helpers shared by the
// single-column kernels (leco_decode.cu) and the batch kernels (leco_batch.cu).
#pragma once
#include <type_traits>

#include "leco_device.cuh"
#include "leco_internal.h"

namespace leco {

// Block model parsed from a header (or a directory entry).
struct BlockHdr {
  uint64_t body_bit;  // absolute bit address of field 0 (raw: of value 0)
  uint32_t l;         // field width; 8*S = raw; 126/127 = 2/1-value sentinels
  double a0, a1, a2;  // model
  uint64_t base;      // FOR minimum / Delta first value
  bool nonneg = false;  // linear model: every prediction of the block lies in [0, 2^51)
};

// Sets h.nonneg for a linear block of len values: the predictions are monotone in
// k, so the two ends bound them all.
template <int CODEC>
__device__ __forceinline__ void mark_nonneg(BlockHdr &h, uint32_t len) {
  if (CODEC == kLinear || CODEC == kLegacy) h.nonneg = preds_nonneg(h.a0, h.a1, len);
}

template <int CODEC, int S>
__device__ __forceinline__ BlockHdr parse_header(const uint8_t *__restrict__ payload, uint64_t off) {
  const uint64_t *words = reinterpret_cast<const uint64_t *>(payload);
  BlockHdr h;
  uint64_t w0 = load_u64_at(words, off);
  h.l = (uint32_t)(w0 & 0xff);
  h.a0 = h.a1 = h.a2 = 0;
  h.base = 0;
  if (CODEC == kLegacy) {  // [u8 l][f64 theta0][f32 theta1][body]; l >= 31: u32 values (raw)
    h.a0 = __longlong_as_double((long long)load_u64_at(words, off + 1));
    h.a1 = (double)__uint_as_float((uint32_t)load_u64_at(words, off + 9));
    h.body_bit = (off + 13) * 8;
    if (h.l == 31) h.l = 32;  // raw: the 32-bit values follow the header
    return h;
  }
  if (h.l == 8u * S || h.l == 126 || h.l == 127) {
    h.body_bit = (off + 1) * 8;
    return h;
  }
  if (CODEC == kLinear || CODEC == kPoly2) {
    h.a0 = __longlong_as_double((long long)load_u64_at(words, off + 1));
    h.a1 = __longlong_as_double((long long)load_u64_at(words, off + 9));
    if (CODEC == kPoly2) h.a2 = __longlong_as_double((long long)load_u64_at(words, off + 17));
  } else {
    uint64_t v = load_u64_at(words, off + 1);
    h.base = S == 8 ? v : (v & 0xffffffffull);
  }
  h.body_bit = (off + Hdr<CODEC, S>::bytes) * 8;
  return h;
}

template <int CODEC, int S>
__device__ __forceinline__ BlockHdr dir_entry_fields(ulonglong2 q0, ulonglong2 q1) {
  BlockHdr h;
  h.body_bit = q0.x & ((1ull << 48) - 1);
  h.l = (uint32_t)(q0.x >> 56);
  h.a0 = __longlong_as_double((long long)q0.y);
  h.a1 = __longlong_as_double((long long)q1.x);
  h.a2 = __longlong_as_double((long long)q1.y);
  h.base = S == 8 ? q0.y : (q0.y & 0xffffffffull);
  return h;
}
template <int CODEC, int S>
__device__ __forceinline__ BlockHdr from_dir(const leco_dir_entry *__restrict__ dir, uint64_t b) {
  const ulonglong2 *p = reinterpret_cast<const ulonglong2 *>(dir + b);
  return dir_entry_fields<CODEC, S>(__ldg(p), __ldg(p + 1));
}
// The same with an L2 eviction policy on the entry's two loads.
template <int CODEC, int S>
__device__ __forceinline__ BlockHdr from_dir_hint(const leco_dir_entry *__restrict__ dir, uint64_t b, uint64_t pol) {
  const ulonglong2 *p = reinterpret_cast<const ulonglong2 *>(dir + b);
  return dir_entry_fields<CODEC, S>(ld_nc_hint_v2(p, pol), ld_nc_hint_v2(p + 1, pol));
}

// Value k of a non-raw, non-Delta block given its field f (bulk decode rules).
template <int CODEC, int S>
__device__ __forceinline__ uint64_t value_from_field(const BlockHdr &h, uint32_t k, uint64_t f) {
  if (CODEC == kFor) return h.base + f;
  int64_t pred;
  if (CODEC == kLinear || CODEC == kLegacy) pred = f2i_x86(pred_linear(h.a0, h.a1, k));
  else pred = f2i_x86(pred_poly2(h.a0, h.a1, h.a2, __uint2double_rn(k)));
  return h.l ? apply_signed((uint64_t)pred, f, h.l) : (uint64_t)pred;
}

// Streams CNT values (a whole number of 16-byte chunks, 16-byte aligned) to out[o0...].
template <typename T, int CNT>
__device__ __forceinline__ void store_vals(T *out, uint64_t o0, const uint64_t *v) {
  if (sizeof(T) == 8) {
#pragma unroll
    for (int c = 0; c < CNT / 2; ++c)
      __stcs(reinterpret_cast<ulonglong2 *>(out + o0 + 2 * c), make_ulonglong2(v[2 * c], v[2 * c + 1]));
  } else {
#pragma unroll
    for (int c = 0; c < CNT / 4; ++c)
      __stcs(reinterpret_cast<uint4 *>(out + o0 + 4 * c),
             make_uint4((uint32_t)v[4 * c], (uint32_t)v[4 * c + 1], (uint32_t)v[4 * c + 2], (uint32_t)v[4 * c + 3]));
  }
}
// The same for a group whose start is 32-byte aligned when CNT values make whole
// 32-byte pieces (the narrow decoders start every thread's group on a 32-byte boundary
// of the output): each piece goes out as one 256-bit store (sm_100).  Other sizes as
// store_vals.  `out` is a generic pointer to global memory, which st.global takes as is:
// a generic address of global memory is its global address.
template <typename T, int CNT>
__device__ __forceinline__ void store_vals32(T *out, uint64_t o0, const uint64_t *v) {
  if constexpr (sizeof(T) * CNT % 32 == 0) {
#pragma unroll
    for (int c = 0; c < (int)(sizeof(T) * CNT / 32); ++c) {
      T *p = out + o0 + c * (32 / sizeof(T));
      if constexpr (sizeof(T) == 8) {
        asm volatile("st.global.cs.v4.u64 [%0], {%1, %2, %3, %4};" ::"l"(p), "l"(v[4 * c]), "l"(v[4 * c + 1]),
                     "l"(v[4 * c + 2]), "l"(v[4 * c + 3])
                     : "memory");
      } else {
        asm volatile("st.global.cs.v8.u32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "r"((uint32_t)v[8 * c]),
                     "r"((uint32_t)v[8 * c + 1]), "r"((uint32_t)v[8 * c + 2]), "r"((uint32_t)v[8 * c + 3]),
                     "r"((uint32_t)v[8 * c + 4]), "r"((uint32_t)v[8 * c + 5]), "r"((uint32_t)v[8 * c + 6]),
                     "r"((uint32_t)v[8 * c + 7])
                     : "memory");
      }
    }
  } else {
    store_vals<T, CNT>(out, o0, v);
  }
}

// Scratch of the Delta scan: two halves of 8 warp totals for each of up to four
// groups of a CTA.  One non-template function, so every kernel holds a single copy
// however many decoder instances it contains.
__device__ __forceinline__ uint64_t *delta_scan_scratch() {
  __shared__ uint64_t s[4 * 16];
  return s;
}

// Signed Delta field i of a block (0 for fields that are not deltas, i.e. i < 0 or
// i >= len - 1), in the value type's modular arithmetic.  The field read is clamped
// into the block's fields and always issued, so a run of these calls keeps all its
// loads in flight; WIDE: fields of more than 32 bits (read through 64-bit words,
// else 32-bit words); SMEM: `words` is a staged copy in shared memory (narrow
// fields only).  Needs l > 0 and len >= 2.
template <typename A, bool WIDE, bool SMEM = false>
__device__ __forceinline__ A delta_field(const uint64_t *__restrict__ words, const BlockHdr &h, uint32_t len, int64_t i) {
  static_assert(!(WIDE && SMEM), "staged Delta blocks have fields of at most 32 bits");
  const uint32_t l = h.l;
  const int64_t ic = i < 0 ? 0 : (i > (int64_t)len - 2 ? (int64_t)len - 2 : i);
  const uint64_t bit = h.body_bit + (uint64_t)ic * l;
  uint64_t f;
  if (WIDE) {
    f = load_field(words, bit, l);
  } else {
    const uint32_t *w = reinterpret_cast<const uint32_t *>(words) + (bit >> 5);
    const uint32_t w0 = SMEM ? w[0] : __ldg(w), w1 = SMEM ? w[1] : __ldg(w + 1);
    f = __funnelshift_r(w0, w1, (uint32_t)(bit & 31)) & (uint32_t)lowmask(l);
  }
  const uint64_t mag = f & lowmask(l - 1);
  const A d = ((f >> (l - 1)) & 1ull) ? (A)mag : (A)(0 - mag);
  return (i >= 0 && i == ic) ? d : (A)0;
}

// This lane's share of the prefix walk of Delta random access (read_Delta_int,
// bit_read.h:1292-1317): the sum of fields lane, lane + 32, ... below k.  Four
// reads in flight per lane; the warp sums the shares.
template <bool WIDE>
__device__ __forceinline__ uint64_t delta_walk_part(const uint64_t *__restrict__ words, const BlockHdr &h, uint32_t k,
                                                    int lane) {
  uint64_t part = 0;
  for (uint32_t j0 = 0; j0 < k; j0 += 128) {  // k >= 1 here, so the block has fields 0 .. k-1
    uint64_t d[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t j = j0 + 32 * q + lane;
      d[q] = delta_field<uint64_t, WIDE>(words, h, k + 1, j);
      if (j >= k) d[q] = 0;
    }
    part += d[0] + d[1] + d[2] + d[3];
  }
  return part;
}

// Delta_int<T>::decodeArray8 (delta_integer_template.h:89-127): value k =
// x0 + sum_{i<k} signed(field_i), mod 2^(8*sizeof(T)); field len-1 is not a delta
// (the reference packs n fields from n-1 deltas, :83).  The block is walked in tiles
// of DS*GS values (GS threads in the group): thread t owns the DS consecutive values
// from k0 = tile start + t*DS, i.e. fields k0-1 .. k0+DS-2, which it keeps in
// registers; one group-wide exclusive scan of the threads' sums (warp shuffles,
// then the warps' totals through shared memory) plus the carry of the tiles before
// gives its first value.  EMIT(k0, v) receives the DS values k0 .. k0+DS-1 (some
// may lie outside [lo, hi) or past the block); the group must call this together.
constexpr int kDeltaSpan = 8;
template <typename T, int G, bool WIDE, bool SMEM, typename Emit>
__device__ __forceinline__ void delta_tiles_w(const uint64_t *__restrict__ words, const BlockHdr &h, uint32_t len,
                                              uint32_t lo, uint32_t hi, Emit emit) {
  using A = typename std::conditional<sizeof(T) == 8, uint64_t, uint32_t>::type;  // arithmetic mod 2^(8S)
  constexpr int DS = kDeltaSpan;
  uint64_t *wtot = delta_scan_scratch() + (GroupOf<G>::sub ? 16 * group_index<G>() : 0);
  const uint32_t tid = group_rank<G>();
  const int lane = tid & 31, warp = tid >> 5;
  const uint32_t GS = group_size<G>(), NW = GS / 32;  // NW <= 8: whole-CTA groups here have <= 256 threads
  const uint32_t TW = DS * GS;                         // values per tile
  const uint32_t t1 = (hi + TW - 1) / TW;               // tiles up to the last value wanted
  const bool any = h.l && len >= 2;                      // a block of one value (or l = 0) has no deltas
  A carry = (A)h.base;
  for (uint32_t tl = 0; tl < t1; ++tl) {
    const uint32_t k0 = tl * TW + tid * DS;
    A v[DS];
#pragma unroll
    for (int j = 0; j < DS; ++j) v[j] = any ? delta_field<A, WIDE, SMEM>(words, h, len, (int64_t)k0 - 1 + j) : (A)0;
#pragma unroll
    for (int j = 1; j < DS; ++j) v[j] += v[j - 1];  // inclusive prefix inside the span
    const A tot = v[DS - 1];
    A incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const A y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    A before = carry, tile_sum;
    if (NW == 1) {
      before += incl - tot;
      tile_sum = __shfl_sync(0xffffffffu, incl, 31);
    } else {
      // one barrier per tile: every warp reads all warp totals of the tile; the two
      // halves of the scratch alternate, so a warp writes a half again only after the
      // next tile's barrier, which every warp passes after its reads of this one
      uint64_t *wt = wtot + 8 * (tl & 1);
      if (lane == 31) wt[warp] = incl;
      group_sync<G>();
      A bw = 0;
      tile_sum = 0;
      for (uint32_t w = 0; w < NW; ++w) {
        const A t = (A)wt[w];
        tile_sum += t;
        if (w < (uint32_t)warp) bw += t;
      }
      before += bw + (incl - tot);
    }
    if (k0 + DS > lo && k0 < hi) {
#pragma unroll
      for (int j = 0; j < DS; ++j) v[j] += before;
      emit(k0, v);
    }
    carry += tile_sum;
  }
}
// SMEM: `words` is a staged copy of the block in shared memory, whose fields are
// at most 32 bits wide.
template <typename T, int G, bool SMEM = false, typename Emit>
__device__ __forceinline__ void delta_tiles(const uint64_t *__restrict__ words, const BlockHdr &h, uint32_t len, uint32_t lo,
                                            uint32_t hi, Emit emit) {
  if (SMEM || h.l <= 32) delta_tiles_w<T, G, false, SMEM>(words, h, len, lo, hi, emit);
  else delta_tiles_w<T, G, true, false>(words, h, len, lo, hi, emit);
}
// Emitter of delta_tiles that stores the values of [lo, hi) to out[obase + k]: for
// a span wholly inside, 256-bit stores when it starts on 32 bytes, 16-byte stores
// when on 16, else one value at a time.
template <typename T>
struct DeltaStore {
  T *out;
  uint64_t obase;
  uint32_t lo, hi;
  template <typename A>
  __device__ __forceinline__ void operator()(uint32_t k0, const A *v) const {
    T *o = out + obase + k0;
    const uintptr_t oa = reinterpret_cast<uintptr_t>(o);
    if (k0 >= lo && k0 + kDeltaSpan <= hi && (oa & 15) == 0) {
      uint64_t w[kDeltaSpan];
#pragma unroll
      for (int j = 0; j < kDeltaSpan; ++j) w[j] = (uint64_t)v[j];
      if ((oa & 31) == 0) store_vals32<T, kDeltaSpan>(out, obase + k0, w);
      else store_vals<T, kDeltaSpan>(out, obase + k0, w);
    } else {
#pragma unroll
      for (int j = 0; j < kDeltaSpan; ++j)
        if (k0 + j >= lo && k0 + j < hi) o[j] = (T)v[j];
    }
  }
};

// True when every prediction of the block is a finite double inside
// (-2^63, 2^63), so the x86 out-of-range rule of f2i_x86 can never apply:
// |a0| + |a1|*(len-1) + |a2|*(len-1)^2 < 2^62 bounds them (rounding moves a
// prediction by a few ulps only).  NaN/inf models fail the comparison.
template <int CODEC>
__device__ __forceinline__ bool pred_in_range(const BlockHdr &h, uint32_t len) {
  const double L = __uint2double_rn(len ? len - 1 : 0);
  double b = fabs(h.a0) + fabs(h.a1) * L;
  if (CODEC == kPoly2) b += fabs(h.a2) * L * L;
  return b < 4611686018427387904.0;
}

// Decodes values [lo, hi) of one block whose fields are at most 32 bits wide
// (raw u32 blocks included).  Each thread produces VEC consecutive values per
// step (U 16-byte chunks, U: the unroll depth; kstart puts every thread's group on
// a 32-byte boundary of the output) and writes them with 256-bit stores.
// SUM: instead of storing, returns this thread's sum of the values (as T).
// The block's case is chosen once, outside the value loop: raw, FOR, a linear block
// whose predictions all lie in [0, 2^51) (both conversions exact on the FP64 pipe),
// or the general prediction (FAST: plain truncation, else the x86 rule).  (With the
// case tested per value and 16-byte stores the storing u64 decoder was 2 % faster
// than this loop with 16-byte stores -- which stalled on the memory-instruction
// queue -- and 1.5 % slower than this loop with 256-bit stores.)
enum : int { kNarrowRaw = 0, kNarrowFor = 1, kNarrowNonneg = 2, kNarrowPred = 3 };
template <typename T, int CODEC, int MODE, bool FAST, bool SMEM, int G, bool SUM, int U>
__device__ __forceinline__ uint64_t decode_narrow_mode(const BlockHdr &h, const uint32_t *__restrict__ words32, T *out,
                                                       uint64_t obase, uint32_t lo, uint32_t hi, int32_t kstart) {
  uint64_t acc = 0;
  constexpr int S = sizeof(T);
  constexpr int VEC = U * 16 / S;  // U 16-byte stores per step
  const uint32_t l = MODE == kNarrowRaw ? 32u : h.l;
  // words32 + body_bit/32: the body's first word (global payload or a staged copy in shared memory)
  const uint32_t *bp = words32 + (h.body_bit >> 5);
  const uint32_t bsh = (uint32_t)(h.body_bit & 31);
  // l == 0: the mask is 0, so every field reads as 0 (the two words read lie inside the
  // image or its slack)
  const uint32_t mask = l >= 32 ? 0xffffffffu : ((1u << l) - 1u);
  const uint32_t sb = l ? l - 1 : 0, m1 = mask >> 1;
  for (int32_t kv = kstart + (int32_t)group_rank<G>() * VEC; kv < (int32_t)hi; kv += (int32_t)group_size<G>() * VEC) {
    uint64_t v[VEC];
#pragma unroll
    for (int j = 0; j < VEC; ++j) {
      const int32_t k = kv + j;
      const uint32_t kk = k < (int32_t)lo ? lo : (uint32_t)k;  // values before lo are not stored
      const uint32_t r = bsh + kk * l;
      const uint32_t *p = bp + (r >> 5);
      const uint32_t w0 = SMEM ? p[0] : __ldg(p), w1 = SMEM ? p[1] : __ldg(p + 1);
      const uint32_t f = __funnelshift_r(w0, w1, r) & mask;
      if constexpr (MODE == kNarrowRaw) {
        v[j] = f;
      } else if constexpr (MODE == kNarrowFor) {
        v[j] = h.base + f;
      } else if constexpr (MODE == kNarrowNonneg) {
        // +mag when the sign bit is set ("data > pred"), else -mag: (mag ^ m) - m with
        // m = 0 or all ones; the magic-number sum holds 2^52 + trunc(prediction)
        const uint32_t m = (f >> sb) - 1u;
        const int32_t d = (int32_t)(((f & m1) ^ m) - m);
        const double q = __dadd_rz(pred_linear_fp64(h.a0, h.a1, kk), 4503599627370496.0);
        v[j] = (uint64_t)__double_as_longlong(q) + (uint64_t)(int64_t)d - 0x4330000000000000ull;
      } else {
        const double pd = (CODEC == kLinear || CODEC == kLegacy) ? pred_linear(h.a0, h.a1, kk)
                                                                 : pred_poly2(h.a0, h.a1, h.a2, __uint2double_rn(kk));
        const int64_t pred = FAST ? __double2ll_rz(pd) : f2i_x86(pd);
        const uint32_t mag = f & m1;
        const int64_t d = ((f >> sb) & 1u) ? (int64_t)mag : -(int64_t)mag;
        v[j] = (uint64_t)(pred + d);
      }
    }
    if (SUM) {
#pragma unroll
      for (int j = 0; j < VEC; ++j)
        if (kv + j >= (int32_t)lo && kv + j < (int32_t)hi) acc += (uint64_t)(T)v[j];
      continue;
    }
    const bool full = kv >= (int32_t)lo && kv + VEC <= (int32_t)hi;
    if (full) {
      store_vals32<T, VEC>(out, obase + kv, v);
    } else {
#pragma unroll
      for (int j = 0; j < VEC; ++j)
        if (kv + j >= (int32_t)lo && kv + j < (int32_t)hi) out[obase + kv + j] = (T)v[j];
    }
  }
  return acc;
}
template <typename T, int CODEC, bool FAST, bool SMEM = false, int G = 256, bool SUM = false, int U = 2>
__device__ __forceinline__ uint64_t decode_narrow(const BlockHdr &h, bool raw, const uint32_t *__restrict__ words32,
                                                  T *out, uint64_t obase, uint32_t lo, uint32_t hi, int32_t kstart) {
  if (raw) return decode_narrow_mode<T, CODEC, kNarrowRaw, FAST, SMEM, G, SUM, U>(h, words32, out, obase, lo, hi, kstart);
  if constexpr (CODEC == kFor) {
    return decode_narrow_mode<T, CODEC, kNarrowFor, FAST, SMEM, G, SUM, U>(h, words32, out, obase, lo, hi, kstart);
  } else {
    if constexpr (FAST && (CODEC == kLinear || CODEC == kLegacy)) {
      if (h.nonneg)
        return decode_narrow_mode<T, CODEC, kNarrowNonneg, FAST, SMEM, G, SUM, U>(h, words32, out, obase, lo, hi, kstart);
    }
    return decode_narrow_mode<T, CODEC, kNarrowPred, FAST, SMEM, G, SUM, U>(h, words32, out, obase, lo, hi, kstart);
  }
}

// ---- bulk / range decode ----------------------------------------------------
// One CTA per block.  Each thread decodes VEC = 16/sizeof(T) consecutive values
// per step from a three-word window of the packed body and writes them with one
// 16-byte store.
// Decodes the values of block b inside [a.first, a.first + a.count) with one
// thread group: the whole CTA (G = 256) or one warp (G = 32, small blocks).
template <typename T, int CODEC, int G = 256, int U = 2>
__device__ __forceinline__ void decode_block(const DecodeLaunch &a, uint64_t b) {
  const uint32_t rank = group_rank<G>();
  constexpr int S = sizeof(T);
  constexpr uint32_t TB = 8u * S;
  constexpr int VEC = 16 / S;
  const uint64_t base = b * a.bs;
  const uint32_t len = (uint32_t)umin64((uint64_t)a.bs, a.n - base);
  // values of this block inside [first, first+count)
  const uint64_t r0 = a.first > base ? a.first : base, r1 = umin64(a.first + a.count, base + len);
  if (r0 >= r1) return;
  const uint32_t lo = (uint32_t)(r0 - base), hi = (uint32_t)(r1 - base);
  T *out = reinterpret_cast<T *>(a.out);
  const uint64_t *words = reinterpret_cast<const uint64_t *>(a.payload);
  BlockHdr h = parse_header<CODEC, S>(a.payload, __ldg(a.offsets + b));
  const uint64_t obase = base - a.first;  // out index of block value 0

  if (h.l == 126 || h.l == 127) {  // sentinel blocks (…_integer_template.h:152-170)
    if (CODEC == kFor || CODEC == kLegacy) { if (rank == 0) atomicOr(a.error, kErrBadHeader); return; }
    if (rank == 0) {
      const uint32_t cnt = h.l == 127 ? 1 : 2;
      for (uint32_t k = lo; k < cnt && k < hi; ++k)
        out[obase + k] = (T)load_field(words, h.body_bit + (uint64_t)k * TB, TB);
    }
    return;
  }
  if (h.l > TB) {
    if (rank == 0) atomicOr(a.error, kErrBadHeader);
    return;
  }
  const bool raw = h.l == TB;

  if (CODEC == kDelta && !raw) {
    delta_tiles<T, G>(words, h, len, lo, hi, DeltaStore<T>{out, obase, lo, hi});
    return;
  }

  // First vector start so that out[obase + kv] is 16-byte aligned (out must be
  // sizeof(T)-aligned); kv may start up to VEC-1 values before lo.
  const uintptr_t oaddr = reinterpret_cast<uintptr_t>(out + obase + lo);
  const int32_t kstart = (int32_t)lo - (int32_t)((oaddr & 31) / S);  // groups start on 32 bytes
  const uint32_t l = raw ? TB : h.l;
  if (l <= 32) {
    // Narrow fields (every u32 block, u64 blocks with l <= 32): 32-bit field
    // extraction; predictions converted without range checks when the block's
    // model keeps every prediction inside int64 (decided once per block).
    const bool fast = (CODEC == kFor) || pred_in_range<CODEC>(h, len);
    const uint32_t *w32 = reinterpret_cast<const uint32_t *>(a.payload);
    if (!raw) mark_nonneg<CODEC>(h, len);
    if (fast) decode_narrow<T, CODEC, true, false, G, false, U>(h, raw, w32, out, obase, lo, hi, kstart);
    else decode_narrow<T, CODEC, false, false, G, false, U>(h, raw, w32, out, obase, lo, hi, kstart);
    return;
  }
  for (int32_t kv = kstart + (int32_t)rank * VEC; kv < (int32_t)hi; kv += (int32_t)group_size<G>() * VEC) {
    uint64_t v[VEC];
    const uint32_t kw = kv < (int32_t)lo ? lo : (uint32_t)kv;  // first value actually needed
    const uint64_t bit0 = h.body_bit + (uint64_t)kw * l;
    const uint64_t w = bit0 >> 6;
    const uint64_t W0 = __ldg(words + w), W1 = __ldg(words + w + 1), W2 = __ldg(words + w + 2);
    const uint32_t sh0 = (uint32_t)(bit0 & 63);
#pragma unroll
    for (int j = 0; j < VEC; ++j) {
      const int32_t k = kv + j;
      const uint32_t rel = sh0 + (uint32_t)(k - (int32_t)kw) * l;  // unused when k < kw
      const uint32_t sh = rel & 63;
      const uint64_t lo64 = rel < 64 ? W0 : (rel < 128 ? W1 : W2);
      const uint64_t hi64 = rel < 64 ? W1 : W2;
      const uint64_t f = funnel64(lo64, hi64, sh) & lowmask(l);
      v[j] = raw ? f : value_from_field<CODEC, S>(h, (uint32_t)k, f);
    }
    const bool full = kv >= (int32_t)lo && kv + VEC <= (int32_t)hi;
    if (full) store_vals<T, VEC>(out, obase + kv, v);
    else {
#pragma unroll
      for (int j = 0; j < VEC; ++j)
        if (kv + j >= (int32_t)lo && kv + j < (int32_t)hi) out[obase + kv + j] = (T)v[j];
    }
  }
}

// Value of one lookup from its block model and field (randomdecodeArray8 rules).
template <int CODEC, int S>
__device__ __forceinline__ uint64_t ra_value(const BlockHdr &h, uint32_t k, uint64_t f, uint32_t *error) {
  constexpr uint32_t TB = 8u * S;
  if (h.l == TB) return f;  // raw (…_integer_template.h:313-317)
  if (h.l > TB) {           // sentinel / corrupt header: the reference's random access has no such case
    atomicOr(error, kErrBadHeader);
    return 0;
  }
  if (CODEC == kFor) return h.l ? h.base + f : h.base;
  const double p = (CODEC == kLinear || CODEC == kLegacy) ? pred_linear(h.a0, h.a1, k)
                                                        : pred_poly2(h.a0, h.a1, h.a2, __uint2double_rn(k));
  if (h.l) return apply_signed((uint64_t)f2i_x86(p), f, h.l);
  return f2T_x86<S>(p);  // l == 0: (T)prediction directly (piecewise_fix_integer_template.h:334, poly :288)
}

// Random access of lookups first_i, first_i + G, ... (G = threads working on
// the index array): each thread keeps U lookups in flight (indices,
// directory entries and payload words are each loaded for all U before any is
// used), lookups i, i+G, i+2G, ... of one thread are strided by the grid so
// index loads and output stores stay coalesced across a warp.
template <typename T, int CODEC>
__device__ __forceinline__ void gather_lookups(const GatherLaunch &a, uint64_t first_i, uint64_t G) {
  constexpr int S = sizeof(T);
  constexpr uint32_t TB = 8u * S;
  constexpr int U = 4;
  const uint64_t *words = reinterpret_cast<const uint64_t *>(a.payload);
  T *out = reinterpret_cast<T *>(a.out);
  const bool small = a.n <= 0xffffffffull;
  const uint64_t stream_pol = l2_evict_first_policy(), dir_pol = l2_evict_last_policy();
  for (uint64_t i0 = first_i; i0 < a.m; i0 += G * U) {
    uint64_t g[U], b[U];
    uint32_t k[U];
    bool live[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint64_t i = i0 + (uint64_t)u * G;
      live[u] = i < a.m;
      g[u] = live[u] ? ld_nc_hint(a.idx + i, stream_pol) : 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (g[u] >= a.n) {
        if (live[u]) {
          out[i0 + (uint64_t)u * G] = 0;
          atomicOr(a.error, kErrBadIndex);
        }
        live[u] = false;
        g[u] = 0;
      }
      if (small) {
        b[u] = (uint32_t)g[u] / a.bs;
        k[u] = (uint32_t)g[u] - (uint32_t)b[u] * a.bs;
      } else {
        b[u] = g[u] / a.bs;
        k[u] = (uint32_t)(g[u] - b[u] * a.bs);
      }
    }
    BlockHdr h[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
      h[u] = a.dir ? from_dir_hint<CODEC, S>(a.dir, b[u], dir_pol)
                   : parse_header<CODEC, S>(a.payload, __ldg(a.offsets + b[u]));
    uint64_t lo[U], hi[U];
    uint32_t sh[U], l[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      l[u] = h[u].l > TB ? 0 : h[u].l;
      const uint64_t bit = h[u].body_bit + (uint64_t)k[u] * l[u];
      sh[u] = (uint32_t)(bit & 63);
      // the second word only when the field crosses into it: a random lookup then
      // touches one DRAM sector instead of two whenever the field sits in one word
      lo[u] = l[u] ? __ldg(words + (bit >> 6)) : 0;
      hi[u] = (l[u] && sh[u] + l[u] > 64) ? __ldg(words + (bit >> 6) + 1) : 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!live[u]) continue;
      const uint64_t f = funnel64(lo[u], hi[u], sh[u]) & lowmask(l[u]);
      st_hint<T>(out + i0 + (uint64_t)u * G, (T)ra_value<CODEC, S>(h[u], k[u], f, a.error), stream_pol);
    }
  }
}

}  // namespace leco
