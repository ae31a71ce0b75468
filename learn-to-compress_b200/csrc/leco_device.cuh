// leco_device.cuh -- device helpers shared by the LeCo sm_100a kernels.
//
// Arithmetic contract (what makes GPU and reference streams interchangeable):
//  * every FP64 step is one IEEE round-to-nearest operation written with an
//    explicit intrinsic (__dadd_rn, __dmul_rn, ...); the library is also built
//    with --fmad=false, so no multiply-add is ever contracted.  The reference is
//    compiled with -ffp-contract=off for the same reason.
//  * double -> integer conversions reproduce what the reference's x86-64 build
//    does, including its out-of-range cases (f2i_x86 / f2u_x86 below).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace leco {

typedef unsigned __int128 u128;
typedef __int128 i128;

constexpr int kLinear = 0, kFor = 1, kDelta = 2, kPoly2 = 3, kVarlen = 4;
// Legacy u32 codec piecewise_fix_op_max (piecewise_fix_op_minimize_maxerror.h:45-186):
// [u8 l][f64 theta0][f32 theta1][body]; raw u32 values after the header when l >= 31.
constexpr int kLegacy = 5;

// Blocks of at most this many values are encoded/decoded by one warp (eight
// per CTA) instead of a whole CTA.
constexpr uint32_t kWarpBlock = 512;

// Error word bits (device error word, read by leco_check).
constexpr uint32_t kErrBadIndex = 1u, kErrBadHeader = 2u, kErrTimeout = 4u, kErrCapacity = 8u, kErrLimit = 16u;

// (int64_t)x as x86-64 CVTTSD2SI computes it: truncation toward zero, and
// INT64_MIN for NaN or |x| >= 2^63 (reference: e.g. piecewise_fix_integer_template.h:54,
// bit_read.h:240).
__device__ __forceinline__ int64_t f2i_x86(double x) {
  return (x >= -9223372036854775808.0 && x < 9223372036854775808.0) ? __double2ll_rz(x)
                                                                     : (int64_t)0x8000000000000000ull;
}
// (uint64_t)x as gcc emits it for x86-64 without AVX-512: below 2^63 (or NaN) the
// signed conversion; otherwise convert x - 2^63 and flip bit 63 (reference:
// piecewise_fix_integer_template.h:334, bit_read.h:530).
__device__ __forceinline__ uint64_t f2u_x86(double x) {
  if (!(x >= 9223372036854775808.0)) return (uint64_t)f2i_x86(x);
  return (uint64_t)f2i_x86(__dsub_rn(x, 9223372036854775808.0)) ^ 0x8000000000000000ull;
}
// (T)x for T of S bytes; uint32_t takes the low half of CVTTSD2SI.
template <int S>
__device__ __forceinline__ uint64_t f2T_x86(double x) {
  if (S == 8) return f2u_x86(x);
  return (uint64_t)(uint32_t)f2i_x86(x);
}

// (__int128)x: truncation toward zero (gcc's __fixdfti) for |x| < 2^127; used where
// the variable-length codec converts its prediction to a 128-bit integer
// (piecewise_cost_merge_integer_template_double_wo_round.h:92,158).
__device__ __forceinline__ i128 f2i128(double x) {
  if (fabs(x) < 9223372036854775808.0) return (i128)__double2ll_rz(x);
  const uint64_t bits = (uint64_t)__double_as_longlong(x);
  const int e = (int)((bits >> 52) & 0x7ff) - 1075;
  const uint64_t m = (bits & ((1ull << 52) - 1)) | (1ull << 52);
  const i128 v = e >= 0 ? ((i128)m << e) : (i128)(m >> (-e));
  return x < 0 ? -v : v;
}

template <typename T>
__device__ __forceinline__ double to_double(T v);
template <>
__device__ __forceinline__ double to_double<uint32_t>(uint32_t v) { return __uint2double_rn(v); }
template <>
__device__ __forceinline__ double to_double<uint64_t>(uint64_t v) { return __ull2double_rn(v); }

// Correctly rounded (to nearest even) u128 -> double.
__device__ __forceinline__ double u128_to_double(u128 x) {
  uint64_t hi = (uint64_t)(x >> 64), lo = (uint64_t)x;
  if (hi == 0) return __ull2double_rn(lo);
  int z = __clzll(hi);                         // 0..63
  u128 y = x << z;                             // top bit at 127
  uint64_t top = (uint64_t)(y >> 64);
  uint64_t rest = (uint64_t)y;
  top |= (rest != 0);                          // sticky bit below the 64-bit window
  double d = __ull2double_rn(top);             // rounds 64 -> 53 bits correctly
  // scale by 2^(64 - z): exact (power of two, no overflow below 2^128)
  return __dmul_rn(d, __longlong_as_double((long long)(1023 + 64 - z) << 52));
}

// Linear prediction theta0 + theta1 * k (one multiply, one add, both rounded).
__device__ __forceinline__ double pred_linear(double t0, double t1, uint32_t k) {
  return __dadd_rn(t0, __dmul_rn(t1, __uint2double_rn(k)));
}

// The same two conversions on the FP64 pipe instead of the conversion unit, exactly:
// (double)k = (2^52 + k) - 2^52 for any 32-bit k, and for 0 <= p < 2^51 the
// round-toward-zero sum 2^52 + p is 2^52 + trunc(p), whose low mantissa bits are
// trunc(p).  pred_linear_fp64 equals pred_linear bit for bit.
__device__ __forceinline__ double u32_to_double_fp64(uint32_t k) {
  return __dsub_rn(__hiloint2double(0x43300000, (int)k), 4503599627370496.0);
}
__device__ __forceinline__ double pred_linear_fp64(double t0, double t1, uint32_t k) {
  return __dadd_rn(t0, __dmul_rn(t1, u32_to_double_fp64(k)));
}
__device__ __forceinline__ int64_t trunc_nonneg_fp64(double p) {
  return __double_as_longlong(__dadd_rz(p, 4503599627370496.0)) - 0x4330000000000000ll;
}
// True when every linear prediction of k = 0..len-1 lies in [0, 2^51): they are
// monotone in k, so the two ends bound them (NaN models fail the comparisons).
__device__ __forceinline__ bool preds_nonneg(double t0, double t1, uint32_t len) {
  const double p0 = pred_linear(t0, t1, 0), p1 = pred_linear(t0, t1, len ? len - 1 : 0);
  return p0 >= 0.0 && p1 >= 0.0 && p0 < 2251799813685248.0 && p1 < 2251799813685248.0;
}
// andviane::Polynomial::operator() for degree 2 (Polynomial.tpp:17-28):
// s = 0; xx = 1; for a in (a0,a1,a2): s = s + xx*a; xx = xx*x.
__device__ __forceinline__ double pred_poly2(double a0, double a1, double a2, double x) {
  double xx = 1.0, s = 0.0;
  s = __dadd_rn(s, __dmul_rn(xx, a0));
  xx = __dmul_rn(xx, x);
  s = __dadd_rn(s, __dmul_rn(xx, a1));
  xx = __dmul_rn(xx, x);
  s = __dadd_rn(s, __dmul_rn(xx, a2));
  return s;
}

__host__ __device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }
__device__ __forceinline__ uint64_t lowmask(uint32_t l) { return l >= 64 ? ~0ull : ((1ull << l) - 1ull); }
__device__ __forceinline__ uint32_t bits_of(uint64_t v) { return v ? 64u - (uint32_t)__clzll(v) : 0u; }

// Two aligned words -> the 64 bits starting at bit `sh` (0..63) of `lo`.
// Branch-free: (hi << 1) << (63 - sh) is hi << (64 - sh) for sh > 0 and 0 for sh == 0.
__device__ __forceinline__ uint64_t funnel64(uint64_t lo, uint64_t hi, uint32_t sh) {
  return (lo >> sh) | ((hi << 1) << (63 - sh));
}

// l bits (l <= 64) at absolute bit address `bit` of an 8-byte aligned byte
// array `words` (LSB-first, the reference's bit order).  Reads 2 words.
__device__ __forceinline__ uint64_t load_field(const uint64_t *__restrict__ words, uint64_t bit, uint32_t l) {
  uint64_t w = bit >> 6;
  uint64_t lo = __ldg(words + w), hi = __ldg(words + w + 1);
  return funnel64(lo, hi, (uint32_t)(bit & 63)) & lowmask(l);
}
// 8 bytes at an arbitrary byte address.
__device__ __forceinline__ uint64_t load_u64_at(const uint64_t *__restrict__ words, uint64_t byte) {
  return load_field(words, byte * 8, 64);
}

// Signed-magnitude field decode: low l-1 bits magnitude, bit l-1 set when the
// value lies above the prediction (bit_read.h:243-255).
__device__ __forceinline__ uint64_t apply_signed(uint64_t pred, uint64_t f, uint32_t l) {
  uint64_t mag = f & lowmask(l - 1);
  return ((f >> (l - 1)) & 1ull) ? pred + mag : pred - mag;
}

// Header sizes of the reference block images.
template <int CODEC, int S>
struct Hdr {
  // bytes before the packed body
  static constexpr uint32_t bytes =
      CODEC == kLinear ? 17u : CODEC == kFor ? 1u + 2u * S : CODEC == kDelta ? 1u + S : CODEC == kLegacy ? 13u : 25u;
};

// Byte size of a block image (headers/bit_write.h:257-323 pad 8-end%8; FOR
// :326-390 pad (32-l)/8 for l <= 32, none above).
template <int CODEC, int S>
__host__ __device__ __forceinline__ uint64_t block_bytes(uint32_t l, uint32_t n) {
  if (CODEC == kLegacy) {  // write_delta_T (bit_write.h:186-245) / write_delta_default (:395-410)
    if (l == 0) return 13;
    if (l >= 31) return 13ull + 4ull * n;
    return 13ull + ((uint64_t)l * n + 7) / 8 + 1 + (32u - l) / 8u;
  }
  if (l == 8u * S) return 1ull + (uint64_t)n * S;
  uint64_t h = CODEC == kLinear ? 17u : CODEC == kFor ? 1u + 2u * S : CODEC == kDelta ? 1u + S : 25u;
  if (l == 0) return h;
  uint64_t end = ((uint64_t)l * n + 7) / 8;
  uint64_t pad = CODEC == kFor ? (l <= 32 ? (32u - l) / 8u : 0u) : 8u - end % 8u;
  return h + end + 1 + pad;
}

// ---- warp / block reductions ------------------------------------------------

__device__ __forceinline__ uint64_t shfl_xor_u64(uint64_t v, int m) {
  return __shfl_xor_sync(0xffffffffu, (unsigned long long)v, m);
}
__device__ __forceinline__ u128 warp_sum_u128(u128 v) {
  for (int m = 16; m; m >>= 1) {
    uint64_t lo = shfl_xor_u64((uint64_t)v, m), hi = shfl_xor_u64((uint64_t)(v >> 64), m);
    v += ((u128)hi << 64) | lo;
  }
  return v;
}
__device__ __forceinline__ uint64_t warp_max_u64(uint64_t v) {
  for (int m = 16; m; m >>= 1) { uint64_t o = shfl_xor_u64(v, m); v = o > v ? o : v; }
  return v;
}
__device__ __forceinline__ uint64_t warp_min_u64(uint64_t v) {
  for (int m = 16; m; m >>= 1) { uint64_t o = shfl_xor_u64(v, m); v = o < v ? o : v; }
  return v;
}
__device__ __forceinline__ int64_t warp_max_i64(int64_t v) {
  for (int m = 16; m; m >>= 1) { int64_t o = (int64_t)shfl_xor_u64((uint64_t)v, m); v = o > v ? o : v; }
  return v;
}
__device__ __forceinline__ int64_t warp_min_i64(int64_t v) {
  for (int m = 16; m; m >>= 1) { int64_t o = (int64_t)shfl_xor_u64((uint64_t)v, m); v = o < v ? o : v; }
  return v;
}
__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
  for (int m = 16; m; m >>= 1) v += shfl_xor_u64(v, m);
  return v;
}

// Block-wide reduction through `red` (>= 32 entries of 16 bytes of shared
// memory); the result is returned to every thread.  OP: 0 sum u128, the rest
// on the low 64 bits: 1 max u64, 2 min u64, 3 max i64, 4 min i64, 5 sum u64.
template <int OP>
__device__ __forceinline__ u128 block_reduce(u128 v, u128 *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  auto wred = [](u128 x) -> u128 {
    switch (OP) {
      case 0: return warp_sum_u128(x);
      case 1: return warp_max_u64((uint64_t)x);
      case 2: return warp_min_u64((uint64_t)x);
      case 3: return (u128)(uint64_t)warp_max_i64((int64_t)(uint64_t)x);
      case 4: return (u128)(uint64_t)warp_min_i64((int64_t)(uint64_t)x);
      default: return warp_sum_u64((uint64_t)x);
    }
  };
  v = wred(v);
  __syncthreads();  // `red` may still be read by a previous reduction
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    u128 ident = OP == 2 ? (u128)~0ull : OP == 3 ? (u128)0x8000000000000000ull : OP == 4 ? (u128)0x7fffffffffffffffull : (u128)0;
    u128 x = lane < nw ? red[lane] : ident;
    x = wred(x);
    if (lane == 0) red[32] = x;
  }
  __syncthreads();
  return red[32];
}

// Two block-wide reductions in one shared-memory round: `red` needs 66 entries.
template <int OPA, int OPB>
__device__ __forceinline__ void block_reduce2(u128 &a, u128 &b, u128 *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  auto wred = [](u128 x, int op) -> u128 {
    switch (op) {
      case 0: return warp_sum_u128(x);
      case 1: return warp_max_u64((uint64_t)x);
      case 2: return warp_min_u64((uint64_t)x);
      case 3: return (u128)(uint64_t)warp_max_i64((int64_t)(uint64_t)x);
      case 4: return (u128)(uint64_t)warp_min_i64((int64_t)(uint64_t)x);
      default: return warp_sum_u64((uint64_t)x);
    }
  };
  auto ident = [](int op) -> u128 {
    return op == 2 ? (u128)~0ull : op == 3 ? (u128)0x8000000000000000ull : op == 4 ? (u128)0x7fffffffffffffffull : (u128)0;
  };
  a = wred(a, OPA);
  b = wred(b, OPB);
  __syncthreads();
  if (lane == 0) {
    red[warp] = a;
    red[33 + warp] = b;
  }
  __syncthreads();
  if (warp == 0) {
    u128 x = lane < nw ? red[lane] : ident(OPA), y = lane < nw ? red[33 + lane] : ident(OPB);
    x = wred(x, OPA);
    y = wred(y, OPB);
    if (lane == 0) {
      red[32] = x;
      red[65] = y;
    }
  }
  __syncthreads();
  a = red[32];
  b = red[65];
}

// ---- thread groups ----------------------------------------------------------
// A block of values is processed by a group of G threads:
//   G = 32        one warp (several blocks per CTA);
//   G = 64, 128   a sub-group of a 256-thread CTA: the CTA holds 256/G groups, group
//                 g synchronises on its own named barrier 8 + g;
//   G = 256       the whole CTA (any blockDim.x).
// These helpers give the rank in the group, synchronise it and reduce over it.
template <int G>
struct GroupOf {
  static constexpr bool warp = G == 32;
  static constexpr bool sub = G == 64 || G == 128;
};
template <int G>
__device__ __forceinline__ uint32_t group_rank() {
  return GroupOf<G>::warp ? (threadIdx.x & 31) : GroupOf<G>::sub ? (threadIdx.x & (G - 1)) : threadIdx.x;
}
template <int G>
__device__ __forceinline__ uint32_t group_size() { return (GroupOf<G>::warp || GroupOf<G>::sub) ? (uint32_t)G : blockDim.x; }
// Index of this thread's group inside the CTA (0 for a whole-CTA group).
template <int G>
__device__ __forceinline__ uint32_t group_index() {
  return GroupOf<G>::warp ? (threadIdx.x >> 5) : GroupOf<G>::sub ? (threadIdx.x / G) : 0u;
}
template <int G>
__device__ __forceinline__ void group_sync() {
  if (GroupOf<G>::warp) __syncwarp();
  else if (GroupOf<G>::sub) asm volatile("bar.sync %0, %1;" ::"r"(8u + threadIdx.x / G), "n"(G) : "memory");
  else __syncthreads();
}
template <int OP>
__device__ __forceinline__ u128 warp_reduce_op(u128 x) {
  switch (OP) {
    case 0: return warp_sum_u128(x);
    case 1: return warp_max_u64((uint64_t)x);
    case 2: return warp_min_u64((uint64_t)x);
    case 3: return (u128)(uint64_t)warp_max_i64((int64_t)(uint64_t)x);
    case 4: return (u128)(uint64_t)warp_min_i64((int64_t)(uint64_t)x);
    default: return warp_sum_u64((uint64_t)x);
  }
}
template <int OP>
__device__ __forceinline__ u128 reduce_identity() {
  return OP == 2 ? (u128)~0ull : OP == 3 ? (u128)0x8000000000000000ull : OP == 4 ? (u128)0x7fffffffffffffffull : (u128)0;
}
// Two reductions over `nw` (<= 32) warps: `warp` is this warp's index among them,
// SYNC synchronises exactly those warps.  `red` as block_reduce2 (66 entries).
template <int OPA, int OPB, typename Sync>
__device__ __forceinline__ void warps_reduce2(u128 &a, u128 &b, u128 *red, int warp, int nw, Sync sync) {
  const int lane = threadIdx.x & 31;
  a = warp_reduce_op<OPA>(a);
  b = warp_reduce_op<OPB>(b);
  sync();  // `red` may still be read by a previous reduction
  if (lane == 0) {
    red[warp] = a;
    red[33 + warp] = b;
  }
  sync();
  if (warp == 0) {
    u128 x = lane < nw ? red[lane] : reduce_identity<OPA>(), y = lane < nw ? red[33 + lane] : reduce_identity<OPB>();
    x = warp_reduce_op<OPA>(x);
    y = warp_reduce_op<OPB>(y);
    if (lane == 0) {
      red[32] = x;
      red[65] = y;
    }
  }
  sync();
  a = red[32];
  b = red[65];
}
template <int OP, int G>
__device__ __forceinline__ u128 group_reduce(u128 v, u128 *red) {
  if (GroupOf<G>::warp) return warp_reduce_op<OP>(v);
  if (GroupOf<G>::sub) {
    u128 none = 0;
    warps_reduce2<OP, 5>(v, none, red, (int)(group_rank<G>() >> 5), G / 32, [] { group_sync<G>(); });
    return v;
  }
  return block_reduce<OP>(v, red);
}

template <int OPA, int OPB, int G>
__device__ __forceinline__ void group_reduce2(u128 &a, u128 &b, u128 *red) {
  if (GroupOf<G>::warp) {
    a = warp_reduce_op<OPA>(a);
    b = warp_reduce_op<OPB>(b);
  } else if (GroupOf<G>::sub) {
    warps_reduce2<OPA, OPB>(a, b, red, (int)(group_rank<G>() >> 5), G / 32, [] { group_sync<G>(); });
  } else {
    block_reduce2<OPA, OPB>(a, b, red);
  }
}

// Reductions over warps 1.. of a CTA while warp 0 runs something else (the
// encoder's look-back): named barrier 1 over blockDim.x - 32 threads, which all
// of warps 1.. must reach.  `red` as block_reduce2 (66 entries).  OP as
// block_reduce.
__device__ __forceinline__ void sub_sync() { asm volatile("bar.sync 1, %0;" ::"r"(blockDim.x - 32) : "memory"); }
template <int OPA, int OPB>
__device__ __forceinline__ void sub_reduce2(u128 &a, u128 &b, u128 *red) {
  warps_reduce2<OPA, OPB>(a, b, red, (int)(threadIdx.x >> 5) - 1, (int)(blockDim.x >> 5) - 1, [] { sub_sync(); });
}
// The same over warps 1.. of a group of G threads (warp 0 of the group runs the
// look-back): a whole CTA uses named barrier 1, a sub-group g barrier 12 + g.
template <int G>
__device__ __forceinline__ void group_sub_sync() {
  if (GroupOf<G>::sub) asm volatile("bar.sync %0, %1;" ::"r"(12u + threadIdx.x / G), "n"(G - 32) : "memory");
  else sub_sync();
}
template <int OPA, int OPB, int G>
__device__ __forceinline__ void group_sub_reduce2(u128 &a, u128 &b, u128 *red) {
  if (GroupOf<G>::sub)
    warps_reduce2<OPA, OPB>(a, b, red, (int)(group_rank<G>() >> 5) - 1, G / 32 - 1, [] { group_sub_sync<G>(); });
  else
    sub_reduce2<OPA, OPB>(a, b, red);
}

// ---- relaxed global word access for the look-back scan ----------------------
__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(uint64_t *p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// ---- L2 eviction priorities for random access ---------------------------------
// A batch of lookups streams its indices in and its results out once, while every
// lookup also reads its block's 32-byte directory entry (a small, hot table).  The
// streams are marked evict-first and the directory evict-last, so the streams do not
// push the directory out of L2 and each lookup pays DRAM only for its payload sector.
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t ld_nc_hint(const uint64_t *p, uint64_t pol) {
  uint64_t v;
  asm("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ ulonglong2 ld_nc_hint_v2(const void *p, uint64_t pol) {
  ulonglong2 v;
  asm("ld.global.nc.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;" : "=l"(v.x), "=l"(v.y) : "l"(p), "l"(pol));
  return v;
}
template <typename T>
__device__ __forceinline__ void st_hint(T *p, T v, uint64_t pol) {
  if constexpr (sizeof(T) == 8)
    asm volatile("st.global.L2::cache_hint.b64 [%0], %1, %2;" ::"l"(p), "l"((uint64_t)v), "l"(pol) : "memory");
  else
    asm volatile("st.global.L2::cache_hint.b32 [%0], %1, %2;" ::"l"(p), "r"((uint32_t)v), "l"(pol) : "memory");
}

}  // namespace leco

namespace leco {
// Normal-equation solve of polynomial_regression_iter for degree 2
// (polynomial_regression_internals.hpp:121-171): B[i][j] = X[i+j], B[i][3] = Y[i];
// row swaps when B[i][i] < B[k][i]; Gaussian elimination; back substitution
// against zero-initialised coefficients.  Same operation order, each step rounded.
__host__ __device__ inline void poly2_solve(const double *X, const double *Y, double *a) {
  double B[3][4];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) B[i][j] = X[i + j];
    B[i][3] = Y[i];
  }
  for (int i = 0; i < 3; ++i)
    for (int k = i + 1; k < 3; ++k)
      if (B[i][i] < B[k][i])
        for (int j = 0; j < 4; ++j) {
          double t = B[i][j];
          B[i][j] = B[k][j];
          B[k][j] = t;
        }
  for (int i = 0; i < 2; ++i)
    for (int k = i + 1; k < 3; ++k) {
#ifdef __CUDA_ARCH__
      double t = __ddiv_rn(B[k][i], B[i][i]);
      for (int j = 0; j < 4; ++j) B[k][j] = __dsub_rn(B[k][j], __dmul_rn(t, B[i][j]));
#else
      double t = B[k][i] / B[i][i];
      for (int j = 0; j < 4; ++j) B[k][j] -= t * B[i][j];
#endif
    }
  a[0] = a[1] = a[2] = 0.0;
  for (int i = 2; i >= 0; --i) {
    a[i] = B[i][3];
    for (int j = 0; j < 3; ++j)
      if (j != i) {
#ifdef __CUDA_ARCH__
        a[i] = __dsub_rn(a[i], __dmul_rn(B[i][j], a[j]));
#else
        a[i] -= B[i][j] * a[j];
#endif
      }
#ifdef __CUDA_ARCH__
    a[i] = __ddiv_rn(a[i], B[i][i]);
#else
    a[i] /= B[i][i];
#endif
  }
}
}  // namespace leco
