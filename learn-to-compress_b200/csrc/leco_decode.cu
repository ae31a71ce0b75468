// leco_decode.cu -- bulk decode, range decode, compressed-domain sum, random
// access and directory build for the LeCo fixed-block codecs.
//
// Bulk decode replaces <Codec>::decodeArray8 per block:
//   Leco_int     piecewise_fix_integer_template.h:142-204 + read_all_bit_fix (bit_read.h:222-275)
//   FOR_int      FOR_integer_template.h:83-112 + read_all_bit_FOR (bit_read.h:1373-1414)
//   Delta_int    delta_integer_template.h:89-127 + read_all_bit_Delta (bit_read.h:1319-1370)
//   Leco_int_poly poly_fix_integer_template.h:93-158 + read_all_bit_fix_poly (bit_read.h:277-330)
// Random access replaces randomdecodeArray8 (piecewise_fix_integer_template.h:305-337,
// FOR_integer_template.h:218-245, delta_integer_template.h:132-154,
// poly_fix_integer_template.h:259-291).
//
// A block is raw iff l == 8*sizeof(T) everywhere (the reference's random-access
// rule).  The reference's bulk decoders also call l == 8*sizeof(T)-1 raw, which
// mis-decodes such packed blocks; this decoder reads them correctly.
#include "leco_device.cuh"
#include "leco_internal.h"

#include <cstdlib>

namespace leco {

// Block model parsed from a header (or a directory entry).
struct BlockHdr {
  uint64_t body_bit;  // absolute bit address of field 0 (raw: of value 0)
  uint32_t l;         // field width; 8*S = raw; 126/127 = 2/1-value sentinels
  double a0, a1, a2;  // model
  uint64_t base;      // FOR minimum / Delta first value
};

template <int CODEC, int S>
__device__ __forceinline__ BlockHdr parse_header(const uint8_t *__restrict__ payload, uint64_t off) {
  const uint64_t *words = reinterpret_cast<const uint64_t *>(payload);
  BlockHdr h;
  uint64_t w0 = load_u64_at(words, off);
  h.l = (uint32_t)(w0 & 0xff);
  h.a0 = h.a1 = h.a2 = 0;
  h.base = 0;
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
__device__ __forceinline__ BlockHdr from_dir(const leco_dir_entry *__restrict__ dir, uint64_t b, uint64_t pol = 0) {
  const ulonglong2 *p = reinterpret_cast<const ulonglong2 *>(dir + b);
  ulonglong2 q0, q1;
  if (pol) {
    q0 = ldg_v2_hint(p, pol);
    q1 = ldg_v2_hint(p + 1, pol);
  } else {
    q0 = __ldg(p);
    q1 = __ldg(p + 1);
  }
  BlockHdr h;
  h.body_bit = q0.x & ((1ull << 48) - 1);
  h.l = (uint32_t)(q0.x >> 56);
  h.a0 = __longlong_as_double((long long)q0.y);
  h.a1 = __longlong_as_double((long long)q1.x);
  h.a2 = __longlong_as_double((long long)q1.y);
  h.base = S == 8 ? q0.y : (q0.y & 0xffffffffull);
  return h;
}

// Value k of a non-raw, non-Delta block given its field f (bulk decode rules).
template <int CODEC, int S>
__device__ __forceinline__ uint64_t value_from_field(const BlockHdr &h, uint32_t k, uint64_t f) {
  if (CODEC == kFor) return h.base + f;
  int64_t pred;
  if (CODEC == kLinear) pred = f2i_x86(pred_linear(h.a0, h.a1, k));
  else pred = f2i_x86(pred_poly2(h.a0, h.a1, h.a2, __uint2double_rn(k)));
  return h.l ? apply_signed((uint64_t)pred, f, h.l) : (uint64_t)pred;
}

// Delta running sum split over the CTA: each thread owns a contiguous chunk
// [k0, k1) of values; a block-wide exclusive scan of the chunks' delta sums
// gives each thread the value at k0.  Must be called by all threads.
struct DeltaChunk {
  uint32_t k0, k1;
  uint64_t run;  // decoded value k0 (mod 2^64)
};
__device__ __forceinline__ DeltaChunk delta_chunk_start(const uint64_t *__restrict__ words, const BlockHdr &h, uint32_t len) {
  __shared__ uint64_t wsum[32];
  const uint32_t nt = blockDim.x, tid = threadIdx.x;
  const uint32_t chunk = (len + nt - 1) / nt;
  DeltaChunk c;
  c.k0 = min(len, tid * chunk);
  c.k1 = min(len, c.k0 + chunk);
  uint64_t local = 0;  // fields k0 .. k1-1 feed values k0+1 .. k1; field len-1 is not a delta
  if (h.l)
    for (uint32_t k = c.k0; k < c.k1 && k + 1 < len; ++k)
      local += apply_signed(0, load_field(words, h.body_bit + (uint64_t)k * h.l, h.l), h.l);
  const int lane = tid & 31, warp = tid >> 5;
  uint64_t incl = local;
  for (int d = 1; d < 32; d <<= 1) {
    uint64_t y = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const int nw = (nt + 31) >> 5;
    uint64_t x = lane < nw ? wsum[lane] : 0, xi = x;
    for (int d = 1; d < 32; d <<= 1) {
      uint64_t y = __shfl_up_sync(0xffffffffu, xi, d);
      if (lane >= d) xi += y;
    }
    if (lane < nw) wsum[lane] = xi - x;
  }
  __syncthreads();
  c.run = h.base + wsum[warp] + (incl - local);
  return c;
}

template <typename T>
__device__ __forceinline__ void store_vals(T *out, uint64_t o0, const uint64_t *v, int cnt, bool full);
template <>
__device__ __forceinline__ void store_vals<uint64_t>(uint64_t *out, uint64_t o0, const uint64_t *v, int, bool full) {
  if (full) __stcs(reinterpret_cast<ulonglong2 *>(out + o0), make_ulonglong2(v[0], v[1]));
}
template <>
__device__ __forceinline__ void store_vals<uint32_t>(uint32_t *out, uint64_t o0, const uint64_t *v, int, bool full) {
  if (full) __stcs(reinterpret_cast<uint4 *>(out + o0), make_uint4((uint32_t)v[0], (uint32_t)v[1], (uint32_t)v[2], (uint32_t)v[3]));
}


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
// step and writes them with one 16-byte store.
template <typename T, int CODEC, bool FAST, bool SMEM = false>
__device__ __forceinline__ void decode_narrow(const BlockHdr &h, bool raw, const uint32_t *__restrict__ words32, T *out,
                                              uint64_t obase, uint32_t lo, uint32_t hi, int32_t kstart) {
  constexpr int S = sizeof(T);
  constexpr int VEC = 16 / S;
  const uint32_t l = raw ? 32u : h.l;
  // words32 + body_bit/32: the body's first word (global payload or a staged copy in shared memory)
  const uint32_t *bp = words32 + (h.body_bit >> 5);
  const uint32_t bsh = (uint32_t)(h.body_bit & 31);
  const uint32_t mask = l >= 32 ? 0xffffffffu : ((1u << l) - 1u);
  const uint32_t sb = l ? l - 1 : 0, m1 = mask >> 1;
  for (int32_t kv = kstart + (int32_t)threadIdx.x * VEC; kv < (int32_t)hi; kv += (int32_t)blockDim.x * VEC) {
    uint64_t v[VEC];
#pragma unroll
    for (int j = 0; j < VEC; ++j) {
      const int32_t k = kv + j;
      const uint32_t kk = k < (int32_t)lo ? lo : (uint32_t)k;  // values before lo are not stored
      const uint32_t r = bsh + kk * l;
      const uint32_t *p = bp + (r >> 5);
      const uint32_t w0 = SMEM ? p[0] : __ldg(p), w1 = SMEM ? p[1] : __ldg(p + 1);
      const uint32_t f = l ? (__funnelshift_r(w0, w1, r) & mask) : 0u;
      if (raw) {
        v[j] = f;
      } else if (CODEC == kFor) {
        v[j] = h.base + f;
      } else {
        const double pd = CODEC == kLinear ? pred_linear(h.a0, h.a1, kk)
                                           : pred_poly2(h.a0, h.a1, h.a2, __uint2double_rn(kk));
        const int64_t pred = FAST ? __double2ll_rz(pd) : f2i_x86(pd);
        const uint32_t mag = f & m1;
        const int64_t d = ((f >> sb) & 1u) ? (int64_t)mag : -(int64_t)mag;
        v[j] = (uint64_t)(pred + d);
      }
    }
    const bool full = kv >= (int32_t)lo && kv + VEC <= (int32_t)hi;
    store_vals<T>(out, obase + kv, v, VEC, full);
    if (!full) {
#pragma unroll
      for (int j = 0; j < VEC; ++j)
        if (kv + j >= (int32_t)lo && kv + j < (int32_t)hi) out[obase + kv + j] = (T)v[j];
    }
  }
}

// ---- bulk / range decode ----------------------------------------------------
// One CTA per block.  Each thread decodes VEC = 16/sizeof(T) consecutive values
// per step from a three-word window of the packed body and writes them with one
// 16-byte store.
template <typename T, int CODEC>
__device__ __forceinline__ void decode_block(const DecodeLaunch &a, uint64_t b) {
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
  const BlockHdr h = parse_header<CODEC, S>(a.payload, __ldg(a.offsets + b));
  const uint64_t obase = base - a.first;  // out index of block value 0

  if (h.l == 126 || h.l == 127) {  // sentinel blocks (…_integer_template.h:152-170)
    if (CODEC == kFor) { if (threadIdx.x == 0) atomicOr(a.error, kErrBadHeader); return; }
    if (threadIdx.x == 0) {
      const uint32_t cnt = h.l == 127 ? 1 : 2;
      for (uint32_t k = lo; k < cnt && k < hi; ++k)
        out[obase + k] = (T)load_field(words, h.body_bit + (uint64_t)k * TB, TB);
    }
    return;
  }
  if (h.l > TB) {
    if (threadIdx.x == 0) atomicOr(a.error, kErrBadHeader);
    return;
  }
  const bool raw = h.l == TB;

  if (CODEC == kDelta && !raw) {
    // Running sum: value k = x0 + sum_{i<k} signed(field_i) (mod 2^(8S)).
    const DeltaChunk c = delta_chunk_start(words, h, len);
    uint64_t run = c.run;
    for (uint32_t k = c.k0; k < c.k1; ++k) {
      if (k >= lo && k < hi) out[obase + k] = (T)run;
      if (h.l && k + 1 < len) run += apply_signed(0, load_field(words, h.body_bit + (uint64_t)k * h.l, h.l), h.l);
    }
    return;
  }

  // First vector start so that out[obase + kv] is 16-byte aligned (out must be
  // sizeof(T)-aligned); kv may start up to VEC-1 values before lo.
  const uintptr_t oaddr = reinterpret_cast<uintptr_t>(out + obase + lo);
  const int32_t kstart = (int32_t)lo - (int32_t)((oaddr & 15) / S);
  const uint32_t l = raw ? TB : h.l;
  if (l <= 32) {
    // Narrow fields (every u32 block, u64 blocks with l <= 32): 32-bit field
    // extraction; predictions converted without range checks when the block's
    // model keeps every prediction inside int64 (decided once per block).
    const bool fast = (CODEC == kFor) || pred_in_range<CODEC>(h, len);
    const uint32_t *w32 = reinterpret_cast<const uint32_t *>(a.payload);
    if (fast) decode_narrow<T, CODEC, true>(h, raw, w32, out, obase, lo, hi, kstart);
    else decode_narrow<T, CODEC, false>(h, raw, w32, out, obase, lo, hi, kstart);
    return;
  }
  for (int32_t kv = kstart + (int32_t)threadIdx.x * VEC; kv < (int32_t)hi; kv += (int32_t)blockDim.x * VEC) {
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
    store_vals<T>(out, obase + kv, v, VEC, full);
    if (!full) {
#pragma unroll
      for (int j = 0; j < VEC; ++j)
        if (kv + j >= (int32_t)lo && kv + j < (int32_t)hi) out[obase + kv + j] = (T)v[j];
    }
  }
}

// Direct decode: one CTA per block of the range, everything read from global memory.
template <typename T, int CODEC>
__global__ void __launch_bounds__(256) decode_kernel(DecodeLaunch a) {
  decode_block<T, CODEC>(a, a.first / a.bs + blockIdx.x);
}

// ---- TMA-staged persistent decode --------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t tx) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(tx) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bulk (non-tensor) TMA copy global -> this CTA's shared memory, completion
// counted on `bar`.  dst/src 16-byte aligned, bytes a multiple of 16.  No
// multicast: the source is always this GPU's own payload.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// Bounded wait on a staging barrier (about a second at most).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  for (uint32_t spins = 0; spins < (1u << 24); ++spins)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

struct StageMeta {
  uint64_t gbase;   // 16-byte aligned global byte address of the staged copy
  uint32_t hoff;    // block header offset inside the staged copy
  uint32_t direct;  // 1: block too large for the buffer, decode from global
};

// Persistent decode of a whole column.  Each CTA walks blocks blockIdx.x,
// blockIdx.x + gridDim.x, ...; thread 0 stages the next block's image (header +
// packed body) into the other half of a double buffer with one cp.async.bulk
// while the CTA decodes the current one out of shared memory.  Blocks that do
// not fit the buffer, wide (l > 32) and Delta blocks take the direct path.
template <typename T, int CODEC>
__global__ void __launch_bounds__(256) decode_staged_kernel(DecodeLaunch a, uint32_t bufcap) {
  constexpr int S = sizeof(T);
  extern __shared__ __align__(128) uint8_t stage[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ StageMeta meta[2];
  const uint32_t tid = threadIdx.x;
  const uint64_t nblk = (a.n + a.bs - 1) / a.bs;
  uint8_t *buf0 = stage, *buf1 = stage + bufcap;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  auto issue = [&](uint64_t b, int which) {  // thread 0 only
    const uint64_t o0 = __ldg(a.offsets + b), o1 = __ldg(a.offsets + b + 1);
    const uint64_t g0 = o0 & ~15ull, g1 = (o1 + 8 + 15) & ~15ull;  // +8: the field reads touch one word past the body
    const uint64_t bytes = g1 - g0;
    StageMeta m;
    m.gbase = g0;
    m.hoff = (uint32_t)(o0 - g0);
    m.direct = bytes > bufcap;
    meta[which] = m;
    if (!m.direct) {
      mbar_arrive_tx(&bar[which], (uint32_t)bytes);
      bulk_g2s(which ? buf1 : buf0, a.payload + g0, (uint32_t)bytes, &bar[which]);
    } else {
      mbar_arrive(&bar[which]);
    }
  };
  uint64_t blk = blockIdx.x;
  if (tid == 0 && blk < nblk) issue(blk, 0);
  uint32_t ph0 = 0, ph1 = 0;
  T *out = reinterpret_cast<T *>(a.out);
  for (int it = 0; blk < nblk; blk += gridDim.x, ++it) {
    const int cur = it & 1;
    const bool has_next = blk + gridDim.x < nblk;
    if (tid == 0 && has_next) issue(blk + gridDim.x, cur ^ 1);
    const bool ok = mbar_wait_bounded(&bar[cur], cur ? ph1 : ph0);
    if (cur) ph1 ^= 1; else ph0 ^= 1;
    if (!ok) {
      if (tid == 0) {
        atomicOr(a.error, kErrTimeout);
        if (has_next) mbar_wait_bounded(&bar[cur ^ 1], cur ? ph0 : ph1);  // let our own copy in flight land
      }
      return;
    }
    const StageMeta m = meta[cur];
    const uint8_t *sb = (cur ? buf1 : buf0);
    const uint32_t l = sb[m.hoff];
    const uint64_t base = blk * a.bs;
    const uint32_t len = (uint32_t)umin64(a.bs, a.n - base);
    const bool raw = l == 8u * S;
    const bool narrow = (CODEC != kDelta) && (l <= 32) && (!raw || S == 4);
    if (m.direct || !narrow) {
      decode_block<T, CODEC>(a, blk);
    } else {
      BlockHdr h;
      h.l = l;
      h.a0 = h.a1 = h.a2 = 0;
      h.base = 0;
      const uint8_t *hb = sb + m.hoff + 1;
      if (!raw) {
        uint64_t w[3] = {0, 0, 0};
        const int nw = CODEC == kPoly2 ? 3 : (CODEC == kLinear ? 2 : 1);
#pragma unroll
        for (int q = 0; q < 3; ++q)
          if (q < nw)
#pragma unroll
            for (int j = 0; j < 8; ++j) w[q] |= (uint64_t)hb[8 * q + j] << (8 * j);
        if (CODEC == kLinear || CODEC == kPoly2) {
          h.a0 = __longlong_as_double((long long)w[0]);
          h.a1 = __longlong_as_double((long long)w[1]);
          h.a2 = __longlong_as_double((long long)w[2]);
        } else {
          h.base = S == 8 ? w[0] : (w[0] & 0xffffffffull);
        }
      }
      h.body_bit = (uint64_t)(m.hoff + (raw ? 1u : Hdr<CODEC, S>::bytes)) * 8;
      const uint32_t *w32 = reinterpret_cast<const uint32_t *>(sb);
      const uintptr_t oaddr = reinterpret_cast<uintptr_t>(out + base);
      const int32_t kstart = -(int32_t)((oaddr & 15) / S);
      const bool fast = (CODEC == kFor) || raw || pred_in_range<CODEC>(h, len);
      if (fast) decode_narrow<T, CODEC, true, true>(h, raw, w32, out, base, 0, len, kstart);
      else decode_narrow<T, CODEC, false, true>(h, raw, w32, out, base, 0, len, kstart);
    }
    __syncthreads();  // everyone is done with this buffer before it is refilled
  }
}

// ---- compressed-domain sum ----------------------------------------------------
// Sum of decoded values mod 2^64 without writing them: reads only the payload.
template <typename T, int CODEC>
__global__ void __launch_bounds__(256) sum_kernel(DecodeLaunch a, uint64_t *d_sum) {
  constexpr int S = sizeof(T);
  constexpr uint32_t TB = 8u * S;
  __shared__ u128 red[33];
  const uint64_t b = blockIdx.x;
  const uint64_t base = b * a.bs;
  const uint32_t len = (uint32_t)umin64((uint64_t)a.bs, a.n - base);
  const uint64_t *words = reinterpret_cast<const uint64_t *>(a.payload);
  const BlockHdr h = parse_header<CODEC, S>(a.payload, __ldg(a.offsets + b));
  const uint64_t tmask = S == 8 ? ~0ull : 0xffffffffull;
  uint64_t acc = 0;
  if (h.l == 126 || h.l == 127 || h.l > TB) {
    if (threadIdx.x == 0) atomicOr(a.error, kErrBadHeader);
    return;
  }
  const bool raw = h.l == TB;
  if (CODEC == kDelta && !raw) {
    const DeltaChunk c = delta_chunk_start(words, h, len);
    uint64_t run = c.run;
    for (uint32_t k = c.k0; k < c.k1; ++k) {
      acc += run & tmask;
      if (h.l && k + 1 < len) run += apply_signed(0, load_field(words, h.body_bit + (uint64_t)k * h.l, h.l), h.l);
    }
  } else {
    const uint32_t l = raw ? TB : h.l;
    for (uint32_t k = threadIdx.x; k < len; k += blockDim.x) {
      uint64_t f = l ? load_field(words, h.body_bit + (uint64_t)k * l, l) : 0;
      acc += (raw ? f : value_from_field<CODEC, S>(h, k, f)) & tmask;
    }
  }
  acc = (uint64_t)block_reduce<5>((u128)acc, red);
  if (threadIdx.x == 0) atomicAdd(reinterpret_cast<unsigned long long *>(d_sum), (unsigned long long)acc);
}

// ---- random access --------------------------------------------------------------
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
  const double p = CODEC == kLinear ? pred_linear(h.a0, h.a1, k) : pred_poly2(h.a0, h.a1, h.a2, __uint2double_rn(k));
  if (h.l) return apply_signed((uint64_t)f2i_x86(p), f, h.l);
  return f2T_x86<S>(p);  // l == 0: (T)prediction directly (piecewise_fix_integer_template.h:334, poly :288)
}

// Batched random access: each thread keeps U lookups in flight (indices,
// directory entries and payload words are each loaded for all U before any is
// used), lookups i, i+G, i+2G, ... of one thread are strided by the grid so
// index loads and output stores stay coalesced across a warp.
template <typename T, int CODEC>
__global__ void __launch_bounds__(256) gather_kernel(GatherLaunch a) {
  constexpr int S = sizeof(T);
  constexpr uint32_t TB = 8u * S;
  constexpr int U = 4;
  const uint64_t *words = reinterpret_cast<const uint64_t *>(a.payload);
  T *out = reinterpret_cast<T *>(a.out);
  const uint64_t G = (uint64_t)gridDim.x * blockDim.x;
  const bool small = a.n <= 0xffffffffull;
  for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < a.m; i0 += G * U) {
    uint64_t g[U], b[U];
    uint32_t k[U];
    bool live[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint64_t i = i0 + (uint64_t)u * G;
      live[u] = i < a.m;
      g[u] = live[u] ? __ldg(a.idx + i) : 0;
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
      h[u] = a.dir ? from_dir<CODEC, S>(a.dir, b[u]) : parse_header<CODEC, S>(a.payload, __ldg(a.offsets + b[u]));
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
      out[i0 + (uint64_t)u * G] = (T)ra_value<CODEC, S>(h[u], k[u], f, a.error);
    }
  }
}

// Delta random access: prefix walk over fields 0..k-1 (bit_read.h:1292-1317).
template <typename T>
__global__ void __launch_bounds__(256) gather_delta_kernel(GatherLaunch a) {
  constexpr int S = sizeof(T);
  constexpr uint32_t TB = 8u * S;
  const uint64_t *words = reinterpret_cast<const uint64_t *>(a.payload);
  T *out = reinterpret_cast<T *>(a.out);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.m; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t g = __ldg(a.idx + i);
    if (g >= a.n) {
      out[i] = 0;
      atomicOr(a.error, kErrBadIndex);
      continue;
    }
    const uint64_t b = g / a.bs;
    const uint32_t k = (uint32_t)(g - b * a.bs);
    const BlockHdr h = a.dir ? from_dir<kDelta, S>(a.dir, b) : parse_header<kDelta, S>(a.payload, __ldg(a.offsets + b));
    uint64_t v;
    if (h.l == TB) {
      v = load_field(words, h.body_bit + (uint64_t)k * TB, TB);
    } else if (h.l > TB) {
      v = 0;
      atomicOr(a.error, kErrBadHeader);
    } else {
      v = h.base;
      if (h.l)
        for (uint32_t j = 0; j < k; ++j) v += apply_signed(0, load_field(words, h.body_bit + (uint64_t)j * h.l, h.l), h.l);
    }
    out[i] = (T)v;
  }
}

// ---- directory ---------------------------------------------------------------------
template <typename T, int CODEC>
__global__ void build_dir_kernel(const uint8_t *payload, const uint64_t *offsets, uint64_t nb, leco_dir_entry *dir) {
  constexpr int S = sizeof(T);
  const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const BlockHdr h = parse_header<CODEC, S>(payload, __ldg(offsets + b));
  leco_dir_entry e;
  e.word0 = h.body_bit | ((uint64_t)h.l << 56) | ((uint64_t)CODEC << 48);
  if (CODEC == kLinear || CODEC == kPoly2) {
    e.a0 = h.a0; e.a1 = h.a1; e.a2 = h.a2;
  } else {
    e.a0 = __longlong_as_double((long long)h.base); e.a1 = 0; e.a2 = 0;
  }
  dir[b] = e;
}

// ---- launchers ------------------------------------------------------------------------

// LECO_DECODE_STAGED=0 selects the direct (one CTA per block) decode kernel.
static bool staged_decode_enabled() {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("LECO_DECODE_STAGED");
    v = (e && e[0] == '0') ? 0 : 1;
  }
  return v == 1;
}

#define LECO_DISPATCH(codec, s, FN, ...)                                   \
  do {                                                                     \
    if ((s) == 4) {                                                        \
      switch (codec) {                                                     \
        case kLinear: FN<uint32_t, kLinear>(__VA_ARGS__); return 0;         \
        case kFor: FN<uint32_t, kFor>(__VA_ARGS__); return 0;               \
        case kDelta: FN<uint32_t, kDelta>(__VA_ARGS__); return 0;           \
        case kPoly2: FN<uint32_t, kPoly2>(__VA_ARGS__); return 0;           \
      }                                                                    \
    } else {                                                               \
      switch (codec) {                                                     \
        case kLinear: FN<uint64_t, kLinear>(__VA_ARGS__); return 0;         \
        case kFor: FN<uint64_t, kFor>(__VA_ARGS__); return 0;               \
        case kDelta: FN<uint64_t, kDelta>(__VA_ARGS__); return 0;           \
        case kPoly2: FN<uint64_t, kPoly2>(__VA_ARGS__); return 0;           \
      }                                                                    \
    }                                                                      \
    return -1;                                                             \
  } while (0)

// Staging buffer per half: enough for 4096-value blocks with fields of up to
// 31 bits (u64) -- larger images are decoded straight from global memory.
constexpr uint32_t kStageBuf = 16640;

template <typename T, int CODEC>
static void run_decode(const DecodeLaunch &L, cudaStream_t st) {
  if (!L.count) return;
  const uint64_t b0 = L.first / L.bs, b1 = (L.first + L.count - 1) / L.bs;
  const uint64_t nblk = b1 - b0 + 1;
  const bool staged = L.first == 0 && L.count == L.n && (reinterpret_cast<uintptr_t>(L.payload) & 15) == 0 &&
                      CODEC != kDelta && nblk >= 1024 && staged_decode_enabled();
  if (!staged) {
    decode_kernel<T, CODEC><<<(unsigned)nblk, 256, 0, st>>>(L);
    return;
  }
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int smem = 2 * kStageBuf + 64;  // +64: field reads may run a few bytes past a full buffer
  cudaFuncSetAttribute(decode_staged_kernel<T, CODEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, decode_staged_kernel<T, CODEC>, 256, smem);
  const uint64_t grid = umin64(nblk, (uint64_t)sms * (uint64_t)(per_sm > 0 ? per_sm : 1));
  decode_staged_kernel<T, CODEC><<<(unsigned)grid, 256, smem, st>>>(L, kStageBuf);
}
int launch_decode(int codec, int s, const DecodeLaunch &L, cudaStream_t st) { LECO_DISPATCH(codec, s, run_decode, L, st); }

template <typename T, int CODEC>
static void run_sum(const DecodeLaunch &L, uint64_t *d_sum, cudaStream_t st) {
  const uint64_t nb = (L.n + L.bs - 1) / L.bs;
  if (nb) sum_kernel<T, CODEC><<<(unsigned)nb, 256, 0, st>>>(L, d_sum);
}
int launch_sum(int codec, int s, const DecodeLaunch &L, uint64_t *d_sum, cudaStream_t st) {
  LECO_DISPATCH(codec, s, run_sum, L, d_sum, st);
}

template <typename T, int CODEC>
static void run_gather(const GatherLaunch &L, cudaStream_t st) {
  if (!L.m) return;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (CODEC == kDelta) {
    const unsigned grid = (unsigned)umin64((L.m + 255) / 256, (uint64_t)sms * 16);
    gather_delta_kernel<T><<<grid, 256, 0, st>>>(L);
    return;
  }
  const uint64_t need = (L.m + 4 * 256 - 1) / (4 * 256);  // 4 lookups in flight per thread
  const unsigned grid = (unsigned)umin64(need, (uint64_t)sms * 8);
  gather_kernel<T, CODEC><<<grid, 256, 0, st>>>(L);
}
int launch_gather(int codec, int s, const GatherLaunch &L, cudaStream_t st) { LECO_DISPATCH(codec, s, run_gather, L, st); }

template <typename T, int CODEC>
static void run_dir(const uint8_t *payload, const uint64_t *offsets, uint64_t nb, leco_dir_entry *dir, cudaStream_t st) {
  if (nb) build_dir_kernel<T, CODEC><<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(payload, offsets, nb, dir);
}
int launch_build_dir(int codec, int s, const uint8_t *payload, const uint64_t *offsets, uint64_t n, uint32_t bs,
                     leco_dir_entry *dir, uint32_t *error, cudaStream_t st) {
  (void)error;
  const uint64_t nb = (n + bs - 1) / bs;
  LECO_DISPATCH(codec, s, run_dir, payload, offsets, nb, dir, st);
}

}  // namespace leco
