// leco_encode.cuh -- per-block encoder shared by the single-column kernels
// (leco_encode.cu) and the persistent multi-column batch kernels (leco_batch.cu).
//
// Reference: Leco_int<T>::encodeArray8_int (piecewise_fix_integer_template.h:27-140),
// FOR_int<T>::encodeArray8_int (FOR_integer_template.h:26-81),
// Delta_int<T>::encodeArray8_int (delta_integer_template.h:26-87),
// Leco_int_poly<T,2>::encodeArray8_int (poly_fix_integer_template.h:28-91),
// packers write_delta_int_T / write_FOR_int_T (bit_write.h:257-390).
#pragma once
#include <type_traits>

#include "leco_device.cuh"
#include "leco_internal.h"

namespace leco {

constexpr uint64_t kFlagAgg = 1ull << 62, kFlagIncl = 2ull << 62, kValMask = (1ull << 62) - 1;
constexpr uint32_t kSpinLimit = 1u << 22;  // x ~32-256 ns backoff: far above any real wait

// Per-block model scratch: the sequential reference fit writes 3 doubles per block.
struct EncodeArgs {
  const void *values;
  uint64_t n;
  uint32_t bs;
  uint64_t nb;
  uint8_t *payload;
  uint64_t payload_cap;
  uint64_t *offsets;
  leco_dir_entry *dir;
  const double *seq_models;  // [nb*3] or null (exact fit in-kernel)
  double polyX[10];          // X sums for full blocks [0..4] and for the tail block [5..9]
  uint64_t *status;          // [nb] look-back words, zeroed
  uint32_t *ticket;          // zeroed
  uint32_t *error;           // error word
  uint32_t rows_area;        // 1: the group's shared memory holds enc_rows_bytes(bs) more bytes after the
                             // values, where u32 LeCo / degree-2 residual rows are packed
};

// Shared-memory layout helper.
template <typename T>
struct EncSmem {
  T *vals;          // [bs] values, later residual magnitudes (linear / poly2)
  uint32_t *signs;  // [bs/32 + 9] sign bits (one word per 32 values, rounded up to 256)
  u128 *red;        // [66]
  uint8_t *hdr;     // [32] header bytes
  uint64_t *bcast;  // [8]
};

template <typename T>
__device__ __forceinline__ EncSmem<T> enc_smem(uint8_t *base, uint32_t bs) {
  EncSmem<T> s;
  s.red = reinterpret_cast<u128 *>(base);                      // 66 * 16 = 1056
  s.bcast = reinterpret_cast<uint64_t *>(base + 1056);         // 8 * 8 = 64
  s.hdr = base + 1120;                                         // 32
  s.signs = reinterpret_cast<uint32_t *>(base + 1152);         // (bs/32+9)*4
  uint32_t soff = 1152 + ((bs / 32 + 9) * 4 + 15) / 16 * 16;
  s.vals = reinterpret_cast<T *>(base + soff);
  return s;
}
// The value region holds round32(bs) values plus 16 bytes: the u64 LeCo path keeps
// round32(bs) staged words and a packed body of up to round32(bs) + 4 words there.
__host__ __device__ inline uint32_t enc_smem_bytes(uint32_t bs, uint32_t s) {
  return 1152 + ((bs / 32 + 9) * 4 + 15) / 16 * 16 + (bs + 31) / 32 * 32 * s + 16;
}
// The packed-rows area of the u32 LeCo / degree-2 encoder: a packed body of at most
// round32(bs) words plus the four zero words after it.
__host__ __device__ inline uint32_t enc_rows_bytes(uint32_t bs) { return (bs + 31) / 32 * 32 * 4 + 16; }

// Decoupled look-back (single-pass prefix sum over per-block totals), run by one
// full warp.  lookback_excl walks back over the predecessors of block b 32 at a
// time (lane i reads block j - i): it needs every block from the nearest one down
// to the first with an inclusive prefix, and waits only while one of those has
// published nothing.  It needs nothing of block b itself, so it can run while the
// block is still being encoded.  Returns the exclusive prefix; on a wait that
// exceeds the spin limit sets kErrTimeout and returns ~0.  lookback_prefix
// publishes block b's total first and its inclusive prefix last.
__device__ __forceinline__ uint64_t lookback_excl(const uint64_t *status, uint64_t b, uint32_t *error,
                                                  uint32_t spin_limit = kSpinLimit) {
  const int lane = threadIdx.x & 31;
  if (b == 0) return 0;
  uint64_t excl = 0;
  int64_t j = (int64_t)b - 1;
  for (;;) {
    const int64_t idx = j - lane;
    uint64_t v = kFlagIncl;  // lanes before block 0 read as "inclusive 0"
    uint32_t spins = 0, ns = 32;
    uint32_t incl;
    int last;  // the farthest lane this window of predecessors needs
    for (;;) {
      if (idx >= 0) v = ld_relaxed(&status[idx]);
      incl = __ballot_sync(0xffffffffu, (v >> 62) == 2);
      last = incl ? __ffs(incl) - 1 : 31;
      const uint32_t need = last == 31 ? 0xffffffffu : ((2u << last) - 1u);
      if (!(__ballot_sync(0xffffffffu, (v >> 62) == 0) & need)) break;
      if (++spins > spin_limit) {
        if (lane == 0) atomicOr(error, kErrTimeout);
        return ~0ull;
      }
      __nanosleep(ns);
      if (ns < 256) ns <<= 1;
    }
    excl += warp_sum_u64(lane <= last ? (v & kValMask) : 0);
    if (incl) break;
    j -= 32;
  }
  return excl;
}
__device__ __forceinline__ uint64_t lookback_prefix(uint64_t *status, uint64_t b, uint64_t my, uint32_t *error,
                                                    uint32_t spin_limit = kSpinLimit) {
  const int lane = threadIdx.x & 31;
  if (b > 0 && lane == 0) st_relaxed(&status[b], kFlagAgg | my);
  const uint64_t excl = lookback_excl(status, b, error, spin_limit);
  if (excl != ~0ull && lane == 0) st_relaxed(&status[b], kFlagIncl | (excl + my));
  return excl;
}

// Prefix publisher, one warp.  A block's own look-back ends at the nearest inclusive
// prefix, but those lag: a block publishes its inclusive prefix only when its own
// look-back is done, so with ~900 blocks in flight each look-back sums long runs of
// totals.  This warp walks the status words in block order (128 per step, lane i
// holding blocks j + 4i .. j + 4i + 3) and turns every published total into an
// inclusive prefix as soon as it and all blocks before it have published, so the blocks
// find one among their nearest predecessors.  Every value it writes is the one the
// block's own look-back would publish.  Block 0's inclusive prefix must be published
// (by this warp) before the call.  Returns after block nb - 1, or sets kErrTimeout on a
// wait that exceeds the spin limit.
__device__ __forceinline__ void publish_prefixes(uint64_t *status, uint64_t nb, uint32_t *error,
                                                 uint32_t spin_limit = kSpinLimit) {
  constexpr int K = 4;
  const int lane = threadIdx.x & 31;
  __syncwarp();
  uint64_t run = ld_relaxed(&status[0]) & kValMask;  // inclusive prefix before block j
  uint64_t j = 1;
  uint32_t spins = 0, ns = 32;
  while (j < nb) {
    uint64_t v[K];
    int first = K * 32;  // this lane's first unpublished position
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const uint64_t idx = j + K * lane + k;
      v[k] = idx < nb ? ld_relaxed(&status[idx]) : 0;
    }
#pragma unroll
    for (int k = K - 1; k >= 0; --k)
      if ((v[k] >> 62) == 0) first = K * lane + k;
    const int n = __reduce_min_sync(0xffffffffu, first);  // published run j .. j + n - 1
    if (n == 0) {
      if (++spins > spin_limit) {
        if (lane == 0) atomicOr(error, kErrTimeout);
        return;
      }
      __nanosleep(ns);
      if (ns < 256) ns <<= 1;
      continue;
    }
    spins = 0;
    ns = 32;
    // Segmented inclusive scan: an inclusive prefix restarts the sum.  Lane-local first...
    uint64_t p[K];
    bool f[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const uint64_t val = v[k] & kValMask;
      const bool fl = (v[k] >> 62) == 2;
      p[k] = (k == 0 || fl) ? val : p[k - 1] + val;
      f[k] = fl || (k > 0 && f[k - 1]);
    }
    // ... then over the lanes' totals
    uint64_t tp = p[K - 1];
    int tf = f[K - 1];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint64_t q = __shfl_up_sync(0xffffffffu, tp, d);
      const int fq = __shfl_up_sync(0xffffffffu, tf, d);
      if (lane >= d && !tf) {
        tp += q;
        tf = fq;
      }
    }
    uint64_t ep = __shfl_up_sync(0xffffffffu, tp, 1);
    int ef = __shfl_up_sync(0xffffffffu, tf, 1);
    if (lane == 0) {
      ep = 0;
      ef = 0;
    }
    if (!ef) ep += run;
    uint64_t last = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const uint64_t fin = f[k] ? p[k] : ep + p[k];
      const int pos = K * lane + k;
      if (pos < n && (v[k] >> 62) == 1) st_relaxed(&status[j + pos], kFlagIncl | fin);
      if (pos == n - 1) last = fin;
    }
    run = __shfl_sync(0xffffffffu, last, (n - 1) / K);
    j += n;
  }
}

// True when every prediction of a len-value block with model (a0, a1, a2) is a
// finite double inside (-2^62, 2^62): the x86 out-of-range rule cannot apply.
__device__ __forceinline__ bool model_in_range(double a0, double a1, double a2, uint32_t len) {
  const double L = __uint2double_rn(len ? len - 1 : 0);
  return fabs(a0) + fabs(a1) * L + fabs(a2) * L * L < 4611686018427387904.0;
}

// Image writer: writes image bytes [0, size) of a block to payload[goff...].
// Image byte i < H is hdr[i]; byte i >= H is byte (i-H) of the LSB-first
// concatenation of fields 0..n-1 (l bits each), zero past the last field.
template <typename FieldFn>
__device__ __forceinline__ uint64_t gather_bits(uint32_t p, uint32_t nbits, uint32_t l, uint32_t n, FieldFn field) {
  uint32_t k = p / l, o = p - k * l;
  u128 acc = k < n ? (u128)(field(k) >> o) : (u128)0;
  uint32_t have = l - o;
  ++k;
  while (have < nbits) {
    if (k < n) acc |= (u128)field(k) << have;
    have += l;
    ++k;
  }
  return (uint64_t)acc & lowmask(nbits);
}

// 128 bits of the body starting at body bit p, for fields of at most 32 bits:
// 32-bit output words assembled in a 64-bit accumulator; k0 = p / l through a
// reciprocal (exact for p < 2^21 and l <= 64).
template <typename FieldFn>
__device__ __forceinline__ uint4 gather128_narrow(uint32_t p, uint32_t l, uint32_t rcp, uint32_t n, FieldFn field) {
  uint32_t k = l == 1 ? p : __umulhi(p, rcp);
  const uint32_t o = p - k * l;
  uint64_t acc = k < n ? ((uint64_t)field(k) >> o) : 0;
  uint32_t have = l - o;
  ++k;
  uint32_t w[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    while (have < 32) {
      if (k < n) acc |= (uint64_t)field(k) << have;
      have += l;
      ++k;
    }
    w[q] = (uint32_t)acc;
    acc >>= 32;
    have -= 32;
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

template <typename FieldFn>
__device__ __forceinline__ void write_image(uint8_t *payload, uint64_t goff, uint64_t size, uint32_t H,
                                            const uint8_t *hdr, uint32_t l, uint32_t nfields, FieldFn field,
                                            uint32_t rank, uint32_t nthreads) {
  const uint64_t gend = goff + size;
  const uint64_t c0 = goff >> 4, c1 = (gend + 15) >> 4;
  const uint64_t body0 = goff + H;  // first body byte (global)
  const uint32_t rcp = l > 1 ? (uint32_t)((0x100000000ull + l - 1) / l) : 0;  // ceil(2^32 / l); l == 1 divides trivially
  for (uint64_t c = c0 + rank; c < c1; c += nthreads) {
    const uint64_t cb = c << 4;
    if (cb >= body0 && cb + 16 <= gend && l) {
      uint32_t p = (uint32_t)((cb - body0) * 8);
      if (l <= 32) {
        *reinterpret_cast<uint4 *>(payload + cb) = gather128_narrow(p, l, rcp, nfields, field);
      } else {
        uint64_t lo = gather_bits(p, 64, l, nfields, field);
        uint64_t hi = gather_bits(p + 64, 64, l, nfields, field);
        *reinterpret_cast<ulonglong2 *>(payload + cb) = make_ulonglong2(lo, hi);
      }
    } else {
      for (int j = 0; j < 16; ++j) {
        uint64_t g = cb + j;
        if (g < goff || g >= gend) continue;
        uint64_t i = g - goff;
        uint8_t byte;
        if (i < H) byte = hdr[i];
        else if (!l) byte = 0;
        else byte = (uint8_t)gather_bits((uint32_t)((i - H) * 8), 8, l, nfields, field);
        payload[g] = byte;
      }
    }
  }
}

// ---- u64 LeCo blocks: residual rows packed in shared memory ------------------------
// Residual i of a row of 32 is kept at column (i ^ row) of its row, so that a warp
// over 32 consecutive residuals and a warp over 32 rows (one residual each) both
// touch 32 distinct banks.
__device__ __forceinline__ uint32_t swz32(uint32_t i) { return i ^ ((i >> 5) & 31u); }

// Packs rows t0, t0 + step, ... of 32 fields each (magnitude res[k] below the sign
// bit l-1, sign bit k of signs[row]) into l 32-bit words per row: row t is body
// words [t*l, t*l + l), the LSB-first field stream of write_delta_int_T
// (bit_write.h:257-323).  Four zero words follow the last row (the image's pad).
__device__ __forceinline__ void pack_rows(const uint32_t *res, const uint32_t *signs, uint32_t *pk, uint32_t len,
                                          uint32_t l, uint32_t t0, uint32_t step) {
  const uint32_t rows = (len + 31) / 32;
  const uint32_t sb = l - 1;
  for (uint32_t t = t0; t < rows; t += step) {
    const uint32_t sg = signs[t], x = t & 31u;
    uint32_t *out = pk + t * l;
    uint64_t acc = 0;
    uint32_t have = 0, q = 0;
#pragma unroll
    for (uint32_t j = 0; j < 32; ++j) {
      const uint32_t f = t * 32 + j < len ? (res[t * 32 + (j ^ x)] | (((sg >> j) & 1u) << sb)) : 0u;
      acc |= (uint64_t)f << have;
      have += l;
      if (have >= 32) {
        out[q++] = (uint32_t)acc;
        acc >>= 32;
        have -= 32;
      }
    }
  }
  if (t0 == 0)
    for (uint32_t j = 0; j < 4; ++j) pk[rows * l + j] = 0;
}

// Writes the image [goff, goff + size) whose body is packed in shared memory
// (pk, at least size - H + 4 bytes readable): 16-byte chunks inside the body by
// funnel shifts, the chunks shared with the header or a neighbouring block byte
// by byte.
__device__ __forceinline__ void write_image_packed(uint8_t *payload, uint64_t goff, uint64_t size, uint32_t H,
                                                   const uint8_t *hdr, const uint32_t *pk, uint32_t rank,
                                                   uint32_t nthreads) {
  const uint64_t gend = goff + size;
  const uint64_t c0 = goff >> 4, c1 = (gend + 15) >> 4;
  const uint64_t body0 = goff + H;
  const uint8_t *pk8 = reinterpret_cast<const uint8_t *>(pk);
  for (uint64_t c = c0 + rank; c < c1; c += nthreads) {
    const uint64_t cb = c << 4;
    if (cb >= body0 && cb + 16 <= gend) {
      const uint32_t q = (uint32_t)(cb - body0), qw = q >> 2, sh = (q & 3u) * 8u;
      const uint32_t w0 = pk[qw], w1 = pk[qw + 1], w2 = pk[qw + 2], w3 = pk[qw + 3], w4 = pk[qw + 4];
      *reinterpret_cast<uint4 *>(payload + cb) = make_uint4(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh),
                                                            __funnelshift_r(w2, w3, sh), __funnelshift_r(w3, w4, sh));
    } else {
      for (int j = 0; j < 16; ++j) {
        const uint64_t g = cb + j;
        if (g < goff || g >= gend) continue;
        const uint64_t i = g - goff;
        payload[g] = i < H ? hdr[i] : pk8[i - H];
      }
    }
  }
}

// (int64_t)(m0 + m1*i) under conversion rule R: 0 = every prediction of the block
// lies in [0, 2^51), both conversions on the FP64 pipe (exact); 1 = in range, plain
// truncation; 2 = the x86 out-of-range rule (f2i_x86).
template <int R>
__device__ __forceinline__ int64_t lin_pred(double m0, double m1, uint32_t i) {
  if (R == 0) return trunc_nonneg_fp64(pred_linear_fp64(m0, m1, i));
  const double p = pred_linear(m0, m1, i);
  return R == 1 ? __double2ll_rz(p) : f2i_x86(p);
}
// Calls fn(std::integral_constant<int, R>) with the cheapest rule valid for the
// block's len predictions, so the loops inside fn carry no per-value test.
template <typename Fn>
__device__ __forceinline__ void with_pred_rule(double m0, double m1, uint32_t len, Fn fn) {
  if (preds_nonneg(m0, m1, len)) fn(std::integral_constant<int, 0>{});
  else if (model_in_range(m0, m1, 0.0, len)) fn(std::integral_constant<int, 1>{});
  else fn(std::integral_constant<int, 2>{});
}

// ---- u64 LeCo blocks, 32-bit path: values staged whole, rows packed in place ---------
// The block's values are copied into shared memory as 16-byte pairs (values 2q, 2q+1)
// with cp.async, every copy of a thread in flight at once.  Rows of 32 values are 256
// bytes; pair j of row t sits in 16-byte slot j ^ (t mod 16) of the row, so that a warp
// over 32 consecutive pairs (two rows) and a warp over 32 rows (the same pair of each)
// both spread over the banks.  The residual pass writes the pair's two signed 32-bit
// residuals over the first 8 bytes of its slot; the packer then turns row t, which
// only its own thread reads, into L words written from word t mod 32 of the row on.
__device__ __forceinline__ uint32_t pair16_slot(uint32_t q) { return q ^ ((q >> 4) & 15u); }

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint4 lds_v4(uint32_t a) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
  return v;
}
__device__ __forceinline__ uint2 lds_v2(uint32_t a) {
  uint2 v;
  asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ void sts_v2(uint32_t a, uint32_t x, uint32_t y) {
  asm volatile("st.shared.v2.u32 [%0], {%1, %2};" ::"r"(a), "r"(x), "r"(y));
}
__device__ __forceinline__ void sts_u32(uint32_t a, uint32_t v) { asm volatile("st.shared.u32 [%0], %1;" ::"r"(a), "r"(v)); }
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Max, min and bitwise or of int32 values over the encoding warps (warps 1.. of the
// group; warp 0 runs the look-back).  `slots`: 96 ints of shared memory that no thread
// still reads (the two reductions of one block use different slots).
template <int G>
__device__ __forceinline__ void enc_reduce3(int32_t &mx, int32_t &mn, uint32_t &ov, int32_t *slots) {
  mx = __reduce_max_sync(0xffffffffu, mx);
  mn = __reduce_min_sync(0xffffffffu, mn);
  ov = __reduce_or_sync(0xffffffffu, ov);
  const uint32_t nw = group_size<G>() / 32 - 1;
  if (nw == 1) {
    __syncwarp();  // orders the warp's shared-memory writes before the next phase
    return;
  }
  const uint32_t w = (group_rank<G>() >> 5) - 1;
  if ((threadIdx.x & 31) == 0) {
    slots[w] = mx;
    slots[32 + w] = mn;
    slots[64 + w] = (int32_t)ov;
  }
  group_sub_sync<G>();
  for (uint32_t k = 0; k < nw; ++k) {
    mx = max(mx, slots[k]);
    mn = min(mn, slots[32 + k]);
    ov |= (uint32_t)slots[64 + k];
  }
}

// Field of signed residual r (|r| < 2^(L-1)): the magnitude with the sign bit
// (r > 0, "data[i] > pred") at bit L-1 (write_delta_int_T, bit_write.h:257-323).
template <int L>
__device__ __forceinline__ uint32_t lin_field(uint32_t r) {
  return (int32_t)r > 0 ? (r | (1u << (L - 1))) : (uint32_t)(-(int32_t)r);
}
// Adds field f of row position j (bits [j*L, j*L + L) of the row's bit stream) to the
// row's words; fields are disjoint and come in increasing j, so adding is or-ing.
template <int L>
__device__ __forceinline__ void place_field(uint32_t (&w)[L], uint32_t f, int j) {
  const int p = j * L, q = p >> 5, s = p & 31;
  w[q] += f << s;
  if (s + L > 32) w[q + 1] += f >> (32 - s);
}
// Packs rows t0, t0 + step, ... < rows (32 signed residuals each, zeros past the
// block's end) into L words, written over row t from word t mod 32 on (bank t + k for
// word k).  Every shift is a compile-time constant.
template <int L>
__device__ __forceinline__ void pack_rows_width(uint32_t vb, uint32_t rows, uint32_t t0, uint32_t step) {
  for (uint32_t t = t0; t < rows; t += step) {
    const uint32_t x = t & 15u, row = vb + t * 256u;
    uint32_t w[L];
#pragma unroll
    for (int k = 0; k < L; ++k) w[k] = 0;
#pragma unroll
    for (int jj = 0; jj < 16; ++jj) {
      const uint2 v = lds_v2(row + (((uint32_t)jj ^ x) << 4));
      place_field<L>(w, lin_field<L>(v.x), 2 * jj);
      place_field<L>(w, lin_field<L>(v.y), 2 * jj + 1);
    }
    const uint32_t o = row + (t & 31u) * 4u;
#pragma unroll
    for (int k = 0; k < L; ++k) sts_u32(o + 4u * k, w[k]);
  }
}
// One call per block and thread: the width is uniform over the block.
static __device__ __noinline__ void pack_rows_dispatch(uint32_t l, uint32_t vb, uint32_t rows, uint32_t t0, uint32_t step) {
  switch (l) {
#define LECO_PACK_CASE(L) \
  case L: pack_rows_width<L>(vb, rows, t0, step); break;
    LECO_PACK_CASE(1) LECO_PACK_CASE(2) LECO_PACK_CASE(3) LECO_PACK_CASE(4) LECO_PACK_CASE(5) LECO_PACK_CASE(6)
    LECO_PACK_CASE(7) LECO_PACK_CASE(8) LECO_PACK_CASE(9) LECO_PACK_CASE(10) LECO_PACK_CASE(11) LECO_PACK_CASE(12)
    LECO_PACK_CASE(13) LECO_PACK_CASE(14) LECO_PACK_CASE(15) LECO_PACK_CASE(16) LECO_PACK_CASE(17)
    LECO_PACK_CASE(18) LECO_PACK_CASE(19) LECO_PACK_CASE(20) LECO_PACK_CASE(21) LECO_PACK_CASE(22)
    LECO_PACK_CASE(23) LECO_PACK_CASE(24) LECO_PACK_CASE(25) LECO_PACK_CASE(26) LECO_PACK_CASE(27)
    LECO_PACK_CASE(28) LECO_PACK_CASE(29) LECO_PACK_CASE(30) LECO_PACK_CASE(31) LECO_PACK_CASE(32)
#undef LECO_PACK_CASE
    default: break;
  }
}

// Stores bytes [lo, hi) of the 16-byte chunk (w0..w3, little-endian) at dst (16-byte
// aligned) with the fewest aligned stores: the chunk's other bytes belong to the
// neighbouring block's image, written by another CTA.
__device__ __forceinline__ void store_chunk_bytes(uint8_t *dst, uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3,
                                                  uint32_t lo, uint32_t hi) {
  for (uint32_t pos = lo; pos < hi;) {
    const uint32_t rem = hi - pos, wi = pos >> 2, sh = (pos & 3u) * 8u;
    const uint32_t w = wi == 0 ? w0 : wi == 1 ? w1 : wi == 2 ? w2 : w3;
    if ((pos & 7u) == 0 && rem >= 8) {
      const uint32_t wn = wi == 0 ? w1 : w3;
      *reinterpret_cast<uint64_t *>(dst + pos) = ((uint64_t)wn << 32) | w;
      pos += 8;
    } else if ((pos & 3u) == 0 && rem >= 4) {
      *reinterpret_cast<uint32_t *>(dst + pos) = w;
      pos += 4;
    } else if ((pos & 1u) == 0 && rem >= 2) {
      *reinterpret_cast<uint16_t *>(dst + pos) = (uint16_t)(w >> sh);
      pos += 2;
    } else {
      dst[pos] = (uint8_t)(w >> sh);
      pos += 1;
    }
  }
}

// Writes the image [goff, goff + size) of a non-raw LeCo block (17-byte header in hdr,
// 4-byte aligned, bytes 17.. zero) whose body rows were packed by pack_rows_dispatch:
// body word k is word k mod L of row t = k / L, at v32[t*64 + t mod 32 + k mod L]; words
// past the last row read as zero (the image's zero tail).  k / L is a multiply-high by
// ceil(2^32 / L), exact for k < 2^16 (a block body has at most 16384 words).  16-byte
// chunks inside the body are funnel-shifted from body words; the chunks holding the
// header or shared with a neighbouring image from image words (header words, then body
// words shifted by the header's 17 bytes), stored byte-exactly.
__device__ __forceinline__ void write_image_rows(uint8_t *payload, uint64_t goff, uint64_t size, const uint8_t *hdr,
                                                 const uint32_t *v32, uint32_t L, uint32_t rows, uint32_t rank,
                                                 uint32_t nthreads) {
  constexpr uint32_t H = 17;
  const uint32_t M = L > 1 ? 0xffffffffu / L + 1u : 0u, nw = rows * L;
  auto word = [&](uint32_t k) -> uint32_t {
    const uint32_t t = L > 1 ? __umulhi(k, M) : k;
    return k < nw ? v32[t * 64u + (t & 31u) + (k - t * L)] : 0u;
  };
  const uint32_t *hw = reinterpret_cast<const uint32_t *>(hdr);
  // image word m: image bytes 4m .. 4m+3 (m < 0: before the image, never stored)
  auto img = [&](int32_t m) -> uint32_t {
    if (m < 0) return 0u;
    if (m < 4) return hw[m];
    if (m == 4) return (hw[4] & 0xffu) | (word(0) << 8);
    return __funnelshift_r(word((uint32_t)m - 5u), word((uint32_t)m - 4u), 24);
  };
  const uint64_t gend = goff + size;
  const uint64_t c0 = goff >> 4, c1 = (gend + 15) >> 4;
  const uint64_t body0 = goff + H;
  for (uint64_t c = c0 + rank; c < c1; c += nthreads) {
    const uint64_t cb = c << 4;
    if (cb >= body0 && cb + 16 <= gend) {
      const uint32_t q = (uint32_t)(cb - body0), qw = q >> 2, sh = (q & 3u) * 8u;
      const uint32_t w0 = word(qw), w1 = word(qw + 1), w2 = word(qw + 2), w3 = word(qw + 3), w4 = word(qw + 4);
      *reinterpret_cast<uint4 *>(payload + cb) = make_uint4(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh),
                                                            __funnelshift_r(w2, w3, sh), __funnelshift_r(w3, w4, sh));
    } else {
      const int32_t e = (int32_t)((int64_t)cb - (int64_t)goff);  // image offset of the chunk (>= -15)
      const int32_t m0 = e >> 2;                                 // floor(e / 4)
      const uint32_t sh = (uint32_t)(e & 3) * 8u;
      const uint32_t i0 = img(m0), i1 = img(m0 + 1), i2 = img(m0 + 2), i3 = img(m0 + 3), i4 = img(m0 + 4);
      const uint32_t lo = cb < goff ? (uint32_t)(goff - cb) : 0u;
      const uint32_t hi = cb + 16 > gend ? (uint32_t)(gend - cb) : 16u;
      if (lo == 0 && hi == 16) {
        *reinterpret_cast<uint4 *>(payload + cb) = make_uint4(__funnelshift_r(i0, i1, sh), __funnelshift_r(i1, i2, sh),
                                                              __funnelshift_r(i2, i3, sh), __funnelshift_r(i3, i4, sh));
      } else {
        store_chunk_bytes(payload + cb, __funnelshift_r(i0, i1, sh), __funnelshift_r(i1, i2, sh),
                          __funnelshift_r(i2, i3, sh), __funnelshift_r(i3, i4, sh), lo, hi);
      }
    }
  }
}

// Leco_int<uint64_t>::encodeArray8_int (piecewise_fix_integer_template.h:27-140)
// for one block with a whole CTA, the same image as the generic encode_block:
//  * warp 0 takes the block's exclusive byte offset by look-back from the start,
//    while warps 1.. encode (the offset needs nothing of the block itself); the
//    block's total is published as soon as it is known, its inclusive prefix
//    once both are;
//  * the low 32 bits of each value are staged (row-swizzled) while the values
//    stream in, and the midpoint pass (:36-46) runs on those same loads;
//  * blocks whose residuals before the shift span < 2^30 and whose predictions lie
//    in [0, 2^51) take their residuals in 32 bits from the staged words (every
//    residual after the shift is below 2^31 in magnitude), overwrite them, and
//    pack rows of 32 into the body in shared memory;
//  * other blocks (wide residuals, negative predictions, raw) recompute their
//    residuals from the values in global memory, which are then L2-resident.
// Needs a group of >= 64 threads (G = 64, 128 or the whole CTA).  Unroll depth U:
// 2U 16-byte loads in flight per thread in the midpoint pass (U in the exact-fit
// moment pass).  Shared memory: enc_smem_bytes(bs, 8) -- staged words and packed
// body take the place of the generic encoder's staged values.
template <int G, int U = 2>
__device__ __forceinline__ void encode_block_l64(const EncodeArgs &a, uint64_t b, uint8_t *smem_raw) {
  constexpr uint32_t TB = 64;
  constexpr int UR = 2 * U, UE = U;
  EncSmem<uint64_t> sm = enc_smem<uint64_t>(smem_raw, a.bs);
  uint32_t *lo = reinterpret_cast<uint32_t *>(sm.vals);  // [round32(bs)] low words, then residuals
  uint32_t *pk = lo + ((a.bs + 31u) & ~31u);              // packed body words
  const uint32_t tid = group_rank<G>(), nt = group_size<G>();
  const uint64_t base = b * a.bs;
  const uint32_t len = (uint32_t)umin64((uint64_t)a.bs, a.n - base);
  const uint64_t *src = reinterpret_cast<const uint64_t *>(a.values) + base;
  double *model = reinterpret_cast<double *>(&sm.bcast[4]);  // m0, m1 for warp 0

  if (tid < 32) {
    // ---- offset by look-back, alongside the encoding ------------------------------
    const uint64_t excl = lookback_excl(a.status, b, a.error);
    if (tid == 0) sm.bcast[1] = excl;
  } else {
    const uint32_t ct = tid - 32, cn = nt - 32;  // encoding threads
    // ---- fit and midpoint shift -----------------------------------------------------
    double m0, m1;
    auto mid_pass = [&](bool stage) -> bool {  // true: residuals before the shift span < 2^30
      int64_t dmax = (int64_t)0x8000000000000000ull, dmin = 0x7fffffffffffffffll;
      // One loop per conversion rule, chosen once per block: predictions in [0, 2^51)
      // take both conversions on the FP64 pipe (exact); other in-range predictions
      // the plain truncation; the rest the x86 out-of-range rule.
      with_pred_rule(m0, m1, len, [&](auto rule) {
        auto visit = [&](uint64_t y, uint32_t i) {
          if (stage) lo[swz32(i)] = (uint32_t)y;
          const int64_t pr = lin_pred<decltype(rule)::value>(m0, m1, i);
          const int64_t d = (int64_t)(y - (uint64_t)pr);
          dmax = d > dmax ? d : dmax;
          dmin = d < dmin ? d : dmin;
        };
        if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {  // 16-byte loads, 2U in flight per thread
          const uint32_t np = len / 2;
#pragma unroll (UR)
          for (uint32_t q = ct; q < np; q += cn) {
            const uint4 v = __ldg(reinterpret_cast<const uint4 *>(src) + q);
            visit(((uint64_t)v.y << 32) | v.x, 2 * q);
            visit(((uint64_t)v.w << 32) | v.z, 2 * q + 1);
          }
          if ((len & 1) && ct == 0) visit(__ldg(src + len - 1), len - 1);
        } else {
          for (uint32_t i = ct; i < len; i += cn) visit(__ldg(src + i), i);
        }
      });
      u128 rmx = (u128)(uint64_t)dmax, rmn = (u128)(uint64_t)dmin;
      group_sub_reduce2<3, 4, G>(rmx, rmn, sm.red);
      dmax = (int64_t)(uint64_t)rmx;
      dmin = (int64_t)(uint64_t)rmn;
      const int64_t mid = (int64_t)((uint64_t)dmax + (uint64_t)dmin);
      m0 = __dadd_rn(m0, __dmul_rn(__ll2double_rn(mid), 0.5));  // x * 0.5 rounds exactly as x / 2.0
      return dmax >= dmin && (uint64_t)(dmax - dmin) < (1ull << 30);
    };
    // ---- 32-bit path (16-byte aligned blocks whose predictions lie in [0, 2^51)) -----
    const uint32_t vb = smem_u32(sm.vals), np = len >> 1;
    // The block's values into their pair slots, every copy of this thread in flight.
    auto stage_pairs = [&]() {
      for (uint32_t q = ct; q < np; q += cn) cp_async16(vb + 16u * pair16_slot(q), src + 2 * q);
      if ((len & 1) && ct == 0) cp_async8(vb + 16u * pair16_slot(np), src + len - 1);
      cp_async_wait_all();
      group_sub_sync<G>();
    };
    // Midpoint pass over the staged values: every d = y - pred is taken in 64 bits but
    // its max and min in 32 bits, with a check that each d fits in an int32 (its high
    // word is the sign extension of its low word).  Returns false (model untouched)
    // when some d does not fit; the 64-bit pass then runs instead.
    int32_t *slots = reinterpret_cast<int32_t *>(sm.red);  // two sets of 96 ints
    bool narrow_range = false;
    auto mid_pass32 = [&]() -> bool {
      int32_t mx = INT32_MIN, mn = INT32_MAX;
      uint32_t bad = 0;
      auto visit = [&](uint64_t y, uint32_t i) {
        const double p = pred_linear_fp64(m0, m1, i);
        // y - trunc(p): the magic-number sum holds 2^52 + trunc(p) (its bits minus 0x433 << 52)
        const uint64_t d = y - (uint64_t)__double_as_longlong(__dadd_rz(p, 4503599627370496.0)) + 0x4330000000000000ull;
        const uint32_t dl = (uint32_t)d;
        bad |= (uint32_t)(d >> 32) ^ (uint32_t)((int32_t)dl >> 31);
        mx = max(mx, (int32_t)dl);
        mn = min(mn, (int32_t)dl);
      };
#pragma unroll 2
      for (uint32_t q = ct; q < np; q += cn) {
        const uint4 v = lds_v4(vb + 16u * pair16_slot(q));
        visit(((uint64_t)v.y << 32) | v.x, 2 * q);
        visit(((uint64_t)v.w << 32) | v.z, 2 * q + 1);
      }
      if ((len & 1) && ct == 0) {
        const uint2 v = lds_v2(vb + 16u * pair16_slot(np));
        visit(((uint64_t)v.y << 32) | v.x, len - 1);
      }
      enc_reduce3<G>(mx, mn, bad, slots);
      if (bad) return false;
      const int64_t mid = (int64_t)mx + (int64_t)mn;
      m0 = __dadd_rn(m0, __dmul_rn(__ll2double_rn(mid), 0.5));  // x * 0.5 rounds exactly as x / 2.0
      narrow_range = (int64_t)mx - (int64_t)mn < (1ll << 30);
      return true;
    };
    const bool al16 = (reinterpret_cast<uintptr_t>(src) & 15) == 0;
    bool pairs = false;  // the 32-bit midpoint pass ran over the staged pairs
    if (a.seq_models) {
      // (issuing the copies before the model is read was measured slower: the model's
      // load then queues behind them)
      m0 = a.seq_models[b * 3 + 0];
      m1 = a.seq_models[b * 3 + 1];
      if (al16 && preds_nonneg(m0, m1, len)) {
        stage_pairs();
        pairs = mid_pass32();
      }
      if (!pairs) narrow_range = mid_pass(true);
    } else {
      // Moments in 32-bit halves of y: a thread sees at most 16384 values, each
      // i*y_lo, i*y_hi < 2^46, so the 64-bit partial sums stay below 2^60.
      uint64_t slo = 0, shi = 0, tlo = 0, thi = 0;
      auto visit = [&](uint64_t y, uint32_t i) {
        const uint32_t yl = (uint32_t)y, yh = (uint32_t)(y >> 32);
        slo += yl;
        shi += yh;
        tlo += (uint64_t)yl * i;
        thi += (uint64_t)yh * i;
      };
      if (al16) {
        stage_pairs();
#pragma unroll (UE)
        for (uint32_t q = ct; q < np; q += cn) {
          const uint4 v = lds_v4(vb + 16u * pair16_slot(q));
          visit(((uint64_t)v.y << 32) | v.x, 2 * q);
          visit(((uint64_t)v.w << 32) | v.z, 2 * q + 1);
        }
        if ((len & 1) && ct == 0) {
          const uint2 v = lds_v2(vb + 16u * pair16_slot(np));
          visit(((uint64_t)v.y << 32) | v.x, len - 1);
        }
      } else {
        for (uint32_t i = ct; i < len; i += cn) visit(__ldg(src + i), i);
      }
      u128 sy = ((u128)shi << 32) + slo, siy = ((u128)thi << 32) + tlo;
      group_sub_reduce2<0, 0, G>(sy, siy, sm.red);
      // lr_int_T::caltheta (lr.h:79-83) on exact moments
      const double md = __uint2double_rn(len);
      const uint64_t m = len;
      const double sumx = __ull2double_rn(m * (m - 1) / 2);
      const double sumxx = u128_to_double((u128)(m - 1) * m * (2 * m - 1) / 6);
      const double sumy = u128_to_double(sy), sumxy = u128_to_double(siy);
      const double ccc = __dsub_rn(__dmul_rn(sumxy, md), __dmul_rn(sumx, sumy));
      const double xxx = __dsub_rn(__dmul_rn(sumxx, md), __dmul_rn(sumx, sumx));
      m1 = __ddiv_rn(ccc, xxx);
      m0 = __ddiv_rn(__dsub_rn(sumy, __dmul_rn(m1, sumx)), md);
      pairs = al16 && preds_nonneg(m0, m1, len) && mid_pass32();
      if (!pairs) narrow_range = mid_pass(true);  // stages the low words in the row layout of pack_rows
    }

    // ---- residuals (:51-72) and width (:108-117) -------------------------------------
    const bool narrow = narrow_range && preds_nonneg(m0, m1, len);
    const bool r32 = narrow && !pairs, r32p = narrow && pairs;
    uint32_t l;
    if (r32p) {
      // Signed 32-bit residuals from the staged low words, written over the first 8
      // bytes of each pair slot; the packer takes magnitude and sign from them.  Every
      // slot of the last row past the block's end holds zeros.
      int32_t rmx = 0, rmn = 0;
#pragma unroll 2
      for (uint32_t q = ct; q < np; q += cn) {
        const uint32_t at = vb + 16u * pair16_slot(q);
        const uint4 v = lds_v4(at);
        const int32_t r0 = (int32_t)(v.x - (uint32_t)trunc_nonneg_fp64(pred_linear_fp64(m0, m1, 2 * q)));
        const int32_t r1 = (int32_t)(v.z - (uint32_t)trunc_nonneg_fp64(pred_linear_fp64(m0, m1, 2 * q + 1)));
        rmx = max(rmx, max(r0, r1));
        rmn = min(rmn, min(r0, r1));
        sts_v2(at, (uint32_t)r0, (uint32_t)r1);
      }
      const uint32_t qend = (len + 31u) / 32u * 16u;  // pairs of the rows
      for (uint32_t q = np + ct; q < qend; q += cn) {
        const uint32_t at = vb + 16u * pair16_slot(q);
        int32_t r0 = 0;
        if (2 * q < len) {  // the odd last value
          r0 = (int32_t)(lds_v2(at).x - (uint32_t)trunc_nonneg_fp64(pred_linear_fp64(m0, m1, 2 * q)));
          rmx = max(rmx, r0);
          rmn = min(rmn, r0);
        }
        sts_v2(at, (uint32_t)r0, 0u);
      }
      uint32_t none = 0;
      enc_reduce3<G>(rmx, rmn, none, slots + 96);
      const uint32_t rm = max((uint32_t)rmx, (uint32_t)(-rmn));  // every |r| < 2^31
      l = rm ? bits_of(rm) + 1 : 0;
    } else if (r32) {
      uint32_t rm32 = 0;
      for (uint32_t i0 = 0; i0 < len; i0 += cn) {
        const uint32_t i = i0 + ct;
        bool pos = false;
        if (i < len) {
          const uint32_t s = swz32(i);
          const int64_t pred = trunc_nonneg_fp64(pred_linear_fp64(m0, m1, i));
          const int32_t d = (int32_t)(lo[s] - (uint32_t)pred);
          pos = d > 0;  // y > pred
          const uint32_t r = pos ? (uint32_t)d : (uint32_t)(-d);
          lo[s] = r;
          rm32 = r > rm32 ? r : rm32;
        }
        const uint32_t ballot = __ballot_sync(0xffffffffu, pos);
        if ((ct & 31) == 0) sm.signs[i0 / 32 + ct / 32] = ballot;
      }
      u128 rmax = rm32, none = 0;
      group_sub_reduce2<1, 5, G>(rmax, none, sm.red);
      l = rmax ? bits_of((uint64_t)rmax) + 1 : 0;
    } else {
      const bool fast = model_in_range(m0, m1, 0.0, len);
      uint64_t rm = 0;
      for (uint32_t i = ct; i < len; i += cn) {
        const uint64_t y = __ldg(src + i);
        const double p = pred_linear(m0, m1, i);
        const int64_t pred = fast ? __double2ll_rz(p) : f2i_x86(p);
        const uint64_t r = y > (uint64_t)pred ? y - (uint64_t)pred : (uint64_t)pred - y;
        rm = r > rm ? r : rm;
      }
      u128 rmax = rm, none = 0;
      group_sub_reduce2<1, 5, G>(rmax, none, sm.red);
      l = rmax ? bits_of((uint64_t)rmax) + 1 : 0;
      if (l > TB) l = TB;
    }
    if (l == TB - 1) l = TB;  // written raw, as the generic encoder explains
    const bool raw = l == TB;
    const uint64_t size = block_bytes<kLinear, 8>(l, len);
    if (ct == 0) {
      if (b > 0) st_relaxed(&a.status[b], kFlagAgg | size);  // successors need not wait for our prefix
      sm.bcast[2] = size;
      sm.bcast[3] = l | ((uint64_t)r32 << 8) | ((uint64_t)r32p << 9);
      model[0] = m0;
      model[1] = m1;
      sm.hdr[0] = (uint8_t)l;
      if (!raw) {
        const uint64_t w0 = (uint64_t)__double_as_longlong(m0), w1 = (uint64_t)__double_as_longlong(m1);
        for (int j = 0; j < 8; ++j) {
          sm.hdr[1 + j] = (uint8_t)(w0 >> (8 * j));
          sm.hdr[9 + j] = (uint8_t)(w1 >> (8 * j));
        }
      }
    }
    // residuals (and signs) are complete: the width reductions ended with a barrier
    if (r32 && l > 0) pack_rows(lo, sm.signs, pk, len, l, ct, cn);
    if (r32p && l > 0) pack_rows_dispatch(l, smem_u32(sm.vals), (len + 31) / 32, ct, cn);
  }
  group_sync<G>();

  const uint64_t size = sm.bcast[2], goff = sm.bcast[1];
  const uint32_t l = (uint32_t)(sm.bcast[3] & 0xff);
  const bool r32 = (sm.bcast[3] >> 8) & 1, raw = l == TB, rows = r32 && l > 0;
  const bool rows_p = ((sm.bcast[3] >> 9) & 1) && l > 0;
  const uint32_t H = raw ? 1u : 17u;
  const double m0 = model[0], m1 = model[1];
  if (goff == ~0ull) return;  // look-back gave up (error word set)
  if (tid == 0) st_relaxed(&a.status[b], kFlagIncl | (goff + size));
  if (goff + size + LECO_PAYLOAD_SLACK > a.payload_cap) {  // never write past the buffer
    if (tid == 0) atomicOr(a.error, kErrCapacity);
    return;
  }

  // ---- body ----------------------------------------------------------------------
  if (raw) {
    write_image(a.payload, goff, size, H, sm.hdr, TB, len, [&](uint32_t k) -> uint64_t { return __ldg(src + k); }, tid, nt);
  } else if (rows_p) {
    write_image_rows(a.payload, goff, size, sm.hdr, lo, l, (len + 31) / 32, tid, nt);
  } else if (rows) {
    write_image_packed(a.payload, goff, size, H, sm.hdr, pk, tid, nt);
  } else {
    const bool fast = model_in_range(m0, m1, 0.0, len);
    const uint32_t sb = l ? l - 1 : 0;
    write_image(a.payload, goff, size, H, sm.hdr, l, len, [&](uint32_t k) -> uint64_t {
      const uint64_t y = __ldg(src + k);
      const double p = pred_linear(m0, m1, k);
      const int64_t pred = fast ? __double2ll_rz(p) : f2i_x86(p);
      const bool pos = y > (uint64_t)pred;
      return (pos ? y - (uint64_t)pred : (uint64_t)pred - y) | ((uint64_t)pos << sb);
    }, tid, nt);
  }

  // ---- offsets and directory -------------------------------------------------------
  if (tid == 0) {
    a.offsets[b] = goff;
    if (b == a.nb - 1) a.offsets[a.nb] = goff + size;
    if (a.dir) {
      leco_dir_entry e;
      e.word0 = ((goff + H) * 8) | ((uint64_t)l << 56) | ((uint64_t)kLinear << 48);
      e.a0 = m0; e.a1 = m1; e.a2 = 0.0;
      a.dir[b] = e;
    }
  }
}

// Legacy u32 format, piecewise_fix_op_max::encodeArray8
// (piecewise_fix_op_minimize_maxerror.h:45-95): the slope is rounded to float,
// residuals are ints against (long long)(theta0 + theta1*i), the midpoint shift
// is taken in int arithmetic, and the width is bits(max |r|) + 1 where a
// residual of -2^31 does not count (the reference's abs() leaves it negative).
// On return vals holds |r| (2^31 for -2^31), signs the bits r > 0, m1 the
// float slope as a double; returns the width.
template <int G, typename T>
__device__ __forceinline__ uint32_t legacy_residuals(const EncSmem<T> &sm, double &m0, double &m1, uint32_t len,
                                                     uint32_t tid, uint32_t nt) {
  m1 = (double)__double2float_rn(m1);
  bool fast = model_in_range(m0, m1, 0.0, len);
  auto resid = [&](uint32_t i) -> int32_t {
    const double p = pred_linear(m0, m1, i);
    return (int32_t)((int64_t)(uint64_t)sm.vals[i] - (fast ? __double2ll_rz(p) : f2i_x86(p)));
  };
  int32_t dmax = INT32_MIN, dmin = INT32_MAX;
  for (uint32_t i = tid; i < len; i += nt) {
    const int32_t d = resid(i);
    dmax = d > dmax ? d : dmax;
    dmin = d < dmin ? d : dmin;
  }
  u128 rmx = (u128)(uint64_t)(int64_t)dmax, rmn = (u128)(uint64_t)(int64_t)dmin;
  group_reduce2<3, 4, G>(rmx, rmn, sm.red);
  const int32_t mid = (int32_t)((uint32_t)(uint64_t)rmx + (uint32_t)(uint64_t)rmn);
  m0 = __dadd_rn(m0, __dmul_rn(__int2double_rn(mid), 0.5));  // x * 0.5 rounds exactly as x / 2.0
  fast = model_in_range(m0, m1, 0.0, len);
  uint32_t emax = 0;
  for (uint32_t i0 = 0; i0 < len; i0 += nt) {
    const uint32_t i = i0 + tid;
    bool pos = false;
    if (i < len) {
      const int32_t d = resid(i);
      pos = d > 0;
      const uint32_t mag = d < 0 ? 0u - (uint32_t)d : (uint32_t)d;
      sm.vals[i] = (T)mag;
      if (d != INT32_MIN && mag > emax) emax = mag;
    }
    const uint32_t ballot = __ballot_sync(0xffffffffu, pos);
    if ((tid & 31) == 0) sm.signs[i0 / 32 + tid / 32] = ballot;
  }
  emax = (uint32_t)(uint64_t)group_reduce<1, G>((u128)emax, sm.red);
  return emax ? bits_of(emax) + 1 : 0;
}

// Encodes block b of the column described by `a` with one thread group: the
// whole CTA (G = 256), a sub-group of 64 or 128 threads, or one warp (G = 32).
// U is the unroll depth of the u64 LeCo path (encode_block_l64).  The caller
// guarantees that every block of the column with a smaller index was handed
// to a group that has already started (ticket order), which makes the
// look-back wait finite.  smem_raw: enc_smem_bytes(a.bs, sizeof(T)) bytes
// owned by this group.  (Running the look-back in the group's first warp from
// the block's start, as the u64 LeCo path does, was measured slower here: the
// other codecs' passes take longer with a warp fewer than the look-back saves.)
template <typename T, int CODEC, int G = 256, int U = 2>
__device__ __forceinline__ void encode_block(const EncodeArgs &a, uint64_t b, uint8_t *smem_raw) {
  if constexpr (CODEC == kLinear && sizeof(T) == 8 && G != 32) {
    encode_block_l64<G, U>(a, b, smem_raw);
    return;
  }
  constexpr int S = sizeof(T);
  constexpr uint32_t TB = 8u * S;
  EncSmem<T> sm = enc_smem<T>(smem_raw, a.bs);
  const uint32_t tid = group_rank<G>(), nt = group_size<G>();
  const uint64_t base = b * a.bs;
  const uint32_t len = (uint32_t)umin64((uint64_t)a.bs, a.n - base);
  const T *src = reinterpret_cast<const T *>(a.values) + base;
  // u32 LeCo / degree-2 blocks with a packed-rows area: residuals are kept row-swizzled
  // (residual i of a row of 32 at column i ^ row) and packed by rows of 32 fields with
  // pack_rows, the image then written from the packed words (write_image_packed)
  // instead of gathering each 16-byte chunk field by field.
  constexpr bool kRowsCodec = S == 4 && (CODEC == kLinear || CODEC == kPoly2) && G != 32;
  const bool rows = kRowsCodec && a.rows_area;
  uint32_t *pk = reinterpret_cast<uint32_t *>(sm.vals) + (a.bs + 31) / 32 * 32;

  // ---- stage the block ------------------------------------------------------
  constexpr uint32_t V = 16 / S;
  if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
    const uint32_t nvec = len / V;
    for (uint32_t i = tid; i < nvec; i += nt)
      reinterpret_cast<uint4 *>(sm.vals)[i] = __ldg(reinterpret_cast<const uint4 *>(src) + i);
    for (uint32_t i = nvec * V + tid; i < len; i += nt) sm.vals[i] = __ldg(src + i);
  } else {
    for (uint32_t i = tid; i < len; i += nt) sm.vals[i] = __ldg(src + i);
  }
  group_sync<G>();

  uint32_t l = 0;
  double m0 = 0, m1 = 0, m2 = 0;  // model (theta0/theta1 or poly a0..a2)
  uint64_t fbase = 0;             // FOR min / Delta first value
  uint32_t H = Hdr<CODEC, S>::bytes;

  bool narrow_range = false;  // residuals before the midpoint shift span < 2^30
  if (CODEC == kLinear || CODEC == kPoly2 || CODEC == kLegacy) {
    // ---- fit -----------------------------------------------------------------
    if (a.seq_models) {
      m0 = a.seq_models[b * 3 + 0];
      m1 = a.seq_models[b * 3 + 1];
      m2 = a.seq_models[b * 3 + 2];
    } else {
      u128 sy = 0, siy = 0, sqy = 0;
      for (uint32_t i = tid; i < len; i += nt) {
        uint64_t y = (uint64_t)sm.vals[i];
        sy += y;
        siy += (u128)y * i;
        if (CODEC == kPoly2) sqy += (u128)y * ((uint64_t)i * i);
      }
      group_reduce2<0, 0, G>(sy, siy, sm.red);
      if (CODEC == kPoly2) sqy = group_reduce<0, G>(sqy, sm.red);
      const double md = __uint2double_rn(len);
      if (CODEC == kLinear || CODEC == kLegacy) {
        // lr_int_T::caltheta (lr.h:79-83; lr_int, lr.h:89-111, is the same) on exact moments
        const uint64_t m = len;
        const double sumx = __ull2double_rn(m * (m - 1) / 2);
        const double sumxx = u128_to_double((u128)(m - 1) * m * (2 * m - 1) / 6);
        const double sumy = u128_to_double(sy), sumxy = u128_to_double(siy);
        const double ccc = __dsub_rn(__dmul_rn(sumxy, md), __dmul_rn(sumx, sumy));
        const double xxx = __dsub_rn(__dmul_rn(sumxx, md), __dmul_rn(sumx, sumx));
        m1 = __ddiv_rn(ccc, xxx);
        m0 = __ddiv_rn(__dsub_rn(sumy, __dmul_rn(m1, sumx)), md);
      } else {
        const double *X = a.polyX + (len == a.bs ? 0 : 5);
        double Y[3] = {u128_to_double(sy), u128_to_double(siy), u128_to_double(sqy)};
        double c[3];
        poly2_solve(X, Y, c);
        m0 = c[0];
        m1 = c[1];
        m2 = c[2];
      }
    }
    if (CODEC == kLegacy) {
      l = legacy_residuals<G>(sm, m0, m1, len, tid, nt);
    } else {
      if (CODEC == kLinear) {
        // ---- midpoint shift (piecewise_fix_integer_template.h:36-46) -----------
        int64_t dmax = (int64_t)0x8000000000000000ull, dmin = 0x7fffffffffffffffll;
        with_pred_rule(m0, m1, len, [&](auto rule) {
          for (uint32_t i = tid; i < len; i += nt) {
            const int64_t pr = lin_pred<decltype(rule)::value>(m0, m1, i);
            int64_t d = (int64_t)((uint64_t)sm.vals[i] - (uint64_t)pr);
            dmax = d > dmax ? d : dmax;
            dmin = d < dmin ? d : dmin;
          }
        });
        u128 rmx = (u128)(uint64_t)dmax, rmn = (u128)(uint64_t)dmin;
        group_reduce2<3, 4, G>(rmx, rmn, sm.red);
        dmax = (int64_t)(uint64_t)rmx;
        dmin = (int64_t)(uint64_t)rmn;
        narrow_range = dmax >= dmin && (uint64_t)(dmax - dmin) < (1ull << 30);
        const int64_t mid = (int64_t)((uint64_t)dmax + (uint64_t)dmin);
        m0 = __dadd_rn(m0, __dmul_rn(__ll2double_rn(mid), 0.5));  // x * 0.5 rounds exactly as x / 2.0
      }
      // ---- residuals (…_integer_template.h:51-72, poly :37-58) -----------------
      uint64_t rmax = 0;
      const bool fast = model_in_range(m0, m1, CODEC == kPoly2 ? m2 : 0.0, len);
      // u64 blocks whose predictions lie in [0, 2^51) (so the reference's unsigned
      // comparison is the signed one) and whose residuals before the midpoint shift
      // spanned less than 2^30: every residual after the shift is below 2^31 in
      // magnitude, so its low 32 bits are the whole of it.  Predictions on the FP64
      // pipe (exact), residual arithmetic in 32 bits.
      const bool r32 = CODEC == kLinear && S == 8 && narrow_range && preds_nonneg(m0, m1, len);
      if (r32) {
        uint32_t rm32 = 0;
        for (uint32_t i0 = 0; i0 < len; i0 += nt) {
          const uint32_t i = i0 + tid;
          bool pos = false;
          if (i < len) {
            const uint64_t y = (uint64_t)sm.vals[i];
            const int64_t pred = trunc_nonneg_fp64(pred_linear_fp64(m0, m1, i));
            const int32_t d = (int32_t)((uint32_t)y - (uint32_t)pred);
            pos = d > 0;  // y > pred
            const uint32_t r = pos ? (uint32_t)d : (uint32_t)(-d);
            sm.vals[i] = (T)r;
            rm32 = r > rm32 ? r : rm32;
          }
          const uint32_t ballot = __ballot_sync(0xffffffffu, pos);
          if ((tid & 31) == 0) sm.signs[i0 / 32 + tid / 32] = ballot;
        }
        rmax = rm32;
      } else {
        auto resid_loop = [&](auto rule) {
          for (uint32_t i0 = 0; i0 < len; i0 += nt) {
            const uint32_t i = i0 + tid;
            bool pos = false;
            uint64_t r = 0;
            if (i < len) {
              const uint64_t y = (uint64_t)sm.vals[i];
              if (CODEC == kLinear) {
                const int64_t pred = lin_pred<decltype(rule)::value>(m0, m1, i);
                pos = S == 8 ? (y > (uint64_t)pred) : ((int64_t)y > pred);
                r = pos ? y - (uint64_t)pred : (uint64_t)pred - y;
              } else {
                const double p = pred_poly2(m0, m1, m2, __uint2double_rn(i));
                const int64_t pred = fast ? __double2ll_rz(p) : f2i_x86(p);
                pos = (int64_t)y > pred;
                r = pos ? y - (uint64_t)pred : (uint64_t)pred - y;
              }
              r &= (S == 8 ? ~0ull : 0xffffffffull);
              rmax = r > rmax ? r : rmax;
            }
            // every lane of the warp (one row of 32) has read its value before any lane
            // writes its residual: the swizzled write lands in another lane's slot
            const uint32_t ballot = __ballot_sync(0xffffffffu, pos);
            if (i < len) sm.vals[kRowsCodec && rows ? swz32(i) : i] = (T)r;
            if ((tid & 31) == 0) sm.signs[i0 / 32 + tid / 32] = ballot;
          }
        };
        if (CODEC == kLinear) with_pred_rule(m0, m1, len, resid_loop);
        else resid_loop(std::integral_constant<int, 2>{});
      }
      rmax = (uint64_t)group_reduce<1, G>((u128)rmax, sm.red);
      l = rmax ? bits_of(rmax) + 1 : 0;
      if (l > TB) l = TB;
    }
  } else if (CODEC == kFor) {
    // ---- frame of reference (FOR_integer_template.h:26-52) --------------------
    uint64_t mn = ~0ull, mx = 0;
    for (uint32_t i = tid; i < len; i += nt) {
      uint64_t y = (uint64_t)sm.vals[i];
      mn = y < mn ? y : mn;
      mx = y > mx ? y : mx;
    }
    u128 rmn = (u128)mn, rmx = (u128)mx;
    group_reduce2<2, 1, G>(rmn, rmx, sm.red);
    mn = (uint64_t)rmn;
    mx = (uint64_t)rmx;
    fbase = mn;
    m1 = __longlong_as_double((long long)mx);
    l = bits_of(mx - mn);
  } else {  // kDelta (delta_integer_template.h:34-66)
    uint64_t rmax = 0;
    for (uint32_t i = tid; i + 1 < len; i += nt) {
      uint64_t x0 = (uint64_t)sm.vals[i], x1 = (uint64_t)sm.vals[i + 1];
      uint64_t r = x1 > x0 ? x1 - x0 : x0 - x1;
      rmax = r > rmax ? r : rmax;
    }
    rmax = (uint64_t)group_reduce<1, G>((u128)rmax, sm.red);
    l = rmax ? bits_of(rmax) + 1 : 0;
    if (l > TB) l = TB;
    fbase = (uint64_t)sm.vals[0];
  }
  // A width of 8*sizeof(T)-1 is written raw: the reference's bulk decoders
  // treat l >= 8*sizeof(T)-1 as raw (piecewise_fix_integer_template.h:171,
  // FOR_integer_template.h:89, poly_fix_integer_template.h:121), so a packed
  // block of that width would not decode there.  Delta has no such rule.
  if (CODEC != kDelta && CODEC != kLegacy && l == TB - 1) l = TB;
  // the legacy format stores widths of 31 and up as raw u32 values after its
  // full header (piecewise_fix_op_minimize_maxerror.h:104-108)
  const bool raw = CODEC == kLegacy ? l >= 31 : l == TB;
  if (raw) {  // residuals overwrote the values: restage them
    group_sync<G>();
    for (uint32_t i = tid; i < len; i += nt) sm.vals[i] = __ldg(src + i);
  }
  const uint64_t size = block_bytes<CODEC, S>(l, len);
  // residuals and signs are complete (the width reduction ended with a barrier)
  if (rows && !raw && l > 0) pack_rows(reinterpret_cast<const uint32_t *>(sm.vals), sm.signs, pk, len, l, tid, nt);

  // ---- offset by look-back ----------------------------------------------------
  if (tid < 32) {
    uint64_t excl = lookback_prefix(a.status, b, size, a.error);
    if (tid == 0) sm.bcast[1] = excl;
  }
  // ---- header bytes ------------------------------------------------------------
  if (tid == 0) {
    sm.hdr[0] = (uint8_t)l;
    if (CODEC == kLegacy) {  // [u8 l][f64 theta0][f32 theta1], raw blocks included
      const uint64_t w0 = (uint64_t)__double_as_longlong(m0);
      const uint32_t w1 = __float_as_uint(__double2float_rn(m1));
      for (int j = 0; j < 8; ++j) sm.hdr[1 + j] = (uint8_t)(w0 >> (8 * j));
      for (int j = 0; j < 4; ++j) sm.hdr[9 + j] = (uint8_t)(w1 >> (8 * j));
    } else if (raw) {
      H = 1;
    } else if (CODEC == kLinear || CODEC == kPoly2) {
      uint64_t w0 = (uint64_t)__double_as_longlong(m0), w1 = (uint64_t)__double_as_longlong(m1),
               w2 = (uint64_t)__double_as_longlong(m2);
      for (int j = 0; j < 8; ++j) {
        sm.hdr[1 + j] = (uint8_t)(w0 >> (8 * j));
        sm.hdr[9 + j] = (uint8_t)(w1 >> (8 * j));
        if (CODEC == kPoly2) sm.hdr[17 + j] = (uint8_t)(w2 >> (8 * j));
      }
    } else if (CODEC == kFor) {
      uint64_t mx = (uint64_t)__double_as_longlong(m1);
      for (int j = 0; j < S; ++j) {
        sm.hdr[1 + j] = (uint8_t)(fbase >> (8 * j));
        sm.hdr[1 + S + j] = (uint8_t)(mx >> (8 * j));
      }
    } else {
      for (int j = 0; j < S; ++j) sm.hdr[1 + j] = (uint8_t)(fbase >> (8 * j));
    }
  }
  group_sync<G>();
  const uint64_t goff = sm.bcast[1];
  if (raw && CODEC != kLegacy) H = 1;
  if (goff == ~0ull) return;                       // look-back gave up (error word set)
  if (goff + size + LECO_PAYLOAD_SLACK > a.payload_cap) {  // never write past the buffer
    if (tid == 0) atomicOr(a.error, kErrCapacity);
    return;
  }

  // ---- body ----------------------------------------------------------------------
  const T *vals = sm.vals;
  const uint32_t *signs = sm.signs;
  if (raw) {
    write_image(a.payload, goff, size, H, sm.hdr, TB, len, [&](uint32_t k) -> uint64_t { return (uint64_t)vals[k]; }, tid, nt);
  } else if (rows && l > 0) {
    write_image_packed(a.payload, goff, size, H, sm.hdr, pk, tid, nt);
  } else if (CODEC == kLegacy) {  // write_delta_T (bit_write.h:186-245): |r| below the sign bit
    const uint32_t sb = l ? l - 1 : 0;
    const uint32_t mm = (1u << sb) - 1u;
    write_image(a.payload, goff, size, H, sm.hdr, l, len, [&](uint32_t k) -> uint64_t {
      return (uint64_t)(((uint32_t)vals[k] & mm) | (((signs[k >> 5] >> (k & 31)) & 1u) << sb));
    }, tid, nt);
  } else if (CODEC == kLinear || CODEC == kPoly2) {
    const uint32_t sb = l ? l - 1 : 0;
    write_image(a.payload, goff, size, H, sm.hdr, l, len, [&](uint32_t k) -> uint64_t {
      return (uint64_t)vals[k] | ((uint64_t)((signs[k >> 5] >> (k & 31)) & 1u) << sb);
    }, tid, nt);
  } else if (CODEC == kFor) {
    const uint64_t mnv = fbase;
    const uint64_t tm = S == 8 ? ~0ull : 0xffffffffull;
    write_image(a.payload, goff, size, H, sm.hdr, l, len, [&](uint32_t k) -> uint64_t { return ((uint64_t)vals[k] - mnv) & tm; }, tid, nt);
  } else {
    const uint32_t sb = l ? l - 1 : 0;
    const uint32_t last = len - 1;
    write_image(a.payload, goff, size, H, sm.hdr, l, len, [&](uint32_t k) -> uint64_t {
      if (k >= last) return 0;  // the reference writes an out-of-bounds field here (delta_integer_template.h:83)
      uint64_t x0 = (uint64_t)vals[k], x1 = (uint64_t)vals[k + 1];
      bool pos = x1 > x0;
      return (pos ? x1 - x0 : x0 - x1) | ((uint64_t)pos << sb);
    }, tid, nt);
  }

  // ---- offsets and directory -------------------------------------------------------
  if (tid == 0) {
    a.offsets[b] = goff;
    if (b == a.nb - 1) a.offsets[a.nb] = goff + size;
    if (a.dir) {
      leco_dir_entry e;
      uint64_t body_bit = (goff + H) * 8;
      const uint32_t dl = CODEC == kLegacy && raw ? 32u : l;  // as the decoder's directory records it
      e.word0 = body_bit | ((uint64_t)dl << 56) | ((uint64_t)CODEC << 48);
      if (CODEC == kLinear || CODEC == kPoly2 || CODEC == kLegacy) {
        e.a0 = m0; e.a1 = m1; e.a2 = m2;
      } else {
        e.a0 = __longlong_as_double((long long)fbase);
        e.a1 = 0; e.a2 = 0;
      }
      a.dir[b] = e;
    }
  }
}

// ---- sequential reference fits (LECO_FIT_REFERENCE) ---------------------------
// One lane per block adds the block's values in the reference's own order and FP64
// operations, so the model is bit-identical to lr_int_T::caltheta (lr.h:66-85) or to
// the Y sums of polynomial_regression_iter (polynomial_regression_internals.hpp:129-137)
// (the kernels: seq_fit_tiled_kernel and seq_fit_ring_kernel in leco_encode.cu,
// batch_seq_fit_kernel in leco_batch.cu).
struct PolyX {
  double x[10];
};

// The model of a len-value block from the sums of the reference's fit loop (linear:
// sum y, sum i*y; poly: the three Y sums): lr_int_T::caltheta (lr.h:79-83) with the
// x sums in closed form -- sum i and sum i*i are exact integers below 2^53 at every
// step of the reference's loop (i < 16384), so these are the same doubles -- or the
// degree-2 solve with the column's X sums (polyX: full block [0..4], tail block [5..9]).
template <int CODEC>
__device__ __forceinline__ void store_seq_model(double *m, double s0, double s1, double s2, uint32_t len, uint32_t bs,
                                                const double *polyX) {
  if (CODEC != kPoly2) {
    const double md = __uint2double_rn(len);
    const uint64_t ml = len;
    const double sumx = __ull2double_rn(ml * (ml - 1) / 2), sumxx = __ull2double_rn((ml - 1) * ml * (2 * ml - 1) / 6);
    const double ccc = __dsub_rn(__dmul_rn(s1, md), __dmul_rn(sumx, s0));
    const double xxx = __dsub_rn(__dmul_rn(sumxx, md), __dmul_rn(sumx, sumx));
    const double t1 = __ddiv_rn(ccc, xxx);
    m[0] = __ddiv_rn(__dsub_rn(s0, __dmul_rn(t1, sumx)), md);
    m[1] = t1;
    m[2] = 0.0;
  } else {
    const double *X = polyX + (len == bs ? 0 : 5);
    double Y[3] = {s0, s1, s2}, c[3];
    poly2_solve(X, Y, c);
    m[0] = c[0];
    m[1] = c[1];
    m[2] = c[2];
  }
}

}  // namespace leco
