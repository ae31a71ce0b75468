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
#include "leco_decode.cuh"
#include "leco_stage.cuh"

#include <cstdlib>

namespace leco {

// Direct decode: one CTA per block of the range, everything read from global memory.
template <typename T, int CODEC>
__global__ void __launch_bounds__(256) decode_kernel(DecodeLaunch a) {
  decode_block<T, CODEC>(a, a.first / a.bs + blockIdx.x);
}

// Small blocks: one warp per block, eight blocks per CTA.
template <typename T, int CODEC>
__global__ void __launch_bounds__(256) decode_kernel_warp(DecodeLaunch a, uint64_t nblk) {
  const uint64_t i = (uint64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  if (i < nblk) decode_block<T, CODEC, 32>(a, a.first / a.bs + i);
}

// Sum of the values of block b, this thread's share (all threads of the CTA
// call it): the values as sum_kernel below computes them, for the staged sum's
// blocks that do not fit its buffer or are wider than 32 bits.
template <typename T, int CODEC>
__device__ __forceinline__ uint64_t sum_block_direct(const DecodeLaunch &a, uint64_t b) {
  constexpr int S = sizeof(T);
  constexpr uint32_t TB = 8u * S;
  const uint64_t base = b * a.bs;
  const uint32_t len = (uint32_t)umin64((uint64_t)a.bs, a.n - base);
  const uint64_t *words = reinterpret_cast<const uint64_t *>(a.payload);
  const BlockHdr h = parse_header<CODEC, S>(a.payload, __ldg(a.offsets + b));
  if (h.l == 126 || h.l == 127 || h.l > TB) {
    if (threadIdx.x == 0) atomicOr(a.error, kErrBadHeader);
    return 0;
  }
  const bool raw = h.l == TB;
  const uint32_t l = raw ? TB : h.l;
  uint64_t acc = 0;
  if (CODEC == kDelta && !raw) {
    delta_tiles<T, 256>(words, h, len, 0, len, [&](uint32_t k0, const auto *v) {
#pragma unroll
      for (int j = 0; j < kDeltaSpan; ++j)
        if (k0 + j < len) acc += (uint64_t)(T)v[j];
    });
    return acc;
  }
  for (uint32_t k = threadIdx.x; k < len; k += blockDim.x) {
    const uint64_t f = l ? load_field(words, h.body_bit + (uint64_t)k * l, l) : 0;
    acc += (uint64_t)(T)(raw ? f : value_from_field<CODEC, S>(h, k, f));
  }
  return acc;
}

// ---- TMA-staged persistent decode --------------------------------------------
struct StageMeta {
  uint64_t gbase;   // 16-byte aligned global byte address of the staged copy
  uint32_t hoff;    // block header offset inside the staged copy
  uint32_t direct;  // 1: block too large for the buffer, decode from global
};

// Persistent decode of a whole column.  Each CTA walks blocks blockIdx.x,
// blockIdx.x + gridDim.x, ...; thread 0 stages the next block's image (header +
// packed body) into the other half of a double buffer with one cp.async.bulk
// while the CTA decodes the current one out of shared memory.  Blocks that do
// not fit the buffer and wide (l > 32) blocks take the direct path.  Delta blocks
// run the row scan (delta_tiles), which synchronises the CTA, so for Delta the
// CTA decodes a block only when every thread's wait succeeded.
// SUM: the compressed-domain sum instead -- the values are added up, not stored,
// and each CTA adds its total to *d_sum once.
template <typename T, int CODEC, bool SUM = false>
__global__ void __launch_bounds__(256) decode_staged_kernel(DecodeLaunch a, uint32_t bufcap, uint64_t *d_sum = nullptr) {
  constexpr int S = sizeof(T);
  extern __shared__ __align__(128) uint8_t stage[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ StageMeta meta[2];
  __shared__ u128 red[SUM ? 33 : 1];
  uint64_t acc = 0;
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
    // a thread whose wait gave up touches neither the buffer nor the output; Delta
    // blocks are decoded by all threads or by none (their scan has CTA barriers)
    const bool go = CODEC == kDelta ? __syncthreads_and(ok) != 0 : ok;
    if (go) {
      const StageMeta m = meta[cur];
      const uint8_t *sb = (cur ? buf1 : buf0);
      const uint32_t l = sb[m.hoff];
      const uint64_t base = blk * a.bs;
      const uint32_t len = (uint32_t)umin64(a.bs, a.n - base);
      const bool raw = l == 8u * S;
      const bool narrow = (l <= 32) && (!raw || S == 4);
      if (m.direct || !narrow) {
        if (SUM) acc += sum_block_direct<T, CODEC>(a, blk);
        else decode_block<T, CODEC>(a, blk);
      } else if (CODEC == kDelta && !raw) {
        BlockHdr h;
        h.l = l;
        h.a0 = h.a1 = h.a2 = 0;
        uint64_t w = 0;
  #pragma unroll
        for (int j = 0; j < S; ++j) w |= (uint64_t)sb[m.hoff + 1 + j] << (8 * j);
        h.base = w;
        h.body_bit = (uint64_t)(m.hoff + Hdr<CODEC, S>::bytes) * 8;
        const uint64_t *sw = reinterpret_cast<const uint64_t *>(sb);
        if (SUM) {
          delta_tiles<T, 256, true>(sw, h, len, 0, len, [&](uint32_t k0, const auto *v) {
  #pragma unroll
            for (int j = 0; j < kDeltaSpan; ++j)
              if (k0 + j < len) acc += (uint64_t)(T)v[j];
          });
        } else {
          delta_tiles<T, 256, true>(sw, h, len, 0, len, DeltaStore<T>{out, base, 0, len});
        }
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
        const int32_t kstart = -(int32_t)((oaddr & 31) / S);  // groups start on 32 bytes
        const bool fast = (CODEC == kFor) || raw || pred_in_range<CODEC>(h, len);
        if (!raw) mark_nonneg<CODEC>(h, len);
        // u64 values: eight per thread step, two 256-bit stores (0.340 ms against 0.345 ms with four
        // for 200M keys); u32 values and the sums keep 32 bytes per step (sixteen u32 values per
        // step took 0.296 ms instead of 0.236 ms for 200M u32 keys, and cost the u32 sums registers)
        constexpr int UD = (S == 8 && !SUM) ? 4 : 2;
        if (fast) acc += decode_narrow<T, CODEC, true, true, 256, SUM, UD>(h, raw, w32, out, base, 0, len, kstart);
        else acc += decode_narrow<T, CODEC, false, true, 256, SUM, UD>(h, raw, w32, out, base, 0, len, kstart);
      }
    }
    // Everyone is done with this buffer before it is refilled; a wait that gave up in
    // any thread ends the CTA's work in all of them together.
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicOr(a.error, kErrTimeout);
        if (has_next) mbar_wait_bounded(&bar[cur ^ 1], cur ? ph0 : ph1);  // let our own copy in flight land
      }
      return;
    }
  }
  if (SUM) {
    acc = (uint64_t)block_reduce<5>((u128)acc, red);
    if (threadIdx.x == 0) atomicAdd(reinterpret_cast<unsigned long long *>(d_sum), (unsigned long long)acc);
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
    delta_tiles<T, 256>(words, h, len, 0, len, [&](uint32_t k0, const auto *v) {
#pragma unroll
      for (int j = 0; j < kDeltaSpan; ++j)
        if (k0 + j < len) acc += (uint64_t)v[j] & tmask;
    });
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
// Batched random access over the whole index array (see gather_lookups).
template <typename T, int CODEC>
__global__ void __launch_bounds__(256) gather_kernel(GatherLaunch a) {
  gather_lookups<T, CODEC>(a, (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, (uint64_t)gridDim.x * blockDim.x);
}

// Delta random access: value k = x0 + the signed fields 0..k-1
// (Delta_int::randomdecodeArray8, delta_integer_template.h:132-154, read_Delta_int
// bit_read.h:1292-1317).  The walk is shared by a warp: lane j adds fields
// j, j+32, ... < k, so each step reads 32 consecutive fields, and a warp sum
// combines the lanes.  Each warp takes lookups in turn (warp-uniform loop).
template <typename T>
__global__ void __launch_bounds__(256) gather_delta_kernel(GatherLaunch a) {
  constexpr int S = sizeof(T);
  constexpr uint32_t TB = 8u * S;
  const uint64_t *words = reinterpret_cast<const uint64_t *>(a.payload);
  T *out = reinterpret_cast<T *>(a.out);
  const int lane = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t i = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < a.m; i += warps) {
    const uint64_t g = __ldg(a.idx + i);
    if (g >= a.n) {
      if (lane == 0) {
        out[i] = 0;
        atomicOr(a.error, kErrBadIndex);
      }
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
      if (lane == 0) atomicOr(a.error, kErrBadHeader);
    } else {
      uint64_t part = 0;  // fields j < k are the deltas before value k
      if (h.l && k) part = h.l > 32 ? delta_walk_part<true>(words, h, k, lane) : delta_walk_part<false>(words, h, k, lane);
      v = h.base + warp_sum_u64(part);
    }
    if (lane == 0) out[i] = (T)v;
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
  if (CODEC == kLinear || CODEC == kPoly2 || CODEC == kLegacy) {
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
        case kLegacy: FN<uint32_t, kLegacy>(__VA_ARGS__); return 0;         \
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
                      CODEC != kLegacy && nblk >= 1024 && L.bs > kWarpBlock && staged_decode_enabled();
  if (!staged) {
    if (L.bs <= kWarpBlock) decode_kernel_warp<T, CODEC><<<(unsigned)((nblk + 7) / 8), 256, 0, st>>>(L, nblk);
    else decode_kernel<T, CODEC><<<(unsigned)nblk, 256, 0, st>>>(L);
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
  if (!nb) return;
  const bool staged = (reinterpret_cast<uintptr_t>(L.payload) & 15) == 0 && CODEC != kLegacy &&
                      nb >= 1024 && L.bs > kWarpBlock && staged_decode_enabled();
  if (!staged) {
    sum_kernel<T, CODEC><<<(unsigned)nb, 256, 0, st>>>(L, d_sum);
    return;
  }
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int smem = 2 * kStageBuf + 64;
  cudaFuncSetAttribute(decode_staged_kernel<T, CODEC, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, decode_staged_kernel<T, CODEC, true>, 256, smem);
  const uint64_t grid = umin64(nb, (uint64_t)sms * (uint64_t)(per_sm > 0 ? per_sm : 1));
  decode_staged_kernel<T, CODEC, true><<<(unsigned)grid, 256, smem, st>>>(L, kStageBuf, d_sum);
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
  if (CODEC == kDelta) {  // one warp per lookup at a time
    const unsigned grid = (unsigned)umin64((L.m + 7) / 8, (uint64_t)sms * 8);
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
