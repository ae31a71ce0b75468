// leco_encode.cu -- single-pass column encoder for the LeCo fixed-block codecs.
//
// One CTA encodes one block per launch slot:
//   1. take a block id from a ticket counter (ids are handed out in start order,
//      so every predecessor of a block is already running or finished),
//   2. stage the block's values in shared memory (read once from HBM),
//   3. fit the model, compute residuals and the bit width l,
//   4. get the block's byte offset from a decoupled look-back prefix sum over
//      the per-block image sizes (status words in the caller's workspace),
//   5. write the exact reference block image (header + LSB-first packed body)
//      straight to its place in the payload with 16-byte stores, byte stores at
//      the two unaligned ends.
//
// Reference: Leco_int<T>::encodeArray8_int (piecewise_fix_integer_template.h:27-140),
// FOR_int<T>::encodeArray8_int (FOR_integer_template.h:26-81),
// Delta_int<T>::encodeArray8_int (delta_integer_template.h:26-87),
// Leco_int_poly<T,2>::encodeArray8_int (poly_fix_integer_template.h:28-91),
// packers write_delta_int_T / write_FOR_int_T (bit_write.h:257-390).
#include "leco_encode.cuh"

#include <string>

namespace leco {

// CTAs per SM the encoder's register budget is set for: six (40 registers) for u64 LeCo
// blocks, whose shared memory allows six, and for the other u32 codecs; five (48) for
// the other u64 codecs; four (64) for degree-2 blocks.
template <typename T, int CODEC>
constexpr int enc_min_ctas() {
  return CODEC == kPoly2 ? 4 : (sizeof(T) == 4 || CODEC == kLinear) ? 6 : 5;
}

template <typename T, int CODEC>
__global__ void __launch_bounds__(256, enc_min_ctas<T, CODEC>()) encode_kernel(EncodeArgs a) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  __shared__ uint64_t ticket;
  if (threadIdx.x == 0) ticket = atomicAdd(a.ticket, 1u);
  __syncthreads();
  const uint64_t b = ticket;
  if (b >= a.nb) return;
  encode_block<T, CODEC>(a, b, smem_raw);
  // block 0 has published its inclusive prefix: its first warp stays on as the prefix
  // publisher for the rest of the column
  if (b == 0 && threadIdx.x < 32 && a.nb > 1) publish_prefixes(a.status, a.nb, a.error);
}

// Small blocks: one warp per block, eight blocks per CTA, each warp with its
// own slice of shared memory and its own ticket.
template <typename T, int CODEC>
__global__ void __launch_bounds__(256) encode_kernel_warp(EncodeArgs a, uint32_t slice) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t t = 0;
  if (lane == 0) t = atomicAdd(a.ticket, 1u);
  const uint64_t b = __shfl_sync(0xffffffffu, t, 0);
  if (b >= a.nb) return;
  encode_block<T, CODEC, 32>(a, b, smem_raw + (size_t)w * slice);
}

// Sequential reference fits, one warp per 32 blocks: each step the warp loads a
// 32 x 32 tile (32 consecutive values of each of its 32 blocks, coalesced) into
// shared memory while the next tile is already in flight to registers; lane j
// then adds the 32 values of block j to its running sums in order, exactly the
// reference's loop (lr.h:72-77; Y sums of polynomial_regression_internals.hpp:129-137).
// A full tile's 32 conversions and products are taken before its adds, so the
// lane's critical path is the add chains alone (the loop that waited on a load and
// a conversion at every step took ~200 us per block of 4096 values).  Twelve warps
// per SM (registers) hold a whole 200M-value column's 1526 warps in one wave, where
// the loads are in flight across warps; a lone warp waits for each next tile.
template <typename T, int CODEC>
__global__ void __launch_bounds__(128) seq_fit_tiled_kernel(const T *__restrict__ values, uint64_t n, uint32_t bs,
                                                            uint64_t nb, PolyX px, double *__restrict__ models) {
  __shared__ T tile[4][32][33];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint64_t b0 = ((uint64_t)blockIdx.x * 4 + w) * 32;
  if (b0 >= nb) return;
  const uint64_t mine = b0 + lane;
  const uint32_t len = mine < nb ? (uint32_t)umin64(bs, n - mine * bs) : 0;
  T nxt[32];
  // value i of row r exists when block b0 + r exists and i < its length
  auto fetch = [&](uint32_t t0) {
    const uint32_t i = t0 + lane;
#pragma unroll
    for (int r = 0; r < 32; ++r) {
      const uint64_t g = (b0 + r) * bs + i;
      nxt[r] = (b0 + r < nb && i < bs && g < n) ? __ldg(values + g) : (T)0;
    }
  };
  double s0 = 0, s1 = 0, s2 = 0;  // linear: sumy sumxy; poly: Y0 Y1 Y2
  uint32_t maxlen = len;
  for (int m = 16; m; m >>= 1) maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, m));
  fetch(0);
  for (uint32_t t0 = 0; t0 < maxlen; t0 += 32) {
#pragma unroll
    for (int r = 0; r < 32; ++r) tile[w][r][lane] = nxt[r];
    __syncwarp();
    if (t0 + 32 < maxlen) fetch(t0 + 32);
    const uint32_t cnt = len > t0 ? (len - t0 < 32 ? len - t0 : 32) : 0;
    const double dt0 = u32_to_double_fp64(t0);
    if (cnt == 32) {
      // y_i * i (linear) or the three Y terms (poly), all before the first add
      double yv[32], pv[32];
#pragma unroll
      for (int c = 0; c < 32; ++c) {
        yv[c] = to_double<T>(tile[w][lane][c]);
        pv[c] = __dmul_rn(__dadd_rn(dt0, (double)c), yv[c]);  // i = t0 + c exactly
      }
      if (CODEC == kLinear) {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          s0 = __dadd_rn(s0, yv[c]);
          s1 = __dadd_rn(s1, pv[c]);
        }
      } else {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const double di = __dadd_rn(dt0, (double)c);
          s0 = __dadd_rn(s0, yv[c]);  // the reference's 1.0 * y is y
          s1 = __dadd_rn(s1, pv[c]);
          s2 = __dadd_rn(s2, __dmul_rn(__dmul_rn(di, di), yv[c]));
        }
      }
    } else {
      for (uint32_t c = 0; c < cnt; ++c) {
        const double di = __dadd_rn(dt0, __uint2double_rn(c)), yi = to_double<T>(tile[w][lane][c]);
        s0 = __dadd_rn(s0, yi);
        s1 = __dadd_rn(s1, __dmul_rn(di, yi));
        if (CODEC != kLinear) s2 = __dadd_rn(s2, __dmul_rn(__dmul_rn(di, di), yi));
      }
    }
    __syncwarp();
  }
  if (len) store_seq_model<CODEC>(models + mine * 3, s0, s1, s2, len, bs, px.x);
}

// The same fits with a deeper pipeline per warp, for columns whose warps fit in one
// wave of this kernel (four CTAs per SM): one warp per CTA, lane j fits block b0 + j,
// and a ring of kFitStages stages holds the next tiles of all 32 blocks (row j: block
// b0 + j, padded by 16 bytes so that the lanes' 16-byte reads of their own rows spread
// over the banks).  A stage is filled by coalesced 16-byte cp.async copies (one group
// per stage) and read after the warp has waited for its group, so a lone warp's add
// chains are no longer held up by its loads (one block of 4096 values: ~60 us instead
// of ~110 us).  Needs 16-byte aligned values and bs * sizeof(T) a multiple of 16.
// Tiles of fewer than 32 values (a block's last when bs is not a multiple of 32, the
// column's short last block) are read from global memory directly.
constexpr int kFitStages = 6;
template <typename T>
__host__ __device__ constexpr uint32_t fit_row_bytes() { return 32u * sizeof(T) + 16u; }
template <typename T>
__host__ __device__ constexpr uint32_t fit_smem_bytes() { return (uint32_t)kFitStages * 32u * fit_row_bytes<T>(); }

template <typename T, int CODEC>
__global__ void __launch_bounds__(32) seq_fit_ring_kernel(const T *__restrict__ values, uint64_t n, uint32_t bs, uint64_t nb,
                                                          PolyX px, double *__restrict__ models) {
  constexpr uint32_t S = sizeof(T), RB = fit_row_bytes<T>(), SB = 32u * RB;
  constexpr uint32_t CPR = 32u * S / 16u;  // 16-byte chunks per row: 16 (u64) or 8 (u32)
  constexpr uint32_t RPI = 32u / CPR;      // rows per copy instruction
  // 16 bytes is all cp.async needs; a larger alignment here would also move the dynamic
  // shared memory of every other kernel in this file (the encoder measured 3-6 % slower)
  extern __shared__ __align__(16) uint8_t ring[];
  const uint32_t lane = threadIdx.x;
  const uint64_t b0 = (uint64_t)blockIdx.x * 32, mine = b0 + lane;
  const uint32_t len = mine < nb ? (uint32_t)umin64(bs, n - mine * bs) : 0;
  const uint32_t ntiles = (__reduce_max_sync(0xffffffffu, len) + 31) / 32;
  const uint32_t sring = smem_u32(ring);
  // tile t of every row whose 32 values all exist; instruction q copies rows
  // RPI*q .. RPI*q + RPI-1, lane k of a row's CPR lanes its k-th 16 bytes
  auto issue = [&](uint32_t t) {
    if (t < ntiles) {
      const uint32_t k = lane % CPR, s = t % kFitStages;
#pragma unroll
      for (uint32_t q = 0; q < CPR; ++q) {
        const uint32_t r = RPI * q + lane / CPR;
        const uint32_t lr = __shfl_sync(0xffffffffu, len, r);
        if (lr >= 32 * (t + 1))
          cp_async16(sring + s * SB + r * RB + 16 * k, values + (b0 + r) * bs + 32 * t + k * (16 / S));
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  for (uint32_t t = 0; t < (uint32_t)kFitStages; ++t) issue(t);
  double s0 = 0, s1 = 0, s2 = 0;  // linear: sumy sumxy; poly: Y0 Y1 Y2
  for (uint32_t t = 0; t < ntiles; ++t) {
    const uint32_t s = t % kFitStages;
    asm volatile("cp.async.wait_group %0;" ::"n"(kFitStages - 1) : "memory");  // tile t's group has landed
    __syncwarp();
    const uint32_t cnt = len > 32 * t ? min(32u, len - 32 * t) : 0u;
    const uint8_t *src = ring + s * SB + lane * RB;
    const double dt0 = u32_to_double_fp64(32 * t);
    if (cnt == 32) {
      double yv[32], pv[32];
#pragma unroll
      for (int q = 0; q < (int)CPR; ++q) {
        const uint4 v = *reinterpret_cast<const uint4 *>(src + 16 * q);
        if (S == 8) {
          yv[2 * q] = to_double<T>((T)(((uint64_t)v.y << 32) | v.x));
          yv[2 * q + 1] = to_double<T>((T)(((uint64_t)v.w << 32) | v.z));
        } else {
          yv[4 * q] = to_double<T>((T)v.x);
          yv[4 * q + 1] = to_double<T>((T)v.y);
          yv[4 * q + 2] = to_double<T>((T)v.z);
          yv[4 * q + 3] = to_double<T>((T)v.w);
        }
      }
#pragma unroll
      for (int c = 0; c < 32; ++c) pv[c] = __dmul_rn(__dadd_rn(dt0, (double)c), yv[c]);  // i = 32t + c exactly
      if (CODEC == kLinear) {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          s0 = __dadd_rn(s0, yv[c]);
          s1 = __dadd_rn(s1, pv[c]);
        }
      } else {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const double di = __dadd_rn(dt0, (double)c);
          s0 = __dadd_rn(s0, yv[c]);  // the reference's 1.0 * y is y
          s1 = __dadd_rn(s1, pv[c]);
          s2 = __dadd_rn(s2, __dmul_rn(__dmul_rn(di, di), yv[c]));
        }
      }
    } else {
      const T *tv = values + mine * bs + 32 * t;  // not staged
      for (uint32_t c = 0; c < cnt; ++c) {
        const double di = __dadd_rn(dt0, __uint2double_rn(c)), yi = to_double<T>(__ldg(tv + c));
        s0 = __dadd_rn(s0, yi);
        s1 = __dadd_rn(s1, __dmul_rn(di, yi));
        if (CODEC != kLinear) s2 = __dadd_rn(s2, __dmul_rn(__dmul_rn(di, di), yi));
      }
    }
    __syncwarp();  // every lane's reads of this stage are done before it is refilled
    issue(t + kFitStages);
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  if (len) store_seq_model<CODEC>(models + mine * 3, s0, s1, s2, len, bs, px.x);
}

// ---- host launchers ---------------------------------------------------------------

template <typename T, int CODEC>
static int launch_encode_t(const EncodeLaunch &L, cudaStream_t st) {
  EncodeArgs a;
  a.values = L.values; a.n = L.n; a.bs = L.bs; a.nb = L.nb;
  a.payload = L.payload; a.payload_cap = L.payload_cap; a.offsets = L.offsets; a.dir = L.dir;
  a.seq_models = nullptr; a.status = L.status; a.ticket = L.ticket; a.error = L.error;
  // u32 LeCo / degree-2 blocks of 513..4096 values pack their residual rows in an area of
  // shared memory after the values (six CTAs per SM are set by registers there anyway)
  a.rows_area = sizeof(T) == 4 && (CODEC == kLinear || CODEC == kPoly2) && L.bs > kWarpBlock && L.bs <= 4096;
  PolyX px;
  for (int i = 0; i < 10; ++i) a.polyX[i] = px.x[i] = L.polyX[i];
  if (L.seq_models && (CODEC == kLinear || CODEC == kPoly2 || CODEC == kLegacy)) {
    // four warps per CTA, 32 blocks per warp (the legacy codec fits as LINEAR does)
    constexpr int FC = CODEC == kLegacy ? kLinear : CODEC;
    const uint64_t warps = (L.nb + 31) / 32;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (warps <= 4ull * (uint64_t)sms && (reinterpret_cast<uintptr_t>(L.values) & 15) == 0 &&
        ((uint64_t)L.bs * sizeof(T)) % 16 == 0) {
      constexpr uint32_t fsm = fit_smem_bytes<T>();
      if (fsm > 48 * 1024)
        cudaFuncSetAttribute(seq_fit_ring_kernel<T, FC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm);
      seq_fit_ring_kernel<T, FC><<<(unsigned)warps, 32, fsm, st>>>(reinterpret_cast<const T *>(L.values), L.n, L.bs,
                                                                   L.nb, px, L.seq_models);
    } else {
      seq_fit_tiled_kernel<T, FC><<<(unsigned)((L.nb + 127) / 128), 128, 0, st>>>(
          reinterpret_cast<const T *>(L.values), L.n, L.bs, L.nb, px, L.seq_models);
    }
    a.seq_models = L.seq_models;
  }
  const uint32_t smem = enc_smem_bytes(L.bs, sizeof(T)) + (a.rows_area ? enc_rows_bytes(L.bs) : 0u);
  if (L.bs <= kWarpBlock) {
    const uint32_t slice = (smem + 15) / 16 * 16;
    encode_kernel_warp<T, CODEC><<<(unsigned)((L.nb + 7) / 8), 256, 8 * slice, st>>>(a, slice);
    return 0;
  }
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(encode_kernel<T, CODEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  encode_kernel<T, CODEC><<<(unsigned)L.nb, 256, smem, st>>>(a);
  return 0;
}

int launch_encode(int codec, int s, const EncodeLaunch &L, cudaStream_t st) {
  if (s == 4) {
    switch (codec) {
      case kLinear: return launch_encode_t<uint32_t, kLinear>(L, st);
      case kFor: return launch_encode_t<uint32_t, kFor>(L, st);
      case kDelta: return launch_encode_t<uint32_t, kDelta>(L, st);
      case kPoly2: return launch_encode_t<uint32_t, kPoly2>(L, st);
      case kLegacy: return launch_encode_t<uint32_t, kLegacy>(L, st);
    }
  } else {
    switch (codec) {
      case kLinear: return launch_encode_t<uint64_t, kLinear>(L, st);
      case kFor: return launch_encode_t<uint64_t, kFor>(L, st);
      case kDelta: return launch_encode_t<uint64_t, kDelta>(L, st);
      case kPoly2: return launch_encode_t<uint64_t, kPoly2>(L, st);
    }
  }
  return -1;
}

// Bounded-wait check: block 1 of a two-block look-back whose block 0 never
// publishes its size (a status word nothing sets).  The wait must give up after
// `spin_limit` polls, set the error word and return.
__global__ void lookback_timeout_probe_kernel(uint64_t *status, uint32_t *error, uint32_t spin_limit, uint64_t *result) {
  if (threadIdx.x < 32) {
    const uint64_t excl = lookback_prefix(status, 1, 16, error, spin_limit);
    if (threadIdx.x == 0) *result = excl;
  }
}

}  // namespace leco

extern "C" int leco_test_bounded_wait(uint32_t spin_limit, uint64_t *h_result) {
  using namespace leco;
  uint32_t *err = nullptr;
  int rc = device_error_word(&err);
  if (rc) return rc;
  uint64_t *buf = nullptr;  // [2] status words + [1] result
  cudaError_t e = cudaMalloc(&buf, 3 * sizeof(uint64_t));
  if (e == cudaSuccess) e = cudaMemset(buf, 0, 3 * sizeof(uint64_t));
  if (e == cudaSuccess) {
    lookback_timeout_probe_kernel<<<1, 32>>>(buf, err, spin_limit, buf + 2);
    e = cudaDeviceSynchronize();
  }
  if (e == cudaSuccess && h_result) e = cudaMemcpy(h_result, buf + 2, sizeof(uint64_t), cudaMemcpyDeviceToHost);
  if (buf) cudaFree(buf);
  if (e != cudaSuccess) return record_error(LECO_ERR_CUDA, std::string("leco_test_bounded_wait: ") + cudaGetErrorString(e));
  return leco_check(nullptr);
}
