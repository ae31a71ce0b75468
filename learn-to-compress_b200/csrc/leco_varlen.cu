// leco_varlen.cu -- variable-length LeCo segments on the GPU: segment encode
// (given the partition), bulk decode, random access and compressed-domain sum.
//
// Segment image (Leco_cost_merge_double_wo_round<uint64_t>,
// headers/piecewise_cost_merge_integer_template_double_wo_round.h:134-272):
//   [u32 start][u8 l][f64 theta0][f32 slope][packed l-bit fields]   (l < 64)
//   [u32 start][u8 64][u64 x n]                                      (raw)
//   [u32 start][u8 127][u64]   one value,  [u32 start][u8 126][u64][u64]  two values
// Prediction theta0 + (double)slope * k.  The encoder converts it to a 128-bit
// integer (:158); bulk decode converts it to uint64_t (bit_read.h:530).
// A column: payload (segment images back to back), offsets[nseg+1], and the
// value index where each segment starts, starts[nseg] (starts[0] = 0).
#include <cuda_runtime.h>

#include <string>

#include "leco_decode.cuh"
#include "leco_encode.cuh"
#include "leco_stage.cuh"

namespace leco {

constexpr uint32_t kVarlenMaxSeg = 16384;  // values per segment the encoder stages in shared memory

struct VarArgs {
  const uint64_t *values;
  uint64_t n;
  const uint64_t *starts;
  uint64_t nseg;
  uint8_t *payload;
  uint64_t payload_cap;
  uint64_t *offsets;
  uint64_t *status;
  uint32_t *ticket;
  uint32_t *error;
  int exact_fit;
  uint32_t max_seg;           // longest segment of this partition (sizes the shared-memory stage)
  const double *seq_models;   // [nseg * 2] reference fits (theta0, theta1) of segments of >= 3 values, or null
};

// The reference's sequential fits of the segments (lr_int_T::caltheta, lr.h:66-85,
// called by newsegment, :140-148), one lane per segment, one warp per 32
// consecutive segments: each step the warp moves a tile of 32 values of each of
// its 32 segments (every row contiguous in memory) into shared memory, with the
// next tile already in flight to registers, and lane j adds row j to its running
// sums in order.  sumx and sumxx are not summed:
// every partial sum of i and of i*i is an integer below 2^53, so they equal their
// closed forms.  Segments that are malformed (empty or longer than 16384 values)
// are skipped; the encoder reports them.
__global__ void __launch_bounds__(128) varlen_seq_fit_kernel(const uint64_t *__restrict__ values, uint64_t n,
                                                             const uint64_t *__restrict__ starts, uint64_t nseg,
                                                             double *__restrict__ models) {
  __shared__ uint64_t tile[4][32][33];
  __shared__ uint64_t rst[4][32];
  __shared__ uint32_t rlen[4][32];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint64_t s0 = ((uint64_t)blockIdx.x * 4 + w) * 32;
  if (s0 >= nseg) return;
  const uint64_t mine = s0 + lane;
  uint64_t st = 0;
  uint32_t len = 0;
  if (mine < nseg) {
    st = __ldg(starts + mine);
    const uint64_t en = mine + 1 < nseg ? __ldg(starts + mine + 1) : n;
    len = (en > st && en <= n && en - st <= kVarlenMaxSeg) ? (uint32_t)(en - st) : 0;
  }
  rst[w][lane] = st;
  rlen[w][lane] = len;
  uint32_t maxlen = len;
  for (int m = 16; m; m >>= 1) maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, m));
  __syncwarp();
  // the next tile's 32 rows are in flight to registers while the current one is summed
  uint64_t nxt[32];
  auto fetch = [&](uint32_t t0) {
    const uint32_t i = t0 + lane;
#pragma unroll
    for (int r = 0; r < 32; ++r) nxt[r] = i < rlen[w][r] ? __ldg(values + rst[w][r] + i) : 0ull;
  };
  double sy = 0, sxy = 0;
  fetch(0);
  for (uint32_t t0 = 0; t0 < maxlen; t0 += 32) {
#pragma unroll
    for (int r = 0; r < 32; ++r) tile[w][r][lane] = nxt[r];
    __syncwarp();
    if (t0 + 32 < maxlen) fetch(t0 + 32);
    const uint32_t cnt = len > t0 ? (len - t0 < 32 ? len - t0 : 32) : 0;
    const uint64_t *row = &tile[w][lane][0];
    if (cnt == 32) {
#pragma unroll
      for (uint32_t h = 0; h < 32; h += 16) {  // 16 conversions issued ahead of their adds
        double y[16];
#pragma unroll
        for (uint32_t c = 0; c < 16; ++c) y[c] = __ull2double_rn(row[h + c]);
#pragma unroll
        for (uint32_t c = 0; c < 16; ++c) {
          sy = __dadd_rn(sy, y[c]);
          sxy = __dadd_rn(sxy, __dmul_rn(__uint2double_rn(t0 + h + c), y[c]));
        }
      }
    } else {
      for (uint32_t c = 0; c < cnt; ++c) {
        const double yi = __ull2double_rn(row[c]);
        sy = __dadd_rn(sy, yi);
        sxy = __dadd_rn(sxy, __dmul_rn(__uint2double_rn(t0 + c), yi));
      }
    }
    __syncwarp();
  }
  if (len < 3) return;
  const uint64_t m = len;
  const double md = __uint2double_rn(len);
  const double sumx = __ull2double_rn(m * (m - 1) / 2), sumxx = __ull2double_rn((m - 1) * m * (2 * m - 1) / 6);
  const double ccc = __dsub_rn(__dmul_rn(sxy, md), __dmul_rn(sumx, sy));
  const double xxx = __dsub_rn(__dmul_rn(sumxx, md), __dmul_rn(sumx, sumx));
  const double th1 = __ddiv_rn(ccc, xxx);
  models[mine * 2 + 0] = __ddiv_rn(__dsub_rn(sy, __dmul_rn(th1, sumx)), md);
  models[mine * 2 + 1] = th1;
}

__device__ __forceinline__ uint64_t seg_bytes(uint32_t l, uint32_t len) {
  if (len == 1) return 13;
  if (len == 2) return 21;
  if (l >= 64) return 5 + 8ull * len;
  if (!l) return 17;
  const uint64_t end = ((uint64_t)l * len + 7) / 8;
  return 17 + end + 1 + (8 - end % 8);
}

// One CTA encodes one segment (newsegment / newsegment_1 / newsegment_2).
__global__ void __launch_bounds__(256) varlen_encode_kernel(VarArgs a) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  __shared__ uint64_t s_ticket, s_off;
  __shared__ u128 red[40];
  __shared__ uint8_t hdr[32];
  __shared__ double s_model[2];
  uint64_t *vals = reinterpret_cast<uint64_t *>(smem_raw);
  uint32_t *signs = reinterpret_cast<uint32_t *>(smem_raw + 8 * (size_t)a.max_seg);
  const uint32_t tid = threadIdx.x, nt = blockDim.x;
  if (tid == 0) s_ticket = atomicAdd(a.ticket, 1u);
  __syncthreads();
  const uint64_t sgi = s_ticket;
  if (sgi >= a.nseg) return;
  const uint64_t st = a.starts[sgi], en = sgi + 1 < a.nseg ? a.starts[sgi + 1] : a.n;
  if (en <= st || en - st > a.max_seg || en > a.n) {  // bad partition: report, keep successors moving
    if (tid < 32) lookback_prefix(a.status, sgi, 0, a.error);
    if (tid == 0) atomicOr(a.error, kErrBadHeader);
    return;
  }
  const uint32_t len = (uint32_t)(en - st);
  for (uint32_t i = tid; i < len; i += nt) vals[i] = __ldg(a.values + st + i);
  __syncthreads();
  uint32_t l = 0;
  double t0 = 0, t1d = 0;
  float slope = 0.f;
  if (len >= 3) {
    if (a.exact_fit) {
      u128 sy = 0, siy = 0;
      for (uint32_t i = tid; i < len; i += nt) {
        sy += vals[i];
        siy += (u128)vals[i] * i;
      }
      sy = block_reduce<0>(sy, red);
      siy = block_reduce<0>(siy, red);
      if (tid == 0) {
        const uint64_t m = len;
        const double md = __uint2double_rn(len);
        const double sumx = __ull2double_rn(m * (m - 1) / 2), sumxx = u128_to_double((u128)(m - 1) * m * (2 * m - 1) / 6);
        const double sumy = u128_to_double(sy), sumxy = u128_to_double(siy);
        const double ccc = __dsub_rn(__dmul_rn(sumxy, md), __dmul_rn(sumx, sumy));
        const double xxx = __dsub_rn(__dmul_rn(sumxx, md), __dmul_rn(sumx, sumx));
        const double th1 = __ddiv_rn(ccc, xxx);
        s_model[1] = th1;
        s_model[0] = __ddiv_rn(__dsub_rn(sumy, __dmul_rn(th1, sumx)), md);
      }
    } else if (tid == 0) {  // the reference's sequential fit, from varlen_seq_fit_kernel
      s_model[0] = a.seq_models[sgi * 2 + 0];
      s_model[1] = a.seq_models[sgi * 2 + 1];
    }
    __syncthreads();
    t0 = s_model[0];
    slope = __double2float_rn(s_model[1]);  // float final_slope = mylr.theta1 (:148)
    t1d = (double)slope;
    uint64_t rmax = 0;
    // Predictions are monotone in i, so the two ends bound them; when all lie in
    // [0, 2^63) the 128-bit residual of :158-166 is the 64-bit one.
    const double pe0 = __dadd_rn(t0, __dmul_rn(t1d, 0.0)), pe1 = __dadd_rn(t0, __dmul_rn(t1d, __uint2double_rn(len - 1)));
    const bool u64pred = pe0 >= 0.0 && pe1 >= 0.0 && pe0 < 9223372036854775808.0 && pe1 < 9223372036854775808.0;
    for (uint32_t i0 = 0; i0 < len; i0 += nt) {
      const uint32_t i = i0 + tid;
      bool pos = false;
      if (i < len) {
        const double p = __dadd_rn(t0, __dmul_rn(t1d, __uint2double_rn(i)));
        uint64_t r;
        if (u64pred) {
          const uint64_t pred = __double2ull_rz(p), y = vals[i];
          pos = y > pred;
          r = pos ? y - pred : pred - y;
        } else {
          const i128 pred = f2i128(p);
          const i128 y = (i128)vals[i];
          pos = y > pred;
          r = (uint64_t)(pos ? y - pred : pred - y);
        }
        vals[i] = r;
        rmax = r > rmax ? r : rmax;
      }
      const uint32_t ballot = __ballot_sync(0xffffffffu, pos);
      if ((tid & 31) == 0) signs[i0 / 32 + tid / 32] = ballot;
    }
    rmax = (uint64_t)block_reduce<1>((u128)rmax, red);
    l = rmax ? bits_of(rmax) + 1 : 0;
    if (l >= 64) {
      l = 64;
      __syncthreads();
      for (uint32_t i = tid; i < len; i += nt) vals[i] = __ldg(a.values + st + i);
    }
  }
  const uint64_t size = seg_bytes(l, len);
  if (tid < 32) {
    const uint64_t excl = lookback_prefix(a.status, sgi, size, a.error);
    if (tid == 0) s_off = excl;
  }
  uint32_t H;
  if (tid == 0) {
    const uint32_t s32 = (uint32_t)st;
    for (int j = 0; j < 4; ++j) hdr[j] = (uint8_t)(s32 >> (8 * j));
    hdr[4] = (uint8_t)(len == 1 ? 127 : len == 2 ? 126 : l);
    if (len >= 3 && l < 64) {
      const uint64_t w0 = (uint64_t)__double_as_longlong(t0);
      const uint32_t w1 = (uint32_t)__float_as_uint(slope);
      for (int j = 0; j < 8; ++j) hdr[5 + j] = (uint8_t)(w0 >> (8 * j));
      for (int j = 0; j < 4; ++j) hdr[13 + j] = (uint8_t)(w1 >> (8 * j));
    }
  }
  __syncthreads();
  const uint64_t goff = s_off;
  if (goff == ~0ull) return;
  if (goff + size + LECO_PAYLOAD_SLACK > a.payload_cap) {
    if (tid == 0) atomicOr(a.error, kErrCapacity);
    return;
  }
  if (len <= 2 || l == 64) {  // values stored as they are
    H = 5;
    write_image(a.payload, goff, size, H, hdr, 64, len, [&](uint32_t k) -> uint64_t { return vals[k]; }, tid, nt);
  } else {
    H = 17;
    const uint32_t sb = l ? l - 1 : 0;
    write_image(a.payload, goff, size, H, hdr, l, len, [&](uint32_t k) -> uint64_t {
      return vals[k] | ((uint64_t)((signs[k >> 5] >> (k & 31)) & 1u) << sb);
    }, tid, nt);
  }
  if (tid == 0) {
    a.offsets[sgi] = goff;
    if (sgi == a.nseg - 1) a.offsets[a.nseg] = goff + size;
  }
}

struct SegHdr {
  uint64_t start;
  uint32_t l;
  double t0, slope;
  uint64_t body_bit;
};

__device__ __forceinline__ SegHdr parse_seg(const uint8_t *payload, uint64_t off) {
  const uint64_t *w = reinterpret_cast<const uint64_t *>(payload);
  const uint64_t h0 = load_u64_at(w, off);
  SegHdr s;
  s.start = h0 & 0xffffffffull;
  s.l = (uint32_t)((h0 >> 32) & 0xff);
  s.t0 = s.slope = 0;
  s.body_bit = (off + 5) * 8;
  if (s.l < 64) {
    s.t0 = __longlong_as_double((long long)load_u64_at(w, off + 5));
    s.slope = (double)__uint_as_float((uint32_t)load_u64_at(w, off + 13));
    s.body_bit = (off + 17) * 8;
  }
  return s;
}

// Value k of a segment of length len (bulk-decode rules; also used for random access).
__device__ __forceinline__ uint64_t seg_value(const uint64_t *words, const SegHdr &h, uint32_t k) {
  if (h.l == 127 || h.l == 126 || h.l == 64) return load_field(words, h.body_bit + (uint64_t)k * 64, 64);
  if (h.l > 64) return 0;
  if (!h.l) return f2u_x86(__dadd_rn(h.t0, __dmul_rn(h.slope, __uint2double_rn(k))));
  const uint64_t pred = f2u_x86(__dadd_rn(h.t0, __dmul_rn(__uint2double_rn(k), h.slope)));
  return apply_signed(pred, load_field(words, h.body_bit + (uint64_t)k * h.l, h.l), h.l);
}

// Bulk decode (Leco_cost_merge_double_wo_round::decodeArray8, :573-626) by
// persistent CTAs over items of kVarGroup consecutive segments: CTA c walks items
// c, c + gridDim.x, ...; warp 0 loads the next item's offsets and starts and
// stages its images (contiguous in the payload) into the other half of a double
// buffer with one cp.async.bulk while the CTA's warps decode the current item's
// segments out of shared memory, one segment per warp.  A segment with fields of at most 32 bits whose
// predictions lie inside (-2^62, 2^62) decodes exactly as a LeCo block with
// theta0 = t0 and theta1 = slope (same prediction, same sign-magnitude fields;
// under that bound the uint64_t conversion of bit_read.h:530 is the truncation the
// block decoder applies), through the block decoder's narrow path; other
// segments, and items larger than the buffer, decode from global memory.
// SUM: the compressed-domain sum instead -- value k of every segment for k below its
// length (seg_value: the bulk decoder's values), added up mod 2^64 without being
// stored, one atomic add per CTA.
constexpr uint32_t kVarGroup = 8;
constexpr uint32_t kVarStageBytes = 24832;  // one buffer: ~8 segments of ~2000 values of 12-bit fields, + slack
struct VarStage {
  uint64_t gbase;                    // staged copy's 16-byte aligned global start
  uint64_t off[kVarGroup];           // image offsets
  uint64_t st[kVarGroup + 1];        // value ranges: segment g is [st[g], st[g+1])
  uint32_t cnt, direct;              // segments in the item; 1: decode from global memory
};

template <bool SUM>
__global__ void __launch_bounds__(256) varlen_decode_kernel(const uint8_t *payload, const uint64_t *offsets,
                                                            const uint64_t *starts, uint64_t nseg, uint64_t n,
                                                            uint64_t *out, uint32_t bufcap, uint32_t *error,
                                                            uint64_t *d_sum) {
  extern __shared__ __align__(128) uint8_t vstage[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ VarStage meta[2];
  __shared__ u128 red[SUM ? 33 : 1];
  uint64_t acc = 0;
  const uint32_t tid = threadIdx.x;
  const uint64_t *words = reinterpret_cast<const uint64_t *>(payload);
  const uint64_t nitems = (nseg + kVarGroup - 1) / kVarGroup;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  auto issue = [&](uint64_t item, int which) {  // warp 0 only
    const uint32_t lane = tid & 31;
    const uint64_t s0 = item * kVarGroup;
    const uint32_t cnt = (uint32_t)umin64(kVarGroup, nseg - s0);
    VarStage &m = meta[which];
    uint64_t o = 0;
    if (lane <= cnt) o = __ldg(offsets + s0 + lane);  // offsets[s0 .. s0 + cnt]
    if (lane < cnt) m.off[lane] = o;
    if (lane <= cnt) m.st[lane] = s0 + lane < nseg ? __ldg(starts + s0 + lane) : n;
    const uint64_t o0 = __shfl_sync(0xffffffffu, o, 0), o1 = __shfl_sync(0xffffffffu, o, cnt);
    if (lane == 0) {
      const uint64_t g0 = o0 & ~15ull, g1 = (o1 + 8 + 15) & ~15ull;  // +8: field reads touch one word past a body
      const uint64_t bytes = g1 - g0;
      m.gbase = g0;
      m.cnt = cnt;
      m.direct = bytes > bufcap;
      if (!m.direct) {
        mbar_arrive_tx(&bar[which], (uint32_t)bytes);
        bulk_g2s(vstage + (size_t)which * bufcap, payload + g0, (uint32_t)bytes, &bar[which]);
      } else {
        mbar_arrive(&bar[which]);
      }
    }
  };
  uint64_t item = blockIdx.x;
  if (tid < 32 && item < nitems) issue(item, 0);
  uint32_t ph0 = 0, ph1 = 0;
  for (int it = 0; item < nitems; item += gridDim.x, ++it) {
    const int cur = it & 1;
    const bool has_next = item + gridDim.x < nitems;
    if (tid < 32 && has_next) issue(item + gridDim.x, cur ^ 1);
    const bool ok = mbar_wait_bounded(&bar[cur], cur ? ph1 : ph0);
    if (cur) ph1 ^= 1;
    else ph0 ^= 1;
    if (ok) {  // a thread whose wait gave up touches neither the buffer nor the output
      const VarStage &m = meta[cur];
      const uint8_t *sb = vstage + (size_t)cur * bufcap;
      const uint32_t lane = tid & 31;
      for (uint32_t g = tid >> 5; g < m.cnt; g += blockDim.x >> 5) {  // one warp per segment
        const uint64_t st = m.st[g], off = m.off[g];
        const uint32_t len = (uint32_t)(m.st[g + 1] - st);
        bool staged = false;
        if (!m.direct) {
          const uint32_t hoff = (uint32_t)(off - m.gbase);
          const uint8_t *hb = sb + hoff;
          const uint32_t start = hb[0] | (uint32_t)hb[1] << 8 | (uint32_t)hb[2] << 16 | (uint32_t)hb[3] << 24;
          const uint32_t l = hb[4];
          if (l >= 1 && l <= 32 && (uint64_t)start == st) {
            uint64_t t0w = 0;
            uint32_t slw = 0;
  #pragma unroll
            for (int j = 0; j < 8; ++j) t0w |= (uint64_t)hb[5 + j] << (8 * j);
  #pragma unroll
            for (int j = 0; j < 4; ++j) slw |= (uint32_t)hb[13 + j] << (8 * j);
            BlockHdr h;
            h.l = l;
            h.a0 = __longlong_as_double((long long)t0w);
            h.a1 = (double)__uint_as_float(slw);
            h.a2 = 0;
            h.base = 0;
            h.body_bit = (uint64_t)(hoff + 17) * 8;
            if (fabs(h.a0) + fabs(h.a1) * __uint2double_rn(len) < 4611686018427387904.0) {
              mark_nonneg<kLinear>(h, len);
              const int32_t kstart = -(int32_t)((reinterpret_cast<uintptr_t>(out + st) & 31) / 8);
              acc += decode_narrow<uint64_t, kLinear, true, true, 32, SUM>(h, false, reinterpret_cast<const uint32_t *>(sb),
                                                                           out, st, 0, len, kstart);
              staged = true;
            }
          }
        }
        if (!staged && SUM) {
          const SegHdr h = parse_seg(payload, off);
          for (uint32_t k = lane; k < len; k += 32) acc += seg_value(words, h, k);
        } else if (!staged) {
          const SegHdr h = parse_seg(payload, off);
          if (h.start != st || (h.l > 64 && h.l != 126 && h.l != 127)) {
            if (lane == 0) atomicOr(error, kErrBadHeader);
          } else {
            const uint32_t c = h.l == 127 ? 1 : h.l == 126 ? 2 : len;
            for (uint32_t k = lane; k < c && k < len; k += 32) __stcs(out + st + k, seg_value(words, h, k));
          }
        }
      }
    }
    // Everyone is done with this buffer before it is refilled; a wait that gave up in
    // any thread ends the CTA's work in all of them together.
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicOr(error, kErrTimeout);
        if (has_next) mbar_wait_bounded(&bar[cur ^ 1], cur ? ph0 : ph1);  // let our own copy in flight land
      }
      return;
    }
  }
  if (SUM) {
    acc = (uint64_t)block_reduce<5>((u128)acc, red);
    if (tid == 0) atomicAdd(reinterpret_cast<unsigned long long *>(d_sum), (unsigned long long)acc);
  }
}

// Launches varlen_decode_kernel<SUM> with its staging buffers.
template <bool SUM>
static cudaError_t launch_varlen_staged(const uint8_t *payload, const uint64_t *offsets, const uint64_t *starts,
                                        uint64_t nseg, uint64_t n, uint64_t *out, uint32_t *err, uint64_t *d_sum,
                                        cudaStream_t st) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int smem = (int)(2 * kVarStageBytes);
  cudaFuncSetAttribute(varlen_decode_kernel<SUM>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, varlen_decode_kernel<SUM>, 256, smem);
  const uint64_t nitems = (nseg + kVarGroup - 1) / kVarGroup;
  const unsigned grid = (unsigned)umin64(nitems, (uint64_t)sms * (uint64_t)(per_sm > 0 ? per_sm : 1));
  varlen_decode_kernel<SUM><<<grid, 256, smem, st>>>(payload, offsets, starts, nseg, n, out, kVarStageBytes, err, d_sum);
  return cudaGetLastError();
}

// Random access (randomdecodeArray8, :636-698; the raw case indexes inside the
// segment): the segment is the last one whose start is <= the index.  Every CTA
// keeps a sample of the start array (every stride-th start, at most kVarSamples)
// in shared memory; a lookup searches the sample there and then only its
// stride-wide window of the start array in global memory.  Each thread carries
// kVarQ lookups through the search level by level, so their loads are in flight
// together.
constexpr uint32_t kVarSamples = 4096, kVarQ = 4;
__global__ void __launch_bounds__(256) varlen_gather_kernel(const uint8_t *payload, const uint64_t *offsets,
                                                            const uint64_t *starts, uint64_t nseg, uint64_t n,
                                                            const uint64_t *idx, uint64_t m, uint64_t *out,
                                                            uint32_t *error) {
  __shared__ uint64_t samp[kVarSamples];
  const uint64_t *words = reinterpret_cast<const uint64_t *>(payload);
  const uint64_t stride = (nseg + kVarSamples - 1) / kVarSamples;
  const uint32_t ns = (uint32_t)((nseg + stride - 1) / stride);
  for (uint32_t i = threadIdx.x; i < ns; i += blockDim.x) samp[i] = __ldg(starts + (uint64_t)i * stride);
  __syncthreads();
  const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < m; i0 += T * kVarQ) {
    uint64_t g[kVarQ], lo[kVarQ], len[kVarQ];
    bool live[kVarQ];
#pragma unroll
    for (uint32_t q = 0; q < kVarQ; ++q) {
      const uint64_t i = i0 + q * T;
      live[q] = i < m;
      g[q] = live[q] ? __ldg(idx + i) : 0;
      if (live[q] && g[q] >= n) {
        out[i] = 0;
        atomicOr(error, kErrBadIndex);
        live[q] = false;
      }
      // sample: largest j with samp[j] <= g (samp[0] = 0)
      uint32_t base = 0, span = ns;
      while (span > 1) {
        const uint32_t half = span / 2;
        base = samp[base + half] <= g[q] ? base + half : base;
        span -= half;
      }
      lo[q] = (uint64_t)base * stride;
      len[q] = umin64(stride, nseg - lo[q]);
    }
    // window: largest s in [lo, lo + len) with starts[s] <= g, all lookups one level at a time
    for (uint64_t span = stride; span > 1; span -= span / 2) {
#pragma unroll
      for (uint32_t q = 0; q < kVarQ; ++q) {
        if (len[q] > 1) {
          const uint64_t half = len[q] / 2;
          lo[q] = __ldg(starts + lo[q] + half) <= g[q] ? lo[q] + half : lo[q];
          len[q] -= half;
        }
      }
    }
    SegHdr h[kVarQ];
#pragma unroll
    for (uint32_t q = 0; q < kVarQ; ++q)
      if (live[q]) h[q] = parse_seg(payload, __ldg(offsets + lo[q]));
#pragma unroll
    for (uint32_t q = 0; q < kVarQ; ++q)
      if (live[q]) out[i0 + q * T] = seg_value(words, h[q], (uint32_t)(g[q] - h[q].start));
  }
}

}  // namespace leco

using namespace leco;

namespace {
int verr(int code, const std::string &m) { return leco::record_error(code, m); }
}  // namespace

extern "C" {

uint64_t leco_varlen_max_payload_bytes(uint64_t n, uint64_t nseg) { return 8 * n + 32 * nseg + LECO_PAYLOAD_SLACK; }
uint64_t leco_varlen_workspace_bytes(uint64_t nseg) { return (nseg * 8 + 255) / 256 * 256 + 256 + (nseg * 16 + 255) / 256 * 256; }
uint64_t leco_varlen_max_segment(void) { return kVarlenMaxSeg; }

int leco_varlen_encode(const uint64_t *d_values, uint64_t n, const uint64_t *d_starts, uint64_t nseg, uint32_t max_segment_len,
                       int fit_mode, uint8_t *d_payload, uint64_t payload_cap, uint64_t *d_offsets, void *d_workspace,
                       uint64_t workspace_bytes, leco_stream_t stream) {
  if (!d_values || !d_starts || !nseg || !n || !d_payload || !d_offsets || !d_workspace)
    return verr(LECO_ERR_ARG, "leco_varlen_encode: null pointer or empty column");
  if (!max_segment_len) max_segment_len = kVarlenMaxSeg;
  if (max_segment_len > kVarlenMaxSeg)
    return verr(LECO_ERR_UNSUPPORTED, "leco_varlen_encode: segments longer than 16384 values are not supported");
  if (workspace_bytes < leco_varlen_workspace_bytes(nseg)) return verr(LECO_ERR_ARG, "leco_varlen_encode: workspace too small");
  if (nseg > 0xffffffffull || n > 0xffffffffull) return verr(LECO_ERR_ARG, "leco_varlen_encode: segments start at 32-bit indices");
  uint32_t *err = nullptr;
  int rc = leco::device_error_word(&err);
  if (rc) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  uint8_t *ws = static_cast<uint8_t *>(d_workspace);
  const uint64_t status_bytes = (nseg * 8 + 255) / 256 * 256;
  const bool exact = fit_mode == LECO_FIT_EXACT;
  double *models = reinterpret_cast<double *>(ws + status_bytes + 256);  // workspace: status, ticket, models
  VarArgs a{d_values, n, d_starts, nseg, d_payload, payload_cap, d_offsets, reinterpret_cast<uint64_t *>(ws),
            reinterpret_cast<uint32_t *>(ws + status_bytes), err, exact, max_segment_len, exact ? nullptr : models};
  cudaError_t e = cudaMemsetAsync(ws, 0, status_bytes + 256, st);
  if (e == cudaSuccess && !exact) varlen_seq_fit_kernel<<<(unsigned)((nseg + 127) / 128), 128, 0, st>>>(d_values, n, d_starts, nseg, models);
  const int smem = 8 * max_segment_len + (max_segment_len / 32 + 9) * 4;
  if (e == cudaSuccess && smem > 48 * 1024)
    e = cudaFuncSetAttribute(varlen_encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess) varlen_encode_kernel<<<(unsigned)nseg, 128, smem, st>>>(a);  // 128 threads: more segments in flight per SM
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? LECO_OK : verr(LECO_ERR_CUDA, std::string("leco_varlen_encode: ") + cudaGetErrorString(e));
}

int leco_varlen_decode(const uint8_t *d_payload, const uint64_t *d_offsets, const uint64_t *d_starts, uint64_t nseg,
                       uint64_t n, uint64_t *d_out, leco_stream_t stream) {
  if (!d_payload || !d_offsets || !d_starts || !d_out || !nseg) return verr(LECO_ERR_ARG, "leco_varlen_decode: null pointer");
  if (reinterpret_cast<uintptr_t>(d_out) & 7)  // values are stored as 32-byte vectors
    return verr(LECO_ERR_ARG, "leco_varlen_decode: d_out must be 8-byte aligned");
  uint32_t *err = nullptr;
  int rc = leco::device_error_word(&err);
  if (rc) return rc;
  const cudaError_t e = launch_varlen_staged<false>(d_payload, d_offsets, d_starts, nseg, n, d_out, err, nullptr,
                                                     reinterpret_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? LECO_OK : verr(LECO_ERR_CUDA, std::string("leco_varlen_decode: ") + cudaGetErrorString(e));
}

int leco_varlen_gather(const uint8_t *d_payload, const uint64_t *d_offsets, const uint64_t *d_starts, uint64_t nseg,
                       uint64_t n, const uint64_t *d_idx, uint64_t m, uint64_t *d_out, leco_stream_t stream) {
  if (!d_payload || !d_offsets || !d_starts || !nseg || (m && (!d_idx || !d_out)))
    return verr(LECO_ERR_ARG, "leco_varlen_gather: null pointer");
  if (!m) return LECO_OK;
  uint32_t *err = nullptr;
  int rc = leco::device_error_word(&err);
  if (rc) return rc;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const unsigned grid = (unsigned)umin64((m + 256 * kVarQ - 1) / (256 * kVarQ), (uint64_t)sms * 4);
  varlen_gather_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(d_payload, d_offsets, d_starts, nseg, n,
                                                                                d_idx, m, d_out, err);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LECO_OK : verr(LECO_ERR_CUDA, std::string("leco_varlen_gather: ") + cudaGetErrorString(e));
}

int leco_varlen_sum(const uint8_t *d_payload, const uint64_t *d_offsets, const uint64_t *d_starts, uint64_t nseg,
                    uint64_t n, uint64_t *d_sum, leco_stream_t stream) {
  if (!d_payload || !d_offsets || !d_starts || !nseg || !d_sum) return verr(LECO_ERR_ARG, "leco_varlen_sum: null pointer");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(d_sum, 0, 8, st);
  uint32_t *err = nullptr;
  int rc = leco::device_error_word(&err);
  if (rc) return rc;
  if (e == cudaSuccess) e = launch_varlen_staged<true>(d_payload, d_offsets, d_starts, nseg, n, nullptr, err, d_sum, st);
  return e == cudaSuccess ? LECO_OK : verr(LECO_ERR_CUDA, std::string("leco_varlen_sum: ") + cudaGetErrorString(e));
}

}  // extern "C"
