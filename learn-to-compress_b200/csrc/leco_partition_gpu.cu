// leco_partition_gpu.cu -- the variable-length segmentation of
// Leco_cost_merge_double_wo_round<uint64_t>::encodeArray8_int on the GPU.
//
// Same segmentation as the host partitioner (leco_partition.cpp) and the
// reference (headers/piecewise_cost_merge_integer_template_double_wo_round.h:283-570,
// cost model newsegment_size :68-131, cal_bits :274-281, fit lr.h:66-85): coarse
// blocks cut as the reference driver does (experiments/leco_double_int_template_wo_round.cpp:85-91),
// inside each
//   1. one-point segments carrying the first difference to their successor and the
//      bit class of the second difference; for each bit class from the smallest up,
//      a segment of that class is merged with its right neighbour when the merged
//      width costs less than `delta` more bits, then grows left and right greedily;
//   2. pairwise merges while the fitted byte size of a pair is below the sum of the
//      two, pass after pass, until a pass saves less than 0.01 % of the coarse
//      block's raw size.
// Both phases are sequential inside a coarse block (every step depends on the
// previous merge), so the parallelism is across coarse blocks: one thread per
// coarse block, persistent threads taking blocks by ticket, each with a private
// scratch slot in global memory (the segment list of phase 1, then the segment
// starts and sizes of phase 2, merged in place).  Every FP64 step is the
// reference's, one rounding each (--fmad=false), so the segment starts are the
// host partitioner's bit for bit.
//
// Output: each coarse block's segment starts go to stage[B0 ...] (at most one per
// value) with their count; a scan of the counts and a gather compact them into the
// caller's starts array.
#include <algorithm>
#include <string>

#include "leco_device.cuh"
#include "leco_internal.h"

namespace leco {

constexpr int kPartThreads = 128;
constexpr int kPartHead = 0;
constexpr int kPartTail = -2;

// A segment of phase 1.  Its successor and bit class live apart, packed in one
// 32-bit word per segment ((next + 2) << 8 | class; class 255 = the reference's
// 10000 sentinel), because the per-class walks read only those: 4 bytes per step
// instead of the whole record.
struct PSeg {
  int32_t start, end, prev, pad;
  int64_t max_delta, min_delta, next_delta;
};
constexpr uint32_t kNoClass = 255;
__device__ __forceinline__ int lk_next(uint32_t w) { return (int)(w >> 8) - 2; }
__device__ __forceinline__ uint32_t lk_class(uint32_t w) { return w & 0xffu; }
__device__ __forceinline__ uint32_t lk_make(int next, uint32_t cls) { return ((uint32_t)(next + 2) << 8) | cls; }

__device__ __forceinline__ uint32_t bits64_d(uint64_t v) { return v ? 64u - (uint32_t)__clzll((long long)v) : 0u; }

// cal_bits(min, max) (…_double_wo_round.h:274-281): bits of ceil(|max - min| / 2) plus one.
__device__ __forceinline__ int cal_bits_d(int64_t mn, int64_t mx) {
  const int64_t diff = (int64_t)((uint64_t)mx - (uint64_t)mn);
  const int64_t ad = diff < 0 ? (int64_t)(0 - (uint64_t)diff) : diff;
  const int64_t range = f2i_x86(ceil(__ddiv_rn(__ll2double_rn(ad), 2.0)));
  return range ? (int)bits64_d((uint64_t)range) + 1 : 0;
}

// newsegment_size (…_double_wo_round.h:68-131) of segment [a, b]: the reference's
// sequential FP64 fit (lr.h:66-85), slope rounded to float, 128-bit prediction.
__device__ uint32_t segment_cost_d(const uint64_t *__restrict__ array, uint32_t a, uint32_t b) {
  if (a == b) return 9;
  if (b == a + 1) return 13;
  const int length = (int)(b - a + 1);
  double sumx = 0, sumy = 0, sumxy = 0, sumxx = 0;
  for (int i = 0; i < length; i++) {
    const double di = (double)i;
    const double y = __ull2double_rn(__ldg(array + a + i));
    sumx = __dadd_rn(sumx, di);
    sumy = __dadd_rn(sumy, y);
    sumxx = __dadd_rn(sumxx, __dmul_rn(di, di));
    sumxy = __dadd_rn(sumxy, __dmul_rn(di, y));
  }
  const double dm = (double)length;
  const double ccc = __dsub_rn(__dmul_rn(sumxy, dm), __dmul_rn(sumx, sumy));
  const double xxx = __dsub_rn(__dmul_rn(sumxx, dm), __dmul_rn(sumx, sumx));
  const double t1 = __ddiv_rn(ccc, xxx);
  const double t0 = __ddiv_rn(__dsub_rn(sumy, __dmul_rn(t1, sumx)), dm);
  const double slope = (double)__double2float_rn(t1);
  uint64_t maxr = 0;
  for (uint32_t j = 0; j < (uint32_t)length; j++) {
    const i128 pred = f2i128(__dadd_rn(t0, __dmul_rn(slope, __uint2double_rn(j))));
    const i128 y = (i128)__ldg(array + a + j);
    const uint64_t r = (uint64_t)(y > pred ? y - pred : pred - y);
    maxr = r > maxr ? r : maxr;
  }
  const uint32_t bits = maxr ? bits64_d(maxr) + 1 : 0;
  if (bits >= 64) return (uint32_t)(5 + 8ull * (uint64_t)length);
  uint64_t overhead = sizeof(float) + sizeof(double) + 5;
  if (bits) overhead += (uint64_t)ceil(__ddiv_rn(__uint2double_rn(bits * (uint32_t)length), 8.0));
  return (uint32_t)overhead;
}

struct PartitionArgs {
  const uint64_t *array;
  uint64_t n;
  uint32_t bs;       // coarse block size
  uint64_t nblocks;  // coarse blocks
  int overhead;      // merge penalty `delta` (bits)
  PSeg *segs;        // per slot: bs + 1 entries
  uint32_t *links;   // per slot: bs + 1 packed (next, class) words
  uint32_t *pidx;    // per slot: bs entries (segment starts, phase 2)
  uint32_t *psz;     // per slot: bs entries (segment sizes, phase 2)
  uint32_t *stage;   // n entries: block b's starts at [b*bs, ...)
  uint32_t *count;   // nblocks entries
  uint32_t *ticket;
};

// Segmentation of coarse block [B0, B0 + len) by one thread.
__device__ void partition_block_d(const PartitionArgs &a, uint32_t B0, uint32_t len, PSeg *s, uint32_t *lk, uint32_t *idx,
                                  uint32_t *sz, uint32_t *out, uint32_t *count) {
  const uint64_t *array = a.array;
  if (len < 2) {  // the reference needs two points per coarse block (it reads array[B0 + 1])
    out[0] = B0;
    *count = 1;
    return;
  }
  // ---- split: linked list of one-point segments (…:286-312) ----
  int ns = 0;
  s[ns] = PSeg{0, 0, -1, 0, 0, 0, 0};  // head
  lk[ns++] = lk_make(-1, kNoClass);
  int min_sb = 10000, max_sb = -1;
  int64_t delta_prev = (int64_t)(__ldg(array + B0 + 1) - __ldg(array + B0));
  int cur = kPartHead;
  for (uint32_t i = B0 + 1; i < B0 + len - 1; i++) {
    const int64_t delta = (int64_t)(__ldg(array + i + 1) - __ldg(array + i));
    const int sdb = cal_bits_d(delta_prev, delta);
    min_sb = min(min_sb, sdb);
    max_sb = max(max_sb, sdb);
    s[ns] = PSeg{(int32_t)i - 1, (int32_t)i - 1, cur, 0, 0, 0, delta_prev};
    lk[ns] = lk_make(-1, (uint32_t)sdb);
    lk[cur] = lk_make(ns, lk_class(lk[cur]));
    cur = ns++;
    delta_prev = delta;
  }
  s[ns] = PSeg{(int32_t)(B0 + len - 2), (int32_t)(B0 + len - 2), cur, 0, 0, 0, delta_prev};
  lk[ns] = lk_make(kPartTail, kNoClass);
  lk[cur] = lk_make(ns, lk_class(lk[cur]));
  ns++;
  const int overhead = a.overhead;

  // ---- merge by bit class (…:326-433) ----
  for (int aim = min_sb; aim <= max_sb; aim++) {
    int c = lk_next(lk[kPartHead]);
    while (c != kPartTail) {
      const uint32_t wc = lk[c];
      int n = lk_next(wc);
      if (n == kPartTail) break;
      if ((int)lk_class(wc) != aim) {
        c = n;
        continue;
      }
      PSeg sc = s[c];
      const PSeg sn = s[n];
      const uint32_t wn = lk[n];
      const int former = sc.start, start = sn.start, now = sn.end;
      const int lbo = cal_bits_d(sc.min_delta, sc.max_delta), rbo = cal_bits_d(sn.min_delta, sn.max_delta);
      const int64_t nmax = max(max(sc.max_delta, sn.max_delta), sc.next_delta);
      const int64_t nmin = min(min(sc.min_delta, sn.min_delta), sc.next_delta);
      const int nb = cal_bits_d(nmin, nmax);
      const int origin_cost = (start - former) * lbo + (now - start + 1) * rbo;
      const int merged_cost = nb * (now - former + 1);
      if (!(merged_cost - origin_cost < overhead)) {
        c = n;
        continue;
      }
      int cnext = lk_next(wn);
      uint32_t ccls = lk_class(wn);
      sc.end = now;
      if (cnext != kPartTail) s[cnext].prev = c;
      sc.next_delta = sn.next_delta;
      sc.max_delta = nmax;
      sc.min_delta = nmin;
      // grow left (never into the first segment of the block)
      int p = sc.prev;
      while (p != kPartHead && s[p].prev != kPartHead) {
        const PSeg sp = s[p];
        const int left = sp.start;
        const int64_t lmax = max(max(sp.max_delta, sc.max_delta), sp.next_delta);
        const int64_t lmin = min(min(sp.min_delta, sc.min_delta), sp.next_delta);
        const int bnew = cal_bits_d(lmin, lmax);
        const int ol = cal_bits_d(sp.min_delta, sp.max_delta), orr = cal_bits_d(sc.min_delta, sc.max_delta);
        const int oc = (sc.start - left) * ol + (sc.end - sc.start + 1) * orr;
        const int mc = bnew * (sc.end - left + 1);
        if (!(mc - oc < overhead)) break;
        sc.start = left;
        sc.prev = sp.prev;
        lk[sp.prev] = lk_make(c, lk_class(lk[sp.prev]));
        sc.min_delta = lmin;
        sc.max_delta = lmax;
        p = sc.prev;
      }
      // grow right (never into the last segment of the block)
      n = cnext;
      while (n != kPartTail) {
        const uint32_t wr = lk[n];
        if (lk_next(wr) == kPartTail) break;
        const PSeg sr = s[n];
        const int right = sr.end;
        const int64_t rmax = max(max(sr.max_delta, sc.max_delta), sc.next_delta);
        const int64_t rmin = min(min(sr.min_delta, sc.min_delta), sc.next_delta);
        const int bnew = cal_bits_d(rmin, rmax);
        const int ol = cal_bits_d(sc.min_delta, sc.max_delta), orr = cal_bits_d(sr.min_delta, sr.max_delta);
        const int oc = (right - sr.start + 1) * orr + (sr.start - sc.start) * ol;
        const int mc = bnew * (right - sc.start + 1);
        if (!(mc - oc < overhead)) break;
        sc.end = right;
        cnext = lk_next(wr);
        ccls = lk_class(wr);
        s[cnext].prev = c;  // cnext is not the tail: the loop stops before the last segment
        sc.max_delta = rmax;
        sc.min_delta = rmin;
        sc.next_delta = sr.next_delta;
        n = cnext;
      }
      s[c] = sc;
      lk[c] = lk_make(cnext, ccls);
      c = cnext;
    }
  }

  // ---- size-driven pairwise merge passes (…:439-483, merge :516-570), in place ----
  uint32_t m = 0;
  for (int c = lk_next(lk[kPartHead]); c != kPartTail; c = lk_next(lk[c])) idx[m++] = (uint32_t)s[c].start;
  const uint32_t endv = B0 + len;
  uint64_t total = 0;
  for (uint32_t i = 0; i < m; i++) {
    sz[i] = segment_cost_d(array, idx[i], (i + 1 < m ? idx[i + 1] : endv) - 1);
    total += sz[i];
  }
  for (;;) {
    const uint64_t before = total;
    uint64_t tnew = 0;
    uint32_t w = 0, k = 0;
    uint32_t start = idx[0];
    while (k < m) {
      if (k == m - 1) {
        const uint32_t z = sz[k];
        idx[w] = idx[k];
        sz[w++] = z;
        tnew += z;
        k++;
        break;
      }
      const uint32_t at2 = k + 2 < m ? idx[k + 2] : endv;
      const uint32_t init_cost = sz[k] + sz[k + 1];
      const uint32_t merge_cost = segment_cost_d(array, start, at2 - 1);
      if (init_cost > merge_cost) {
        idx[w] = start;
        sz[w++] = merge_cost;
        tnew += merge_cost;
        start = at2;
        k += 2;
      } else {
        const uint32_t at1 = idx[k + 1], z = sz[k];
        idx[w] = idx[k];
        sz[w++] = z;
        tnew += z;
        start = at1;
        k++;
      }
    }
    m = w;
    total = tnew;
    const uint64_t decline = before - total;  // unsigned, as in the reference
    const double pct = __ddiv_rn(__dmul_rn(__ull2double_rn(decline), 100.0), __dmul_rn((double)sizeof(uint64_t), (double)a.bs));
    if (!(decline > 0) || pct < 0.01) break;
  }
  for (uint32_t i = 0; i < m; i++) out[i] = idx[i];
  *count = m;
}

__global__ void __launch_bounds__(kPartThreads) partition_kernel(PartitionArgs a) {
  const uint64_t slot = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  PSeg *s = a.segs + slot * (a.bs + 1);
  uint32_t *lk = a.links + slot * (a.bs + 1);
  uint32_t *idx = a.pidx + slot * a.bs, *sz = a.psz + slot * a.bs;
  for (;;) {
    const uint64_t b = atomicAdd(a.ticket, 1u);
    if (b >= a.nblocks) return;
    const uint64_t B0 = b * a.bs;
    const uint32_t len = (uint32_t)(b == a.nblocks - 1 ? a.n - B0 : a.bs);
    partition_block_d(a, (uint32_t)B0, len, s, lk, idx, sz, a.stage + B0, a.count + b);
  }
}

// Exclusive scan of the per-block counts (one CTA, chunks of 1024), then each
// block's starts are copied to their place in the caller's array.
__global__ void __launch_bounds__(1024) count_scan_kernel(const uint32_t *count, uint64_t nb, uint64_t *base, uint64_t *total) {
  __shared__ uint64_t wsum[32];
  __shared__ uint64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint64_t c0 = 0; c0 < nb; c0 += 1024) {
    const uint64_t i = c0 + threadIdx.x;
    const uint64_t x = i < nb ? count[i] : 0;
    uint64_t inc = x;
    for (int d = 1; d < 32; d <<= 1) {
      const uint64_t y = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += y;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      const uint64_t v = wsum[lane];
      uint64_t vi = v;
      for (int d = 1; d < 32; d <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, vi, d);
        if (lane >= d) vi += y;
      }
      wsum[lane] = vi - v;
    }
    __syncthreads();
    if (i < nb) base[i] = carry + wsum[warp] + inc - x;
    __syncthreads();
    if (threadIdx.x == 1023) carry += wsum[31] + inc;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(256) starts_gather_kernel(const uint32_t *stage, const uint32_t *count, const uint64_t *base,
                                                            uint64_t nb, uint32_t bs, uint64_t *starts, uint64_t cap,
                                                            uint32_t *error) {
  for (uint64_t b = blockIdx.x; b < nb; b += gridDim.x) {
    const uint32_t c = count[b];
    const uint64_t o = base[b];
    for (uint32_t j = threadIdx.x; j < c; j += blockDim.x) {
      if (o + j < cap) starts[o + j] = stage[b * bs + j];
      else atomicOr(error, kErrCapacity);
    }
  }
}

static void part_layout(uint64_t n, uint32_t coarse_blocks, uint32_t &bs, uint64_t &nb, uint64_t &slots) {
  uint64_t b = n / coarse_blocks;
  if (!b) b = 1;
  bs = (uint32_t)b;
  nb = n / b;
  if (nb * b < n) nb++;
  slots = std::min<uint64_t>((nb + kPartThreads - 1) / kPartThreads, 148 * 4) * kPartThreads;
}

static uint64_t align256(uint64_t x) { return (x + 255) / 256 * 256; }

}  // namespace leco

using namespace leco;

extern "C" {

uint64_t leco_varlen_partition_workspace_bytes(uint64_t n, uint32_t coarse_blocks) {
  if (!coarse_blocks || n < 2) return 0;
  uint32_t bs;
  uint64_t nb, slots;
  part_layout(n, coarse_blocks, bs, nb, slots);
  return align256(slots * (bs + 1) * sizeof(PSeg)) + align256(slots * (bs + 1) * 4ull) + 2 * align256(slots * bs * 4ull) +
         align256(n * 4) +
         align256(nb * 4) + align256(nb * 8) + 256;
}

int leco_varlen_partition_device(const uint64_t *d_values, uint64_t n, uint32_t coarse_blocks, int64_t delta,
                                 uint64_t *d_starts, uint64_t starts_cap, uint64_t *d_nseg, void *d_ws, uint64_t ws_bytes,
                                 leco_stream_t stream) {
  if (!d_values || !d_starts || !d_nseg || !coarse_blocks || n < 2)
    return record_error(LECO_ERR_ARG, "leco_varlen_partition_device: need values (n >= 2), starts and a block count");
  if (n > 0xffffffffull) return record_error(LECO_ERR_ARG, "leco_varlen_partition_device: segments start at 32-bit indices");
  if (n / coarse_blocks >= (1ull << 24) - 4)
    return record_error(LECO_ERR_ARG, "leco_varlen_partition_device: coarse blocks of at most 2^24 - 5 values");
  if (!d_ws || ws_bytes < leco_varlen_partition_workspace_bytes(n, coarse_blocks) || (reinterpret_cast<uintptr_t>(d_ws) & 255))
    return record_error(LECO_ERR_ARG, "leco_varlen_partition_device: workspace must be leco_varlen_partition_workspace_bytes(), 256-byte aligned");
  uint32_t *err = nullptr;
  int rc = device_error_word(&err);
  if (rc) return rc;
  uint32_t bs;
  uint64_t nb, slots;
  part_layout(n, coarse_blocks, bs, nb, slots);
  uint8_t *w = static_cast<uint8_t *>(d_ws);
  PartitionArgs A;
  A.array = d_values;
  A.n = n;
  A.bs = bs;
  A.nblocks = nb;
  A.overhead = (int)delta;
  A.segs = reinterpret_cast<PSeg *>(w);
  w += align256(slots * (bs + 1) * sizeof(PSeg));
  A.links = reinterpret_cast<uint32_t *>(w);
  w += align256(slots * (bs + 1) * 4ull);
  A.pidx = reinterpret_cast<uint32_t *>(w);
  w += align256(slots * bs * 4ull);
  A.psz = reinterpret_cast<uint32_t *>(w);
  w += align256(slots * bs * 4ull);
  A.stage = reinterpret_cast<uint32_t *>(w);
  w += align256(n * 4);
  A.count = reinterpret_cast<uint32_t *>(w);
  w += align256(nb * 4);
  uint64_t *base = reinterpret_cast<uint64_t *>(w);
  w += align256(nb * 8);
  A.ticket = reinterpret_cast<uint32_t *>(w);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(A.ticket, 0, 4, st) != cudaSuccess) return record_error(LECO_ERR_CUDA, "leco_varlen_partition_device: memset");
  partition_kernel<<<(unsigned)(slots / kPartThreads), kPartThreads, 0, st>>>(A);
  count_scan_kernel<<<1, 1024, 0, st>>>(A.count, nb, base, d_nseg);
  starts_gather_kernel<<<(unsigned)std::min<uint64_t>(nb, 148 * 8), 256, 0, st>>>(A.stage, A.count, base, nb, bs, d_starts,
                                                                                   starts_cap, err);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return record_error(LECO_ERR_CUDA, std::string("leco_varlen_partition_device: ") + cudaGetErrorString(e));
  return LECO_OK;
}

}  // extern "C"
