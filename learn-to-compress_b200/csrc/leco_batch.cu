// leco_batch.cu -- batch engine: thousands of columns of uneven length, mixed
// uint32/uint64 and mixed LeCo/FOR/Delta/poly codecs, encoded and decoded by
// one persistent launch per pass.
//
// Work queue: the batch's blocks are listed column by column as work items of
// 256/G consecutive blocks, G being the column's threads per block (32, 64, 128
// or 256): one block per item for G = 256, eight for G = 32 (one warp each).
// Every CTA (256 threads) of a persistent grid takes the next item from an atomic
// ticket and runs the per-block encoder or decoder instance for that column's
// codec, value type, G and unroll depth in each of its 256/G groups.  Items
// are handed out in order and every CTA of the grid is resident, so the
// encoder's per-column look-back (byte offsets) only ever waits on blocks that
// are already being processed.
//
// The reference has no counterpart: its drivers loop over blocks of one column
// (experiments/leco_int_fix_template.cpp:111-127, :145-153).  The per-column
// path (leco_batch_*_per_column) is what a caller of leco_encode / leco_decode
// does without the batch engine, kept as the baseline.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "leco_batch.cuh"

namespace leco {

// Sequential reference fits for every block of the columns that need them, one warp
// per 32 consecutive blocks of the batch (lane j: block g0 + j, whatever its column):
// each step the warp loads 32 consecutive values of each of its blocks (one row per
// block, coalesced; u32 and u64 rows mix) into shared memory while the next step's
// values are already in flight to registers, and lane j adds its block's values to
// its running sums in order -- the reference's loop (lr.h:72-77; Y sums of
// polynomial_regression_internals.hpp:129-137), as seq_fit_tiled_kernel does for one
// column.  A full step's conversions and products are taken before its adds.  (One
// thread per block with its own loads waited ~50 ns per value on each load.)
__global__ void __launch_bounds__(128) batch_seq_fit_kernel(BatchArgs B) {
  __shared__ uint64_t tile[4][32][33];
  __shared__ const uint8_t *row_ptr[4][32];
  __shared__ uint32_t row_len[4][32], row_s[4][32];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint64_t g0 = ((uint64_t)blockIdx.x * 4 + w) * 32, gb = g0 + lane;
  if (g0 >= B.total) return;
  uint32_t len = 0, s = 8, bs = 1;
  int codec = kLinear;
  const uint8_t *vals = nullptr;
  const double *polyX = nullptr;
  double *model = nullptr;
  if (gb < B.total) {
    const uint32_t ci = find_column(B.prefix, B.ncols, gb);
    const DevCol &c = B.cols[ci];
    if (c.seq) {
      const uint64_t b = gb - __ldg(B.prefix + ci);
      len = (uint32_t)umin64(c.bs, c.n - b * c.bs);
      s = (uint32_t)c.dtype;
      bs = c.bs;
      codec = c.codec;
      vals = reinterpret_cast<const uint8_t *>(c.values) + b * c.bs * s;
      polyX = c.polyX;
      model = B.models + gb * 3;
    }
  }
  row_ptr[w][lane] = vals;
  row_len[w][lane] = len;
  row_s[w][lane] = s;
  const bool poly = codec == kPoly2;
  const bool any_poly = __any_sync(0xffffffffu, poly && len);
  const uint32_t maxlen = __reduce_max_sync(0xffffffffu, len);
  uint64_t nxt[32];
  auto fetch = [&](uint32_t t0) {
    const uint32_t i = t0 + lane;
#pragma unroll
    for (int r = 0; r < 32; ++r) {
      const uint32_t lr = row_len[w][r];
      uint64_t v = 0;
      if (i < lr) {
        const uint8_t *vr = row_ptr[w][r];
        v = row_s[w][r] == 8 ? __ldg(reinterpret_cast<const uint64_t *>(vr) + i)
                             : (uint64_t)__ldg(reinterpret_cast<const uint32_t *>(vr) + i);
      }
      nxt[r] = v;
    }
  };
  __syncwarp();
  double s0 = 0, s1 = 0, s2 = 0;  // linear: sumy sumxy; poly: Y0 Y1 Y2
  if (maxlen) fetch(0);
  for (uint32_t t0 = 0; t0 < maxlen; t0 += 32) {
#pragma unroll
    for (int r = 0; r < 32; ++r) tile[w][r][lane] = nxt[r];
    __syncwarp();
    if (t0 + 32 < maxlen) fetch(t0 + 32);
    const uint32_t cnt = len > t0 ? (len - t0 < 32 ? len - t0 : 32) : 0;
    const double dt0 = u32_to_double_fp64(t0);
    if (cnt == 32) {
      double yv[32];
#pragma unroll
      for (int c = 0; c < 32; ++c) yv[c] = __ull2double_rn(tile[w][lane][c]);  // a u32 value converts the same way
      if (!any_poly) {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          s0 = __dadd_rn(s0, yv[c]);
          s1 = __dadd_rn(s1, __dmul_rn(__dadd_rn(dt0, (double)c), yv[c]));  // i = t0 + c exactly
        }
      } else {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const double di = __dadd_rn(dt0, (double)c);
          s0 = __dadd_rn(s0, yv[c]);  // the reference's 1.0 * y is y
          s1 = __dadd_rn(s1, __dmul_rn(di, yv[c]));
          s2 = __dadd_rn(s2, __dmul_rn(__dmul_rn(di, di), yv[c]));
        }
      }
    } else {
      for (uint32_t c = 0; c < cnt; ++c) {
        const double di = __dadd_rn(dt0, __uint2double_rn(c)), yi = __ull2double_rn(tile[w][lane][c]);
        s0 = __dadd_rn(s0, yi);
        s1 = __dadd_rn(s1, __dmul_rn(di, yi));
        if (poly) s2 = __dadd_rn(s2, __dmul_rn(__dmul_rn(di, di), yi));
      }
    }
    __syncwarp();
  }
  if (!len) return;
  if (poly) store_seq_model<kPoly2>(model, s0, s1, s2, len, bs, polyX);
  else store_seq_model<kLinear>(model, s0, s1, s2, len, bs, polyX);
}

}  // namespace leco

using namespace leco;

struct leco_batch {
  std::vector<leco_column_desc> cols;
  std::vector<uint64_t> prefix;
  int fit_mode = LECO_FIT_REFERENCE;
  bool any_seq = false;
  int device = 0;
  DevCol *d_cols = nullptr;
  uint64_t *d_prefix = nullptr;
  uint64_t *d_items = nullptr;
  uint64_t nitems = 0;
  uint8_t *d_ws = nullptr;  // status [total] | ticket | models [total*3]
  uint64_t ws_bytes = 0, status_bytes = 0, models_off = 0;
  uint32_t enc_smem = 0;
  int enc_grid = 0, dec_grid = 0;
  uint32_t *err = nullptr;               // library error word on this device
  cudaStream_t capture_stream = nullptr;  // graphs are captured here (the caller's stream may be the legacy default stream)
  cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
};

namespace {

// Shared memory one work item may take (the CTA limit is 227 KB).
constexpr uint32_t kBatchMaxSmem = 200 * 1024;

int berr(int code, const std::string &m) { return leco::record_error(code, m); }

bool needs_seq(int codec, int dtype, uint32_t bs, int fit_mode) {
  if (fit_mode != LECO_FIT_REFERENCE) return false;
  if (codec == kLinear) return !(dtype == LECO_U32 && bs <= 2048);
  return codec == kPoly2;
}

BatchArgs args_of(const leco_batch *b, uint32_t *err) {
  BatchArgs B;
  B.cols = b->d_cols;
  B.prefix = b->d_prefix;
  B.items = b->d_items;
  B.nitems = b->nitems;
  B.ncols = (uint32_t)b->cols.size();
  B.total = b->prefix.back();
  B.status = reinterpret_cast<uint64_t *>(b->d_ws);
  B.ticket = reinterpret_cast<unsigned long long *>(b->d_ws + b->status_bytes);
  B.models = reinterpret_cast<double *>(b->d_ws + b->models_off);
  B.error = err;
  return B;
}

}  // namespace

extern "C" {

int leco_batch_create(const leco_column_desc *h_cols, uint32_t ncols, int fit_mode, leco_batch **out) {
  if (!h_cols || !ncols || !out) return berr(LECO_ERR_ARG, "leco_batch_create: null pointer or empty batch");
  if (fit_mode != LECO_FIT_REFERENCE && fit_mode != LECO_FIT_EXACT) return berr(LECO_ERR_ARG, "leco_batch_create: bad fit_mode");
  auto *b = new leco_batch();
  b->cols.assign(h_cols, h_cols + ncols);
  b->fit_mode = fit_mode;
  cudaGetDevice(&b->device);
  b->prefix.resize(ncols + 1);
  std::vector<DevCol> dc(ncols);
  uint64_t total = 0;
  uint32_t max_smem = 0;
  for (uint32_t i = 0; i < ncols; ++i) {
    const leco_column_desc &c = h_cols[i];
    if (c.codec < kLinear || c.codec > kPoly2 || (c.dtype != 4 && c.dtype != 8) || !c.block_size ||
        c.block_size > LECO_MAX_BLOCK || !c.n || !c.d_payload || !c.d_offsets) {
      delete b;
      return berr(LECO_ERR_ARG, "leco_batch_create: bad descriptor for column " + std::to_string(i));
    }
    b->prefix[i] = total;
    total += leco_num_blocks(c.n, c.block_size);
    DevCol &d = dc[i];
    d.codec = c.codec;
    d.dtype = c.dtype;
    d.bs = c.block_size;
    d.seq = needs_seq(c.codec, c.dtype, c.block_size, fit_mode);
    b->any_seq |= d.seq != 0;
    d.n = c.n;
    d.values = c.d_values;
    d.out = c.d_out;
    d.payload = c.d_payload;
    d.payload_cap = c.payload_cap;
    d.offsets = c.d_offsets;
    d.dir = c.d_dir;
    for (int k = 0; k < 10; ++k) d.polyX[k] = 0;
    if (c.codec == kPoly2) {
      const uint64_t nb = leco_num_blocks(c.n, c.block_size);
      poly2_x_sums((uint32_t)std::min<uint64_t>(c.n, c.block_size), d.polyX);
      poly2_x_sums((uint32_t)(c.n - (nb - 1) * c.block_size), d.polyX + 5);
    }
    d.group = c.group_threads ? c.group_threads : (c.block_size <= kWarpBlock ? 32u : 256u);
    d.unroll = c.unroll ? c.unroll : 2u;
    d.pad = 0;
    if ((d.group != 32 && d.group != 64 && d.group != 128 && d.group != 256) ||
        (d.unroll != 1 && d.unroll != 2 && d.unroll != 4)) {
      delete b;
      return berr(LECO_ERR_ARG, "leco_batch_create: column " + std::to_string(i) +
                                    ": group_threads must be 0, 32, 64, 128 or 256 and unroll 0, 1, 2 or 4");
    }
    d.slice = (enc_smem_bytes(c.block_size, (uint32_t)c.dtype) + 15) / 16 * 16;
    const uint32_t item_smem = d.slice * (256 / d.group);
    if (item_smem > kBatchMaxSmem) {
      delete b;
      return berr(LECO_ERR_ARG, "leco_batch_create: column " + std::to_string(i) + ": " + std::to_string(256 / d.group) +
                                    " groups of " + std::to_string(d.slice) + " bytes of shared memory exceed the " +
                                    std::to_string(kBatchMaxSmem) + " a CTA may use");
    }
    max_smem = std::max(max_smem, item_smem);
  }
  // work items: (column << 32) | first block, 256/G blocks per item
  std::vector<uint64_t> items;
  for (uint32_t i = 0; i < ncols; ++i) {
    const uint64_t nb = leco_num_blocks(h_cols[i].n, h_cols[i].block_size);
    const uint64_t step = 256 / dc[i].group;
    for (uint64_t blk = 0; blk < nb; blk += step) items.push_back(((uint64_t)i << 32) | blk);
  }
  b->nitems = items.size();
  b->prefix[ncols] = total;
  if (total > 0xffffffffull) {
    delete b;
    return berr(LECO_ERR_ARG, "leco_batch_create: more than 2^32 blocks");
  }
  b->status_bytes = (total * 8 + 255) / 256 * 256;
  b->models_off = b->status_bytes + 256;
  b->ws_bytes = b->models_off + (b->any_seq ? (total * 24 + 255) / 256 * 256 : 0);
  b->enc_smem = max_smem;
  cudaError_t e = cudaMalloc(&b->d_cols, ncols * sizeof(DevCol));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_prefix, (ncols + 1) * sizeof(uint64_t));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_ws, b->ws_bytes);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_cols, dc.data(), ncols * sizeof(DevCol), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_prefix, b->prefix.data(), (ncols + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_items, std::max<size_t>(1, items.size()) * sizeof(uint64_t));
  if (e == cudaSuccess) e = cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(uint64_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && leco::device_error_word(&b->err)) e = cudaErrorUnknown;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess && max_smem > 48 * 1024)
    e = cudaFuncSetAttribute(batch_encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
  int sms = 148, per_enc = 1, per_dec = 1;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_enc, batch_encode_kernel, 256, max_smem);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_dec, batch_decode_kernel, 256, 0);
  if (e != cudaSuccess || per_enc < 1 || per_dec < 1) {
    leco_batch_destroy(b);
    return berr(e != cudaSuccess ? LECO_ERR_CUDA : LECO_ERR_ARG,
                std::string("leco_batch_create: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "no resident CTA fits"));
  }
  // every CTA of the persistent grid must be resident (the look-back waits on them)
  b->enc_grid = (int)std::min<uint64_t>(b->nitems, (uint64_t)sms * per_enc);
  b->dec_grid = (int)std::min<uint64_t>(b->nitems, (uint64_t)sms * per_dec);
  *out = b;
  return LECO_OK;
}

int leco_batch_destroy(leco_batch *b) {
  if (!b) return LECO_OK;
  for (auto &g : b->graph)
    if (g) cudaGraphExecDestroy(g);
  if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
  if (b->d_cols) cudaFree(b->d_cols);
  if (b->d_prefix) cudaFree(b->d_prefix);
  if (b->d_items) cudaFree(b->d_items);
  if (b->d_ws) cudaFree(b->d_ws);
  delete b;
  return LECO_OK;
}

uint64_t leco_batch_total_blocks(const leco_batch *b) { return b ? b->prefix.back() : 0; }

int leco_batch_encode(leco_batch *b, leco_stream_t stream) {
  if (!b) return berr(LECO_ERR_ARG, "leco_batch_encode: null batch");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const BatchArgs B = args_of(b, b->err);
  cudaError_t e = cudaMemsetAsync(b->d_ws, 0, b->status_bytes + 256, st);  // look-back words + ticket
  if (e == cudaSuccess && b->any_seq)
    batch_seq_fit_kernel<<<(unsigned)((B.total + 127) / 128), 128, 0, st>>>(B);  // four warps of 32 blocks
  if (e == cudaSuccess) batch_encode_kernel<<<b->enc_grid, 256, b->enc_smem, st>>>(B);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? LECO_OK : berr(LECO_ERR_CUDA, std::string("leco_batch_encode: ") + cudaGetErrorString(e));
}

int leco_batch_decode(leco_batch *b, leco_stream_t stream) {
  if (!b) return berr(LECO_ERR_ARG, "leco_batch_decode: null batch");
  for (const auto &c : b->cols) {
    if (!c.d_out) return berr(LECO_ERR_ARG, "leco_batch_decode: a column has no output buffer");
    if (reinterpret_cast<uintptr_t>(c.d_out) & (uint64_t)(c.dtype - 1))  // values are stored as 16/32-byte vectors
      return berr(LECO_ERR_ARG, "leco_batch_decode: a column's output buffer is not aligned to its value size");
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const BatchArgs B = args_of(b, b->err);
  cudaError_t e = cudaMemsetAsync(b->d_ws + b->status_bytes, 0, 256, st);  // ticket
  if (e == cudaSuccess) batch_decode_kernel<<<b->dec_grid, 256, 0, st>>>(B);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? LECO_OK : berr(LECO_ERR_CUDA, std::string("leco_batch_decode: ") + cudaGetErrorString(e));
}

int leco_batch_run_graph(leco_batch *b, int passes, leco_stream_t stream) {
  if (!b || passes < 1 || passes > 3) return berr(LECO_ERR_ARG, "leco_batch_run_graph: passes must be 1 (encode), 2 (decode) or 3");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (!b->graph[passes]) {
    cudaGraph_t g = nullptr;
    cudaStream_t cs = b->capture_stream;
    leco_stream_t lcs = reinterpret_cast<leco_stream_t>(cs);
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return berr(LECO_ERR_CUDA, std::string("leco_batch_run_graph: ") + cudaGetErrorString(e));
    int rc = LECO_OK;
    if (passes & 1) rc = leco_batch_encode(b, lcs);
    if (!rc && (passes & 2)) rc = leco_batch_decode(b, lcs);
    e = cudaStreamEndCapture(cs, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph[passes], g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) return berr(LECO_ERR_CUDA, std::string("leco_batch_run_graph: ") + cudaGetErrorString(e));
  }
  cudaError_t e = cudaGraphLaunch(b->graph[passes], st);
  return e == cudaSuccess ? LECO_OK : berr(LECO_ERR_CUDA, std::string("leco_batch_run_graph: ") + cudaGetErrorString(e));
}

// Baseline: one leco_encode call per column (the batch's workspace is reused;
// each call resets it).
int leco_batch_encode_per_column(leco_batch *b, leco_stream_t stream) {
  if (!b) return berr(LECO_ERR_ARG, "null batch");
  for (const auto &c : b->cols) {
    int rc = leco_encode(c.codec, c.dtype, c.d_values, c.n, c.block_size, b->fit_mode, c.d_payload, c.payload_cap,
                         c.d_offsets, c.d_dir, b->d_ws, b->ws_bytes, stream);
    if (rc) return rc;
  }
  return LECO_OK;
}

int leco_batch_decode_per_column(leco_batch *b, leco_stream_t stream) {
  if (!b) return berr(LECO_ERR_ARG, "null batch");
  for (const auto &c : b->cols) {
    int rc = leco_decode(c.codec, c.dtype, c.d_payload, c.d_offsets, c.n, c.block_size, c.d_out, stream);
    if (rc) return rc;
  }
  return LECO_OK;
}

}  // extern "C"
