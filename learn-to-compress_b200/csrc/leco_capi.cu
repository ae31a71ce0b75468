// leco_capi.cu -- the C ABI (include/leco.h): argument checks, workspace
// layout, launches, host-buffer pipelines and the per-block drop-in calls.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "leco_device.cuh"
#include "leco_internal.h"

namespace leco {

static thread_local std::string g_last_error;

static int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}
int record_error(int code, const std::string &msg) { return fail(code, msg); }

static int cuda_fail(cudaError_t e, const char *where) {
  return fail(LECO_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define LECO_CUDA(call)                                   \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
  } while (0)

// Library-wide device error word: a file-scope __device__ variable, so no
// allocation is needed.  Host code obtains its device address once per device.
__device__ uint32_t g_error_word;
static uint32_t *g_error_ptr[64];

static int error_ptr(uint32_t **p) {
  int dev = 0;
  LECO_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(LECO_ERR_ARG, "device ordinal out of range");
  if (!g_error_ptr[dev]) LECO_CUDA(cudaGetSymbolAddress((void **)&g_error_ptr[dev], g_error_word));
  *p = g_error_ptr[dev];
  return LECO_OK;
}

int device_error_word(uint32_t **p) { return error_ptr(p); }

static bool codec_ok(int codec) { return codec >= kLinear && codec <= kPoly2; }
// Codecs the read side (decode, random access, sum, directory, zone map, validation) accepts.
static bool codec_read_ok(int codec, int dtype) { return codec_ok(codec) || (codec == kLegacy && dtype == LECO_U32); }
static bool dtype_ok(int dtype) { return dtype == LECO_U32 || dtype == LECO_U64; }
// Codecs the encoder writes: the four block codecs, and the legacy format for u32.
static bool codec_write_ok(int codec, int dtype) { return codec_read_ok(codec, dtype); }

void poly2_x_sums(uint32_t N, double X[5]) {
  for (int k = 0; k < 5; ++k) {
    double acc = 0;
    for (uint32_t j = 0; j < N; ++j) {
      double xr = 1.0, xj = (double)j;
      if (k >= 1) xr = xj;
      for (int d = 2; d <= k; ++d) xr = xr * xj;
      acc += xr;
    }
    X[k] = acc;
  }
}

// Workspace layout of leco_encode.
struct EncWs {
  uint64_t status_off, ticket_off, models_off, total;
};
static EncWs enc_ws(uint64_t nb, bool seq) {
  EncWs w;
  w.status_off = 0;
  w.ticket_off = (nb * 8 + 255) / 256 * 256;
  w.models_off = w.ticket_off + 256;
  w.total = w.models_off + (seq ? (nb * 24 + 255) / 256 * 256 : 0);
  return w;
}
// Whether LECO_FIT_REFERENCE needs the sequential fit kernel: for u32 linear
// blocks of at most 2048 values every partial FP64 sum of lr.h:72-77 is an
// exact integer, so the exact in-kernel moments reproduce it bit for bit.
static bool needs_seq_fit(int codec, int dtype, uint32_t bs, int fit_mode) {
  if (fit_mode != LECO_FIT_REFERENCE) return false;
  if (codec == kLinear || codec == kLegacy) return !(dtype == LECO_U32 && bs <= 2048);
  return codec == kPoly2;
}

// Chunk-relative offsets on the device (leco_decode_host): off[0..cnt] -= base.
__global__ void rebase_offsets_kernel(uint64_t *off, uint64_t cnt, uint64_t base) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k <= cnt; k += (uint64_t)gridDim.x * blockDim.x)
    off[k] -= base;
}

}  // namespace leco

using namespace leco;

extern "C" {

const char *leco_last_error(void) { return g_last_error.c_str(); }
const char *leco_version(void) { return "leco-b200 0.1 (sm_100a)"; }

uint64_t leco_num_blocks(uint64_t n, uint32_t block_size) { return block_size ? (n + block_size - 1) / block_size : 0; }

uint64_t leco_block_bytes(int codec, int dtype, uint32_t l, uint32_t nvalues) {
  if (dtype == LECO_U32) {
    switch (codec) {
      case kLinear: return block_bytes<kLinear, 4>(l, nvalues);
      case kFor: return block_bytes<kFor, 4>(l, nvalues);
      case kDelta: return block_bytes<kDelta, 4>(l, nvalues);
      case kPoly2: return block_bytes<kPoly2, 4>(l, nvalues);
      case kLegacy: return block_bytes<kLegacy, 4>(l, nvalues);
    }
  } else if (dtype == LECO_U64) {
    switch (codec) {
      case kLinear: return block_bytes<kLinear, 8>(l, nvalues);
      case kFor: return block_bytes<kFor, 8>(l, nvalues);
      case kDelta: return block_bytes<kDelta, 8>(l, nvalues);
      case kPoly2: return block_bytes<kPoly2, 8>(l, nvalues);
    }
  }
  return 0;
}

uint64_t leco_max_payload_bytes(int codec, int dtype, uint64_t n, uint32_t block_size) {
  if (!codec_write_ok(codec, dtype) || !dtype_ok(dtype) || !block_size) return 0;
  const uint64_t nb = leco_num_blocks(n, block_size);
  // Worst block: raw (1 + n*s) or the widest packed image; the packed image
  // with l = 8s-1 never exceeds raw + header + 16 bytes.
  return n * (uint64_t)dtype + nb * 48 + LECO_PAYLOAD_SLACK;
}

uint64_t leco_encode_workspace_bytes(int codec, int dtype, uint64_t n, uint32_t block_size, int fit_mode) {
  const uint64_t nb = leco_num_blocks(n, block_size);
  return enc_ws(nb, needs_seq_fit(codec, dtype, block_size, fit_mode)).total;
}

int leco_encode(int codec, int dtype, const void *d_values, uint64_t n, uint32_t block_size, int fit_mode,
                uint8_t *d_payload, uint64_t payload_cap, uint64_t *d_offsets, leco_dir_entry *d_dir,
                void *d_workspace, uint64_t workspace_bytes, leco_stream_t stream) {
  if (!codec_write_ok(codec, dtype))
    return fail(LECO_ERR_UNSUPPORTED, "leco_encode: codec must be LINEAR, FOR, DELTA, POLY2 or LINEAR_F32 (u32)");
  if (!dtype_ok(dtype)) return fail(LECO_ERR_ARG, "leco_encode: dtype must be LECO_U32 or LECO_U64");
  if (!block_size || block_size > LECO_MAX_BLOCK) return fail(LECO_ERR_ARG, "leco_encode: block_size must be in 1..16384");
  if (n == 0) return fail(LECO_ERR_ARG, "leco_encode: n must be > 0");
  if (!d_values || !d_payload || !d_offsets || !d_workspace) return fail(LECO_ERR_ARG, "leco_encode: null pointer");
  if ((reinterpret_cast<uintptr_t>(d_payload) & 15) || (reinterpret_cast<uintptr_t>(d_values) & (dtype - 1)))
    return fail(LECO_ERR_ARG, "leco_encode: payload must be 16-byte aligned and values aligned to their size");
  if (fit_mode != LECO_FIT_REFERENCE && fit_mode != LECO_FIT_EXACT) return fail(LECO_ERR_ARG, "leco_encode: bad fit_mode");
  const uint64_t nb = leco_num_blocks(n, block_size);
  if (nb > 0xffffffffull) return fail(LECO_ERR_ARG, "leco_encode: too many blocks");
  const bool seq = needs_seq_fit(codec, dtype, block_size, fit_mode);
  const EncWs w = enc_ws(nb, seq);
  if (workspace_bytes < w.total) return fail(LECO_ERR_ARG, "leco_encode: workspace too small");
  uint32_t *err = nullptr;
  int rc = error_ptr(&err);
  if (rc) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  uint8_t *ws = static_cast<uint8_t *>(d_workspace);
  LECO_CUDA(cudaMemsetAsync(ws, 0, w.models_off, st));  // status words + ticket
  EncodeLaunch L;
  L.values = d_values; L.n = n; L.bs = block_size; L.nb = nb;
  L.payload = d_payload; L.payload_cap = payload_cap; L.offsets = d_offsets; L.dir = d_dir;
  L.seq_models = seq ? reinterpret_cast<double *>(ws + w.models_off) : nullptr;
  L.status = reinterpret_cast<uint64_t *>(ws + w.status_off);
  L.ticket = reinterpret_cast<uint32_t *>(ws + w.ticket_off);
  L.error = err;
  for (int i = 0; i < 10; ++i) L.polyX[i] = 0;
  if (codec == kPoly2) {
    poly2_x_sums(std::min<uint64_t>(n, block_size), L.polyX);
    const uint64_t tail = n - (nb - 1) * block_size;
    poly2_x_sums((uint32_t)tail, L.polyX + 5);
  }
  if (launch_encode(codec, dtype, L, st)) return fail(LECO_ERR_UNSUPPORTED, "leco_encode: no kernel");
  LECO_CUDA(cudaGetLastError());
  return LECO_OK;
}

static int check_column(const char *fn, int codec, int dtype, const void *payload, const void *offsets, uint32_t bs) {
  if (!codec_read_ok(codec, dtype))
    return fail(LECO_ERR_UNSUPPORTED, std::string(fn) + ": codec must be LINEAR, FOR, DELTA, POLY2 or LINEAR_F32 (u32)");
  if (!dtype_ok(dtype)) return fail(LECO_ERR_ARG, std::string(fn) + ": dtype must be LECO_U32 or LECO_U64");
  if (!bs || bs > LECO_MAX_BLOCK) return fail(LECO_ERR_ARG, std::string(fn) + ": block_size must be in 1..16384");
  if (!payload || !offsets) return fail(LECO_ERR_ARG, std::string(fn) + ": null pointer");
  if (reinterpret_cast<uintptr_t>(payload) & 7) return fail(LECO_ERR_ARG, std::string(fn) + ": payload must be 8-byte aligned");
  return LECO_OK;
}

int leco_decode(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
                uint32_t block_size, void *d_out, leco_stream_t stream) {
  return leco_decode_range(codec, dtype, d_payload, d_offsets, n, block_size, 0, n, d_out, stream);
}

int leco_decode_range(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
                      uint32_t block_size, uint64_t first, uint64_t count, void *d_out, leco_stream_t stream) {
  int rc = check_column("leco_decode", codec, dtype, d_payload, d_offsets, block_size);
  if (rc) return rc;
  if (!d_out || (reinterpret_cast<uintptr_t>(d_out) & (dtype - 1))) return fail(LECO_ERR_ARG, "leco_decode: out null or misaligned");
  if (first > n || count > n - first) return fail(LECO_ERR_ARG, "leco_decode: range outside the column");
  if (!count) return LECO_OK;
  uint32_t *err = nullptr;
  if ((rc = error_ptr(&err))) return rc;
  DecodeLaunch L{d_payload, d_offsets, n, block_size, first, count, d_out, err};
  if (launch_decode(codec, dtype, L, reinterpret_cast<cudaStream_t>(stream))) return fail(LECO_ERR_UNSUPPORTED, "no kernel");
  LECO_CUDA(cudaGetLastError());
  return LECO_OK;
}

int leco_build_directory(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
                         uint32_t block_size, leco_dir_entry *d_dir, leco_stream_t stream) {
  int rc = check_column("leco_build_directory", codec, dtype, d_payload, d_offsets, block_size);
  if (rc) return rc;
  if (!d_dir) return fail(LECO_ERR_ARG, "leco_build_directory: null directory");
  uint32_t *err = nullptr;
  if ((rc = error_ptr(&err))) return rc;
  if (launch_build_dir(codec, dtype, d_payload, d_offsets, n, block_size, d_dir, err, reinterpret_cast<cudaStream_t>(stream)))
    return fail(LECO_ERR_UNSUPPORTED, "no kernel");
  LECO_CUDA(cudaGetLastError());
  return LECO_OK;
}

int leco_gather(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets,
                const leco_dir_entry *d_dir, uint64_t n, uint32_t block_size, const uint64_t *d_idx, uint64_t m,
                void *d_out, leco_stream_t stream) {
  int rc = check_column("leco_gather", codec, dtype, d_payload, d_offsets, block_size);
  if (rc) return rc;
  if (m && (!d_idx || !d_out)) return fail(LECO_ERR_ARG, "leco_gather: null pointer");
  if (!m) return LECO_OK;
  uint32_t *err = nullptr;
  if ((rc = error_ptr(&err))) return rc;
  GatherLaunch L{d_payload, d_offsets, d_dir, n, block_size, d_idx, m, d_out, err};
  if (launch_gather(codec, dtype, L, reinterpret_cast<cudaStream_t>(stream))) return fail(LECO_ERR_UNSUPPORTED, "no kernel");
  LECO_CUDA(cudaGetLastError());
  return LECO_OK;
}

uint64_t leco_sum_workspace_bytes(uint64_t n, uint32_t block_size) {
  (void)n;
  (void)block_size;
  return 0;
}

int leco_sum(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
             uint32_t block_size, uint64_t *d_sum, void *d_partials, leco_stream_t stream) {
  (void)d_partials;
  int rc = check_column("leco_sum", codec, dtype, d_payload, d_offsets, block_size);
  if (rc) return rc;
  if (!d_sum) return fail(LECO_ERR_ARG, "leco_sum: null output");
  uint32_t *err = nullptr;
  if ((rc = error_ptr(&err))) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  LECO_CUDA(cudaMemsetAsync(d_sum, 0, sizeof(uint64_t), st));
  DecodeLaunch L{d_payload, d_offsets, n, block_size, 0, n, nullptr, err};
  if (launch_sum(codec, dtype, L, d_sum, st)) return fail(LECO_ERR_UNSUPPORTED, "no kernel");
  LECO_CUDA(cudaGetLastError());
  return LECO_OK;
}

// ---- predicate pushdown -------------------------------------------------------------

uint64_t leco_filter_workspace_bytes(uint64_t n, uint32_t block_size) {
  const uint64_t nb = leco_num_blocks(n, block_size);
  return (nb + (nb + 31) / 32) * 8 + 64;  // per-block counts, per-group totals
}

static int filter_setup(const char *fn, int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets,
                        uint64_t n, uint32_t block_size, uint32_t *d_out, uint64_t out_cap, uint64_t *d_count,
                        void *d_ws, uint64_t ws_bytes, cudaStream_t st, FilterLaunch &L) {
  int rc = check_column(fn, codec, dtype, d_payload, d_offsets, block_size);
  if (rc) return rc;
  if (codec != kLinear && codec != kFor)
    return fail(LECO_ERR_UNSUPPORTED, std::string(fn) + ": the reference filters LINEAR and FOR columns only");
  if (n >= (1ull << 32)) return fail(LECO_ERR_ARG, std::string(fn) + ": output indices are uint32 (n < 2^32)");
  if (!d_count || (out_cap && !d_out)) return fail(LECO_ERR_ARG, std::string(fn) + ": null output");
  const uint64_t nb = leco_num_blocks(n, block_size);
  if (!d_ws || ws_bytes < leco_filter_workspace_bytes(n, block_size) || (reinterpret_cast<uintptr_t>(d_ws) & 7))
    return fail(LECO_ERR_ARG, std::string(fn) + ": workspace must be leco_filter_workspace_bytes() bytes, 8-byte aligned");
  uint32_t *err = nullptr;
  if ((rc = error_ptr(&err))) return rc;
  L = FilterLaunch{};
  L.payload = d_payload;
  L.offsets = d_offsets;
  L.n = n;
  L.bs = block_size;
  L.nb = nb;
  L.out = d_out;
  L.cap = d_out ? out_cap : 0;
  L.count = d_count;
  L.counts = reinterpret_cast<uint64_t *>(d_ws);
  L.group_tot = L.counts + nb;
  L.error = err;
  L.max_windows = 65536;
  L.vec_out = (reinterpret_cast<uintptr_t>(d_out) & 15) == 0;
  if (!nb) LECO_CUDA(cudaMemsetAsync(d_count, 0, 8, st));
  return LECO_OK;
}

int leco_filter_range(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
                      uint32_t block_size, uint64_t filter, const uint64_t *d_zone_min, const uint64_t *d_zone_max,
                      uint32_t *d_out, uint64_t out_cap, uint64_t *d_count, void *d_ws, uint64_t ws_bytes,
                      leco_stream_t stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  FilterLaunch L;
  int rc = filter_setup("leco_filter_range", codec, dtype, d_payload, d_offsets, n, block_size, d_out, out_cap, d_count,
                        d_ws, ws_bytes, st, L);
  if (rc) return rc;
  L.f1 = filter;
  L.zone = d_zone_max;
  L.zone_lo = d_zone_min;
  const int lrc = launch_filter(codec, dtype, L, 0, st);
  if (lrc > 0) return fail(LECO_ERR_UNSUPPORTED, "leco_filter_range: no kernel");
  if (lrc < 0) return cuda_fail((cudaError_t)-lrc, "leco_filter_range: launch");
  LECO_CUDA(cudaGetLastError());
  return LECO_OK;
}

int leco_filter_range_close(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
                            uint32_t block_size, uint64_t filter1, uint64_t filter2, uint64_t base,
                            const uint64_t *d_zone_min, uint32_t *d_out, uint64_t out_cap, uint64_t *d_count,
                            void *d_ws, uint64_t ws_bytes, leco_stream_t stream) {
  if (base < 1 || base > 0x7fffffffull) return fail(LECO_ERR_ARG, "leco_filter_range_close: base must be in 1..INT32_MAX");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  FilterLaunch L;
  int rc = filter_setup("leco_filter_range_close", codec, dtype, d_payload, d_offsets, n, block_size, d_out, out_cap,
                        d_count, d_ws, ws_bytes, st, L);
  if (rc) return rc;
  L.f1 = filter1;
  L.f2 = filter2;
  L.base = base;
  L.zone = codec == kLinear ? d_zone_min : nullptr;
  const int lrc = launch_filter(codec, dtype, L, 1, st);
  if (lrc > 0) return fail(LECO_ERR_UNSUPPORTED, "leco_filter_range_close: no kernel");
  if (lrc < 0) return cuda_fail((cudaError_t)-lrc, "leco_filter_range_close: launch");
  LECO_CUDA(cudaGetLastError());
  return LECO_OK;
}

int leco_zonemap(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
                 uint32_t block_size, uint64_t *d_min, uint64_t *d_max, leco_stream_t stream) {
  int rc = check_column("leco_zonemap", codec, dtype, d_payload, d_offsets, block_size);
  if (rc) return rc;
  if (!d_min || !d_max) return fail(LECO_ERR_ARG, "leco_zonemap: null output");
  uint32_t *err = nullptr;
  if ((rc = error_ptr(&err))) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  DecodeLaunch L{d_payload, d_offsets, n, block_size, 0, n, nullptr, err};
  if (launch_zonemap(codec, dtype, L, d_min, d_max, st)) return fail(LECO_ERR_UNSUPPORTED, "leco_zonemap: no kernel");
  LECO_CUDA(cudaGetLastError());
  return LECO_OK;
}

int leco_check(leco_stream_t stream) {
  uint32_t *err = nullptr;
  int rc = error_ptr(&err);
  if (rc) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  uint32_t h = 0;
  LECO_CUDA(cudaMemcpyAsync(&h, err, 4, cudaMemcpyDeviceToHost, st));
  LECO_CUDA(cudaStreamSynchronize(st));
  if (h) LECO_CUDA(cudaMemsetAsync(err, 0, 4, st));
  LECO_CUDA(cudaStreamSynchronize(st));
  if (h & kErrTimeout) return fail(LECO_ERR_TIMEOUT, "device wait gave up (look-back or queue)");
  if (h & kErrCapacity) return fail(LECO_ERR_CAPACITY, "payload buffer smaller than the encoded column");
  if (h & kErrBadHeader) return fail(LECO_ERR_CORRUPT, "invalid block header");
  if (h & kErrBadIndex) return fail(LECO_ERR_CORRUPT, "index outside the column");
  if (h & kErrLimit) return fail(LECO_ERR_UNSUPPORTED, "close-range filter: a block needs more than 65536 windows");
  return LECO_OK;
}

// ---- host-side validation ------------------------------------------------------------

int leco_validate_host(int codec, int dtype, const uint8_t *h_payload, uint64_t payload_bytes,
                       const uint64_t *h_offsets, uint64_t n, uint32_t block_size, uint64_t *bad_block) {
  int rc = check_column("leco_validate_host", codec, dtype, h_payload, h_offsets, block_size);
  if (rc) return rc;
  const uint64_t nb = leco_num_blocks(n, block_size);
  const uint32_t tb = 8u * (uint32_t)dtype;
  for (uint64_t b = 0; b < nb; ++b) {
    const uint64_t o = h_offsets[b], e = h_offsets[b + 1];
    const uint32_t len = (uint32_t)std::min<uint64_t>(block_size, n - b * block_size);
    bool ok = o < e && e <= payload_bytes;
    if (ok) {
      const uint32_t l = h_payload[o];
      bool sentinel = (l == 126 || l == 127) && codec != kFor && codec != kLegacy;
      if (sentinel) ok = e - o >= 1 + (uint64_t)dtype * (l == 127 ? 1 : 2);
      else ok = l <= tb && (e - o) == leco_block_bytes(codec, dtype, l, len);
      if (ok && codec == kFor && l > 0 && l < tb) {
        // FOR: header max - min must need exactly l bits (FOR_integer_template.h:43-49)
        uint64_t mn = 0, mx = 0;
        memcpy(&mn, h_payload + o + 1, dtype);
        memcpy(&mx, h_payload + o + 1 + dtype, dtype);
        ok = mx >= mn;
      }
    }
    if (!ok) {
      if (bad_block) *bad_block = b;
      return fail(LECO_ERR_CORRUPT, "leco_validate_host: block " + std::to_string(b) + " is not a valid image");
    }
  }
  return LECO_OK;
}

// ---- host-buffer pipelines -------------------------------------------------------------

// Device memory of the host-buffer calls (leco_*_host) comes from a memory pool of this
// library, one per device, that keeps up to kHostPoolKeep bytes mapped between calls.
// From the default pool (release threshold 0) every call mapped its buffers afresh once
// the previous call's stream had synchronised.  If the pool cannot be made, the default
// pool is used.
constexpr uint64_t kHostPoolKeep = 1ull << 30;
cudaMemPool_t host_pool() {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  static bool tried[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!tried[dev]) {
    tried[dev] = true;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) == cudaSuccess) {
      uint64_t keep = kHostPoolKeep;
      if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) == cudaSuccess) pools[dev] = pool;
      else cudaMemPoolDestroy(pool);
    }
    cudaGetLastError();  // a failed attempt leaves no sticky error behind
  }
  return pools[dev];
}

struct DevBuf {
  void *p = nullptr;
  cudaStream_t st = nullptr;
  ~DevBuf() {
    if (p) cudaFreeAsync(p, st);
  }
  cudaError_t alloc(size_t bytes, cudaStream_t s) {
    st = s;
    cudaMemPool_t pool = host_pool();
    return pool ? cudaMallocFromPoolAsync(&p, bytes ? bytes : 1, pool, s) : cudaMallocAsync(&p, bytes ? bytes : 1, s);
  }
};

int leco_encode_host(int codec, int dtype, const void *h_values, uint64_t n, uint32_t block_size, int fit_mode,
                     uint8_t *h_payload, uint64_t payload_cap, uint64_t *h_offsets, uint64_t *out_bytes) {
  if (!h_values || !h_payload || !h_offsets) return fail(LECO_ERR_ARG, "leco_encode_host: null pointer");
  if (!codec_write_ok(codec, dtype) || !dtype_ok(dtype) || !block_size || block_size > LECO_MAX_BLOCK || !n)
    return fail(LECO_ERR_ARG, "leco_encode_host: bad codec/dtype/block_size/n");
  cudaStream_t st;
  LECO_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  int rc = LECO_OK;
  {
    const uint64_t nb = leco_num_blocks(n, block_size);
    const uint64_t cap = leco_max_payload_bytes(codec, dtype, n, block_size);
    const uint64_t wsb = leco_encode_workspace_bytes(codec, dtype, n, block_size, fit_mode);
    DevBuf dv, dp, doff, dws;
    if (dv.alloc(n * dtype, st) || dp.alloc(cap, st) || doff.alloc((nb + 1) * 8, st) || dws.alloc(wsb, st)) {
      rc = fail(LECO_ERR_NOMEM, "leco_encode_host: device allocation failed");
    } else {
      cudaMemcpyAsync(dv.p, h_values, n * dtype, cudaMemcpyHostToDevice, st);
      rc = leco_encode(codec, dtype, dv.p, n, block_size, fit_mode, (uint8_t *)dp.p, cap, (uint64_t *)doff.p, nullptr,
                       dws.p, wsb, reinterpret_cast<leco_stream_t>(st));
      if (!rc) {
        cudaMemcpyAsync(h_offsets, doff.p, (nb + 1) * 8, cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        rc = leco_check(reinterpret_cast<leco_stream_t>(st));
      }
      if (!rc) {
        const uint64_t total = h_offsets[nb];
        if (out_bytes) *out_bytes = total;
        if (total > payload_cap) rc = fail(LECO_ERR_CAPACITY, "leco_encode_host: payload_cap too small");
        else cudaMemcpyAsync(h_payload, dp.p, total, cudaMemcpyDeviceToHost, st);
      }
    }
  }
  cudaError_t e = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (!rc && e != cudaSuccess) rc = cuda_fail(e, "leco_encode_host");
  return rc;
}

// Decodes a host column in chunks of whole blocks on four streams, so the
// host->device copy of one chunk, the decode of another and the device->host
// copy of a third overlap.
int leco_decode_host(int codec, int dtype, const uint8_t *h_payload, const uint64_t *h_offsets, uint64_t n,
                     uint32_t block_size, void *h_out) {
  int rc = check_column("leco_decode_host", codec, dtype, h_payload, h_offsets, block_size);
  if (rc) return rc;
  if (!h_out) return fail(LECO_ERR_ARG, "leco_decode_host: null output");
  const uint64_t nb = leco_num_blocks(n, block_size);
  if (!nb) return LECO_OK;
  const uint64_t total = h_offsets[nb];
  // chunk = ~32 MiB of decoded values, whole blocks; four streams keep the
  // device->host copies queued back to back even when this thread is slow to
  // enqueue the next chunk
  uint64_t bpc = std::max<uint64_t>(1, (32ull << 20) / ((uint64_t)block_size * dtype));
  bpc = std::min(bpc, nb);
  const int NS = 4;
  cudaStream_t st[NS];
  for (int i = 0; i < NS; ++i) LECO_CUDA(cudaStreamCreateWithFlags(&st[i], cudaStreamNonBlocking));
  DevBuf pay[NS], off[NS], out[NS];
  uint64_t max_chunk_bytes = 0;
  for (uint64_t b0 = 0; b0 < nb; b0 += bpc) {
    uint64_t b1 = std::min(nb, b0 + bpc);
    max_chunk_bytes = std::max(max_chunk_bytes, h_offsets[b1] - h_offsets[b0]);
  }
  for (int i = 0; i < NS && !rc; ++i) {
    if (pay[i].alloc(max_chunk_bytes + LECO_PAYLOAD_SLACK + 8, st[i]) || off[i].alloc((bpc + 1) * 8, st[i]) ||
        out[i].alloc(bpc * block_size * (uint64_t)dtype, st[i]))
      rc = fail(LECO_ERR_NOMEM, "leco_decode_host: device allocation failed");
  }
  uint64_t chunk = 0;
  for (uint64_t b0 = 0; b0 < nb && !rc; b0 += bpc, ++chunk) {
    const int i = (int)(chunk % NS);
    cudaStream_t s = st[i];
    const uint64_t b1 = std::min(nb, b0 + bpc), cb = b1 - b0;
    const uint64_t pbase = h_offsets[b0] & ~7ull;  // keep the 8-byte word alignment of bit addresses
    cudaStreamSynchronize(s);                       // the buffers are reused
    const uint64_t nbytes = h_offsets[b1] - pbase;
    cudaMemcpyAsync(pay[i].p, h_payload + pbase, std::min<uint64_t>(nbytes + 8, total - pbase), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(off[i].p, h_offsets + b0, (cb + 1) * 8, cudaMemcpyHostToDevice, s);
    rebase_offsets_kernel<<<(unsigned)std::min<uint64_t>((cb + 256) / 256, 64), 256, 0, s>>>((uint64_t *)off[i].p, cb, pbase);
    const uint64_t v0 = b0 * block_size, nv = std::min<uint64_t>(n, b1 * block_size) - v0;
    rc = leco_decode(codec, dtype, (const uint8_t *)pay[i].p, (const uint64_t *)off[i].p, nv, block_size, out[i].p,
                     reinterpret_cast<leco_stream_t>(s));
    cudaMemcpyAsync(static_cast<uint8_t *>(h_out) + v0 * dtype, out[i].p, nv * dtype, cudaMemcpyDeviceToHost, s);
  }
  for (int i = 0; i < NS; ++i) {
    cudaError_t e = cudaStreamSynchronize(st[i]);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "leco_decode_host");
  }
  if (!rc) rc = leco_check(reinterpret_cast<leco_stream_t>(st[0]));
  for (int i = 0; i < NS; ++i) {
    pay[i].~DevBuf(); pay[i].p = nullptr;
    off[i].~DevBuf(); off[i].p = nullptr;
    out[i].~DevBuf(); out[i].p = nullptr;
    cudaStreamSynchronize(st[i]);
    cudaStreamDestroy(st[i]);
  }
  return rc;
}

int leco_gather_host(int codec, int dtype, const uint8_t *h_payload, const uint64_t *h_offsets, uint64_t n,
                     uint32_t block_size, const uint64_t *h_idx, uint64_t m, void *h_out) {
  int rc = check_column("leco_gather_host", codec, dtype, h_payload, h_offsets, block_size);
  if (rc) return rc;
  if (m && (!h_idx || !h_out)) return fail(LECO_ERR_ARG, "leco_gather_host: null pointer");
  const uint64_t nb = leco_num_blocks(n, block_size);
  cudaStream_t st;
  LECO_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  {
    const uint64_t total = h_offsets[nb];
    DevBuf dp, doff, ddir, didx, dout;
    if (dp.alloc(total + LECO_PAYLOAD_SLACK, st) || doff.alloc((nb + 1) * 8, st) || ddir.alloc(nb * sizeof(leco_dir_entry), st) ||
        didx.alloc(m * 8, st) || dout.alloc(m * dtype, st)) {
      rc = fail(LECO_ERR_NOMEM, "leco_gather_host: device allocation failed");
    } else {
      cudaMemsetAsync((uint8_t *)dp.p + total, 0, LECO_PAYLOAD_SLACK, st);
      cudaMemcpyAsync(dp.p, h_payload, total, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(doff.p, h_offsets, (nb + 1) * 8, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(didx.p, h_idx, m * 8, cudaMemcpyHostToDevice, st);
      leco_stream_t ls = reinterpret_cast<leco_stream_t>(st);
      rc = leco_build_directory(codec, dtype, (const uint8_t *)dp.p, (const uint64_t *)doff.p, n, block_size,
                                (leco_dir_entry *)ddir.p, ls);
      if (!rc)
        rc = leco_gather(codec, dtype, (const uint8_t *)dp.p, (const uint64_t *)doff.p, (const leco_dir_entry *)ddir.p, n,
                         block_size, (const uint64_t *)didx.p, m, dout.p, ls);
      if (!rc) cudaMemcpyAsync(h_out, dout.p, m * dtype, cudaMemcpyDeviceToHost, st);
      if (!rc) rc = leco_check(ls);
    }
  }
  cudaError_t e = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (!rc && e != cudaSuccess) rc = cuda_fail(e, "leco_gather_host");
  return rc;
}

// ---- per-block drop-in -----------------------------------------------------------------
// The reference's drivers call the codec once per block.  Each calling thread keeps one
// stream, one device buffer and one pinned host buffer (both only grow) for these calls,
// created on its first per-block call on a device and kept until leco_thread_release()
// or the process ends, so a call costs its copies, one launch and one synchronize.

namespace {

struct BlockCtx {
  int device = -1;
  cudaStream_t st = nullptr;
  uint8_t *d = nullptr;  // device buffer
  uint64_t dcap = 0;
  uint8_t *h = nullptr;  // pinned host staging
  uint64_t hcap = 0;
};
thread_local BlockCtx t_block;

void block_ctx_free(BlockCtx &c) {
  if (c.st) cudaStreamSynchronize(c.st);
  if (c.d) cudaFree(c.d);
  if (c.h) cudaFreeHost(c.h);
  if (c.st) cudaStreamDestroy(c.st);
  c = BlockCtx{};
}

uint64_t round256(uint64_t x) { return (x + 255) & ~255ull; }

// The calling thread's context on the current device, with at least dev_bytes of device
// and host_bytes of pinned host memory.
int block_ctx(uint64_t dev_bytes, uint64_t host_bytes, BlockCtx *&out) {
  int dev = 0;
  LECO_CUDA(cudaGetDevice(&dev));
  BlockCtx &c = t_block;
  if (c.device != dev) {
    if (c.device >= 0) {  // the thread moved to another device: free on the old one
      LECO_CUDA(cudaSetDevice(c.device));
      block_ctx_free(c);
      LECO_CUDA(cudaSetDevice(dev));
    }
    LECO_CUDA(cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking));
    c.device = dev;
  }
  if (c.dcap < dev_bytes) {
    if (c.d) LECO_CUDA(cudaFree(c.d));
    c.d = nullptr;
    c.dcap = 0;
    const uint64_t cap = std::max<uint64_t>(dev_bytes, 1ull << 20);
    if (cudaMalloc(&c.d, cap) != cudaSuccess) return fail(LECO_ERR_NOMEM, "per-block call: device allocation failed");
    c.dcap = cap;
  }
  if (c.hcap < host_bytes) {
    if (c.h) LECO_CUDA(cudaFreeHost(c.h));
    c.h = nullptr;
    c.hcap = 0;
    const uint64_t cap = std::max<uint64_t>(host_bytes, 1ull << 20);
    if (cudaHostAlloc(&c.h, cap, cudaHostAllocDefault) != cudaSuccess)
      return fail(LECO_ERR_NOMEM, "per-block call: pinned host allocation failed");
    c.hcap = cap;
  }
  out = &c;
  return LECO_OK;
}

// Copies a block image to the start of the context's device buffer with LECO_PAYLOAD_SLACK
// zero bytes after it, then offsets {0, in_bytes} and `extra` (nextra words) at
// round256(in_bytes + slack): one pinned staging copy, one upload.
void stage_block(BlockCtx &c, const uint8_t *h_in, uint64_t in_bytes, const uint64_t *extra = nullptr, int nextra = 0) {
  const uint64_t pb = round256(in_bytes + LECO_PAYLOAD_SLACK);
  memcpy(c.h, h_in, in_bytes);
  memset(c.h + in_bytes, 0, pb - in_bytes);
  uint64_t *tail = reinterpret_cast<uint64_t *>(c.h + pb);
  tail[0] = 0;
  tail[1] = in_bytes;
  for (int i = 0; i < nextra; ++i) tail[2 + i] = extra[i];
  cudaMemcpyAsync(c.d, c.h, pb + 8 * (2 + nextra), cudaMemcpyHostToDevice, c.st);
}

}  // namespace

int leco_thread_release(void) {
  if (t_block.device < 0) return LECO_OK;
  int dev = 0;
  LECO_CUDA(cudaGetDevice(&dev));
  LECO_CUDA(cudaSetDevice(t_block.device));
  block_ctx_free(t_block);
  LECO_CUDA(cudaSetDevice(dev));
  return LECO_OK;
}

int64_t leco_block_encode(int codec, int dtype, const void *h_values, uint32_t length, int fit_mode, uint8_t *h_out) {
  if (!h_values || !h_out) return fail(LECO_ERR_ARG, "leco_block_encode: null pointer");
  if (!length || length > LECO_MAX_BLOCK) return fail(LECO_ERR_ARG, "leco_block_encode: length must be in 1..16384");
  if (!dtype_ok(dtype)) return fail(LECO_ERR_ARG, "leco_block_encode: dtype must be LECO_U32 or LECO_U64");
  const uint64_t vb = round256((uint64_t)length * dtype);
  const uint64_t cap = leco_max_payload_bytes(codec, dtype, length, length);
  const uint64_t wsb = leco_encode_workspace_bytes(codec, dtype, length, length, fit_mode);
  BlockCtx *c = nullptr;
  int rc = block_ctx(vb + 256 + round256(cap) + round256(wsb), vb + 256 + round256(cap), c);
  if (rc) return rc;
  uint8_t *dv = c->d, *doff = c->d + vb, *dp = doff + 256, *dws = dp + round256(cap);
  memcpy(c->h, h_values, (uint64_t)length * dtype);
  cudaMemcpyAsync(dv, c->h, (uint64_t)length * dtype, cudaMemcpyHostToDevice, c->st);
  const leco_stream_t ls = reinterpret_cast<leco_stream_t>(c->st);
  rc = leco_encode(codec, dtype, dv, length, length, fit_mode, dp, cap, reinterpret_cast<uint64_t *>(doff), nullptr, dws,
                   wsb, ls);
  if (rc) return rc;
  // offsets and the image come back in one copy: [offsets (256)][image (cap)]
  cudaMemcpyAsync(c->h, doff, 256 + cap, cudaMemcpyDeviceToHost, c->st);
  if ((rc = leco_check(ls)) != LECO_OK) return rc;  // synchronizes the stream
  uint64_t off[2];
  memcpy(off, c->h, 16);
  const uint64_t bytes = off[1];
  if (bytes > cap) return fail(LECO_ERR_CORRUPT, "leco_block_encode: image larger than its bound");
  memcpy(h_out, c->h + 256, bytes);
  return (int64_t)bytes;
}

int leco_block_decode(int codec, int dtype, const uint8_t *h_in, uint64_t in_bytes, uint32_t length, void *h_out) {
  if (!h_in || !h_out || !length) return fail(LECO_ERR_ARG, "leco_block_decode: bad argument");
  if (!dtype_ok(dtype)) return fail(LECO_ERR_ARG, "leco_block_decode: dtype must be LECO_U32 or LECO_U64");
  const uint64_t pb = round256(in_bytes + LECO_PAYLOAD_SLACK), ob = (uint64_t)length * dtype;
  BlockCtx *c = nullptr;
  int rc = block_ctx(pb + 256 + ob, std::max(pb + 256, ob), c);
  if (rc) return rc;
  uint8_t *dp = c->d, *dout = c->d + pb + 256;
  uint64_t *doff = reinterpret_cast<uint64_t *>(c->d + pb);
  stage_block(*c, h_in, in_bytes);
  const leco_stream_t ls = reinterpret_cast<leco_stream_t>(c->st);
  rc = leco_decode(codec, dtype, dp, doff, length, length, dout, ls);
  if (rc) return rc;
  cudaMemcpyAsync(c->h, dout, ob, cudaMemcpyDeviceToHost, c->st);
  if ((rc = leco_check(ls)) != LECO_OK) return rc;  // synchronizes the stream
  memcpy(h_out, c->h, ob);
  return LECO_OK;
}

int64_t leco_block_filter(int codec, int dtype, const uint8_t *h_in, uint64_t in_bytes, uint32_t length,
                          uint32_t block_start, int close, uint64_t filter1, uint64_t filter2, uint64_t base,
                          uint32_t *h_out, uint64_t out_cap) {
  if (!h_in || !in_bytes || !length || length > LECO_MAX_BLOCK || (out_cap && !h_out))
    return fail(LECO_ERR_ARG, "leco_block_filter: bad argument");
  cudaStream_t st;
  LECO_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  int64_t rc = 0;
  {
    std::vector<uint8_t> tmp(in_bytes + LECO_PAYLOAD_SLACK, 0);
    memcpy(tmp.data(), h_in, in_bytes);
    const uint64_t off[2] = {0, in_bytes};
    const uint64_t wsb = leco_filter_workspace_bytes(length, length);
    DevBuf pay, doff, out, cnt, ws;
    if (pay.alloc(tmp.size(), st) || doff.alloc(16, st) || out.alloc(out_cap * 4, st) || cnt.alloc(8, st) ||
        ws.alloc(wsb, st)) {
      rc = fail(LECO_ERR_NOMEM, "leco_block_filter: device allocation failed");
    } else {
      cudaMemcpyAsync(pay.p, tmp.data(), tmp.size(), cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(doff.p, off, 16, cudaMemcpyHostToDevice, st);
      const leco_stream_t ls = reinterpret_cast<leco_stream_t>(st);
      rc = close ? leco_filter_range_close(codec, dtype, (const uint8_t *)pay.p, (const uint64_t *)doff.p, length, length,
                                           filter1, filter2, base, nullptr, (uint32_t *)out.p, out_cap,
                                           (uint64_t *)cnt.p, ws.p, wsb, ls)
                 : leco_filter_range(codec, dtype, (const uint8_t *)pay.p, (const uint64_t *)doff.p, length, length,
                                     filter1, nullptr, nullptr, (uint32_t *)out.p, out_cap, (uint64_t *)cnt.p, ws.p,
                                     wsb, ls);
      uint64_t c = 0;
      if (!rc) {
        cudaMemcpyAsync(&c, cnt.p, 8, cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = cuda_fail(e, "leco_block_filter");
      }
      if (!rc && (rc = leco_check(ls)) == 0) {
        const uint64_t w = std::min<uint64_t>(c, out_cap);
        if (w) {
          cudaMemcpyAsync(h_out, out.p, w * 4, cudaMemcpyDeviceToHost, st);
          cudaError_t e = cudaStreamSynchronize(st);
          if (e != cudaSuccess) rc = cuda_fail(e, "leco_block_filter");
          for (uint64_t i = 0; i < w && !rc; ++i) h_out[i] += block_start;
        }
        if (!rc) rc = (int64_t)c;
      }
    }
  }
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return rc;
}

int leco_block_random(int codec, int dtype, const uint8_t *h_in, uint64_t in_bytes, uint32_t length,
                      uint32_t to_find, void *h_value) {
  if (!h_in || !h_value || to_find >= length) return fail(LECO_ERR_ARG, "leco_block_random: bad argument");
  if (!dtype_ok(dtype)) return fail(LECO_ERR_ARG, "leco_block_random: dtype must be LECO_U32 or LECO_U64");
  const uint64_t pb = round256(in_bytes + LECO_PAYLOAD_SLACK);
  BlockCtx *c = nullptr;
  int rc = block_ctx(pb + 512, pb + 256, c);
  if (rc) return rc;
  uint8_t *dp = c->d;
  uint64_t *doff = reinterpret_cast<uint64_t *>(c->d + pb);
  uint64_t *didx = doff + 2, *dout = doff + 4;
  const uint64_t idx = to_find;
  stage_block(*c, h_in, in_bytes, &idx, 1);  // the index lands at didx
  const leco_stream_t ls = reinterpret_cast<leco_stream_t>(c->st);
  rc = leco_gather(codec, dtype, dp, doff, nullptr, length, length, didx, 1, dout, ls);
  if (rc) return rc;
  cudaMemcpyAsync(c->h, dout, 8, cudaMemcpyDeviceToHost, c->st);
  if ((rc = leco_check(ls)) != LECO_OK) return rc;  // synchronizes the stream
  memcpy(h_value, c->h, (uint64_t)dtype);
  return LECO_OK;
}

}  // extern "C"
