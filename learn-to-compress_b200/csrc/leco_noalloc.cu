// leco_noalloc.cu -- leco_encode for callers that cannot allocate device memory.
//
// leco_encode needs a few bytes of device scratch per block (the look-back status words and
// ticket that give each block its byte offset, and in reference-fit mode the per-block models
// of the sequential fit), which its caller normally passes as a workspace.  Some callers have no
// way to provide it: an engine whose buffer manager owns all device memory and lends the codec
// only the input and output buffers it reserved, or a latency-critical thread that must never
// call cudaMalloc/cudaFree because those can synchronize the whole device and stall other
// streams.  leco_encode_noalloc serves them from a fixed array compiled into this library.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "leco_internal.h"

namespace {

// Largest column leco_encode_noalloc accepts, in blocks (e.g. 134M values at 4096 per block).
constexpr uint64_t kNoallocMaxBlocks = 32768;
// Encoder scratch for that many blocks: 8-byte status word per block, the ticket line, and
// 24 bytes of sequential-fit model per block (reference fit mode), each part 256-byte aligned.
constexpr uint64_t kNoallocScratchBytes = kNoallocMaxBlocks * 8 + 256 + kNoallocMaxBlocks * 24;

// The scratch itself.  Every GPU that loads this library holds these bytes until the process
// exits.  In host code the name is only a stand-in, not a device address: the address is
// obtained per device with cudaGetSymbolAddress below.
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoallocScratchBytes];

std::mutex g_setup_mutex;
void *g_scratch_ptr[64] = {};

// Per-device set-up: resolves the scratch array's device address once, with the device
// current.  Runs on the first call on each device.
int scratch_for_current_device(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return leco::record_error(LECO_ERR_CUDA, std::string("leco_encode_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return leco::record_error(LECO_ERR_ARG, "leco_encode_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return leco::record_error(LECO_ERR_CUDA, std::string("leco_encode_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return LECO_OK;
}

}  // namespace

extern "C" int leco_encode_noalloc(int codec, int dtype, const void *d_values, uint64_t n, uint32_t block_size,
                                   int fit_mode, uint8_t *d_payload, uint64_t payload_cap, uint64_t *d_offsets,
                                   leco_dir_entry *d_dir, leco_stream_t stream) {
  if (!block_size) return leco::record_error(LECO_ERR_ARG, "leco_encode_noalloc: block_size must be in 1..16384");
  const uint64_t nb = leco_num_blocks(n, block_size);
  if (nb > kNoallocMaxBlocks)
    return leco::record_error(LECO_ERR_ARG, "leco_encode_noalloc: column has " + std::to_string(nb) +
                                                " blocks; the built-in scratch holds at most " +
                                                std::to_string(kNoallocMaxBlocks) + " (use leco_encode with a workspace)");
  if (leco_encode_workspace_bytes(codec, dtype, n, block_size, fit_mode) > kNoallocScratchBytes)
    return leco::record_error(LECO_ERR_ARG, "leco_encode_noalloc: column exceeds the built-in scratch");
  void *scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  return leco_encode(codec, dtype, d_values, n, block_size, fit_mode, d_payload, payload_cap, d_offsets, d_dir, scratch,
                     kNoallocScratchBytes, stream);
}

extern "C" uint64_t leco_encode_noalloc_max_blocks(void) { return kNoallocMaxBlocks; }
