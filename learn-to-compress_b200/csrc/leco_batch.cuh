// leco_batch.cuh -- types shared by the batch engine's host code (leco_batch.cu)
// and its persistent kernels (leco_batch_encode.cu, leco_batch_decode.cu), which
// are compiled as separate translation units.
#pragma once
#include <cuda_runtime.h>

#include "leco_decode.cuh"
#include "leco_encode.cuh"

namespace leco {

struct DevCol {
  int32_t codec, dtype;
  uint32_t bs, seq;
  uint32_t group, unroll;  // threads per block (32, 64, 128, 256), unroll depth (1, 2, 4)
  uint32_t slice, pad;     // encoder shared memory per group (bytes)
  uint64_t n;
  const void *values;
  void *out;
  uint8_t *payload;
  uint64_t payload_cap;
  uint64_t *offsets;
  leco_dir_entry *dir;
  double polyX[10];
};

__device__ __forceinline__ uint32_t find_column(const uint64_t *__restrict__ prefix, uint32_t ncols, uint64_t gb) {
  uint32_t lo = 0, hi = ncols;  // largest c with prefix[c] <= gb
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(prefix + mid) <= gb) lo = mid;
    else hi = mid;
  }
  return lo;
}

#define LECO_BATCH_DISPATCH(codec, dtype, FN, ...)                 \
  do {                                                             \
    if ((dtype) == 4) {                                            \
      switch (codec) {                                             \
        case kLinear: FN<uint32_t, kLinear>(__VA_ARGS__); break;   \
        case kFor: FN<uint32_t, kFor>(__VA_ARGS__); break;         \
        case kDelta: FN<uint32_t, kDelta>(__VA_ARGS__); break;     \
        case kPoly2: FN<uint32_t, kPoly2>(__VA_ARGS__); break;     \
      }                                                            \
    } else {                                                       \
      switch (codec) {                                             \
        case kLinear: FN<uint64_t, kLinear>(__VA_ARGS__); break;   \
        case kFor: FN<uint64_t, kFor>(__VA_ARGS__); break;         \
        case kDelta: FN<uint64_t, kDelta>(__VA_ARGS__); break;     \
        case kPoly2: FN<uint64_t, kPoly2>(__VA_ARGS__); break;     \
      }                                                            \
    }                                                              \
  } while (0)

struct BatchArgs {
  const DevCol *cols;
  const uint64_t *prefix;  // [ncols + 1] blocks before each column
  const uint64_t *items;   // [nitems] (column << 32) | first block
  uint32_t ncols;
  uint64_t nitems;
  uint64_t total;          // blocks in the batch
  uint64_t *status;        // [total] look-back words (zeroed per encode pass)
  unsigned long long *ticket;  // zeroed per pass
  double *models;          // [total * 3] sequential-fit models
  uint32_t *error;
};

// Persistent kernels (one ticket = one work item), defined in leco_batch_encode.cu
// and leco_batch_decode.cu.
__global__ void __launch_bounds__(256, 3) batch_encode_kernel(BatchArgs B);
__global__ void __launch_bounds__(256, 4) batch_decode_kernel(BatchArgs B);

}  // namespace leco
