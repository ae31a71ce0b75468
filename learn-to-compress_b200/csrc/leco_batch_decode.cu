// leco_batch_decode.cu -- the batch engine's persistent decode kernel (see
// leco_batch.cu for the work queue), a translation unit of its own like the
// encoder's.
#include "leco_batch.cuh"

namespace leco {

template <typename T, int CODEC, int G, int U>
__device__ __forceinline__ void batch_decode_one(const BatchArgs &B, const DevCol &c, uint64_t b) {
  DecodeLaunch a{c.payload, c.offsets, c.n, c.bs, 0, c.n, c.out, B.error};
  decode_block<T, CODEC, G, U>(a, b);
}
// The unroll depth changes the narrow-field decoder; Delta blocks take one instance.
template <typename T, int CODEC, int G>
__device__ __forceinline__ void batch_decode_u(const BatchArgs &B, const DevCol &c, uint64_t b) {
  if constexpr (CODEC != kDelta) {
    switch (c.unroll) {
      case 1: batch_decode_one<T, CODEC, G, 1>(B, c, b); return;
      case 4: batch_decode_one<T, CODEC, G, 4>(B, c, b); return;
      default: batch_decode_one<T, CODEC, G, 2>(B, c, b); return;
    }
  } else {
    batch_decode_one<T, CODEC, G, 2>(B, c, b);
  }
}
template <typename T, int CODEC>
__device__ __forceinline__ void batch_decode_any(const BatchArgs &B, const DevCol &c, uint64_t b) {
  switch (c.group) {
    case 32: batch_decode_u<T, CODEC, 32>(B, c, b); return;
    case 64: batch_decode_u<T, CODEC, 64>(B, c, b); return;
    case 128: batch_decode_u<T, CODEC, 128>(B, c, b); return;
    default: batch_decode_u<T, CODEC, 256>(B, c, b); return;
  }
}

// Persistent decode: one ticket = one work item, as the encoder.
__global__ void __launch_bounds__(256, 4) batch_decode_kernel(BatchArgs B) {
  __shared__ unsigned long long item;
  for (;;) {
    if (threadIdx.x == 0) item = atomicAdd(B.ticket, 1ull);
    __syncthreads();
    const uint64_t it = item;
    __syncthreads();
    if (it >= B.nitems) break;
    const uint64_t e = __ldg(B.items + it);
    const uint32_t ci = (uint32_t)(e >> 32);
    const DevCol &c = B.cols[ci];
    const uint64_t b = (e & 0xffffffffull) + threadIdx.x / c.group;
    if (b < __ldg(B.prefix + ci + 1) - __ldg(B.prefix + ci)) LECO_BATCH_DISPATCH(c.codec, c.dtype, batch_decode_any, B, c, b);
    __syncthreads();  // the Delta row scan's shared scratch is reused by the next item
  }
}

}  // namespace leco
