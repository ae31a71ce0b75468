// leco_batch_encode.cu -- the batch engine's persistent encode kernel (see
// leco_batch.cu for the work queue).  A translation unit of its own: its many
// per-codec, per-group and per-unroll encoder instances compile in parallel with
// the decoder's.
#include "leco_batch.cuh"

namespace leco {

template <typename T, int CODEC, int G, int U>
__device__ __forceinline__ void batch_encode_one(const BatchArgs &B, const DevCol &c, uint32_t ci, uint64_t b,
                                                 uint8_t *smem) {
  EncodeArgs a;
  a.values = c.values;
  a.n = c.n;
  a.bs = c.bs;
  const uint64_t p0 = __ldg(B.prefix + ci);
  a.nb = __ldg(B.prefix + ci + 1) - p0;
  a.payload = c.payload;
  a.payload_cap = c.payload_cap;
  a.offsets = c.offsets;
  a.dir = c.dir;
  a.seq_models = c.seq ? B.models + p0 * 3 : nullptr;
  for (int i = 0; i < 10; ++i) a.polyX[i] = c.polyX[i];
  a.status = B.status + p0;
  a.ticket = nullptr;
  a.error = B.error;
  a.rows_area = 0;  // the batch's per-group slices hold the values only
  encode_block<T, CODEC, G, U>(a, b, smem);
}
// The unroll depth changes only the u64 LeCo encoder; other codecs take one instance.
template <typename T, int CODEC, int G>
__device__ __forceinline__ void batch_encode_u(const BatchArgs &B, const DevCol &c, uint32_t ci, uint64_t b, uint8_t *smem) {
  if constexpr (CODEC == kLinear && sizeof(T) == 8 && G != 32) {
    switch (c.unroll) {
      case 1: batch_encode_one<T, CODEC, G, 1>(B, c, ci, b, smem); return;
      case 4: batch_encode_one<T, CODEC, G, 4>(B, c, ci, b, smem); return;
      default: batch_encode_one<T, CODEC, G, 2>(B, c, ci, b, smem); return;
    }
  } else {
    batch_encode_one<T, CODEC, G, 2>(B, c, ci, b, smem);
  }
}
template <typename T, int CODEC>
__device__ __forceinline__ void batch_encode_any(const BatchArgs &B, const DevCol &c, uint32_t ci, uint64_t b, uint8_t *smem) {
  switch (c.group) {
    case 32: batch_encode_u<T, CODEC, 32>(B, c, ci, b, smem); return;
    case 64: batch_encode_u<T, CODEC, 64>(B, c, ci, b, smem); return;
    case 128: batch_encode_u<T, CODEC, 128>(B, c, ci, b, smem); return;
    default: batch_encode_u<T, CODEC, 256>(B, c, ci, b, smem); return;
  }
}

// Persistent encode: one ticket = one work item; group g of the CTA takes block
// first + g of the item with its own slice of shared memory.
__global__ void __launch_bounds__(256, 3) batch_encode_kernel(BatchArgs B) {
  extern __shared__ __align__(16) uint8_t smem[];
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
    const uint32_t gi = threadIdx.x / c.group;
    const uint64_t b = (e & 0xffffffffull) + gi;
    if (b < __ldg(B.prefix + ci + 1) - __ldg(B.prefix + ci))
      LECO_BATCH_DISPATCH(c.codec, c.dtype, batch_encode_any, B, c, ci, b, smem + (size_t)gi * c.slice);
    __syncthreads();  // shared memory is reused by the next item
  }
}

}  // namespace leco
