// Reference-style driver for the C++ drop-in (include/leco_codecs.hpp): the same per-block
// loop as the reference's experiment drivers (encode every block into its own buffer, decode
// every block, random-access sampled positions, check everything against the input), run on
// the GPU codec.  Writes the concatenated block images to argv[1] for the pytest that compares
// them with the oracle.  Exit status 0 = every self-check passed.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "leco_codecs.hpp"

template <typename Codec, typename T>
static int run(const char *name, std::vector<T> &data, int blocks, FILE *out) {
  Codec codec;
  const int N = (int)data.size();
  int block_size = N / blocks;
  blocks = N / block_size;
  if (blocks * block_size < N) blocks++;
  codec.init(blocks, block_size);
  std::vector<uint8_t *> block_start_vec;
  std::vector<uint32_t> sizes;
  for (int i = 0; i < blocks; i++) {
    int len = (i == blocks - 1) ? N - (blocks - 1) * block_size : block_size;
    uint8_t *descriptor = (uint8_t *)malloc((size_t)len * sizeof(T) * 4 + 64);
    uint8_t *end = codec.encodeArray8_int(data.data() + (size_t)i * block_size, len, descriptor, i);
    sizes.push_back((uint32_t)(end - descriptor));
    block_start_vec.push_back(descriptor);
  }
  int bad = 0;
  std::vector<T> recover(N);
  for (int i = 0; i < blocks; i++) {
    int len = (i == blocks - 1) ? N - (blocks - 1) * block_size : block_size;
    codec.decodeArray8(block_start_vec[i], len, recover.data() + (size_t)i * block_size, i);
  }
  for (int j = 0; j < N; j++) bad += recover[j] != data[j];
  uint64_t state = 12345;
  for (int r = 0; r < 2000; r++) {
    state = state * 6364136223846793005ull + 1442695040888963407ull;
    int idx = (int)((state >> 33) % (uint64_t)N);
    T v = codec.randomdecodeArray8(block_start_vec[idx / block_size], idx % block_size, nullptr, N);
    bad += v != data[idx];
  }
  uint32_t nb = (uint32_t)blocks;
  fwrite(&nb, 4, 1, out);
  fwrite(sizes.data(), 4, nb, out);
  for (int i = 0; i < blocks; i++) fwrite(block_start_vec[i], 1, sizes[i], out);
  for (auto *p : block_start_vec) free(p);
  printf("%s: %d blocks, %d mismatches\n", name, blocks, bad);
  return bad;
}

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  FILE *out = fopen(argv[1], "wb");
  if (!out) return 2;
  const int N = 200000;
  std::vector<uint32_t> k32(N);
  std::vector<uint64_t> k64(N);
  uint64_t state = 7;
  for (int i = 0; i < N; i++) {
    state = state * 6364136223846793005ull + 1442695040888963407ull;
    k32[i] = (uint32_t)(1000ull * i + ((state >> 40) & 255));
    k64[i] = 5000000000ull + 77ull * i * i / 64 + ((state >> 20) & 4095);
  }
  int bad = 0;
  bad += run<Codecset::Leco_int<uint32_t>>("leco_u32", k32, 200, out);
  bad += run<Codecset::Leco_int<uint64_t>>("leco_u64", k64, 49, out);
  bad += run<Codecset::FOR_int<uint64_t>>("for_u64", k64, 49, out);
  bad += run<Codecset::Delta_int<uint32_t>>("delta_u32", k32, 200, out);
  bad += run<Codecset::Leco_int_poly<uint64_t, 2>>("poly2_u64", k64, 25, out);
  // column extension: one launch for the whole column
  Codecset::Leco_int<uint64_t> col;
  col.init(0, 4096);
  std::vector<uint8_t> payload;
  std::vector<uint64_t> offsets;
  col.encodeColumn(k64.data(), N, payload, offsets);
  std::vector<uint64_t> back(N);
  col.decodeColumn(payload.data(), offsets.data(), N, back.data());
  for (int i = 0; i < N; i++) bad += back[i] != k64[i];
  std::vector<uint64_t> idx = {0, 1, 4095, 4096, 199999}, got(idx.size());
  col.gather(payload.data(), offsets.data(), N, idx.data(), idx.size(), got.data());
  for (size_t i = 0; i < idx.size(); i++) bad += got[i] != k64[idx[i]];
  fclose(out);
  printf("total mismatches %d\n", bad);
  return bad ? 1 : 0;
}
