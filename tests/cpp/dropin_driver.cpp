// Reference-style driver for the C++ drop-in (include/leco_codecs.hpp): the same per-block
// loop as the reference's experiment drivers (encode every block into its own buffer, decode
// every block, random-access sampled positions, check everything against the input), run on
// the GPU codec.  Writes the concatenated block images to argv[1] for the pytest that compares
// them with the oracle.  Exit status 0 = every self-check passed.
#include <algorithm>
#include <cmath>
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

// The legacy u32 codec's driver loop (experiments/fix_int.cpp:57,75,108,153: init with three
// arguments and encodeArray8 / decodeArray8 / randomdecodeArray8 on uint32_t blocks).
static int run_legacy(const char *name, std::vector<uint32_t> &data, int blocks, FILE *out) {
  Codecset::piecewise_fix_op_max codec;
  const int N = (int)data.size();
  int block_size = N / blocks;
  blocks = N / block_size;
  if (blocks * block_size < N) blocks++;
  codec.init(blocks, block_size, 0);
  std::vector<uint8_t *> block_start_vec;
  std::vector<uint32_t> sizes;
  for (int i = 0; i < blocks; i++) {
    int len = (i == blocks - 1) ? N - (blocks - 1) * block_size : block_size;
    uint8_t *descriptor = (uint8_t *)malloc((size_t)len * 4 * 4 + 64);
    uint8_t *end = codec.encodeArray8(data.data() + (size_t)i * block_size, len, descriptor, i);
    sizes.push_back((uint32_t)(end - descriptor));
    block_start_vec.push_back(descriptor);
  }
  int bad = 0;
  std::vector<uint32_t> recover(N);
  for (int i = 0; i < blocks; i++) {
    int len = (i == blocks - 1) ? N - (blocks - 1) * block_size : block_size;
    codec.decodeArray8(block_start_vec[i], len, recover.data() + (size_t)i * block_size, i);
  }
  for (int j = 0; j < N; j++) bad += recover[j] != data[j];
  uint64_t state = 99;
  for (int r = 0; r < 2000; r++) {
    state = state * 6364136223846793005ull + 1442695040888963407ull;
    int idx = (int)((state >> 33) % (uint64_t)N);
    bad += codec.randomdecodeArray8(block_start_vec[idx / block_size], idx % block_size, nullptr, N) != data[idx];
  }
  uint32_t nb = (uint32_t)blocks;
  fwrite(&nb, 4, 1, out);
  fwrite(sizes.data(), 4, nb, out);
  for (int i = 0; i < blocks; i++) fwrite(block_start_vec[i], 1, sizes[i], out);
  for (auto *p : block_start_vec) free(p);
  printf("%s: %d blocks, %d mismatches\n", name, blocks, bad);
  return bad;
}

// The reference's filter experiments (experiments/leco_int_fix_template.cpp:216-326,
// FOR_int_fix_template.cpp:226-322) on the drop-in classes: zone map from the data, the
// filter_range loop with its zone-map skip, the close-range loop with LeCo's per-block window
// start.  Writes (count, indices) of both loops to `out` for the pytest to compare with the
// oracle.
template <typename Codec>
static void filter_experiment(const std::vector<uint64_t> &data, int blocks, uint64_t filter1, uint64_t filter2,
                              uint64_t base, bool leco, FILE *out) {
  Codec codec;
  const int N = (int)data.size();
  int block_size = N / blocks;
  blocks = N / block_size;
  if (blocks * block_size < N) blocks++;
  codec.init(blocks, block_size);
  std::vector<uint8_t *> block_start_vec;
  std::vector<std::pair<uint64_t, uint64_t>> zonemap;
  for (int i = 0; i < blocks; i++) {
    int len = (i == blocks - 1) ? N - (blocks - 1) * block_size : block_size;
    uint8_t *descriptor = (uint8_t *)malloc((size_t)len * 8 * 4 + 64);
    codec.encodeArray8_int(data.data() + (size_t)i * block_size, len, descriptor, i);
    block_start_vec.push_back(descriptor);
    uint64_t lo = UINT64_MAX, hi = 0;
    for (int j = 0; j < len; j++) {
      lo = std::min(lo, data[(size_t)i * block_size + j]);
      hi = std::max(hi, data[(size_t)i * block_size + j]);
    }
    zonemap.emplace_back(lo, hi);
  }
  std::vector<uint32_t> bit_pos(data.size() + blocks);
  int total_counter = 0;
  for (int i = 0; i < blocks; i++) {
    if (zonemap[i].second <= filter1) continue;
    int len = (i == blocks - 1) ? N - (blocks - 1) * block_size : block_size;
    total_counter += codec.filter_range(block_start_vec[i], len, filter1, bit_pos.data() + total_counter, i);
  }
  fwrite(&total_counter, 4, 1, out);
  fwrite(bit_pos.data(), 4, total_counter, out);
  total_counter = 0;
  for (int i = 0; i < blocks && base; i++) {
    int len = (i == blocks - 1) ? N - (blocks - 1) * block_size : block_size;
    uint64_t f1 = filter1, f2 = filter2;
    if (leco) {
      f1 = ceil((double)(zonemap[i].first - filter1) / (double)base) * base + filter1;
      f2 = ceil((double)(zonemap[i].first - filter1) / (double)base) * base + filter2;
      if (zonemap[i].first % base < filter2 && zonemap[i].first % base > filter1) {
        f1 -= base;
        f2 -= base;
      }
    }
    total_counter += codec.filter_range_close(block_start_vec[i], len, bit_pos.data() + total_counter, i, f1, f2, (int)base);
  }
  fwrite(&total_counter, 4, 1, out);
  fwrite(bit_pos.data(), 4, total_counter, out);
  for (auto *p : block_start_vec) free(p);
}

int main(int argc, char **argv) {
  if (argc < 3) return 2;
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
  bad += run_legacy("legacy_u32", k32, 200, out);
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
  FILE *fout = fopen(argv[2], "wb");
  if (!fout) return 2;
  const uint64_t median = k64[N / 2];
  filter_experiment<Codecset::Leco_int<uint64_t>>(k64, 49, median, median, 0, true, fout);
  filter_experiment<Codecset::Leco_int<uint64_t>>(k64, 49, 1ull << 28, 1ull << 29, 1ull << 30, true, fout);
  filter_experiment<Codecset::FOR_int<uint64_t>>(k64, 49, 1000, 40000, 65536, false, fout);
  fclose(fout);
  printf("total mismatches %d\n", bad);
  return bad ? 1 : 0;
}
