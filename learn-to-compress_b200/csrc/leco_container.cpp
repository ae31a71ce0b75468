// leco_container.cpp -- the column container on disk, and import/export of the
// reference's per-block byte strings.
//
// The reference keeps every block as a separate malloc'ed byte string and has no
// file format (its drivers encode, measure and free; experiments/leco_int_fix_template.cpp:108-127).
// A column here is payload (block images back to back) + offsets[nunits+1]
// (+ starts[nunits] for variable-length segments); the container stores exactly
// that, little-endian, behind a 64-byte header:
//
//   0  char[8] "LECOCOL1"         32 u64 nunits (blocks or segments)
//   8  u32 version (1)            40 u64 payload bytes
//  12  u32 codec                  48 u64 flags (bit 0: starts present)
//  16  u32 dtype (bytes/value)    56 u64 checksum of the rest of the file and header bytes 0-55
//  20  u32 block size (0: varlen)
//  24  u64 n (values)
//
// then offsets[nunits+1] (u64), starts[nunits] (u64, when flagged) and the payload
// padded to a multiple of 8 bytes.  The checksum is a four-lane multiply-rotate
// hash over 8-byte words (defined below), so a flipped or truncated byte is caught
// before any block is handed to a kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "leco_internal.h"

namespace {

constexpr char kMagic[8] = {'L', 'E', 'C', 'O', 'C', 'O', 'L', '1'};
constexpr uint32_t kVersion = 1;

struct FileHeader {
  char magic[8];
  uint32_t version, codec, dtype, block_size;
  uint64_t n, nunits, payload_bytes, flags, checksum;
};
static_assert(sizeof(FileHeader) == 64, "header layout");

inline uint64_t rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

// Four independent lanes over consecutive 8-byte words, folded at the end.
struct Hasher {
  static constexpr uint64_t P1 = 0x9E3779B185EBCA87ull, P2 = 0xC2B2AE3D27D4EB4Full, P3 = 0x165667B19E3779F9ull;
  uint64_t lane[4] = {P1, P2, P3, P1 ^ P2};
  uint64_t words = 0;
  uint8_t tail[32];
  size_t ntail = 0;
  void mix_block(const uint8_t *p) {
    for (int i = 0; i < 4; ++i) {
      uint64_t w;
      memcpy(&w, p + 8 * i, 8);
      lane[i] = rotl(lane[i] + w * P2, 31) * P1;
    }
    words += 4;
  }
  void update(const void *data, size_t len) {
    const uint8_t *p = static_cast<const uint8_t *>(data);
    if (ntail) {
      const size_t take = std::min(len, 32 - ntail);
      memcpy(tail + ntail, p, take);
      ntail += take;
      p += take;
      len -= take;
      if (ntail == 32) {
        mix_block(tail);
        ntail = 0;
      }
    }
    for (; len >= 32; p += 32, len -= 32) mix_block(p);
    memcpy(tail, p, len);
    ntail = len;
  }
  uint64_t digest() {
    uint64_t h = rotl(lane[0], 1) + rotl(lane[1], 7) + rotl(lane[2], 12) + rotl(lane[3], 18);
    h ^= words * 32 + ntail;
    for (size_t i = 0; i < ntail; ++i) h = rotl(h ^ (tail[i] * P3), 11) * P1;
    h ^= h >> 33;
    h *= P2;
    h ^= h >> 29;
    h *= P3;
    h ^= h >> 32;
    return h;
  }
};

int fail(int code, const std::string &msg) { return leco::record_error(code, msg); }

struct File {
  FILE *f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

uint64_t pad8(uint64_t x) { return (x + 7) & ~7ull; }

int check_info(const leco_container_info *info) {
  if (!info) return fail(LECO_ERR_ARG, "container: null info");
  if (info->codec < LECO_CODEC_LINEAR || info->codec > LECO_CODEC_VARLEN) return fail(LECO_ERR_ARG, "container: bad codec");
  if (info->dtype != LECO_U32 && info->dtype != LECO_U64) return fail(LECO_ERR_ARG, "container: bad dtype");
  if (info->codec == LECO_CODEC_VARLEN) {
    if (info->dtype != LECO_U64 || !info->has_starts) return fail(LECO_ERR_ARG, "container: variable-length columns are u64 with starts");
  } else {
    if (!info->block_size || info->block_size > LECO_MAX_BLOCK) return fail(LECO_ERR_ARG, "container: bad block size");
    if (info->nunits != leco_num_blocks(info->n, info->block_size)) return fail(LECO_ERR_ARG, "container: nunits != blocks of n");
  }
  return LECO_OK;
}

// Reads and checks the header and the offsets/starts arrays; leaves the file at the payload.
int read_head(FILE *f, const char *path, FileHeader &h, std::vector<uint64_t> &off, std::vector<uint64_t> &starts, Hasher &hs) {
  if (fread(&h, sizeof h, 1, f) != 1) return fail(LECO_ERR_CORRUPT, std::string("container: short header in ") + path);
  if (memcmp(h.magic, kMagic, 8) != 0) return fail(LECO_ERR_CORRUPT, std::string("container: not a LECOCOL1 file: ") + path);
  if (h.version != kVersion) return fail(LECO_ERR_UNSUPPORTED, "container: unknown version");
  leco_container_info info{(int)h.codec, (int)h.dtype, h.block_size, h.n, h.nunits, h.payload_bytes, (int)(h.flags & 1)};
  if (check_info(&info)) return fail(LECO_ERR_CORRUPT, std::string("container: inconsistent header in ") + path);
  if (h.nunits > (1ull << 40) || h.payload_bytes > (1ull << 46)) return fail(LECO_ERR_CORRUPT, "container: sizes out of range");
  hs.update(&h, offsetof(FileHeader, checksum));
  off.resize(h.nunits + 1);
  if (fread(off.data(), 8, off.size(), f) != off.size()) return fail(LECO_ERR_CORRUPT, "container: truncated offsets");
  hs.update(off.data(), off.size() * 8);
  if (off[0] != 0 || off[h.nunits] != h.payload_bytes) return fail(LECO_ERR_CORRUPT, "container: offsets do not span the payload");
  for (uint64_t i = 0; i < h.nunits; ++i)
    if (off[i] >= off[i + 1]) return fail(LECO_ERR_CORRUPT, "container: offsets not increasing");
  if (h.flags & 1) {
    starts.resize(h.nunits);
    if (fread(starts.data(), 8, starts.size(), f) != starts.size()) return fail(LECO_ERR_CORRUPT, "container: truncated starts");
    hs.update(starts.data(), starts.size() * 8);
    for (uint64_t i = 0; i < h.nunits; ++i)
      if ((i == 0 ? starts[0] != 0 : starts[i] <= starts[i - 1]) || starts[i] >= h.n)
        return fail(LECO_ERR_CORRUPT, "container: segment starts not increasing within the column");
  }
  return LECO_OK;
}

int read_payload(FILE *f, const FileHeader &h, uint8_t *dst, Hasher &hs) {
  const uint64_t padded = pad8(h.payload_bytes);
  if (fread(dst, 1, h.payload_bytes, f) != h.payload_bytes) return fail(LECO_ERR_CORRUPT, "container: truncated payload");
  hs.update(dst, h.payload_bytes);
  uint8_t zeros[8] = {0}, pad[8];
  const size_t np = (size_t)(padded - h.payload_bytes);
  if (np && fread(pad, 1, np, f) != np) return fail(LECO_ERR_CORRUPT, "container: truncated payload padding");
  hs.update(zeros, np);
  if (hs.digest() != h.checksum) return fail(LECO_ERR_CORRUPT, "container: checksum mismatch");
  return LECO_OK;
}

}  // namespace

extern "C" {

int leco_container_write(const char *path, const leco_container_info *info, const uint8_t *h_payload,
                         const uint64_t *h_offsets, const uint64_t *h_starts) {
  int rc = check_info(info);
  if (rc) return rc;
  if (!path || !h_payload || !h_offsets || (info->has_starts && !h_starts))
    return fail(LECO_ERR_ARG, "leco_container_write: null argument");
  if (h_offsets[0] != 0 || h_offsets[info->nunits] != info->payload_bytes)
    return fail(LECO_ERR_ARG, "leco_container_write: offsets do not span payload_bytes");
  FileHeader h{};
  memcpy(h.magic, kMagic, 8);
  h.version = kVersion;
  h.codec = (uint32_t)info->codec;
  h.dtype = (uint32_t)info->dtype;
  h.block_size = info->codec == LECO_CODEC_VARLEN ? 0 : info->block_size;
  h.n = info->n;
  h.nunits = info->nunits;
  h.payload_bytes = info->payload_bytes;
  h.flags = info->has_starts ? 1 : 0;
  Hasher hs;
  hs.update(&h, offsetof(FileHeader, checksum));
  hs.update(h_offsets, (info->nunits + 1) * 8);
  if (info->has_starts) hs.update(h_starts, info->nunits * 8);
  hs.update(h_payload, info->payload_bytes);
  const uint8_t zeros[8] = {0};
  const size_t np = (size_t)(pad8(info->payload_bytes) - info->payload_bytes);
  hs.update(zeros, np);
  h.checksum = hs.digest();
  const std::string tmp = std::string(path) + ".tmp";
  {
    File fh;
    fh.f = fopen(tmp.c_str(), "wb");
    if (!fh.f) return fail(LECO_ERR_ARG, std::string("leco_container_write: cannot open ") + tmp);
    bool ok = fwrite(&h, sizeof h, 1, fh.f) == 1 &&
              fwrite(h_offsets, 8, info->nunits + 1, fh.f) == info->nunits + 1 &&
              (!info->has_starts || fwrite(h_starts, 8, info->nunits, fh.f) == info->nunits) &&
              fwrite(h_payload, 1, info->payload_bytes, fh.f) == info->payload_bytes &&
              (!np || fwrite(zeros, 1, np, fh.f) == np);
    ok = ok && fflush(fh.f) == 0;
    if (!ok) return fail(LECO_ERR_ARG, "leco_container_write: write failed");
  }
  // the file appears under its name only when complete
  if (rename(tmp.c_str(), path) != 0) return fail(LECO_ERR_ARG, "leco_container_write: rename failed");
  return LECO_OK;
}

int leco_container_info_read(const char *path, leco_container_info *info) {
  if (!path || !info) return fail(LECO_ERR_ARG, "leco_container_info_read: null argument");
  File fh;
  fh.f = fopen(path, "rb");
  if (!fh.f) return fail(LECO_ERR_ARG, std::string("leco_container_info_read: cannot open ") + path);
  FileHeader h;
  std::vector<uint64_t> off, starts;
  Hasher hs;
  int rc = read_head(fh.f, path, h, off, starts, hs);
  if (rc) return rc;
  *info = leco_container_info{(int)h.codec, (int)h.dtype, h.block_size, h.n, h.nunits, h.payload_bytes, (int)(h.flags & 1)};
  return LECO_OK;
}

int leco_container_read(const char *path, uint8_t *h_payload, uint64_t payload_cap, uint64_t *h_offsets, uint64_t *h_starts) {
  if (!path || !h_payload || !h_offsets) return fail(LECO_ERR_ARG, "leco_container_read: null argument");
  File fh;
  fh.f = fopen(path, "rb");
  if (!fh.f) return fail(LECO_ERR_ARG, std::string("leco_container_read: cannot open ") + path);
  FileHeader h;
  std::vector<uint64_t> off, starts;
  Hasher hs;
  int rc = read_head(fh.f, path, h, off, starts, hs);
  if (rc) return rc;
  if (payload_cap < h.payload_bytes) return fail(LECO_ERR_CAPACITY, "leco_container_read: payload buffer too small");
  if ((h.flags & 1) && !h_starts) return fail(LECO_ERR_ARG, "leco_container_read: the column has segment starts");
  if ((rc = read_payload(fh.f, h, h_payload, hs))) return rc;
  memcpy(h_offsets, off.data(), off.size() * 8);
  if (h.flags & 1) memcpy(h_starts, starts.data(), starts.size() * 8);
  if (h.codec != LECO_CODEC_VARLEN) {
    uint64_t bad = 0;
    if ((rc = leco_validate_host((int)h.codec, (int)h.dtype, h_payload, h.payload_bytes, h_offsets, h.n, h.block_size, &bad)))
      return rc;
  }
  return LECO_OK;
}

// Device buffers: the column is staged through host memory (one copy each way).
int leco_container_save_device(const char *path, const leco_container_info *info, const uint8_t *d_payload,
                               const uint64_t *d_offsets, const uint64_t *d_starts, leco_stream_t stream) {
  int rc = check_info(info);
  if (rc) return rc;
  if (!d_payload || !d_offsets || (info->has_starts && !d_starts)) return fail(LECO_ERR_ARG, "leco_container_save_device: null argument");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  std::vector<uint8_t> pay(info->payload_bytes);
  std::vector<uint64_t> off(info->nunits + 1), starts(info->has_starts ? info->nunits : 0);
  if (cudaMemcpyAsync(off.data(), d_offsets, off.size() * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(pay.data(), d_payload, pay.size(), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      (info->has_starts && cudaMemcpyAsync(starts.data(), d_starts, starts.size() * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return fail(LECO_ERR_CUDA, "leco_container_save_device: copy from the device failed");
  return leco_container_write(path, info, pay.data(), off.data(), info->has_starts ? starts.data() : nullptr);
}

int leco_container_load_device(const char *path, uint8_t *d_payload, uint64_t payload_cap, uint64_t *d_offsets,
                               uint64_t *d_starts, leco_stream_t stream) {
  leco_container_info info;
  int rc = leco_container_info_read(path, &info);
  if (rc) return rc;
  if (!d_payload || !d_offsets || (info.has_starts && !d_starts)) return fail(LECO_ERR_ARG, "leco_container_load_device: null argument");
  if (payload_cap < info.payload_bytes + LECO_PAYLOAD_SLACK)
    return fail(LECO_ERR_CAPACITY, "leco_container_load_device: payload buffer needs payload_bytes + LECO_PAYLOAD_SLACK");
  std::vector<uint8_t> pay(info.payload_bytes + LECO_PAYLOAD_SLACK, 0);
  std::vector<uint64_t> off(info.nunits + 1), starts(info.has_starts ? info.nunits : 0);
  if ((rc = leco_container_read(path, pay.data(), pay.size(), off.data(), info.has_starts ? starts.data() : nullptr))) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(d_payload, pay.data(), pay.size(), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_offsets, off.data(), off.size() * 8, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      (info.has_starts && cudaMemcpyAsync(d_starts, starts.data(), starts.size() * 8, cudaMemcpyHostToDevice, st) != cudaSuccess) ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return fail(LECO_ERR_CUDA, "leco_container_load_device: copy to the device failed");
  return LECO_OK;
}

int leco_import_blocks(const uint8_t *const *h_blocks, const uint64_t *h_sizes, uint64_t nblocks, uint8_t *h_payload,
                       uint64_t payload_cap, uint64_t *h_offsets) {
  if (!h_blocks || !h_sizes || !h_payload || !h_offsets) return fail(LECO_ERR_ARG, "leco_import_blocks: null argument");
  uint64_t pos = 0;
  for (uint64_t b = 0; b < nblocks; ++b) {
    if (!h_blocks[b] || !h_sizes[b]) return fail(LECO_ERR_ARG, "leco_import_blocks: empty block");
    if (pos + h_sizes[b] > payload_cap) return fail(LECO_ERR_CAPACITY, "leco_import_blocks: payload buffer too small");
    h_offsets[b] = pos;
    memcpy(h_payload + pos, h_blocks[b], h_sizes[b]);
    pos += h_sizes[b];
  }
  h_offsets[nblocks] = pos;
  return LECO_OK;
}

int leco_export_blocks(const uint8_t *h_payload, const uint64_t *h_offsets, uint64_t nblocks, uint8_t *const *h_blocks,
                       uint64_t *h_sizes) {
  if (!h_payload || !h_offsets || !h_sizes) return fail(LECO_ERR_ARG, "leco_export_blocks: null argument");
  for (uint64_t b = 0; b < nblocks; ++b) {
    if (h_offsets[b + 1] <= h_offsets[b]) return fail(LECO_ERR_CORRUPT, "leco_export_blocks: offsets not increasing");
    h_sizes[b] = h_offsets[b + 1] - h_offsets[b];
    if (h_blocks) {
      if (!h_blocks[b]) return fail(LECO_ERR_ARG, "leco_export_blocks: null block buffer");
      memcpy(h_blocks[b], h_payload + h_offsets[b], h_sizes[b]);
    }
  }
  return LECO_OK;
}

}  // extern "C"
