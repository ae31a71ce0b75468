// leco_codecs.hpp -- C++ drop-in for the reference's per-block codec classes.
//
// Same namespace, class names and method signatures as
//   Codecset::Leco_int<T>          headers/piecewise_fix_integer_template.h:14-338
//   Codecset::FOR_int<T>           headers/FOR_integer_template.h:14-249
//   Codecset::Delta_int<T>         headers/delta_integer_template.h:14-158
//   Codecset::Leco_int_poly<T, 2>  headers/poly_fix_integer_template.h:15-292
// so code written against the reference (e.g. experiments/leco_int_fix_template.cpp) compiles
// unchanged after swapping the include.  Every call runs on the GPU through include/leco.h and
// writes / reads the reference's byte format; encodeArray8_int with the default fit mode returns
// the same bytes as the reference (a block whose width would be 8*sizeof(T)-1 is written raw,
// because the reference's own bulk decoder reads such widths as raw).
//
// Per-block calls pay a kernel launch and two copies each; whole columns belong in the column
// API (encodeColumn / decodeColumn / gather below, or leco_encode / leco_decode on device buffers).
// Errors (which the reference leaves undefined) throw std::runtime_error.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "leco.h"

namespace Codecset {
namespace leco_detail {

inline void check(int64_t rc, const char *what) {
  if (rc < 0) throw std::runtime_error(std::string(what) + ": " + leco_last_error());
}

// Bytes of a block image starting at `in`, from its header byte: the whole image for
// bulk decode; for random access only the prefix that holds field `upto`.
inline uint64_t image_bytes(int codec, int dtype, const uint8_t *in, uint32_t length) {
  const uint32_t l = in[0];
  if (l == 127) return 1 + (uint64_t)dtype;
  if (l == 126) return 1 + 2 * (uint64_t)dtype;
  return leco_block_bytes(codec, dtype, l, length);
}

}  // namespace leco_detail

template <typename T, int CODEC>
class LecoBlockCodec {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "T must be uint32_t or uint64_t");

 public:
  std::vector<std::pair<int, int>> mul_add_diff_set;  // always empty; kept for source compatibility
  int blocks = 0;
  int block_size = 0;
  int fit_mode = LECO_FIT_REFERENCE;

  void init(int block, int block_s) {
    blocks = block;
    block_size = block_s;
  }

  // Writes the block image of data[0..length) to res; returns the end pointer.
  uint8_t *encodeArray8_int(const T *data, const size_t length, uint8_t *res, size_t /*nvalue*/) {
    int64_t nb = leco_block_encode(CODEC, (int)sizeof(T), data, (uint32_t)length, fit_mode, res);
    leco_detail::check(nb, "encodeArray8_int");
    return res + nb;
  }

  // Decodes `length` values of the block image `in` into out; returns out.
  T *decodeArray8(const uint8_t *in, const size_t length, T *out, size_t /*nvalue*/) {
    const uint64_t bytes = leco_detail::image_bytes(CODEC, (int)sizeof(T), in, (uint32_t)length);
    leco_detail::check(leco_block_decode(CODEC, (int)sizeof(T), in, bytes, (uint32_t)length, out), "decodeArray8");
    return out;
  }

  // Value `to_find` of the block image `in`.  Like the reference, it reads only the bytes
  // up to that value's field, so the block length is not needed.
  T randomdecodeArray8(const uint8_t *in, int to_find, uint32_t * /*out*/, size_t /*nvalue*/) {
    const uint32_t n = (uint32_t)to_find + 1;
    const uint32_t l = in[0];
    uint64_t bytes = (l == 8 * sizeof(T)) ? 1 + (uint64_t)n * sizeof(T) : leco_detail::image_bytes(CODEC, (int)sizeof(T), in, n);
    T v = 0;
    leco_detail::check(leco_block_random(CODEC, (int)sizeof(T), in, bytes, n, (uint32_t)to_find, &v), "randomdecodeArray8");
    return v;
  }

  // Indices block_id*block_size + k of the values above `filter` (Leco_int / FOR_int
  // only; piecewise_fix_integer_template.h:206-252, FOR_integer_template.h:115-160).
  // Like the reference, `out` must have room for every match; returns the count.
  int filter_range(uint8_t *in, const size_t length, T filter, uint32_t *out, size_t block_id) {
    return run_filter(in, length, out, block_id, 0, (uint64_t)filter, 0, 0);
  }
  // Close range: windows (filter1 + p*base, filter2 + p*base) for Leco_int, residues
  // filter1 < v % base < filter2 for FOR_int (:254-303, FOR :166-215).  Indices of every
  // window are appended (the reference overwrites earlier windows' for l > 0); the count
  // is the reference's.
  int filter_range_close(uint8_t *in, const size_t length, uint32_t *out, size_t block_id, T filter1, T filter2,
                         int base) {
    return run_filter(in, length, out, block_id, 1, (uint64_t)filter1, (uint64_t)filter2, (uint64_t)(int64_t)base);
  }

  // ---- column extensions (one launch per column) -------------------------------------
  // Encodes data[0..n) in blocks of block_size: payload = concatenated block images,
  // offsets[b] = byte offset of block b, offsets[nblocks] = total.
  void encodeColumn(const T *data, size_t n, std::vector<uint8_t> &payload, std::vector<uint64_t> &offsets) const {
    const uint64_t cap = leco_max_payload_bytes(CODEC, (int)sizeof(T), n, (uint32_t)block_size);
    payload.resize(cap);
    offsets.resize(leco_num_blocks(n, (uint32_t)block_size) + 1);
    uint64_t bytes = 0;
    leco_detail::check(leco_encode_host(CODEC, (int)sizeof(T), data, n, (uint32_t)block_size, fit_mode, payload.data(), cap,
                                        offsets.data(), &bytes),
                       "encodeColumn");
    payload.resize(bytes + LECO_PAYLOAD_SLACK);
  }
  void decodeColumn(const uint8_t *payload, const uint64_t *offsets, size_t n, T *out) const {
    leco_detail::check(leco_decode_host(CODEC, (int)sizeof(T), payload, offsets, n, (uint32_t)block_size, out), "decodeColumn");
  }
  void gather(const uint8_t *payload, const uint64_t *offsets, size_t n, const uint64_t *idx, size_t m, T *out) const {
    leco_detail::check(leco_gather_host(CODEC, (int)sizeof(T), payload, offsets, n, (uint32_t)block_size, idx, m, out), "gather");
  }

 private:
  int run_filter(const uint8_t *in, size_t length, uint32_t *out, size_t block_id, int close, uint64_t f1, uint64_t f2,
                 uint64_t base) {
    const uint64_t bytes = leco_detail::image_bytes(CODEC, (int)sizeof(T), in, (uint32_t)length);
    const uint32_t start = (uint32_t)(block_id * (size_t)block_size);
    uint64_t cap = length + 1;  // every index once, plus the l == 0 window end
    int64_t c = leco_block_filter(CODEC, (int)sizeof(T), in, bytes, (uint32_t)length, start, close, f1, f2, base, out, cap);
    leco_detail::check(c, close ? "filter_range_close" : "filter_range");
    if ((uint64_t)c > cap) {  // overlapping windows counted an index more than once
      c = leco_block_filter(CODEC, (int)sizeof(T), in, bytes, (uint32_t)length, start, close, f1, f2, base, out, (uint64_t)c);
      leco_detail::check(c, "filter_range_close");
    }
    return (int)c;
  }
};

template <typename T>
class Leco_int : public LecoBlockCodec<T, LECO_CODEC_LINEAR> {};

template <typename T>
class FOR_int : public LecoBlockCodec<T, LECO_CODEC_FOR> {};

template <typename T>
class Delta_int : public LecoBlockCodec<T, LECO_CODEC_DELTA> {};

// The reference's legacy u32 codec (piecewise_fix_op_minimize_maxerror.h:20-186).
// encodeArray8 writes the reference's block image (:45-119) byte for byte.  The encoder's
// difference lists (mul_add_diff_set, :79-84) stay empty: decodeArray8 returns the stored
// values, whereas the reference's own bulk decoder accumulates the prediction by addition and
// its drivers then correct it with those lists (experiments/fix_int.cpp:110-117).
class piecewise_fix_op_max {
 public:
  std::vector<int> mul_add_diff_set, mul_add_diff_set_minus;  // always empty: nothing to correct
  int block_num = 0;
  int block_size = 0;
  void init(int blocks, int blocksize, int /*extra*/) {
    block_num = blocks;
    block_size = blocksize;
  }
  int fit_mode = LECO_FIT_REFERENCE;
  // Writes the block image of in[0..length) to res; returns the end pointer.
  uint8_t *encodeArray8(uint32_t *in, const size_t length, uint8_t *res, size_t /*nvalue*/) {
    int64_t nb = leco_block_encode(LECO_CODEC_LINEAR_F32, LECO_U32, in, (uint32_t)length, fit_mode, res);
    leco_detail::check(nb, "encodeArray8");
    return res + nb;
  }
  uint32_t *decodeArray8(uint8_t *in, const size_t length, uint32_t *out, size_t /*nvalue*/) {
    const uint64_t bytes = leco_block_bytes(LECO_CODEC_LINEAR_F32, LECO_U32, in[0], (uint32_t)length);
    leco_detail::check(leco_block_decode(LECO_CODEC_LINEAR_F32, LECO_U32, in, bytes, (uint32_t)length, out), "decodeArray8");
    return out;
  }
  uint32_t randomdecodeArray8(uint8_t *in, const size_t l, uint32_t * /*out*/, size_t /*nvalue*/) {
    const uint32_t n = (uint32_t)l + 1;
    const uint64_t bytes = leco_block_bytes(LECO_CODEC_LINEAR_F32, LECO_U32, in[0], n);
    uint32_t v = 0;
    leco_detail::check(leco_block_random(LECO_CODEC_LINEAR_F32, LECO_U32, in, bytes, n, (uint32_t)l, &v), "randomdecodeArray8");
    return v;
  }
};

template <typename T, int degree>
class Leco_int_poly : public LecoBlockCodec<T, LECO_CODEC_POLY2> {
  static_assert(degree == 2, "the B200 codec provides the degree-2 polynomial model");
};

}  // namespace Codecset
