// Test infrastructure only: a C-ABI wrapper around the UNMODIFIED reference codec
// headers (yhliu918/Learn-to-Compress, headers/*_integer_template.h), compiled
// from where they lie by oracle/Makefile into oracle/_ref/libleco_ref.so.  It is
// the checker that pins the plain-C restatement (oracle/leco_oracle.c) and the
// reference arm of bench.py; nothing in the product links it.
//
// Every function forwards to the reference class method named in its comment and
// adds only the per-block loop of the reference drivers
// (experiments/leco_int_fix_template.cpp:108-127 encode, :142-153 decode,
// :189-207 random access).
#include "piecewise_fix_integer_template.h"
#include "FOR_integer_template.h"
#include "delta_integer_template.h"
#include "poly_fix_integer_template.h"
#include "piecewise_cost_merge_integer_template_double_wo_round.h"

#include <atomic>
#include <thread>
#include <vector>

using namespace Codecset;

namespace {

enum { C_LECO = 0, C_FOR = 1, C_DELTA = 2, C_POLY2 = 3 };

template <typename T>
size_t enc_block(int codec, const T *data, size_t len, uint8_t *out, size_t block_id) {
  uint8_t *end = out;
  switch (codec) {
    case C_LECO: { Leco_int<T> c; end = c.encodeArray8_int(data, len, out, block_id); break; }
    case C_FOR: { FOR_int<T> c; end = c.encodeArray8_int(data, len, out, block_id); break; }
    case C_DELTA: { Delta_int<T> c; end = c.encodeArray8_int(const_cast<T *>(data), len, out, block_id); break; }
    case C_POLY2: { Leco_int_poly<T, 2> c; end = c.encodeArray8_int(data, len, out, block_id); break; }
    default: return 0;
  }
  return (size_t)(end - out);
}

template <typename T>
void dec_block(int codec, const uint8_t *in, size_t len, T *out, size_t block_id) {
  switch (codec) {
    case C_LECO: { Leco_int<T> c; c.decodeArray8(in, len, out, block_id); break; }
    case C_FOR: { FOR_int<T> c; c.decodeArray8(in, len, out, block_id); break; }
    case C_DELTA: { Delta_int<T> c; c.decodeArray8(const_cast<uint8_t *>(in), len, out, block_id); break; }
    case C_POLY2: { Leco_int_poly<T, 2> c; c.decodeArray8(in, len, out, block_id); break; }
    default: break;
  }
}

template <typename T>
T ra_block(int codec, const uint8_t *in, int k) {
  switch (codec) {
    case C_LECO: { Leco_int<T> c; return c.randomdecodeArray8(in, k, nullptr, 0); }
    case C_FOR: { FOR_int<T> c; return c.randomdecodeArray8(in, k, nullptr, 0); }
    case C_DELTA: { Delta_int<T> c; return c.randomdecodeArray8(const_cast<uint8_t *>(in), k, nullptr, 0); }
    case C_POLY2: { Leco_int_poly<T, 2> c; return c.randomdecodeArray8(in, k, nullptr, 0); }
    default: return 0;
  }
}

// Runs fn(lo, hi) over [0, n) split into `threads` contiguous ranges.
template <typename F>
void parallel_ranges(size_t n, int threads, F fn) {
  if (threads <= 1 || n < 2) { fn((size_t)0, n); return; }
  std::vector<std::thread> pool;
  size_t per = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    size_t lo = (size_t)t * per, hi = std::min(n, lo + per);
    if (lo >= hi) break;
    pool.emplace_back([=] { fn(lo, hi); });
  }
  for (auto &th : pool) th.join();
}

template <typename T>
size_t col_encode(int codec, const T *data, size_t n, uint32_t bs, uint8_t *out, uint64_t *offsets) {
  size_t nb = (n + bs - 1) / bs, pos = 0;
  for (size_t b = 0; b < nb; ++b) {
    size_t len = std::min<size_t>(bs, n - b * bs);
    offsets[b] = pos;
    pos += enc_block<T>(codec, data + b * bs, len, out + pos, b);
  }
  offsets[nb] = pos;
  return pos;
}

// col_encode over `threads` contiguous block ranges: each range is encoded into its own
// buffer, then the images are placed back to back in `out` (same bytes as col_encode).
template <typename T>
size_t col_encode_mt(int codec, const T *data, size_t n, uint32_t bs, uint8_t *out, uint64_t *offsets, int threads) {
  const size_t nb = (n + bs - 1) / bs;
  if (threads <= 1 || nb < 2) return col_encode<T>(codec, data, n, bs, out, offsets);
  const size_t per = (nb + threads - 1) / threads;
  const size_t parts = (nb + per - 1) / per;
  std::vector<std::vector<uint8_t>> buf(parts);
  std::vector<size_t> used(parts, 0);
  parallel_ranges(parts, (int)parts, [&](size_t lo, size_t hi) {
    for (size_t p = lo; p < hi; ++p) {
      const size_t b0 = p * per, b1 = std::min(nb, b0 + per);
      const size_t v0 = b0 * bs, v1 = std::min(n, b1 * (size_t)bs);
      buf[p].resize((v1 - v0) * sizeof(T) * 2 + (b1 - b0) * 64 + 64);
      size_t pos = 0;
      for (size_t b = b0; b < b1; ++b) {
        const size_t len = std::min<size_t>(bs, n - b * bs);
        offsets[b] = pos;  // relative to the range; rebased below
        pos += enc_block<T>(codec, data + b * bs, len, buf[p].data() + pos, b);
      }
      used[p] = pos;
    }
  });
  std::vector<size_t> base(parts + 1, 0);
  for (size_t p = 0; p < parts; ++p) base[p + 1] = base[p] + used[p];
  parallel_ranges(parts, (int)parts, [&](size_t lo, size_t hi) {
    for (size_t p = lo; p < hi; ++p) {
      memcpy(out + base[p], buf[p].data(), used[p]);
      const size_t b0 = p * per, b1 = std::min(nb, b0 + per);
      for (size_t b = b0; b < b1; ++b) offsets[b] += base[p];
    }
  });
  offsets[nb] = base[parts];
  return base[parts];
}

template <typename T>
void col_decode(int codec, const uint8_t *payload, const uint64_t *offsets, size_t n, uint32_t bs, T *out, int threads) {
  size_t nb = (n + bs - 1) / bs;
  parallel_ranges(nb, threads, [&](size_t lo, size_t hi) {
    for (size_t b = lo; b < hi; ++b) {
      size_t len = std::min<size_t>(bs, n - b * bs);
      dec_block<T>(codec, payload + offsets[b], len, out + b * bs, b);
    }
  });
}

template <typename T>
void col_random(int codec, const uint8_t *payload, const uint64_t *offsets, uint32_t bs, const uint64_t *idx, size_t m, T *out, int threads) {
  parallel_ranges(m, threads, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i) {
      uint64_t g = idx[i];
      out[i] = ra_block<T>(codec, payload + offsets[g / bs], (int)(g % bs));
    }
  });
}

}  // namespace

extern "C" {

// One block through <Codec>::encodeArray8_int; returns the bytes written.
size_t ref_encode_block_u32(int codec, const uint32_t *d, size_t len, uint8_t *out) { return enc_block<uint32_t>(codec, d, len, out, 0); }
size_t ref_encode_block_u64(int codec, const uint64_t *d, size_t len, uint8_t *out) { return enc_block<uint64_t>(codec, d, len, out, 0); }
// One block through <Codec>::decodeArray8.
void ref_decode_block_u32(int codec, const uint8_t *in, size_t len, uint32_t *out) { dec_block<uint32_t>(codec, in, len, out, 0); }
void ref_decode_block_u64(int codec, const uint8_t *in, size_t len, uint64_t *out) { dec_block<uint64_t>(codec, in, len, out, 0); }
// One value through <Codec>::randomdecodeArray8.
uint32_t ref_random_u32(int codec, const uint8_t *in, int k) { return ra_block<uint32_t>(codec, in, k); }
uint64_t ref_random_u64(int codec, const uint8_t *in, int k) { return ra_block<uint64_t>(codec, in, k); }

// Whole column, blocks of `bs` values, concatenated block images + byte offsets[nb+1].
size_t ref_column_encode_u32(int codec, const uint32_t *d, size_t n, uint32_t bs, uint8_t *out, uint64_t *off) { return col_encode<uint32_t>(codec, d, n, bs, out, off); }
size_t ref_column_encode_u64(int codec, const uint64_t *d, size_t n, uint32_t bs, uint8_t *out, uint64_t *off) { return col_encode<uint64_t>(codec, d, n, bs, out, off); }
// The same column encoded with `threads` host threads over contiguous block ranges.
size_t ref_column_encode_mt_u32(int codec, const uint32_t *d, size_t n, uint32_t bs, uint8_t *out, uint64_t *off, int threads) { return col_encode_mt<uint32_t>(codec, d, n, bs, out, off, threads); }
size_t ref_column_encode_mt_u64(int codec, const uint64_t *d, size_t n, uint32_t bs, uint8_t *out, uint64_t *off, int threads) { return col_encode_mt<uint64_t>(codec, d, n, bs, out, off, threads); }
void ref_column_decode_u32(int codec, const uint8_t *p, const uint64_t *off, size_t n, uint32_t bs, uint32_t *out, int threads) { col_decode<uint32_t>(codec, p, off, n, bs, out, threads); }
void ref_column_decode_u64(int codec, const uint8_t *p, const uint64_t *off, size_t n, uint32_t bs, uint64_t *out, int threads) { col_decode<uint64_t>(codec, p, off, n, bs, out, threads); }
void ref_column_random_u32(int codec, const uint8_t *p, const uint64_t *off, uint32_t bs, const uint64_t *idx, size_t m, uint32_t *out, int threads) { col_random<uint32_t>(codec, p, off, bs, idx, m, out, threads); }
void ref_column_random_u64(int codec, const uint8_t *p, const uint64_t *off, uint32_t bs, const uint64_t *idx, size_t m, uint64_t *out, int threads) { col_random<uint64_t>(codec, p, off, bs, idx, m, out, threads); }

// ---- Variable-length cost-merge codec, u64 (Leco_cost_merge_double_wo_round) ----
// Drives the class the way experiments/leco_double_int_template_wo_round.cpp does:
// init(blocks, block_size, delta), encodeArray8_int per coarse block over the whole
// array, then hands out the segment images.  The handle owns the codec object.
void *ref_varlen_encode_u64(const uint64_t *d, size_t n, int blocks, int64_t delta) {
  auto *c = new Leco_cost_merge_double_wo_round<uint64_t>();
  int block_size = (int)(n / (size_t)blocks);
  int nb = (int)(n / (size_t)block_size);
  if ((size_t)nb * block_size < n) nb++;
  c->init(nb, block_size, (uint64_t)delta);
  std::vector<uint8_t> scratch(n * sizeof(uint64_t) * 4 + 64);
  for (int i = 0; i < nb; ++i) {
    size_t len = (size_t)block_size;
    if (i == nb - 1) len = n - (size_t)(nb - 1) * block_size;
    c->encodeArray8_int(const_cast<uint64_t *>(d), len, scratch.data(), (size_t)i);
  }
  return c;
}
size_t ref_varlen_segments(void *h) { return ((Leco_cost_merge_double_wo_round<uint64_t> *)h)->block_start_vec_total.size(); }
// Copies segment starts (value index), byte sizes and the concatenated images.
size_t ref_varlen_export(void *h, uint32_t *starts, uint64_t *byte_off, uint8_t *payload) {
  auto *c = (Leco_cost_merge_double_wo_round<uint64_t> *)h;
  size_t ns = c->block_start_vec_total.size(), pos = 0;
  for (size_t i = 0; i < ns; ++i) {
    if (starts) starts[i] = c->segment_index_total[i];
    if (byte_off) byte_off[i] = pos;
    if (payload) memcpy(payload + pos, c->block_start_vec_total[i], c->segment_length_total[i]);
    pos += c->segment_length_total[i];
  }
  if (byte_off) byte_off[ns] = pos;
  return pos;
}
// Leco_cost_merge_double_wo_round::decodeArray8 over all segments.
void ref_varlen_decode(void *h, size_t n, uint64_t *out) {
  auto *c = (Leco_cost_merge_double_wo_round<uint64_t> *)h;
  c->decodeArray8(n, out, n);
  c->segment_index_total.pop_back();  // decodeArray8 appends n; undo so the handle stays reusable
}
// get_segment_id (ALEX upper_bound) + randomdecodeArray8 for each index.
void ref_varlen_random(void *h, const uint64_t *idx, size_t m, uint64_t *out) {
  auto *c = (Leco_cost_merge_double_wo_round<uint64_t> *)h;
  for (size_t i = 0; i < m; ++i) {
    int sid = c->get_segment_id((int)idx[i]);
    out[i] = c->randomdecodeArray8(sid, c->block_start_vec_total[sid], (int)idx[i], nullptr, 0);
  }
}
void ref_varlen_free(void *h) {
  auto *c = (Leco_cost_merge_double_wo_round<uint64_t> *)h;
  for (auto *p : c->block_start_vec_total) free(p);
  delete c;
}

}  // extern "C"

// ---- predicate pushdown ----------------------------------------------------
// The filter experiments' loops (experiments/leco_int_fix_template.cpp:244-256 and
// :290-322, FOR_int_fix_template.cpp:254-266 and :303-322) around the codecs'
// filter_range / filter_range_close.  zmax / zmin: the zone map (per-block maximum
// / minimum); zmax may be null (no skipping).  For LeCo close-range, zmin null
// passes filter1/filter2 to every block unchanged.  Returns the count; `out`
// is what the codec methods left there.
namespace {
template <typename T>
size_t col_filter(int codec, const uint8_t *p, const uint64_t *off, size_t n, uint32_t bs, T filter, const uint64_t *zmax,
                  uint32_t *out) {
  size_t nb = (n + bs - 1) / bs;
  Leco_int<T> lc;
  FOR_int<T> fc;
  lc.init((int)nb, (int)bs);
  fc.init((int)nb, (int)bs);
  size_t total = 0;
  for (size_t i = 0; i < nb; ++i) {
    if (zmax && (T)zmax[i] <= filter) continue;
    size_t len = std::min<size_t>(bs, n - i * bs);
    uint8_t *in = const_cast<uint8_t *>(p + off[i]);
    total += codec == C_LECO ? lc.filter_range(in, len, filter, out + total, (int)i)
                             : fc.filter_range(in, len, filter, out + total, i);
  }
  return total;
}

template <typename T>
void window_start(T lo, T filter1, T filter2, T base, T *a, T *b) {
  T f1 = ceil((double)(T)(lo - filter1) / (double)base) * base + filter1;
  T f2 = ceil((double)(T)(lo - filter1) / (double)base) * base + filter2;
  if (lo % base < filter2 && lo % base > filter1) {
    f1 -= base;
    f2 -= base;
  }
  *a = f1;
  *b = f2;
}
template <typename T>
size_t col_filter_close(int codec, const uint8_t *p, const uint64_t *off, size_t n, uint32_t bs, T filter1, T filter2,
                        T base, const uint64_t *zmin, uint32_t *out) {
  size_t nb = (n + bs - 1) / bs;
  Leco_int<T> lc;
  FOR_int<T> fc;
  lc.init((int)nb, (int)bs);
  fc.init((int)nb, (int)bs);
  size_t total = 0;
  for (size_t i = 0; i < nb; ++i) {
    size_t len = std::min<size_t>(bs, n - i * bs);
    uint8_t *in = const_cast<uint8_t *>(p + off[i]);
    if (codec == C_LECO) {
      T f1 = filter1, f2 = filter2;
      if (zmin) window_start<T>((T)zmin[i], filter1, filter2, base, &f1, &f2);
      total += lc.filter_range_close(in, len, out + total, (int)i, f1, f2, (int)base);
    } else {
      total += fc.filter_range_close(in, len, out + total, i, filter1, filter2, (int)base);
    }
  }
  return total;
}
}  // namespace

extern "C" {
size_t ref_column_filter_u32(int codec, const uint8_t *p, const uint64_t *off, size_t n, uint32_t bs, uint32_t f, const uint64_t *zmax, uint32_t *out) { return col_filter<uint32_t>(codec, p, off, n, bs, f, zmax, out); }
size_t ref_column_filter_u64(int codec, const uint8_t *p, const uint64_t *off, size_t n, uint32_t bs, uint64_t f, const uint64_t *zmax, uint32_t *out) { return col_filter<uint64_t>(codec, p, off, n, bs, f, zmax, out); }
size_t ref_column_filter_close_u32(int codec, const uint8_t *p, const uint64_t *off, size_t n, uint32_t bs, uint32_t f1, uint32_t f2, uint32_t base, const uint64_t *zmin, uint32_t *out) { return col_filter_close<uint32_t>(codec, p, off, n, bs, f1, f2, base, zmin, out); }
size_t ref_column_filter_close_u64(int codec, const uint8_t *p, const uint64_t *off, size_t n, uint32_t bs, uint64_t f1, uint64_t f2, uint64_t base, const uint64_t *zmin, uint32_t *out) { return col_filter_close<uint64_t>(codec, p, off, n, bs, f1, f2, base, zmin, out); }
}  // extern "C"

// One block through <Codec>::filter_range / filter_range_close with the codec's
// block_size = bs and the given block_id (the index base is block_id*bs).
// ref_close_window_start_*: the LeCo close-range experiment's per-block window
// start from the block minimum (experiments/leco_int_fix_template.cpp:299-304).
namespace {
template <typename T>
size_t blk_filter(int codec, const uint8_t *in, size_t len, uint32_t bs, int block_id, T f, uint32_t *out) {
  uint8_t *p = const_cast<uint8_t *>(in);
  if (codec == C_LECO) { Leco_int<T> c; c.init(block_id + 1, (int)bs); return c.filter_range(p, len, f, out, block_id); }
  FOR_int<T> c;
  c.init(block_id + 1, (int)bs);
  return c.filter_range(p, len, f, out, (size_t)block_id);
}
template <typename T>
size_t blk_filter_close(int codec, const uint8_t *in, size_t len, uint32_t bs, int block_id, T f1, T f2, int base, uint32_t *out) {
  uint8_t *p = const_cast<uint8_t *>(in);
  if (codec == C_LECO) { Leco_int<T> c; c.init(block_id + 1, (int)bs); return c.filter_range_close(p, len, out, block_id, f1, f2, base); }
  FOR_int<T> c;
  c.init(block_id + 1, (int)bs);
  return c.filter_range_close(p, len, out, (size_t)block_id, f1, f2, base);
}
}  // namespace

extern "C" {
size_t ref_block_filter_u32(int codec, const uint8_t *in, size_t len, uint32_t bs, int bid, uint32_t f, uint32_t *out) { return blk_filter<uint32_t>(codec, in, len, bs, bid, f, out); }
size_t ref_block_filter_u64(int codec, const uint8_t *in, size_t len, uint32_t bs, int bid, uint64_t f, uint32_t *out) { return blk_filter<uint64_t>(codec, in, len, bs, bid, f, out); }
size_t ref_block_filter_close_u32(int codec, const uint8_t *in, size_t len, uint32_t bs, int bid, uint32_t f1, uint32_t f2, int base, uint32_t *out) { return blk_filter_close<uint32_t>(codec, in, len, bs, bid, f1, f2, base, out); }
size_t ref_block_filter_close_u64(int codec, const uint8_t *in, size_t len, uint32_t bs, int bid, uint64_t f1, uint64_t f2, int base, uint32_t *out) { return blk_filter_close<uint64_t>(codec, in, len, bs, bid, f1, f2, base, out); }
void ref_close_window_start_u32(uint32_t lo, uint32_t f1, uint32_t f2, uint32_t base, uint32_t *a, uint32_t *b) { window_start<uint32_t>(lo, f1, f2, base, a, b); }
void ref_close_window_start_u64(uint64_t lo, uint64_t f1, uint64_t f2, uint64_t base, uint64_t *a, uint64_t *b) { window_start<uint64_t>(lo, f1, f2, base, a, b); }
}  // extern "C"

// ---- legacy u32 codec piecewise_fix_op_max (piecewise_fix_op_minimize_maxerror.h) ----
#include "piecewise_fix_op_minimize_maxerror.h"
extern "C" {
// encodeArray8 on one block; diff_plus/diff_minus (n bytes, nullable) get the block's
// mul_add_diff_set / mul_add_diff_set_minus membership.  Returns bytes written.
size_t ref_legacy_encode_block(const uint32_t *in, size_t n, uint8_t *out, uint8_t *diff_plus, uint8_t *diff_minus) {
  piecewise_fix_op_max c;
  c.init(1, (int)n, 0);
  uint8_t *end = c.encodeArray8(const_cast<uint32_t *>(in), n, out, 0);
  if (diff_plus) for (int i : c.mul_add_diff_set) diff_plus[i] = 1;
  if (diff_minus) for (int i : c.mul_add_diff_set_minus) diff_minus[i] = 1;
  return (size_t)(end - out);
}
void ref_legacy_decode_block(const uint8_t *in, size_t n, uint32_t *out) {
  piecewise_fix_op_max c;
  c.decodeArray8(const_cast<uint8_t *>(in), n, out, 0);
}
uint32_t ref_legacy_random(const uint8_t *in, int k) {
  piecewise_fix_op_max c;
  return c.randomdecodeArray8(const_cast<uint8_t *>(in), (size_t)k, nullptr, 0);
}
}  // extern "C"
