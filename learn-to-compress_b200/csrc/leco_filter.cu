// leco_filter.cu -- predicate pushdown on compressed columns: the indices of the
// values that pass a filter, found without decoding the column to memory.
//
// Semantics are those of the reference's per-block filters, called block after
// block as its filter experiments do:
//   range (values above f):  Leco_int<T>::filter_range   piecewise_fix_integer_template.h:206-252
//                            FOR_int<T>::filter_range    FOR_integer_template.h:115-160
//   close range (windows):   Leco_int<T>::filter_range_close  piecewise_fix_integer_template.h:254-303
//                            FOR_int<T>::filter_range_close   FOR_integer_template.h:166-215
//   column loops:            experiments/leco_int_fix_template.cpp:244-256, :290-322
//                            experiments/FOR_int_fix_template.cpp:254-266, :303-322
// The output is uint32 global indices b*block_size + k, blocks in order, each
// block's indices in the order the reference emits them.
//
// Three launches: a counting pass (one warp per 32 blocks), an exclusive scan of
// the per-group totals, and a writing pass (one warp per block with matches),
// whose output position is its group's prefix plus the counts of the group's
// earlier blocks.  Before reading any field, a block (or window) is classified
// from its model's value bounds, its FOR header or the zone map: all indices
// match, none do, or the values must be read.  Read blocks (and window loops)
// are evaluated in both passes; every other block reads only its plan.
#include <algorithm>

#include "leco_decode.cuh"
#include "leco_encode.cuh"

namespace leco {

constexpr int kFT = 256;                              // threads per CTA
constexpr int kFU = 4;                                // 32-item groups per lane per step

// (int)x as x86-64 compiles it (32-bit CVTTSD2SI): NaN and values outside the
// int range give INT_MIN.  The filters keep their index thresholds in int
// (piecewise_fix_integer_template.h:226,275-276).
__device__ __forceinline__ int32_t f2i32_x86(double x) {
  return (x > -2147483649.0 && x < 2147483648.0) ? __double2int_rz(x) : (int32_t)0x80000000;
}
// std::max / std::min as the filters use them: (a < b) ? b : a, (b < a) ? b : a.
__device__ __forceinline__ double std_max(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double std_min(double a, double b) { return b < a ? b : a; }

// A decoded value against a bound of type T: uint64_t compares unsigned; for
// uint32_t the bound is promoted to int64_t and the comparison is signed
// (bit_read.h:421,477).
template <int S>
__device__ __forceinline__ bool cmp_gt(uint64_t v, uint64_t f) { return S == 8 ? v > f : (int64_t)v > (int64_t)f; }
template <int S>
__device__ __forceinline__ bool cmp_lt(uint64_t v, uint64_t f) { return S == 8 ? v < f : (int64_t)v < (int64_t)f; }

// (double)(f + c) for f of type T and an int64_t offset c: T = uint64_t wraps
// modulo 2^64 and converts unsigned; T = uint32_t is widened to int64_t first.
template <int S>
__device__ __forceinline__ double bound_plus(uint64_t f, int64_t c) {
  if (S == 8) return __ull2double_rn(f + (uint64_t)c);
  return __ll2double_rn((int64_t)(uint32_t)f + c);
}

// Value k of a block as the filter readers compute it: raw values as stored,
// FOR min + offset, LeCo (long long)(theta0 + k*theta1) -/+ the magnitude in
// wrapping 64-bit arithmetic (bit_read.h:409-420; l == 0: the prediction).
template <int S, int CODEC>
__device__ __forceinline__ uint64_t filter_value(const uint64_t *__restrict__ words, const BlockHdr &h, bool raw, uint32_t k) {
  constexpr uint32_t TB = 8u * S;
  if (raw) return load_field(words, h.body_bit + (uint64_t)k * TB, TB);
  if (CODEC == kFor) {
    const uint64_t v = h.l ? h.base + load_field(words, h.body_bit + (uint64_t)k * h.l, h.l) : h.base;
    return S == 8 ? v : (v & 0xffffffffull);
  }
  uint64_t v = (uint64_t)f2i_x86(pred_linear(h.a0, h.a1, k));
  if (h.l) v = apply_signed(v, load_field(words, h.body_bit + (uint64_t)k * h.l, h.l), h.l);
  return v;
}

// What one block evaluates.
enum : int {
  kPredAbove = 0,   // v > f1
  kPredModulo = 1,  // f1 < v % base < f2 (FOR close range)
  kPredAnyWin = 2,  // raw LeCo block, close range: v in some window (f1 + p*base, f2 + p*base)
  kPredWindows = 3  // packed LeCo block, close range: the reference's window loop
};

template <int S>
__device__ __forceinline__ bool single_pred(int pred, uint64_t v, uint64_t f1, uint64_t f2, uint64_t base) {
  if (pred == kPredAbove) return cmp_gt<S>(v, f1);
  if (pred == kPredModulo) {
    const uint64_t r = v % base;
    return r > f1 && r < f2;
  }
  // kPredAnyWin: the largest window start below v is v - ((v - f1 - 1) % base) - 1
  return v > f1 && f2 > f1 && ((v - f1 - 1) % base) + 1 < f2 - f1;
}

constexpr int kFB = kFT / 32;            // warps per CTA
constexpr uint32_t kFWin = 32;           // windows per chunk (close range), one per lane

// How a window's values relate to its bounds, decided from the block model
// (or header / zone map) before any field is read.
enum : int { kNone = 0, kAll = 1, kEval = 2 };

// Per-warp plan of one block.
struct BlockPlan {
  BlockHdr h;
  uint64_t vbase;
  uint32_t len, lo, hi;
  uint32_t ra;    // single window, kEval: every index in [ra, hi) matches without reading (ra == hi: none)
  int pred;
  int mode;       // single window: kNone / kAll / kEval
  bool raw;
  bool bounded;   // LeCo: every prediction of the block lies inside (-2^62, 2^62) and l <= 61
  uint64_t f1, f2;
};

// Bounds of the values of a packed LeCo block at indices [k0, k1] (k0 <= k1):
// the predictions are monotone in k when every one lies inside (-2^62, 2^62),
// and a value differs from its prediction by at most 2^(l-1) - 1.
__device__ __forceinline__ void leco_value_bounds(const BlockHdr &h, uint32_t k0, uint32_t k1, int64_t &vmin, int64_t &vmax) {
  const int64_t pa = __double2ll_rz(pred_linear(h.a0, h.a1, k0)), pb = __double2ll_rz(pred_linear(h.a0, h.a1, k1));
  const int64_t m = h.l ? (((int64_t)1 << (h.l - 1)) - 1) : 0;
  vmin = (pa < pb ? pa : pb) - m;
  vmax = (pa < pb ? pb : pa) + m;
}

// Window classification against (w1, w2) (w2 = none: range filter v > w1) in
// the comparison domain of T.  For T = uint64_t a negative int64 value wraps
// to a huge unsigned one, so only blocks whose values are all non-negative are
// classified.
template <int S>
__device__ __forceinline__ int classify(int64_t vmin, int64_t vmax, uint64_t w1, uint64_t w2, bool two_sided) {
  if (S == 8 && vmin < 0) return kEval;
  const bool gt_all = S == 8 ? (uint64_t)vmin > w1 : vmin > (int64_t)w1;
  const bool gt_none = S == 8 ? (uint64_t)vmax <= w1 : vmax <= (int64_t)w1;
  if (!two_sided) return gt_all ? kAll : (gt_none ? kNone : kEval);
  const bool lt_all = S == 8 ? (uint64_t)vmax < w2 : vmax < (int64_t)w2;
  const bool lt_none = S == 8 ? (uint64_t)vmin >= w2 : vmin >= (int64_t)w2;
  if (gt_none || lt_none) return kNone;
  return gt_all && lt_all ? kAll : kEval;
}

// Per-index forms of the window classification for a bounded packed LeCo
// block: every value at k is above w1 (resp. below w2).  Monotone in k because
// the predictions are.
template <int S>
__device__ __forceinline__ bool surely_above(const BlockHdr &h, int64_t m, uint32_t k, uint64_t w1) {
  const int64_t v = __double2ll_rz(pred_linear(h.a0, h.a1, k)) - m;
  return S == 8 ? (v >= 0 && (uint64_t)v > w1) : v > (int64_t)w1;
}
template <int S>
__device__ __forceinline__ bool surely_below(const BlockHdr &h, int64_t m, uint32_t k, uint64_t w2) {
  const int64_t v = __double2ll_rz(pred_linear(h.a0, h.a1, k)) + m;
  return S == 8 ? (w2 > 0x7fffffffffffffffull || v < (int64_t)w2) : v < (int64_t)w2;
}
// First k in [lo, hi) where a monotone predicate changes from `from` to its
// opposite (hi when it never does).
template <typename P>
__device__ __forceinline__ uint32_t first_change(uint32_t lo, uint32_t hi, bool from, P pred) {
  while (lo < hi) {
    const uint32_t mid = lo + ((hi - lo) >> 1);
    if (pred(mid) == from) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}
// The indices [ia, ib) of window [k0, k1) whose values all lie inside
// (w1, w2); the rest of the window must be read.  ia == ib: none.
template <int S>
__device__ __forceinline__ void surely_inside(const BlockHdr &h, uint32_t k0, uint32_t k1, uint64_t w1, uint64_t w2,
                                              uint32_t &ia, uint32_t &ib) {
  const int64_t m = h.l ? (((int64_t)1 << (h.l - 1)) - 1) : 0;
  auto above = [&](uint32_t k) { return surely_above<S>(h, m, k, w1); };
  auto below = [&](uint32_t k) { return surely_below<S>(h, m, k, w2); };
  if (h.a1 >= 0) {  // predictions non-decreasing: above turns true, below turns false
    ia = first_change(k0, k1, false, above);
    ib = first_change(ia, k1, true, below);
  } else {          // non-increasing: below turns true, above turns false
    ia = first_change(k0, k1, false, below);
    ib = first_change(ia, k1, true, above);
  }
}

template <int S, int CODEC>
__device__ __forceinline__ BlockPlan plan_block(const FilterLaunch &a, uint64_t b, int close) {
  constexpr uint32_t TB = 8u * S;
  constexpr uint64_t TM = S == 8 ? ~0ull : 0xffffffffull;
  const uint64_t *words = reinterpret_cast<const uint64_t *>(a.payload);
  BlockPlan p;
  p.vbase = b * a.bs;
  p.len = (uint32_t)umin64((uint64_t)a.bs, a.n - p.vbase);
  const uint64_t off = __ldg(a.offsets + b);
  p.h = parse_header<CODEC, S>(a.payload, off);
  p.raw = p.h.l == TB;
  p.pred = kPredAbove;
  p.mode = kEval;
  p.lo = p.hi = p.ra = 0;
  p.f1 = a.f1 & TM;
  p.f2 = a.f2 & TM;
  p.bounded = CODEC == kLinear && !p.raw && p.h.l <= 61 && pred_in_range<kLinear>(p.h, p.len + 1);
  const uint64_t step = a.base & TM;
  if (p.h.l > TB) {  // sentinel or corrupt header: no case in the reference's filters
    if ((threadIdx.x & 31) == 0) atomicOr(a.error, kErrBadHeader);
    p.mode = kNone;
    return p;
  }
  if (!close) {
    p.hi = p.ra = p.len;
    if (a.zone && __ldg(a.zone + b) <= p.f1) {  // the experiment's zone-map skip (:247-249)
      p.mode = kNone;
    } else if (!p.raw && CODEC == kFor) {
      const uint64_t mx = load_u64_at(words, off + 1 + S) & TM;  // header maximum (FOR_integer_template.h:143)
      if (mx <= p.f1) p.mode = kNone;
      else if (p.h.base > p.f1) p.mode = kAll;                   // the header minimum is above the filter
    } else if (!p.raw) {  // the model's threshold index (piecewise_fix_integer_template.h:221-230)
      const int64_t di = p.h.l ? (int64_t)1 << (p.h.l - 1) : 0;
      const double q = __ddiv_rn(__dsub_rn(bound_plus<S>((p.f1 + 1) & TM, -di), p.h.a0), p.h.a1);
      const int32_t thre = f2i32_x86(std_max(q, 0.));
      if ((uint64_t)(int64_t)thre >= p.len) {
        p.mode = kNone;
      } else {
        p.lo = (uint32_t)thre;
        if (a.zone_lo && __ldg(a.zone_lo + b) > p.f1) {
          p.mode = kAll;  // every value is above the filter: indices [thre, len)
        } else if (p.bounded) {
          int64_t vmin, vmax;
          leco_value_bounds(p.h, p.lo, p.hi - 1, vmin, vmax);
          p.mode = classify<S>(vmin, vmax, p.f1, 0, false);
          if (p.mode == kEval && p.h.a1 > 0) {
            // predictions increase with k, so "every value at k is above the filter" turns
            // true at one index and stays true: only the indices before it are read
            const int64_t m = p.h.l ? (((int64_t)1 << (p.h.l - 1)) - 1) : 0;
            p.ra = first_change(p.lo, p.hi, false, [&](uint32_t k) { return surely_above<S>(p.h, m, k, p.f1); });
          }
        }
      }
    }
    if (p.mode == kNone) p.hi = p.lo;
    if (p.mode != kEval || p.ra < p.lo || p.ra > p.hi) p.ra = p.hi;  // a split only for read blocks
    return p;
  }
  p.hi = p.ra = p.len;
  if (CODEC == kFor) {
    p.pred = kPredModulo;
    return p;
  }
  if (a.zone) {  // first window from the block minimum (leco_int_fix_template.cpp:299-304)
    const uint64_t zmin = __ldg(a.zone + b) & TM;
    const double db = __ull2double_rn(step);
    const double qb = __dmul_rn(ceil(__ddiv_rn(__ull2double_rn((zmin - p.f1) & TM), db)), db);
    uint64_t w1 = f2T_x86<S>(__dadd_rn(qb, __ull2double_rn(p.f1)));
    uint64_t w2 = f2T_x86<S>(__dadd_rn(qb, __ull2double_rn(p.f2)));
    const uint64_t r = zmin % step;
    if (r < p.f2 && r > p.f1) {
      w1 = (w1 - step) & TM;
      w2 = (w2 - step) & TM;
    }
    p.f1 = w1;
    p.f2 = w2;
  }
  p.pred = p.raw ? kPredAnyWin : kPredWindows;
  return p;
}

// Writes the consecutive indices idx0 .. idx0+cnt-1 to out[pos ...] (positions
// at or past cap are dropped), by one warp: 16-byte stores once pos is aligned
// when the output buffer itself is 16-byte aligned.
__device__ __forceinline__ void write_run(const FilterLaunch &a, uint64_t pos, uint32_t idx0, uint32_t cnt) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t head = cnt;
  if (a.vec_out) head = min(cnt, (uint32_t)((4u - (uint32_t)(pos & 3)) & 3u));
  for (uint32_t j = lane; j < head; j += 32)
    if (pos + j < a.cap) a.out[pos + j] = idx0 + j;
  if (head == cnt) return;
  pos += head;
  idx0 += head;
  cnt -= head;
  const uint32_t nvec = cnt >> 2;
  uint4 *o4 = reinterpret_cast<uint4 *>(a.out + pos);
  for (uint32_t v = lane; v < nvec; v += 32) {
    const uint64_t q = pos + 4ull * v;
    const uint32_t x = idx0 + 4 * v;
    if (q + 4 <= a.cap) {
      __stcs(o4 + v, make_uint4(x, x + 1, x + 2, x + 3));
    } else {
      for (uint32_t t = 0; t < 4; ++t)
        if (q + t < a.cap) a.out[q + t] = x + t;
    }
  }
  const uint32_t rem = cnt & 3;
  if (lane < rem) {
    const uint64_t q = pos + 4ull * nvec + lane;
    if (q < a.cap) a.out[q] = idx0 + 4 * nvec + lane;
  }
}

// Close range on a packed LeCo block, by one warp: the reference's window loop
// (piecewise_fix_integer_template.h:275-298), windows in chunks of 32 (one per
// lane).  Window p = (f1 + p*base, f2 + p*base) (bounds wrap in T) covers
// indices [thre1, thre2) ([thre1, thre2] for l == 0); the loop ends at the
// first window with thre1 >= len or thre2 <= 0.  A window whose value bounds lie
// inside (outside) its bounds matches every (no) index without reading fields;
// the others are evaluated 32 indices at a time.  Counts, or (write) stores the
// matches from out position `run` on.
template <int S, int CODEC, bool WRITE>
__device__ uint64_t window_loop(const FilterLaunch &a, const BlockPlan &p, uint64_t run) {
  constexpr uint64_t TM = S == 8 ? ~0ull : 0xffffffffull;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t *words = reinterpret_cast<const uint64_t *>(a.payload);
  const uint64_t step = a.base & TM;
  const int64_t di = p.h.l ? (int64_t)1 << (p.h.l - 1) : 0;
  const double dlen = __uint2double_rn(p.len);
  uint64_t total = 0;
  for (uint32_t q0 = 0;; q0 += kFWin) {
    const uint64_t q = q0 + lane;
    const uint64_t w1 = (p.f1 + q * step) & TM, w2 = (p.f2 + q * step) & TM;
    const int32_t t1 = f2i32_x86(std_max(__dsub_rn(__ddiv_rn(__dsub_rn(bound_plus<S>(w1, -di), p.h.a0), p.h.a1), 1.0), 0.));
    const int32_t t2 = f2i32_x86(std_min(__dadd_rn(__ddiv_rn(__dsub_rn(bound_plus<S>(w2, di), p.h.a0), p.h.a1), 1.0), dlen));
    const bool ok = (uint64_t)(int64_t)t1 < p.len && t2 > 0;
    const uint32_t fails = __ballot_sync(0xffffffffu, !ok);
    const uint32_t nwin = fails ? (uint32_t)(__ffs(fails) - 1) : kFWin;
    if (q0 >= a.max_windows) {  // the loop would go on past the window limit
      if (nwin && lane == 0 && !WRITE) atomicOr(a.error, kErrLimit);
      break;
    }
    // window [k0, e): read [k0, ia) and [ib, e), all of [ia, ib) matches
    uint32_t k0 = 0, e = 0, ia = 0, ib = 0;
    if (lane < nwin) {
      const int32_t ee = p.h.l ? t2 : t2 + 1;  // one past the window's last index
      if (ee > t1) {
        k0 = (uint32_t)t1;
        e = (uint32_t)ee;
        ia = ib = e;  // undecided: read everything
        if (p.bounded) {
          int64_t vmin, vmax;
          leco_value_bounds(p.h, k0, e - 1, vmin, vmax);
          const int mode = classify<S>(vmin, vmax, w1, w2, true);
          if (mode == kNone) e = ia = ib = k0;
          else if (mode == kAll) ia = k0;
          else surely_inside<S>(p.h, k0, e, w1, w2, ia, ib);
          if (ib <= ia) ia = ib = e;
        }
      }
    }
    for (uint32_t w = 0; w < nwin; ++w) {
      const uint32_t wk0 = __shfl_sync(0xffffffffu, k0, w), we = __shfl_sync(0xffffffffu, e, w);
      if (we <= wk0) continue;
      const uint32_t wa = __shfl_sync(0xffffffffu, ia, w), wb = __shfl_sync(0xffffffffu, ib, w);
      const uint64_t lo1 = __shfl_sync(0xffffffffu, w1, w), hi2 = __shfl_sync(0xffffffffu, w2, w);
      // three runs in index order: read [wk0, wa), all of [wa, wb), read [wb, we)
      for (int part = 0; part < 3; ++part) {
        const uint32_t r0 = part == 0 ? wk0 : (part == 1 ? wa : wb);
        const uint32_t r1 = part == 0 ? wa : (part == 1 ? wb : we);
        if (r1 <= r0) continue;
        if (part == 1) {
          if (WRITE) write_run(a, run + total, (uint32_t)(p.vbase + r0), r1 - r0);
          total += r1 - r0;
          continue;
        }
        for (uint32_t k1 = r0; k1 < r1; k1 += 32) {
          const uint32_t k = k1 + lane;
          bool fl = false;
          if (k < r1) {
            const uint64_t v = filter_value<S, CODEC>(words, p.h, false, k);
            fl = cmp_gt<S>(v, lo1) && cmp_lt<S>(v, hi2);
          }
          const uint32_t m = __ballot_sync(0xffffffffu, fl);
          if (WRITE && fl) {
            const uint64_t pos = run + total + __popc(m & ((1u << lane) - 1u));
            if (pos < a.cap) a.out[pos] = (uint32_t)(p.vbase + k);
          }
          total += __popc(m);
        }
      }
    }
    if (nwin < kFWin) break;
  }
  return total;
}

__device__ __forceinline__ BlockPlan shfl_plan(const BlockPlan &q, int src) {
  BlockPlan p;
  p.h.body_bit = __shfl_sync(0xffffffffu, q.h.body_bit, src);
  p.h.l = __shfl_sync(0xffffffffu, q.h.l, src);
  p.h.a0 = __shfl_sync(0xffffffffu, q.h.a0, src);
  p.h.a1 = __shfl_sync(0xffffffffu, q.h.a1, src);
  p.h.a2 = 0;
  p.h.base = __shfl_sync(0xffffffffu, q.h.base, src);
  p.vbase = __shfl_sync(0xffffffffu, q.vbase, src);
  p.len = __shfl_sync(0xffffffffu, q.len, src);
  p.lo = __shfl_sync(0xffffffffu, q.lo, src);
  p.hi = __shfl_sync(0xffffffffu, q.hi, src);
  p.ra = __shfl_sync(0xffffffffu, q.ra, src);
  p.pred = __shfl_sync(0xffffffffu, q.pred, src);
  p.mode = __shfl_sync(0xffffffffu, q.mode, src);
  p.raw = __shfl_sync(0xffffffffu, (int)q.raw, src) != 0;
  p.bounded = __shfl_sync(0xffffffffu, (int)q.bounded, src) != 0;
  p.f1 = __shfl_sync(0xffffffffu, q.f1, src);
  p.f2 = __shfl_sync(0xffffffffu, q.f2, src);
  return p;
}

// Evaluates a read single-window block [p.lo, p.hi) 32*kFU indices per step,
// all fields of a step in flight.  Counts; with WRITE also stores the matches
// from out position `run` on (positions at or past cap are dropped).
template <int S, int CODEC, bool WRITE>
__device__ __forceinline__ uint64_t eval_block(const FilterLaunch &a, const BlockPlan &p, uint32_t k0, uint32_t k1,
                                               uint64_t run) {
  const uint32_t lane = threadIdx.x & 31, lt = (1u << lane) - 1u;
  const uint64_t *words = reinterpret_cast<const uint64_t *>(a.payload);
  const uint64_t step = a.base & (S == 8 ? ~0ull : 0xffffffffull);
  uint64_t cnt = 0;
  for (uint32_t s0 = k0; s0 < k1; s0 += 32 * kFU) {
    uint32_t m[kFU];
#pragma unroll
    for (int u = 0; u < kFU; ++u) {
      const uint32_t k = s0 + u * 32 + lane;
      bool fl = false;
      if (k < k1) fl = single_pred<S>(p.pred, filter_value<S, CODEC>(words, p.h, p.raw, k), p.f1, p.f2, step);
      m[u] = __ballot_sync(0xffffffffu, fl);
    }
#pragma unroll
    for (int u = 0; u < kFU; ++u) {
      if (WRITE && ((m[u] >> lane) & 1u)) {
        const uint64_t pos = run + cnt + __popc(m[u] & lt);
        if (pos < a.cap) a.out[pos] = (uint32_t)(p.vbase + s0 + u * 32 + lane);
      }
      cnt += __popc(m[u]);
    }
  }
  return cnt;
}

// Matches of one block (warp-uniform).
template <int S, int CODEC>
__device__ __forceinline__ uint64_t count_block(const FilterLaunch &a, const BlockPlan &p) {
  if (p.pred == kPredWindows) return window_loop<S, CODEC, false>(a, p, 0);
  if (p.mode == kAll) return p.hi - p.lo;
  if (p.mode != kEval) return 0;
  return eval_block<S, CODEC, false>(a, p, p.lo, p.ra, 0) + (p.hi - p.ra);
}

// Writes the matches of one block from output position `run` on (warp-uniform).
template <int S, int CODEC>
__device__ __forceinline__ void write_block(const FilterLaunch &a, const BlockPlan &p, uint64_t run) {
  if (p.pred == kPredWindows) {
    window_loop<S, CODEC, true>(a, p, run);
    return;
  }
  if (p.mode == kAll) {
    write_run(a, run, (uint32_t)(p.vbase + p.lo), p.hi - p.lo);
    return;
  }
  if (p.mode == kEval) {
    run += eval_block<S, CODEC, true>(a, p, p.lo, p.ra, run);
    if (p.ra < p.hi) write_run(a, run, (uint32_t)(p.vbase + p.ra), p.hi - p.ra);
  }
}

// counts[b]: the block's match count in the low 40 bits; a block whose matches are
// one run of indices [lo, lo + count) known from its plan alone also carries
// kRunFlag and lo (bits 40..62), so the writing pass needs no second plan for it.
constexpr uint64_t kCountMask = (1ull << 40) - 1, kRunFlag = 1ull << 63;

// ---- pass 1: match counts --------------------------------------------------------
// One warp per group of 32 consecutive blocks: lane j plans block j (all header,
// offset and zone-map loads of the group in flight at once); blocks decided by
// their plan are counted from it, the others (read blocks, window loops) by the
// whole warp one after another.  Writes counts[b] and the group's total.
// The three passes are chained by programmatic dependent launch: each lets the next
// one be launched as soon as all its CTAs run, and the next one waits for the whole
// previous grid (griddepcontrol.wait: completed, its writes visible) before it reads
// anything that grid writes.  The launch gaps between the passes are hidden that way.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait_prior_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <int S, int CODEC>
__global__ void __launch_bounds__(kFT) filter_count_kernel(FilterLaunch a, int close) {
  pdl_launch_dependents();
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t g = (uint64_t)blockIdx.x * kFB + (threadIdx.x >> 5);
  const uint64_t b0 = g * 32;
  if (b0 >= a.nb) return;  // whole warps only
  const uint32_t nblk = (uint32_t)umin64(32, a.nb - b0);
  BlockPlan mine;
  uint64_t mycnt = 0;
  bool read = false;
  if (lane < nblk) {
    mine = plan_block<S, CODEC>(a, b0 + lane, close);
    read = mine.pred == kPredWindows || mine.mode == kEval;
    if (!read && mine.mode == kAll) mycnt = mine.hi - mine.lo;
  }
  for (uint32_t need = __ballot_sync(0xffffffffu, read); need; need &= need - 1) {
    const int j = __ffs(need) - 1;
    const BlockPlan p = shfl_plan(mine, j);
    const uint64_t c = count_block<S, CODEC>(a, p);
    if (lane == (uint32_t)j) mycnt = c;
  }
  if (lane < nblk) {
    const bool run = !read && mine.mode == kAll && mycnt;
    a.counts[b0 + lane] = mycnt | (run ? kRunFlag | ((uint64_t)mine.lo << 40) : 0);
  }
  const uint64_t tot = warp_sum_u64(mycnt);
  if (lane == 0) a.group_tot[g] = tot;
}

// ---- pass 2: exclusive scan of the group totals (one CTA of 1024 threads) ----------
// group_tot[g] becomes the output position of group g's first match; *count the
// total number of matches.  (A decoupled look-back over the groups inside pass 1
// was measured slower: its chain of waits took longer than this launch.)
__global__ void __launch_bounds__(1024) filter_scan_kernel(uint64_t *group_tot, uint64_t ngroups, uint64_t *count) {
  __shared__ uint64_t wsum[33];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  pdl_launch_dependents();
  pdl_wait_prior_grid();  // every group total is written
  uint64_t carry = 0;
  for (uint64_t base = 0; base < ngroups; base += 1024) {
    const uint64_t i = base + tid;
    const uint64_t v = i < ngroups ? group_tot[i] : 0;
    uint64_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const uint64_t x = wsum[lane];
      uint64_t xi = x;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, xi, o);
        if (lane >= (uint32_t)o) xi += y;
      }
      wsum[lane] = xi - x;
      if (lane == 31) wsum[32] = xi;
    }
    __syncthreads();
    if (i < ngroups) group_tot[i] = carry + wsum[warp] + incl - v;
    carry += wsum[32];
    __syncthreads();  // wsum is rewritten by the next chunk
  }
  if (tid == 0) *count = carry;
}

// ---- pass 3: writing ------------------------------------------------------------------
// One warp per block with matches: its output position is its group's prefix plus
// the counts of the group's earlier blocks.  A single run of indices is written
// straight from counts[b] (16-byte stores); other blocks are planned again and
// their matches written (read blocks and window loops evaluated again).
template <int S, int CODEC>
__global__ void __launch_bounds__(kFT) filter_write_kernel(FilterLaunch a, int close) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t b = (uint64_t)blockIdx.x * kFB + (threadIdx.x >> 5);
  pdl_wait_prior_grid();  // the scan (and the counting pass before it) are complete
  if (b >= a.nb) return;  // whole warps only
  const uint64_t w = __ldg(a.counts + b);
  if (!(w & kCountMask)) return;
  const uint64_t g = b >> 5;
  const uint32_t j = (uint32_t)(b & 31);
  const uint64_t before = lane < j ? __ldg(a.counts + (g << 5) + lane) & kCountMask : 0;
  const uint64_t run = __ldg(a.group_tot + g) + warp_sum_u64(before);
  if (w & kRunFlag) {
    write_run(a, run, (uint32_t)(b * a.bs + ((w >> 40) & 0x7fffff)), (uint32_t)(w & kCountMask));
    return;
  }
  BlockPlan mine;
  if (lane == 0) mine = plan_block<S, CODEC>(a, b, close);
  write_block<S, CODEC>(a, shfl_plan(mine, 0), run);
}

// ---- zone map: per-block minimum and maximum of the decoded values -------------------
template <typename T, int CODEC>
__global__ void __launch_bounds__(256) zonemap_kernel(DecodeLaunch a, uint64_t *zmin, uint64_t *zmax) {
  constexpr int S = sizeof(T);
  constexpr uint32_t TB = 8u * S;
  constexpr uint64_t TM = S == 8 ? ~0ull : 0xffffffffull;
  __shared__ u128 red[66];
  const uint64_t b = blockIdx.x;
  const uint64_t base = b * a.bs;
  const uint32_t len = (uint32_t)umin64((uint64_t)a.bs, a.n - base);
  const uint64_t *words = reinterpret_cast<const uint64_t *>(a.payload);
  const uint64_t off = __ldg(a.offsets + b);
  const BlockHdr h = parse_header<CODEC, S>(a.payload, off);
  if (h.l == 126 || h.l == 127 || h.l > TB) {
    if (threadIdx.x == 0) {
      atomicOr(a.error, kErrBadHeader);
      zmin[b] = 0;
      zmax[b] = 0;
    }
    return;
  }
  const bool raw = h.l == TB;
  if (CODEC == kFor && !raw) {  // the header holds both
    if (threadIdx.x == 0) {
      zmin[b] = h.base;
      zmax[b] = load_u64_at(words, off + 1 + S) & TM;
    }
    return;
  }
  uint64_t mn = ~0ull, mx = 0;
  if (CODEC == kDelta && !raw) {
    delta_tiles<T, 256>(words, h, len, 0, len, [&](uint32_t k0, const auto *vs) {
#pragma unroll
      for (int j = 0; j < kDeltaSpan; ++j)
        if (k0 + j < len) {
          const uint64_t v = (uint64_t)vs[j] & TM;
          mn = v < mn ? v : mn;
          mx = v > mx ? v : mx;
        }
    });
  } else {
    const uint32_t l = raw ? TB : h.l;
    for (uint32_t k = threadIdx.x; k < len; k += blockDim.x) {
      const uint64_t f = l ? load_field(words, h.body_bit + (uint64_t)k * l, l) : 0;
      const uint64_t v = (raw ? f : value_from_field<CODEC, S>(h, k, f)) & TM;
      mn = v < mn ? v : mn;
      mx = v > mx ? v : mx;
    }
  }
  u128 A = mn, B = mx;
  block_reduce2<2, 1>(A, B, red);
  if (threadIdx.x == 0) {
    zmin[b] = (uint64_t)A;
    zmax[b] = (uint64_t)B;
  }
}

template <int S, int CODEC>
static int run_filter(FilterLaunch L, int close, cudaStream_t st) {
  const uint64_t groups = (L.nb + 31) / 32;
  filter_count_kernel<S, CODEC><<<(unsigned)((groups + kFB - 1) / kFB), kFT, 0, st>>>(L, close);
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr.val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.stream = st;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(1);
  cfg.blockDim = dim3(1024);
  cudaError_t e = cudaLaunchKernelEx(&cfg, filter_scan_kernel, L.group_tot, groups, L.count);
  cfg.gridDim = dim3((unsigned)((L.nb + kFB - 1) / kFB));
  cfg.blockDim = dim3(kFT);
  if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, filter_write_kernel<S, CODEC>, L, close);
  return e == cudaSuccess ? 0 : -(int)e;
}

int launch_filter(int codec, int s, const FilterLaunch &L, int close, cudaStream_t st) {
  if (!L.nb) return 0;
  if (s == 4) {
    if (codec == kLinear) return run_filter<4, kLinear>(L, close, st);
    if (codec == kFor) return run_filter<4, kFor>(L, close, st);
  } else {
    if (codec == kLinear) return run_filter<8, kLinear>(L, close, st);
    if (codec == kFor) return run_filter<8, kFor>(L, close, st);
  }
  return 1;
}

template <typename T, int CODEC>
static void run_zonemap(const DecodeLaunch &L, uint64_t nb, uint64_t *zmin, uint64_t *zmax, cudaStream_t st) {
  if (nb) zonemap_kernel<T, CODEC><<<(unsigned)nb, 256, 0, st>>>(L, zmin, zmax);
}
int launch_zonemap(int codec, int s, const DecodeLaunch &L, uint64_t *zmin, uint64_t *zmax, cudaStream_t st) {
  const uint64_t nb = (L.n + L.bs - 1) / L.bs;
  if (s == 4) {
    switch (codec) {
      case kLinear: run_zonemap<uint32_t, kLinear>(L, nb, zmin, zmax, st); return 0;
      case kFor: run_zonemap<uint32_t, kFor>(L, nb, zmin, zmax, st); return 0;
      case kDelta: run_zonemap<uint32_t, kDelta>(L, nb, zmin, zmax, st); return 0;
      case kPoly2: run_zonemap<uint32_t, kPoly2>(L, nb, zmin, zmax, st); return 0;
      case kLegacy: run_zonemap<uint32_t, kLegacy>(L, nb, zmin, zmax, st); return 0;
    }
  } else {
    switch (codec) {
      case kLinear: run_zonemap<uint64_t, kLinear>(L, nb, zmin, zmax, st); return 0;
      case kFor: run_zonemap<uint64_t, kFor>(L, nb, zmin, zmax, st); return 0;
      case kDelta: run_zonemap<uint64_t, kDelta>(L, nb, zmin, zmax, st); return 0;
      case kPoly2: run_zonemap<uint64_t, kPoly2>(L, nb, zmin, zmax, st); return 0;
    }
  }
  return 1;
}

}  // namespace leco
