// leco_partition.cpp -- host partitioner for variable-length LeCo segments.
//
// Restates the segmentation of Leco_cost_merge_double_wo_round<uint64_t>::encodeArray8_int
// (headers/piecewise_cost_merge_integer_template_double_wo_round.h:283-515, merge :516-570,
// cost model newsegment_size :68-131, cal_bits :274-281).  The column is cut into coarse
// blocks exactly as the reference driver does (experiments/leco_double_int_template_wo_round.cpp:85-91);
// inside each coarse block:
//   1. every point starts as its own segment; each carries the first difference to its
//      successor and the bit class of the second difference (cal_bits of two neighbouring
//      first differences),
//   2. for each bit class from the smallest to the largest, a segment of that class is
//      merged with its right neighbour when the merged width costs less than `delta` more
//      bits than the two apart, and the merge then grows left and right greedily,
//   3. the segments are then merged pairwise while the fitted byte size of the pair is
//      smaller than the sum of their sizes, pass after pass, until a pass saves less than
//      0.01 % of the coarse block's raw size.
// The segment byte images are written by the GPU (leco_varlen_encode).  Coarse blocks
// are independent, so they are partitioned in parallel on the host cores.
//
// Arithmetic follows the reference: the fit is its sequential FP64 loop (this file is
// compiled with -ffp-contract=off), the slope is rounded to float, the prediction is
// converted to a 128-bit integer.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "leco_internal.h"

namespace {

typedef __int128 i128;

uint32_t bits64(uint64_t v) { return v ? 64u - (uint32_t)__builtin_clzll(v) : 0u; }

// cal_bits(min, max) (…_double_wo_round.h:274-281): bits of ceil(|max - min| / 2) plus one.
int cal_bits(int64_t mn, int64_t mx) {
  const int64_t diff = (int64_t)((uint64_t)mx - (uint64_t)mn);
  const int64_t ad = diff < 0 ? (int64_t)(0 - (uint64_t)diff) : diff;
  const double half = std::ceil((double)ad / 2.);
  int64_t range;
  if (half >= -9223372036854775808.0 && half < 9223372036854775808.0) range = (int64_t)half;
  else range = INT64_MIN;  // x86 CVTTSD2SI for out-of-range values
  return range ? (int)bits64((uint64_t)range) + 1 : 0;
}

// lr_int_T<uint64_t>::caltheta (lr.h:66-85) on y[0..m).
void fit_seq(const uint64_t *y, int m, double *t0, double *t1) {
  double sumx = 0, sumy = 0, sumxy = 0, sumxx = 0;
  for (int i = 0; i < m; i++) {
    sumx = sumx + (double)i;
    sumy = sumy + (double)y[i];
    sumxx = sumxx + (double)i * i;
    sumxy = sumxy + (double)i * y[i];
  }
  const double ccc = sumxy * m - sumx * sumy;
  const double xxx = sumxx * m - sumx * sumx;
  *t1 = ccc / xxx;
  *t0 = (sumy - *t1 * sumx) / (double)m;
}

// newsegment_size (…_double_wo_round.h:68-131): the cost model of segment [a, b].
uint64_t segment_cost(const uint64_t *array, uint32_t a, uint32_t b) {
  if (a == b) return 9;
  if (b == a + 1) return 13;
  const int length = (int)(b - a + 1);
  uint64_t overhead = sizeof(float) + sizeof(double) + 5;
  double t0, t1;
  fit_seq(array + a, length, &t0, &t1);
  const float slope = (float)t1;
  uint64_t maxr = 0;
  for (uint32_t j = a; j <= b; j++) {
    const i128 pred = (i128)(t0 + (double)slope * (double)(j - a));
    const i128 y = (i128)array[j];
    const uint64_t r = (uint64_t)(y > pred ? y - pred : pred - y);
    if (r > maxr) maxr = r;
  }
  uint32_t bits = maxr ? bits64(maxr) + 1 : 0;
  if (bits >= 64) return 5 + 8ull * (uint64_t)length;
  if (bits) overhead += (uint64_t)std::ceil((double)(bits * length) / 8.0);
  return overhead;
}

struct Seg {
  int start, end;
  int64_t max_delta, min_delta, next_delta;
  int ddn;  // bit class of the second difference towards the next segment
  int prev, next;
};

// Segmentation of one coarse block [B0, B0 + len): appends segment starts to `out`.
void partition_block(const uint64_t *array, uint32_t B0, uint32_t len, uint32_t block_size, int overhead,
                     std::vector<uint32_t> &out) {
  if (len < 2) {  // the reference needs two points per coarse block (it reads array[B0 + 1])
    out.push_back(B0);
    return;
  }
  // ---- split: linked list of one-point segments (…:286-312) ----
  std::vector<Seg> s;
  s.reserve(len + 1);
  const int HEAD = 0;
  s.push_back(Seg{0, 0, 0, 0, 0, 10000, -1, -1});  // head
  int tail_idx = -2;                               // the tail sentinel is index -2
  int min_sb = 10000, max_sb = -1;
  int64_t delta_prev = (int64_t)(array[B0 + 1] - array[B0]);
  int cur = HEAD;
  for (uint32_t i = B0 + 1; i < B0 + len - 1; i++) {
    const int64_t delta = (int64_t)(array[i + 1] - array[i]);
    const int sdb = cal_bits(delta_prev, delta);
    min_sb = std::min(min_sb, sdb);
    max_sb = std::max(max_sb, sdb);
    s.push_back(Seg{(int)i - 1, (int)i - 1, 0, 0, delta_prev, sdb, cur, -1});
    s[cur].next = (int)s.size() - 1;
    cur = (int)s.size() - 1;
    delta_prev = delta;
  }
  s.push_back(Seg{(int)(B0 + len - 2), (int)(B0 + len - 2), 0, 0, delta_prev, 10000, cur, tail_idx});
  s[cur].next = (int)s.size() - 1;
  const int last = (int)s.size() - 1;
  (void)last;
  auto is_tail = [&](int x) { return x == tail_idx; };
  auto nxt = [&](int x) { return s[x].next; };

  // ---- merge by bit class (…:326-433) ----
  for (int aim = min_sb; aim <= max_sb; aim++) {
    int c = s[HEAD].next;
    while (!is_tail(c) && !is_tail(nxt(c))) {
      if (s[c].ddn != aim) {
        c = nxt(c);
        continue;
      }
      int n = nxt(c);
      const int former = s[c].start, start = s[n].start, now = s[n].end;
      const int lbo = cal_bits(s[c].min_delta, s[c].max_delta), rbo = cal_bits(s[n].min_delta, s[n].max_delta);
      const int64_t nmax = std::max(std::max(s[c].max_delta, s[n].max_delta), s[c].next_delta);
      const int64_t nmin = std::min(std::min(s[c].min_delta, s[n].min_delta), s[c].next_delta);
      const int nb = cal_bits(nmin, nmax);
      const int origin_cost = (start - former) * lbo + (now - start + 1) * rbo;
      const int merged_cost = nb * (now - former + 1);
      if (!(merged_cost - origin_cost < overhead)) {
        c = nxt(c);
        continue;
      }
      s[c].end = now;
      s[c].next = s[n].next;
      if (!is_tail(s[n].next)) s[s[n].next].prev = c;
      s[c].next_delta = s[n].next_delta;
      s[c].max_delta = nmax;
      s[c].min_delta = nmin;
      s[c].ddn = s[n].ddn;
      // grow left (never into the first segment of the block)
      int p = s[c].prev;
      while (p != HEAD && s[p].prev != HEAD) {
        const int left = s[p].start;
        const int64_t lmax = std::max(std::max(s[p].max_delta, s[c].max_delta), s[p].next_delta);
        const int64_t lmin = std::min(std::min(s[p].min_delta, s[c].min_delta), s[p].next_delta);
        const int bnew = cal_bits(lmin, lmax);
        const int ol = cal_bits(s[p].min_delta, s[p].max_delta), orr = cal_bits(s[c].min_delta, s[c].max_delta);
        const int oc = (s[c].start - left) * ol + (s[c].end - s[c].start + 1) * orr;
        const int mc = bnew * (s[c].end - left + 1);
        if (!(mc - oc < overhead)) break;
        s[c].start = left;
        s[c].prev = s[p].prev;
        s[s[p].prev].next = c;
        s[c].min_delta = lmin;
        s[c].max_delta = lmax;
        p = s[c].prev;
      }
      // grow right (never into the last segment of the block)
      n = nxt(c);
      while (!is_tail(n) && !is_tail(nxt(n))) {
        const int right = s[n].end;
        const int64_t rmax = std::max(std::max(s[n].max_delta, s[c].max_delta), s[c].next_delta);
        const int64_t rmin = std::min(std::min(s[n].min_delta, s[c].min_delta), s[c].next_delta);
        const int bnew = cal_bits(rmin, rmax);
        const int ol = cal_bits(s[c].min_delta, s[c].max_delta), orr = cal_bits(s[n].min_delta, s[n].max_delta);
        const int oc = (right - s[n].start + 1) * orr + (s[n].start - s[c].start) * ol;
        const int mc = bnew * (right - s[c].start + 1);
        if (!(mc - oc < overhead)) break;
        s[c].end = right;
        s[c].next = s[n].next;
        if (!is_tail(s[n].next)) s[s[n].next].prev = c;
        s[c].max_delta = rmax;
        s[c].min_delta = rmin;
        s[c].ddn = s[n].ddn;
        s[c].next_delta = s[n].next_delta;
        n = nxt(c);
      }
      c = nxt(c);
    }
  }

  // ---- size-driven pairwise merge passes (…:439-483, merge :516-570) ----
  std::vector<uint32_t> idx, sz;
  for (int c = s[HEAD].next; !is_tail(c); c = nxt(c)) idx.push_back((uint32_t)s[c].start);
  const uint32_t endv = B0 + len;
  for (size_t i = 0; i < idx.size(); i++) sz.push_back((uint32_t)segment_cost(array, idx[i], (i + 1 < idx.size() ? idx[i + 1] : endv) - 1));
  uint64_t total = 0;
  for (uint32_t v : sz) total += v;
  for (;;) {
    const uint64_t before = total;
    std::vector<uint32_t> nidx, nsz;
    uint64_t tnew = 0;
    const size_t ns = idx.size();
    uint32_t start = idx[0];
    size_t k = 0;
    auto at = [&](size_t j) { return j < ns ? idx[j] : endv; };
    while (k < ns) {
      if (k == ns - 1) {
        nidx.push_back(idx[k]);
        nsz.push_back(sz[k]);
        tnew += sz[k];
        k++;
        break;
      }
      const uint32_t init_cost = sz[k] + sz[k + 1];
      const uint32_t merge_cost = (uint32_t)segment_cost(array, start, at(k + 2) - 1);
      if (init_cost > merge_cost) {
        nidx.push_back(start);
        nsz.push_back(merge_cost);
        tnew += merge_cost;
        start = at(k + 2);
        k += 2;
      } else {
        nidx.push_back(idx[k]);
        nsz.push_back(sz[k]);
        tnew += sz[k];
        start = at(k + 1);
        k++;
      }
    }
    idx.swap(nidx);
    sz.swap(nsz);
    total = tnew;
    const uint64_t decline = before - total;  // unsigned, as in the reference
    const double pct = decline * 100.0 / (sizeof(uint64_t) * block_size * 1.0);
    if (!(decline > 0) || pct < 0.01) break;
  }
  out.insert(out.end(), idx.begin(), idx.end());
}

}  // namespace

extern "C" {

int leco_varlen_partition(const uint64_t *h_values, uint64_t n, uint32_t coarse_blocks, int64_t delta,
                          uint64_t *h_starts, uint64_t starts_cap, uint64_t *nseg, int threads) {
  if (!h_values || !h_starts || !nseg || !coarse_blocks || n < 2)
    return leco::record_error(LECO_ERR_ARG, "leco_varlen_partition: need values (n >= 2), starts and a block count");
  if (n > 0xffffffffull) return leco::record_error(LECO_ERR_ARG, "leco_varlen_partition: segments start at 32-bit indices");
  // coarse blocks as experiments/leco_double_int_template_wo_round.cpp:85-91
  uint64_t block_size = n / coarse_blocks;
  if (!block_size) block_size = 1;
  uint64_t blocks = n / block_size;
  if (blocks * block_size < n) blocks++;
  std::vector<std::vector<uint32_t>> parts(blocks);
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  std::vector<std::thread> pool;
  std::atomic<uint64_t> nextb{0};
  auto work = [&]() {
    for (;;) {
      const uint64_t b = nextb.fetch_add(1);
      if (b >= blocks) return;
      const uint64_t B0 = b * block_size;
      const uint64_t len = (b == blocks - 1) ? n - B0 : block_size;
      partition_block(h_values, (uint32_t)B0, (uint32_t)len, (uint32_t)block_size, (int)delta, parts[b]);
    }
  };
  for (int t = 0; t < threads; ++t) pool.emplace_back(work);
  for (auto &t : pool) t.join();
  uint64_t k = 0;
  for (const auto &p : parts) {
    if (k + p.size() > starts_cap) return leco::record_error(LECO_ERR_CAPACITY, "leco_varlen_partition: starts_cap too small");
    for (uint32_t v : p) h_starts[k++] = v;
  }
  *nseg = k;
  return LECO_OK;
}

}  // extern "C"
