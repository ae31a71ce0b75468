// leco_serve.cu -- request loop over compressed columns resident in HBM.
//
// Point-lookup and range-scan requests arrive from any number of client
// threads (leco_server_submit).  A server thread keeps up to `slots` batches in
// flight, each on its own stream: whenever a slot is free it admits pending
// requests in arrival order as long as their index and output buffers fit in
// the device arena (admission by free device memory), turns them into one item
// table -- a chunk of up to 4096 lookups or one block of a range scan per CTA --
// and runs the whole batch as ONE kernel launch, bracketed by the index upload
// and the per-request copies of the results to the clients' host buffers.  A
// host callback stamps each request's completion time; the arena space is
// returned when the batch retires, and requests that arrived meanwhile are
// admitted into the next batch while the previous ones are still on the GPU
// (continuous batching).  With slots = 1 and one request per batch the same
// loop is the plain per-request launch path used as the baseline.
//
// The reference has no counterpart (its random access is a per-index CPU loop,
// experiments/leco_int_fix_template.cpp:189-207); per lookup this runs the same
// randomdecodeArray8 rules as leco_gather.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "leco_decode.cuh"

namespace leco {

struct ServeCol {
  int32_t codec, dtype;
  uint32_t bs, pad;
  uint64_t n;
  const uint8_t *payload;
  const uint64_t *offsets;
  const leco_dir_entry *dir;
};

// kind 0: lookups  a = device index pointer, b = count (<= kServeChunk), out = results
// kind 1: range    a = first value, b = count, c = block index, out = the request's output
struct ServeItem {
  uint32_t kind, col;
  uint64_t a, b, c;
  void *out;
};
constexpr uint32_t kServeChunk = 4096;

// Delta lookups: the prefix walk of each lookup is shared by a warp (lane j adds
// fields j, j+32, ...), the CTA's warps taking the chunk's lookups in turn.
template <typename T>
__device__ __forceinline__ void delta_lookups(const ServeCol &c, const uint64_t *idx, uint64_t m, T *out, uint32_t *error) {
  constexpr int S = sizeof(T);
  constexpr uint32_t TB = 8u * S;
  const uint64_t *words = reinterpret_cast<const uint64_t *>(c.payload);
  const int lane = threadIdx.x & 31;
  for (uint64_t i = threadIdx.x >> 5; i < m; i += blockDim.x >> 5) {
    const uint64_t g = __ldg(idx + i);
    if (g >= c.n) {
      if (lane == 0) {
        out[i] = 0;
        atomicOr(error, kErrBadIndex);
      }
      continue;
    }
    const uint64_t b = g / c.bs;
    const uint32_t k = (uint32_t)(g - b * c.bs);
    const BlockHdr h = c.dir ? from_dir<kDelta, S>(c.dir, b) : parse_header<kDelta, S>(c.payload, __ldg(c.offsets + b));
    uint64_t v = h.base;
    if (h.l == TB) {
      v = load_field(words, h.body_bit + (uint64_t)k * TB, TB);
    } else if (h.l > TB) {
      if (lane == 0) atomicOr(error, kErrBadHeader);
    } else {
      uint64_t part = 0;  // fields j < k are the deltas before value k
      if (h.l && k) part = h.l > 32 ? delta_walk_part<true>(words, h, k, lane) : delta_walk_part<false>(words, h, k, lane);
      v += warp_sum_u64(part);
    }
    if (lane == 0) out[i] = (T)v;
  }
}

template <typename T, int CODEC>
__device__ __forceinline__ void serve_one(const ServeCol &c, const ServeItem &it, uint32_t *error) {
  if (it.kind == 0) {
    const uint64_t *idx = reinterpret_cast<const uint64_t *>(it.a);
    if (CODEC == kDelta) {
      delta_lookups<T>(c, idx, it.b, reinterpret_cast<T *>(it.out), error);
    } else {
      GatherLaunch g{c.payload, c.offsets, c.dir, c.n, c.bs, idx, it.b, it.out, error};
      gather_lookups<T, CODEC>(g, threadIdx.x, blockDim.x);
    }
  } else {
    DecodeLaunch d{c.payload, c.offsets, c.n, c.bs, it.a, it.b, it.out, error};
    decode_block<T, CODEC, 256>(d, it.c);
  }
}

__global__ void __launch_bounds__(256) serve_kernel(const ServeCol *__restrict__ cols, const ServeItem *__restrict__ items,
                                                    uint32_t *error) {
  const ServeItem it = items[blockIdx.x];
  const ServeCol c = cols[it.col];
  if (c.dtype == 4) {
    switch (c.codec) {
      case kLinear: serve_one<uint32_t, kLinear>(c, it, error); break;
      case kFor: serve_one<uint32_t, kFor>(c, it, error); break;
      case kDelta: serve_one<uint32_t, kDelta>(c, it, error); break;
      case kPoly2: serve_one<uint32_t, kPoly2>(c, it, error); break;
    }
  } else {
    switch (c.codec) {
      case kLinear: serve_one<uint64_t, kLinear>(c, it, error); break;
      case kFor: serve_one<uint64_t, kFor>(c, it, error); break;
      case kDelta: serve_one<uint64_t, kDelta>(c, it, error); break;
      case kPoly2: serve_one<uint64_t, kPoly2>(c, it, error); break;
    }
  }
}

// First-fit allocator over one device buffer (the output/index budget).
class Arena {
 public:
  // Every allocation is a multiple of 256 bytes, so only that much of `size` is usable.
  void init(uint64_t size) {
    size &= ~255ull;
    size_ = size;
    free_.clear();
    free_[0] = size;
    used_ = 0;
  }
  static uint64_t round(uint64_t bytes) { return (bytes + 255) & ~255ull; }
  // Offset of `bytes` (rounded to 256) or ~0 when nothing fits.
  uint64_t alloc(uint64_t bytes) {
    bytes = round(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        const uint64_t off = it->first, rest = it->second - bytes;
        free_.erase(it);
        if (rest) free_[off + bytes] = rest;
        used_ += bytes;
        return off;
      }
    }
    return ~0ull;
  }
  void release(uint64_t off, uint64_t bytes) {
    bytes = round(bytes);
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  uint64_t size() const { return size_; }
  uint64_t used() const { return used_; }

 private:
  uint64_t size_ = 0, used_ = 0;
  std::map<uint64_t, uint64_t> free_;
};

using Clock = std::chrono::steady_clock;

struct Req {
  uint64_t id = 0;
  leco_request r{};
  Clock::time_point t_submit, t_done;
  uint64_t off = 0, bytes = 0;  // arena space: [indices][results]
  std::atomic<int> done{0};       // results are in the client's buffer (set by the batch callback)
  bool retired = false;           // the server loop no longer references this request (under mu)
};

struct Slot {
  struct ::leco_server *server = nullptr;
  cudaStream_t st = nullptr;
  ServeItem *h_items = nullptr;  // pinned
  ServeItem *d_items = nullptr;
  std::vector<Req *> reqs;
  std::atomic<int> busy{0};
  std::atomic<int> finished{0};
};

}  // namespace leco

using namespace leco;

struct leco_server {
  std::vector<leco_column_desc> cols;
  ServeCol *d_cols = nullptr;
  leco_server_options opt{};
  uint8_t *arena_base = nullptr;
  Arena arena;
  std::vector<Slot *> slots;
  uint32_t max_items = 0;
  uint32_t *err = nullptr;
  std::mutex mu;
  std::condition_variable cv;       // submissions and batch completions
  std::condition_variable cv_done;  // request completions
  std::deque<Req *> pending;
  std::map<uint64_t, Req *> live;
  uint64_t next_id = 1;
  bool stop = false;
  std::thread loop;
  // statistics
  uint64_t completed = 0, lookups = 0, scanned = 0, batches = 0, max_batch = 0;
  std::vector<double> lat_us;
  std::string fail_msg;
};

namespace {

int serr(int code, const std::string &m) { return leco::record_error(code, m); }

uint64_t req_bytes(const leco_request &r, int dtype) {
  const uint64_t idx = r.kind == LECO_REQ_LOOKUP ? ((r.count * 8 + 255) & ~255ull) : 0;
  return idx + r.count * (uint64_t)dtype;
}

uint32_t req_items(const leco_request &r, uint32_t bs) {
  if (r.kind == LECO_REQ_LOOKUP) return (uint32_t)((r.count + kServeChunk - 1) / kServeChunk);
  if (!r.count) return 0;
  return (uint32_t)((r.first + r.count - 1) / bs - r.first / bs + 1);
}

void CUDART_CB batch_done(void *p) {
  auto *s = static_cast<Slot *>(p);
  const auto now = Clock::now();
  for (Req *r : s->reqs) {
    r->t_done = now;
    r->done.store(1, std::memory_order_release);
  }
  s->finished.store(1, std::memory_order_release);
  // taking the lock orders this store before the loop's check-then-wait, so the wake-up
  // below cannot fall between them and be lost
  { std::lock_guard<std::mutex> lk(s->server->mu); }
  s->server->cv.notify_one();  // wake the server loop to retire the batch
}

// Issues one batch on slot s.  Called by the server thread only.
void issue(leco_server *sv, Slot *s) {
  cudaStream_t st = s->st;
  uint32_t ni = 0;
  for (Req *q : s->reqs) {
    const leco_request &r = q->r;
    const leco_column_desc &c = sv->cols[r.column];
    uint8_t *base = sv->arena_base + q->off;
    if (r.kind == LECO_REQ_LOOKUP) {
      const uint64_t idx_bytes = (r.count * 8 + 255) & ~255ull;
      cudaMemcpyAsync(base, r.h_idx, r.count * 8, cudaMemcpyHostToDevice, st);
      uint8_t *out = base + idx_bytes;
      for (uint64_t i = 0; i < r.count; i += kServeChunk) {
        ServeItem &it = s->h_items[ni++];
        it.kind = 0;
        it.col = r.column;
        it.a = reinterpret_cast<uint64_t>(base) + i * 8;
        it.b = std::min<uint64_t>(kServeChunk, r.count - i);
        it.c = 0;
        it.out = out + i * (uint64_t)c.dtype;
      }
    } else {
      const uint64_t b0 = r.first / c.block_size, b1 = (r.first + r.count - 1) / c.block_size;
      for (uint64_t b = b0; b <= b1; ++b) {
        ServeItem &it = s->h_items[ni++];
        it.kind = 1;
        it.col = r.column;
        it.a = r.first;
        it.b = r.count;
        it.c = b;
        it.out = base;
      }
    }
  }
  cudaMemcpyAsync(s->d_items, s->h_items, ni * sizeof(ServeItem), cudaMemcpyHostToDevice, st);
  if (ni) serve_kernel<<<ni, 256, 0, st>>>(sv->d_cols, s->d_items, sv->err);
  for (Req *q : s->reqs) {
    const leco_request &r = q->r;
    const int dt = sv->cols[r.column].dtype;
    const uint64_t idx_bytes = r.kind == LECO_REQ_LOOKUP ? ((r.count * 8 + 255) & ~255ull) : 0;
    cudaMemcpyAsync(r.h_out, sv->arena_base + q->off + idx_bytes, r.count * (uint64_t)dt, cudaMemcpyDeviceToHost, st);
  }
  s->finished.store(0);
  cudaLaunchHostFunc(st, batch_done, s);
}

void server_loop(leco_server *sv) {
  const uint32_t max_req = std::max<uint32_t>(1, sv->opt.max_requests_per_batch);
  uint64_t tried_id = 0;  // next_id when admission into a free slot was last tried
  for (;;) {
    bool worked = false;
    // retire finished batches
    for (Slot *s : sv->slots) {
      if (s->busy.load() && s->finished.load(std::memory_order_acquire)) {
        std::lock_guard<std::mutex> lk(sv->mu);
        for (Req *q : s->reqs) {
          sv->arena.release(q->off, q->bytes);
          sv->completed++;
          if (q->r.kind == LECO_REQ_LOOKUP) sv->lookups += q->r.count;
          else sv->scanned += q->r.count;
          sv->lat_us.push_back(std::chrono::duration<double, std::micro>(q->t_done - q->t_submit).count());
          q->retired = true;
        }
        s->reqs.clear();
        s->busy.store(0);
        worked = true;
        sv->cv_done.notify_all();
      }
    }
    // admit into a free slot
    for (Slot *s : sv->slots) {
      if (s->busy.load()) continue;
      {
        std::lock_guard<std::mutex> lk(sv->mu);
        tried_id = sv->next_id;
        uint32_t items = 0;
        while (!sv->pending.empty() && s->reqs.size() < max_req) {
          Req *q = sv->pending.front();
          const leco_column_desc &c = sv->cols[q->r.column];
          const uint32_t ni = req_items(q->r, c.block_size);
          if (items + ni > sv->max_items) break;
          const uint64_t off = sv->arena.alloc(q->bytes);
          if (off == ~0ull) break;  // wait for memory to free up (arrival order is kept)
          q->off = off;
          items += ni;
          s->reqs.push_back(q);
          sv->pending.pop_front();
        }
      }
      if (s->reqs.empty()) break;
      s->busy.store(1);
      issue(sv, s);
      sv->batches++;
      sv->max_batch = std::max<uint64_t>(sv->max_batch, s->reqs.size());
      worked = true;
    }
    if (!worked) {
      std::unique_lock<std::mutex> lk(sv->mu);
      bool inflight = false;
      for (Slot *s : sv->slots) inflight |= s->busy.load() != 0;
      if (sv->stop && sv->pending.empty() && !inflight) return;
      // Nothing was retired or admitted in this pass: the requests that were pending then
      // wait for a slot or for arena space, which come back only when a batch finishes.  Go
      // round again at once only for a finished batch, or for requests that arrived after the
      // last admission try while a slot is free.  Batch callbacks and submissions notify `cv`
      // under `mu`, so the wait misses neither; its timeout is only a backstop.
      bool ready = false, free_slot = false;
      for (Slot *s : sv->slots) {
        ready |= s->busy.load() && s->finished.load();
        free_slot |= !s->busy.load();
      }
      ready |= free_slot && !sv->pending.empty() && sv->next_id != tried_id;
      if (!ready) sv->cv.wait_for(lk, std::chrono::milliseconds(2));
    }
  }
}

}  // namespace

extern "C" {

int leco_server_create(const leco_column_desc *h_cols, uint32_t ncols, const leco_server_options *opt, leco_server **out) {
  if (!h_cols || !ncols || !out) return serr(LECO_ERR_ARG, "leco_server_create: null pointer or no columns");
  auto *sv = new leco_server();
  sv->cols.assign(h_cols, h_cols + ncols);
  if (opt) sv->opt = *opt;
  if (!sv->opt.slots) sv->opt.slots = 4;
  if (!sv->opt.max_requests_per_batch) sv->opt.max_requests_per_batch = 1024;
  if (!sv->opt.max_items_per_batch) sv->opt.max_items_per_batch = 65536;
  sv->max_items = sv->opt.max_items_per_batch;
  std::vector<ServeCol> dc(ncols);
  for (uint32_t i = 0; i < ncols; ++i) {
    const leco_column_desc &c = h_cols[i];
    if (c.codec < kLinear || c.codec > kPoly2 || (c.dtype != 4 && c.dtype != 8) || !c.block_size || !c.n || !c.d_payload ||
        !c.d_offsets) {
      delete sv;
      return serr(LECO_ERR_ARG, "leco_server_create: bad descriptor for column " + std::to_string(i));
    }
    dc[i] = ServeCol{c.codec, c.dtype, c.block_size, 0, c.n, c.d_payload, c.d_offsets, c.d_dir};
  }
  size_t fr = 0, tot = 0;
  cudaError_t e = cudaMemGetInfo(&fr, &tot);
  uint64_t budget = sv->opt.hbm_budget_bytes ? sv->opt.hbm_budget_bytes : (uint64_t)(fr / 4);
  // admission never plans on more than the device can give now (keep 1 GiB spare)
  if (e == cudaSuccess && budget + (1ull << 30) > fr) budget = fr > (2ull << 30) ? fr - (1ull << 30) : fr / 2;
  if (e == cudaSuccess) e = cudaMalloc(&sv->arena_base, budget);
  if (e == cudaSuccess) e = cudaMalloc(&sv->d_cols, ncols * sizeof(ServeCol));
  if (e == cudaSuccess) e = cudaMemcpy(sv->d_cols, dc.data(), ncols * sizeof(ServeCol), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && leco::device_error_word(&sv->err)) e = cudaErrorUnknown;
  for (uint32_t i = 0; e == cudaSuccess && i < sv->opt.slots; ++i) {
    auto *s = new Slot();
    s->server = sv;
    sv->slots.push_back(s);
    e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaHostAlloc(&s->h_items, sv->max_items * sizeof(ServeItem), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_items, sv->max_items * sizeof(ServeItem));
  }
  if (e != cudaSuccess) {
    leco_server_destroy(sv);
    return serr(LECO_ERR_NOMEM, std::string("leco_server_create: ") + cudaGetErrorString(e));
  }
  sv->arena.init(budget);
  sv->loop = std::thread(server_loop, sv);
  *out = sv;
  return LECO_OK;
}

int leco_server_submit(leco_server *sv, const leco_request *req, uint64_t *req_id) {
  if (!sv || !req || !req_id) return serr(LECO_ERR_ARG, "leco_server_submit: null pointer");
  if (req->column >= sv->cols.size()) return serr(LECO_ERR_ARG, "leco_server_submit: no such column");
  const leco_column_desc &c = sv->cols[req->column];
  if (req->kind != LECO_REQ_LOOKUP && req->kind != LECO_REQ_RANGE) return serr(LECO_ERR_ARG, "leco_server_submit: bad kind");
  if (!req->count || !req->h_out || (req->kind == LECO_REQ_LOOKUP && !req->h_idx))
    return serr(LECO_ERR_ARG, "leco_server_submit: empty request or null buffer");
  if (req->kind == LECO_REQ_RANGE && (req->first > c.n || req->count > c.n - req->first))
    return serr(LECO_ERR_ARG, "leco_server_submit: range outside the column");
  const uint64_t bytes = req_bytes(*req, c.dtype);
  // compared as the arena will allocate it (rounded up to 256 bytes): a request that could
  // never be admitted is refused here instead of blocking every request behind it
  if (Arena::round(bytes) > sv->arena.size() || req_items(*req, c.block_size) > sv->max_items)
    return serr(LECO_ERR_NOMEM, "leco_server_submit: request larger than the server's device budget");
  auto *q = new Req();
  q->r = *req;
  q->bytes = bytes;
  q->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    q->id = sv->next_id++;
    sv->pending.push_back(q);
    sv->live[q->id] = q;
  }
  sv->cv.notify_one();
  *req_id = q->id;
  return LECO_OK;
}

int leco_server_wait(leco_server *sv, uint64_t req_id, double *latency_us) {
  if (!sv) return serr(LECO_ERR_ARG, "leco_server_wait: null server");
  Req *q = nullptr;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->live.find(req_id);
    if (it == sv->live.end()) return serr(LECO_ERR_ARG, "leco_server_wait: unknown request id");
    q = it->second;
  }
  std::unique_lock<std::mutex> lk(sv->mu);
  // completion is published by the batch callback; the loop retires the batch
  sv->cv_done.wait(lk, [&] { return q->retired; });
  if (latency_us) *latency_us = std::chrono::duration<double, std::micro>(q->t_done - q->t_submit).count();
  sv->live.erase(req_id);
  lk.unlock();
  delete q;
  return LECO_OK;
}

int leco_server_drain(leco_server *sv) {
  if (!sv) return serr(LECO_ERR_ARG, "leco_server_drain: null server");
  std::unique_lock<std::mutex> lk(sv->mu);
  sv->cv_done.wait(lk, [&] {
    bool inflight = false;
    for (Slot *s : sv->slots) inflight |= s->busy.load() != 0;
    return sv->pending.empty() && !inflight;
  });
  return LECO_OK;
}

int leco_server_get_stats(leco_server *sv, leco_server_stats *out) {
  if (!sv || !out) return serr(LECO_ERR_ARG, "leco_server_get_stats: null pointer");
  std::lock_guard<std::mutex> lk(sv->mu);
  out->completed = sv->completed;
  out->lookups = sv->lookups;
  out->scanned_values = sv->scanned;
  out->batches = sv->batches;
  out->max_requests_in_batch = sv->max_batch;
  out->arena_bytes = sv->arena.size();
  std::vector<double> v = sv->lat_us;
  std::sort(v.begin(), v.end());
  auto pct = [&](double p) { return v.empty() ? 0.0 : v[(size_t)std::min<double>(v.size() - 1, p * (v.size() - 1) + 0.5)]; };
  out->p50_us = pct(0.50);
  out->p99_us = pct(0.99);
  out->max_us = v.empty() ? 0.0 : v.back();
  double sum = 0;
  for (double x : v) sum += x;
  out->mean_us = v.empty() ? 0.0 : sum / v.size();
  return LECO_OK;
}

int leco_server_reset_stats(leco_server *sv) {
  if (!sv) return serr(LECO_ERR_ARG, "null server");
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->completed = sv->lookups = sv->scanned = sv->batches = sv->max_batch = 0;
  sv->lat_us.clear();
  return LECO_OK;
}

int leco_server_destroy(leco_server *sv) {
  if (!sv) return LECO_OK;
  if (sv->loop.joinable()) {
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->stop = true;
    }
    sv->cv.notify_all();
    sv->loop.join();
  }
  for (Slot *s : sv->slots) {
    if (s->st) cudaStreamSynchronize(s->st);
    if (s->st) cudaStreamDestroy(s->st);
    if (s->h_items) cudaFreeHost(s->h_items);
    if (s->d_items) cudaFree(s->d_items);
    delete s;
  }
  for (auto &kv : sv->live) delete kv.second;
  if (sv->arena_base) cudaFree(sv->arena_base);
  if (sv->d_cols) cudaFree(sv->d_cols);
  delete sv;
  return LECO_OK;
}

}  // extern "C"
