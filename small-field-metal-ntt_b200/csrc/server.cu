// server.cu -- serving LDE / blow-up requests with continuous batching.
//
// A server owns `slots` CUDA streams and one device arena of `budget` bytes
// (allocated once, at creation; requests never call cudaMalloc).  Requests are
// queued in arrival order; sfntt_server_poll retires finished requests
// (event query, arena space returned) and admits queued ones, in order, while
// a slot is free, the arena has room for the request, and the GPU has room:
// a request's width is the fraction of the GPU its widest pass fills
// (min(1, tiles / (2 * SMs)), 2^13-word tiles), and requests run together only
// while their widths add up to at most one.  A request that fills the GPU by
// itself therefore runs alone, as in the plain loop; small requests that
// arrive while others run are packed beside them and overlap on the device.
// Twiddle and multiplier tables stay resident in the context across requests.
//
// sfntt_serve_trace replays a request trace against the wall clock: request i
// is submitted at arrival_s[i] after the start; with slots = 1 the server is
// the plain sequential per-request loop (one request in flight, the next one
// admitted when it finishes), with slots > 1 it batches continuously.
#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <vector>

#include "context.hpp"

namespace {

// First-fit allocator over [0, size) in 256-byte units.
class Arena {
 public:
  explicit Arena(size_t size) { free_[0] = size; }
  bool alloc(size_t bytes, size_t* off) {
    bytes = (bytes + 255) & ~size_t(255);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes;
        const size_t base = it->first;
        free_.erase(it);
        if (rest) free_[base + bytes] = rest;
        used_[*off] = bytes;
        return true;
      }
    }
    return false;
  }
  void release(size_t off) {
    auto u = used_.find(off);
    if (u == used_.end()) return;
    size_t start = off, len = u->second;
    used_.erase(u);
    auto next = free_.lower_bound(start);
    if (next != free_.end() && next->first == start + len) {
      len += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == start) {
        start = prev->first;
        len += prev->second;
        free_.erase(prev);
      }
    }
    free_[start] = len;
  }

 private:
  std::map<size_t, size_t> free_, used_;
};

struct Request {
  uint64_t ticket;
  double width = 1.0;  // fraction of the GPU the request fills
  sfntt_lde_item item;
  const uint32_t* h_in = nullptr;  // host request: input copied into the arena
  uint32_t* h_out = nullptr;       // host request: result copied back here
  size_t off = 0;                  // arena block: [input (host requests)] output
  int slot = -1;
};

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct sfntt_server {
  sfntt_ctx* ctx = nullptr;
  uint8_t* arena_base = nullptr;
  size_t budget = 0;
  Arena* arena = nullptr;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;
  std::vector<int64_t> slot_req;  // ticket running on each slot, -1 if free
  std::deque<Request> queue;
  std::map<uint64_t, Request> running, finished;
  std::deque<uint64_t> ready;  // finished, not yet reported by poll
  bool exclusive_running = false;
  double occupancy = 0;  // sum of the running requests' widths
  uint64_t next_ticket = 1;
};

namespace {

using sfntt::Status;

size_t in_bytes(const sfntt_lde_item& it) { return ((size_t)it.batch << it.log_n) * 4; }
size_t out_bytes(const sfntt_lde_item& it) { return ((size_t)it.batch << (it.log_n + it.added_bits)) * 4; }
size_t round256(size_t b) { return (b + 255) & ~size_t(255); }
size_t arena_bytes(const Request& r) { return (r.h_in ? round256(in_bytes(r.item)) : 0) + out_bytes(r.item); }

// BabyBear / KoalaBear items outside the fused LDE's range run the unfused
// composition through the context's one scratch buffer, so they run alone on
// the device.
bool exclusive(const sfntt_lde_item& it) {
  return sfntt::is_monty(it.field) && it.batch && !(it.log_n >= 1 && it.log_n <= 24 && it.added_bits <= 4);
}

Status admit(sfntt_server* sv) {
  while (!sv->queue.empty()) {
    int slot = -1;
    for (size_t s = 0; s < sv->slot_req.size(); ++s)
      if (sv->slot_req[s] < 0) { slot = (int)s; break; }
    if (slot < 0) return {};
    Request& r = sv->queue.front();
    if (!sv->running.empty() && (exclusive(r.item) || sv->exclusive_running)) return {};
    if (!sv->running.empty() && sv->occupancy + r.width > 1.0 + 1e-9) return {};  // the GPU is full
    size_t off = 0;
    if (!sv->arena->alloc(arena_bytes(r), &off)) return {};  // in order: wait for memory
    r.off = off;
    r.slot = slot;
    sfntt_lde_item it = r.item;
    uint8_t* block = sv->arena_base + off;
    cudaStream_t st = sv->streams[slot];
    Status s = [&]() -> Status {
      if (r.h_in) {
        it.d_in = reinterpret_cast<const uint32_t*>(block);
        block += round256(in_bytes(it));
        SFNTT_CU(cudaMemcpyAsync(const_cast<uint32_t*>(it.d_in), r.h_in, in_bytes(it), cudaMemcpyHostToDevice, st));
      }
      it.d_out = reinterpret_cast<uint32_t*>(block);
      SFNTT_TRY(sfntt::run_item(sv->ctx, it, st));
      if (r.h_out) SFNTT_CU(cudaMemcpyAsync(r.h_out, it.d_out, out_bytes(it), cudaMemcpyDeviceToHost, st));
      SFNTT_CU(cudaEventRecord(sv->events[slot], st));
      return {};
    }();
    if (!s.ok()) {
      sv->arena->release(off);
      return s;
    }
    sv->slot_req[slot] = (int64_t)r.ticket;
    sv->exclusive_running = exclusive(r.item);
    sv->occupancy += r.width;
    r.item.d_out = it.d_out;
    sv->running.emplace(r.ticket, r);
    sv->queue.pop_front();
  }
  return {};
}

Status retire(sfntt_server* sv) {
  for (size_t s = 0; s < sv->slot_req.size(); ++s) {
    if (sv->slot_req[s] < 0) continue;
    cudaError_t e = cudaEventQuery(sv->events[s]);
    if (e == cudaErrorNotReady) continue;
    if (e != cudaSuccess) return {sfntt::map_cuda_error(e), std::string("request: ") + cudaGetErrorString(e)};
    const uint64_t t = (uint64_t)sv->slot_req[s];
    sv->slot_req[s] = -1;
    auto it = sv->running.find(t);
    sv->occupancy = std::max(0.0, sv->occupancy - it->second.width);
    sv->finished.emplace(t, it->second);
    sv->running.erase(it);
    if (sv->running.empty()) {
      sv->exclusive_running = false;
      sv->occupancy = 0;
    }
    sv->ready.push_back(t);
  }
  return {};
}

// Makes the tables of a request resident (no-op once cached) and waits for
// them, so that slot streams can read them.
Status prepare_request(sfntt_ctx* ctx, const sfntt_lde_item& req, const void* any) {
  sfntt_lde_item probe = req;
  if (!probe.d_in) probe.d_in = static_cast<const uint32_t*>(any);  // buffers are not touched
  probe.d_out = static_cast<uint32_t*>(const_cast<void*>(any));
  SFNTT_TRY(sfntt::prepare_item(ctx, probe, ctx->stream));
  SFNTT_CU(cudaStreamSynchronize(ctx->stream));
  return {};
}

int finish(sfntt_ctx* ctx, const Status& s) {
  if (ctx) ctx->last_error = s.ok() ? std::string() : s.msg;
  return s.code;
}

}  // namespace

extern "C" {

int sfntt_server_create(sfntt_ctx* ctx, size_t budget_bytes, int slots, sfntt_server** out) {
  if (!ctx || !out || slots < 1 || slots > 64 || budget_bytes == 0) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->device);
  auto* sv = new sfntt_server();
  sv->ctx = ctx;
  sv->budget = budget_bytes;
  Status s = [&]() -> Status {
    SFNTT_CU(cudaMalloc(reinterpret_cast<void**>(&sv->arena_base), budget_bytes));
    sv->arena = new Arena(budget_bytes);
    sv->streams.resize(slots, nullptr);
    sv->events.resize(slots, nullptr);
    sv->slot_req.assign(slots, -1);
    for (int i = 0; i < slots; ++i) {
      SFNTT_CU(cudaStreamCreateWithFlags(&sv->streams[i], cudaStreamNonBlocking));
      SFNTT_CU(cudaEventCreateWithFlags(&sv->events[i], cudaEventDisableTiming));
    }
    return {};
  }();
  if (prev >= 0) cudaSetDevice(prev);
  if (!s.ok()) {
    cudaGetLastError();
    sfntt_server_destroy(sv);
    return finish(ctx, s);
  }
  *out = sv;
  return finish(ctx, {});
}

void sfntt_server_destroy(sfntt_server* sv) {
  if (!sv) return;
  int prev = -1;
  cudaGetDevice(&prev);
  if (sv->ctx) cudaSetDevice(sv->ctx->device);
  for (cudaStream_t s : sv->streams)
    if (s) cudaStreamSynchronize(s);
  for (cudaEvent_t e : sv->events)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t s : sv->streams)
    if (s) cudaStreamDestroy(s);
  if (sv->arena_base) cudaFree(sv->arena_base);
  delete sv->arena;
  if (prev >= 0) cudaSetDevice(prev);
  delete sv;
}

}  // extern "C"

namespace {

int submit(sfntt_server* sv, const sfntt_lde_item* req, const uint32_t* h_in, uint32_t* h_out, uint64_t* ticket) {
  if (!sv || !req || !ticket) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(sv->ctx->mu);
  if (!sfntt::valid_field(req->field)) return SFNTT_INVALID_ARGUMENT;
  Request r;
  r.item = *req;
  r.h_in = h_in;
  r.h_out = h_out;
  if (h_in) r.item.d_in = nullptr;
  r.item.d_out = nullptr;
  if (r.item.batch && !h_in && !r.item.d_in) return SFNTT_INVALID_ARGUMENT;
  if (!sfntt::ext_fits(r.item.log_n, r.item.added_bits, 30))
    return finish(sv->ctx, {SFNTT_INVALID_SIZE, "log_n + added_bits > 30"});
  const double tiles = (double)((uint64_t)r.item.batch << (r.item.log_n + r.item.added_bits)) / 8192.0;
  r.width = std::min(1.0, tiles / (2.0 * sv->ctx->sm_count));
  if (arena_bytes(r) > sv->budget)
    return finish(sv->ctx, {SFNTT_ALLOC_FAILED, "request exceeds the server's HBM budget"});
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(sv->ctx->device);
  Status s = prepare_request(sv->ctx, r.item, sv->arena_base);
  if (prev >= 0) cudaSetDevice(prev);
  if (!s.ok()) return finish(sv->ctx, s);
  r.ticket = sv->next_ticket++;
  sv->queue.push_back(r);
  *ticket = r.ticket;
  return SFNTT_OK;
}

}  // namespace

extern "C" {

int sfntt_server_submit(sfntt_server* sv, const sfntt_lde_item* req, uint64_t* ticket) {
  return submit(sv, req, nullptr, nullptr, ticket);
}

int sfntt_server_submit_host(sfntt_server* sv, const sfntt_lde_item* req, const uint32_t* h_in, uint32_t* h_out,
                             uint64_t* ticket) {
  if (req && req->batch && (!h_in || !h_out)) return SFNTT_INVALID_ARGUMENT;
  return submit(sv, req, h_in, h_out, ticket);
}

int sfntt_server_poll(sfntt_server* sv, uint64_t* done, size_t cap, size_t* n_done) {
  if (!sv || !n_done) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(sv->ctx->mu);
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(sv->ctx->device);
  Status s = retire(sv);
  if (s.ok()) s = admit(sv);
  if (prev >= 0) cudaSetDevice(prev);
  *n_done = 0;
  while (done && *n_done < cap && !sv->ready.empty()) {
    done[(*n_done)++] = sv->ready.front();
    sv->ready.pop_front();
  }
  return finish(sv->ctx, s);
}

int sfntt_server_result(sfntt_server* sv, uint64_t ticket, uint32_t** d_out) {
  if (!sv || !d_out) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(sv->ctx->mu);
  auto it = sv->finished.find(ticket);
  if (it == sv->finished.end()) return SFNTT_INVALID_ARGUMENT;
  *d_out = it->second.item.d_out;
  return SFNTT_OK;
}

int sfntt_server_release(sfntt_server* sv, uint64_t ticket) {
  if (!sv) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(sv->ctx->mu);
  auto it = sv->finished.find(ticket);
  if (it == sv->finished.end()) return SFNTT_INVALID_ARGUMENT;
  sv->arena->release(it->second.off);
  sv->finished.erase(it);
  return SFNTT_OK;
}

size_t sfntt_server_pending(const sfntt_server* sv) {
  return sv ? sv->queue.size() + sv->running.size() : 0;
}

int sfntt_serve_trace(sfntt_ctx* ctx, const sfntt_lde_item* reqs, const uint32_t* const* h_in,
                      uint32_t* const* h_out, const double* arrival_s, size_t count, int slots, size_t budget_bytes,
                      double* latency_s, double* makespan_s) {
  if (!ctx || (count && (!reqs || !arrival_s || !latency_s)) || !makespan_s) return SFNTT_INVALID_ARGUMENT;
  if ((h_in == nullptr) != (h_out == nullptr)) return SFNTT_INVALID_ARGUMENT;
  for (size_t i = 1; i < count; ++i)
    if (arrival_s[i] < arrival_s[i - 1]) return finish(ctx, {SFNTT_INVALID_ARGUMENT, "arrivals must be sorted"});
  sfntt_server* sv = nullptr;
  int st = sfntt_server_create(ctx, budget_bytes, slots, &sv);
  if (st) return st;
  {  // tables of every request resident before the clock starts
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(ctx->device);
    for (size_t i = 0; i < count && st == SFNTT_OK; ++i) st = finish(ctx, prepare_request(ctx, reqs[i], sv->arena_base));
    if (prev >= 0) cudaSetDevice(prev);
  }
  std::map<uint64_t, size_t> index;
  std::vector<uint64_t> done(64);
  size_t next = 0, completed = 0;
  const double t0 = now_s();
  while (st == SFNTT_OK && completed < count) {
    const double t = now_s() - t0;
    while (next < count && arrival_s[next] <= t) {
      uint64_t ticket = 0;
      st = h_in ? sfntt_server_submit_host(sv, &reqs[next], h_in[next], h_out[next], &ticket)
                : sfntt_server_submit(sv, &reqs[next], &ticket);
      if (st) break;
      index[ticket] = next++;
    }
    if (st) break;
    size_t nd = 0;
    st = sfntt_server_poll(sv, done.data(), done.size(), &nd);
    const double tc = now_s() - t0;
    for (size_t k = 0; k < nd; ++k) {
      const size_t i = index[done[k]];
      latency_s[i] = tc - arrival_s[i];
      sfntt_server_release(sv, done[k]);
      ++completed;
    }
  }
  *makespan_s = now_s() - t0;
  sfntt_server_destroy(sv);
  return st;
}

}  // extern "C"
