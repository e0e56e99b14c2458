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
// Requests of one shape (field, sizes, shift, plan) that each leave part of
// the GPU idle can also share a launch (sfntt_server_set_packing): the request
// at the front of the queue takes queued requests of its shape along as
// further columns of one batch -- the reference's pattern of encoding many
// columns into one command buffer (src/ntt/babybear/metal_ct_gs_r4.rs:181-246)
// applied across requests.  Their inputs are gathered into one arena block,
// one LDE runs over all the columns, and each request's output is its slice
// of the launch's output block.
//
// sfntt_serve_trace replays a request trace against the wall clock: request i
// is submitted at arrival_s[i] after the start; with slots = 1 the server is
// the plain sequential per-request loop (one request in flight, the next one
// admitted when it finishes), with slots > 1 it batches continuously
// (sfntt_serve_trace_packed: and packs up to max_pack requests per launch).
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
  uint64_t group = 0;              // the launch (and arena block) the request ran in
  int slot = -1;
};

// One launch: a request alone, or requests of one shape packed as the columns
// of one batch.  Its arena block holds [packed input] output; the block is
// returned when the last of its requests is released.
struct Group {
  size_t off = 0;
  int refs = 0;
  double width = 0;
  bool exclusive = false;
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
  std::vector<std::vector<uint64_t>> slot_req;  // tickets running on each slot (one launch), empty if free
  std::vector<uint64_t> slot_group;
  std::deque<Request> queue;
  std::map<uint64_t, Request> running, finished;
  std::map<uint64_t, Group> groups;
  std::deque<uint64_t> ready;  // finished, not yet reported by poll
  bool exclusive_running = false;
  double occupancy = 0;  // sum of the running launches' widths
  uint64_t next_ticket = 1, next_group = 1;
  int max_pack = 1;         // requests per launch (1: every request launches alone)
  uint64_t launches = 0;    // launches (groups) admitted
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

double width_of(const sfntt_server* sv, const sfntt_lde_item& it) {
  const double tiles = (double)((uint64_t)it.batch << (it.log_n + it.added_bits)) / 8192.0;
  return std::min(1.0, tiles / (2.0 * sv->ctx->sm_count));
}

// Requests that may share one launch: the same field, sizes, shift and plan,
// each short of filling the GPU alone.
bool packable(const Request& r) { return r.width < 1.0 && r.item.batch > 0 && !exclusive(r.item); }
bool same_shape(const sfntt_lde_item& a, const sfntt_lde_item& b) {
  return a.field == b.field && a.log_n == b.log_n && a.added_bits == b.added_bits &&
         a.shift_monty == b.shift_monty && a.plan == b.plan;
}

// Admits queued requests in order while a slot is free, the GPU has room and
// the arena has room.  The request at the front of the queue launches; with
// packing on, queued requests of its shape (up to max_pack) join it as
// further columns of the same batch: their inputs are gathered into one arena block (host
// requests copy there from the host, device requests from d_in), one LDE runs
// over all the columns, and each request's output is its slice of the
// launch's output block (copied back to the host for host requests).
Status admit(sfntt_server* sv) {
  while (!sv->queue.empty()) {
    int slot = -1;
    for (size_t s = 0; s < sv->slot_req.size(); ++s)
      if (sv->slot_req[s].empty()) { slot = (int)s; break; }
    if (slot < 0) return {};
    const Request& front = sv->queue.front();
    if (!sv->running.empty() && (exclusive(front.item) || sv->exclusive_running)) return {};
    const double room = sv->running.empty() ? 1.0 : 1.0 - sv->occupancy;
    if (!sv->running.empty() && front.width > room + 1e-9) return {};  // the GPU is full
    // members of the launch: the front, then same-shape requests behind it
    std::vector<size_t> members{0};
    uint32_t cols = front.item.batch;
    if (sv->max_pack > 1 && packable(front)) {
      // Same-shape requests join until max_pack: one launch of their columns
      // never takes longer than their launches one after another, so the
      // launch may be wider than the GPU's free width (it then runs as
      // running work drains); the front request alone decided admission.
      for (size_t q = 1; q < sv->queue.size() && (int)members.size() < sv->max_pack; ++q) {
        const Request& c = sv->queue[q];
        if (!packable(c) || !same_shape(c.item, front.item)) continue;
        members.push_back(q);
        cols += c.item.batch;
      }
    }
    const bool packed = members.size() > 1;
    sfntt_lde_item it = front.item;
    it.batch = cols;
    const bool stage_in = packed || front.h_in;
    const size_t in_b = stage_in ? round256(in_bytes(it)) : 0;
    size_t off = 0;
    if (!sv->arena->alloc(in_b + out_bytes(it), &off)) return {};  // in order: wait for memory
    uint8_t* block = sv->arena_base + off;
    cudaStream_t st = sv->streams[slot];
    const uint64_t n_words = 1ull << it.log_n, ext_words = 1ull << (it.log_n + it.added_bits);
    Status s = [&]() -> Status {
      if (stage_in) {
        uint32_t* dst = reinterpret_cast<uint32_t*>(block);
        for (size_t q : members) {
          const Request& r = sv->queue[q];
          const size_t b = in_bytes(r.item);
          if (r.h_in) SFNTT_CU(cudaMemcpyAsync(dst, r.h_in, b, cudaMemcpyHostToDevice, st));
          else SFNTT_CU(cudaMemcpyAsync(dst, r.item.d_in, b, cudaMemcpyDeviceToDevice, st));
          dst += (size_t)r.item.batch * n_words;
        }
        it.d_in = reinterpret_cast<const uint32_t*>(block);
      }
      it.d_out = reinterpret_cast<uint32_t*>(block + in_b);
      SFNTT_TRY(sfntt::run_item(sv->ctx, it, st));
      uint32_t* src = it.d_out;
      for (size_t q : members) {
        const Request& r = sv->queue[q];
        if (r.h_out) SFNTT_CU(cudaMemcpyAsync(r.h_out, src, out_bytes(r.item), cudaMemcpyDeviceToHost, st));
        src += (size_t)r.item.batch * ext_words;
      }
      SFNTT_CU(cudaEventRecord(sv->events[slot], st));
      return {};
    }();
    if (!s.ok()) {
      sv->arena->release(off);
      return s;
    }
    const uint64_t gid = sv->next_group++;
    Group& g = sv->groups[gid];
    g.off = off;
    g.refs = (int)members.size();
    g.width = std::min(std::max(width_of(sv, it), front.width), std::max(room, front.width));
    g.exclusive = exclusive(it);
    sv->slot_group[slot] = gid;
    sv->exclusive_running = g.exclusive;
    sv->occupancy += g.width;
    ++sv->launches;
    uint32_t* out = it.d_out;
    for (size_t q : members) {
      Request r = sv->queue[q];
      r.group = gid;
      r.slot = slot;
      r.item.d_out = out;
      out += (size_t)r.item.batch * ext_words;
      sv->slot_req[slot].push_back(r.ticket);
      sv->running.emplace(r.ticket, r);
    }
    for (auto q = members.rbegin(); q != members.rend(); ++q) sv->queue.erase(sv->queue.begin() + (ptrdiff_t)*q);
  }
  return {};
}

Status retire(sfntt_server* sv) {
  for (size_t s = 0; s < sv->slot_req.size(); ++s) {
    if (sv->slot_req[s].empty()) continue;
    cudaError_t e = cudaEventQuery(sv->events[s]);
    if (e == cudaErrorNotReady) continue;
    if (e != cudaSuccess) return {sfntt::map_cuda_error(e), std::string("request: ") + cudaGetErrorString(e)};
    const auto g = sv->groups.find(sv->slot_group[s]);
    if (g != sv->groups.end()) sv->occupancy = std::max(0.0, sv->occupancy - g->second.width);
    for (uint64_t t : sv->slot_req[s]) {
      auto it = sv->running.find(t);
      sv->finished.emplace(t, it->second);
      sv->running.erase(it);
      sv->ready.push_back(t);
    }
    sv->slot_req[s].clear();
    if (sv->running.empty()) {
      sv->exclusive_running = false;
      sv->occupancy = 0;
    }
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
    sv->slot_req.assign(slots, {});
    sv->slot_group.assign(slots, 0);
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
  r.width = width_of(sv, r.item);
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
  auto g = sv->groups.find(it->second.group);
  if (g != sv->groups.end() && --g->second.refs <= 0) {
    sv->arena->release(g->second.off);
    sv->groups.erase(g);
  }
  sv->finished.erase(it);
  return SFNTT_OK;
}

int sfntt_server_set_packing(sfntt_server* sv, int max_requests) {
  if (!sv || max_requests < 1) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(sv->ctx->mu);
  sv->max_pack = max_requests;
  return SFNTT_OK;
}

uint64_t sfntt_server_launches(const sfntt_server* sv) { return sv ? sv->launches : 0; }

size_t sfntt_server_pending(const sfntt_server* sv) {
  return sv ? sv->queue.size() + sv->running.size() : 0;
}

int sfntt_serve_trace(sfntt_ctx* ctx, const sfntt_lde_item* reqs, const uint32_t* const* h_in,
                      uint32_t* const* h_out, const double* arrival_s, size_t count, int slots, size_t budget_bytes,
                      double* latency_s, double* makespan_s) {
  return sfntt_serve_trace_packed(ctx, reqs, h_in, h_out, arrival_s, count, slots, 1, budget_bytes, latency_s,
                                  makespan_s, nullptr);
}

int sfntt_serve_trace_packed(sfntt_ctx* ctx, const sfntt_lde_item* reqs, const uint32_t* const* h_in,
                             uint32_t* const* h_out, const double* arrival_s, size_t count, int slots, int max_pack,
                             size_t budget_bytes, double* latency_s, double* makespan_s, uint64_t* launches) {
  if (!ctx || (count && (!reqs || !arrival_s || !latency_s)) || !makespan_s || max_pack < 1)
    return SFNTT_INVALID_ARGUMENT;
  if ((h_in == nullptr) != (h_out == nullptr)) return SFNTT_INVALID_ARGUMENT;
  for (size_t i = 1; i < count; ++i)
    if (arrival_s[i] < arrival_s[i - 1]) return finish(ctx, {SFNTT_INVALID_ARGUMENT, "arrivals must be sorted"});
  sfntt_server* sv = nullptr;
  int st = sfntt_server_create(ctx, budget_bytes, slots, &sv);
  if (st) return st;
  sv->max_pack = max_pack;
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
  if (launches) *launches = sv->launches;
  sfntt_server_destroy(sv);
  return st;
}

}  // extern "C"
