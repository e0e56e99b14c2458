// batch.cu -- uneven batches of LDE / blow-up work items in one graph launch,
// with an autotuned plan per (field, log n, columns, blow-up).
//
// An item is one polynomial batch: `batch` SoA columns of 2^log_n points in
// either field, extended by 2^added_bits (0 = evaluate on the same-size coset).
// BabyBear items run the coset LDE of src/lde/mod.rs:43-107; M31 items run the
// composition inverse(odds(log n)) -> zero-pad -> forward(odds(log n + b)).
//
// * sfntt_batch_run: one item after another on one stream (the plain
//   per-polynomial loop).
// * sfntt_batch_graph_create / sfntt_graph_launch: every item captured once
//   into a CUDA graph, items spread over `lanes` forked streams so that
//   independent items overlap on the device; replaying the graph is one launch
//   for the whole batch.
// * sfntt_autotune: for each distinct key (field, log n, columns rounded up to
//   a power of two, blow-up) time the candidate plans on the first item with
//   that key and keep the fastest; the table can be saved and loaded as text.
//   Plans: the persistent TMA engine with per-position strided twiddles, the
//   same with four-step strided passes, or the first (non-TMA) tile engine.
#include <algorithm>
#include <cstdio>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "context.hpp"
#include "host_field.hpp"
#include "worklist.cuh"

struct sfntt_graph {
  int device = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t kernels = 0;
  void* work = nullptr;  // persistent form: the device work lists and their counters
};

namespace sfntt {
namespace {

struct Knobs {
  bool no_tma, ntt_plain, lde_plain, split_c12;
  int tma_ctas;
};

// A plan is an engine (SFNTT_PLAN_TMA / _TMA_FOUR_STEP / _TILE) plus optional
// flags: SFNTT_PLAN_SPLIT12 (layer ranges above 12 layers: a 12-layer
// contiguous pass, the rest in strided passes) and SFNTT_PLAN_ONE_CTA (one
// persistent CTA per SM instead of the kernel's full residency).
Knobs plan_knobs(int plan, const sfntt_ctx* ctx) {
  const bool split = (plan & SFNTT_PLAN_SPLIT12) != 0;
  const int ctas = (plan & SFNTT_PLAN_ONE_CTA) ? 1 : 0;
  switch (plan & SFNTT_PLAN_ENGINE_MASK) {
    case SFNTT_PLAN_TMA: return {false, true, false, split, ctas};
    case SFNTT_PLAN_TMA_FOUR_STEP: return {false, true, true, split, ctas};
    case SFNTT_PLAN_TILE: return {true, false, false, false, 0};
    default: return {ctx->no_tma, ctx->ntt_plain, ctx->lde_plain, ctx->split_c12, ctx->tma_ctas};
  }
}

bool valid_plan(int plan) {
  if (plan & ~(SFNTT_PLAN_ENGINE_MASK | SFNTT_PLAN_SPLIT12 | SFNTT_PLAN_ONE_CTA)) return false;
  const int e = plan & SFNTT_PLAN_ENGINE_MASK;
  if (e == SFNTT_PLAN_AUTO) return plan == SFNTT_PLAN_AUTO;
  return e != SFNTT_PLAN_TILE || plan == SFNTT_PLAN_TILE;
}

uint32_t pow2_ceil(uint32_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

std::string key_of(const sfntt_lde_item& it) {
  char buf[96];
  const char* tag = it.field == SFNTT_BABYBEAR ? "bb" : (it.field == SFNTT_KOALABEAR ? "kb" : "m31");
  std::snprintf(buf, sizeof buf, "%s/%u/%u/%u", tag, it.log_n,
                pow2_ceil(it.batch ? it.batch : 1), it.added_bits);
  return buf;
}

Status check_item(const sfntt_lde_item& it) {
  if (!valid_field(it.field)) return {SFNTT_INVALID_ARGUMENT, "item: unknown field"};
  if (!ext_fits(it.log_n, it.added_bits, 30)) return {SFNTT_INVALID_SIZE, "item: log_n + added_bits too large"};
  if (it.batch && (!it.d_in || !it.d_out)) return {SFNTT_INVALID_ARGUMENT, "item: null buffer"};
  return {};
}

}  // namespace

// Runs one item on stream s under its plan (tuned, explicit or default).
Status run_item(sfntt_ctx* ctx, const sfntt_lde_item& it, cudaStream_t s) {
  SFNTT_TRY(check_item(it));
  int plan = it.plan;
  if (plan == SFNTT_PLAN_AUTO) {
    auto f = ctx->tuned.find(key_of(it));
    plan = f == ctx->tuned.end() ? SFNTT_PLAN_AUTO : f->second;
  }
  if (!valid_plan(plan)) return {SFNTT_INVALID_ARGUMENT, "item: unknown plan " + std::to_string(plan)};
  const Knobs saved{ctx->no_tma, ctx->ntt_plain, ctx->lde_plain, ctx->split_c12, ctx->tma_ctas};
  const Knobs k = plan_knobs(plan, ctx);
  ctx->no_tma = k.no_tma;
  ctx->ntt_plain = k.ntt_plain;
  ctx->lde_plain = k.lde_plain;
  ctx->split_c12 = k.split_c12;
  ctx->tma_ctas = k.tma_ctas;
  Status st = is_monty(it.field)
                  ? monty_lde_dev(ctx, it.field, it.d_in, it.d_out, it.log_n, it.batch, it.added_bits,
                                  it.shift_monty, SFNTT_LDE_FUSED, s)
                  : m31_lde_dev(ctx, it.d_in, it.d_out, it.log_n, it.batch, it.added_bits, s);
  ctx->no_tma = saved.no_tma;
  ctx->ntt_plain = saved.ntt_plain;
  ctx->lde_plain = saved.lde_plain;
  ctx->split_c12 = saved.split_c12;
  ctx->tma_ctas = saved.tma_ctas;
  return st;
}

Status prepare_item(sfntt_ctx* ctx, const sfntt_lde_item& it, cudaStream_t s) {
  SFNTT_TRY(check_item(it));
  const uint2* t = nullptr;
  const uint32_t ext = it.log_n + it.added_bits;
  if (is_monty(it.field)) {
    const int f = it.field;
    const uint32_t adicity = host::monty_field(f).two_adicity;
    if (ext + 1 > adicity) return {SFNTT_INVALID_SIZE, "log_n + added_bits must be <= " + std::to_string(adicity - 1)};
    if (it.log_n) SFNTT_TRY(monty_twiddles(ctx, f, true, it.log_n, s, &t));
    if (ext) SFNTT_TRY(monty_twiddles(ctx, f, false, ext, s, &t));
    if (it.added_bits <= 4) {
      SFNTT_TRY(monty_lde_table(ctx, f, it.log_n, it.added_bits, it.shift_monty, 0, s, &t));
      if (it.log_n >= 13) SFNTT_TRY(monty_lde_table(ctx, f, it.log_n, it.added_bits, it.shift_monty, 2, s, &t));
    }
    SFNTT_TRY(monty_lde_table(ctx, f, it.log_n, it.added_bits, it.shift_monty, 1, s, &t));
    if (it.log_n >= 13) {
      SFNTT_TRY(monty_twist_table(ctx, f, it.log_n - 8, 8, true, s, &t));
      SFNTT_TRY(monty_twist_table(ctx, f, it.log_n - 8, 8, false, s, &t));
    }
    // strided-pass twists of the four-step plain-NTT plans inside [0, log_n - 8)
    // (both layer splits: a graph captured later may use either)
    for (uint32_t top : {it.log_n, ext}) {
      const uint32_t lo = top >= 13 ? top - 8 : 0;
      if (lo > 12) {
        for (bool c12 : {false, true}) {
          uint32_t plo[4], pcnt[4];
          const int k = tma_split(0, lo, plo, pcnt, c12, 14u);  // Montgomery fields
          for (int i = 1; i < k; ++i) {
            const bool compact = twist_compact_for(plo[i], pcnt[i]);
            SFNTT_TRY(monty_twist_table(ctx, f, plo[i], pcnt[i], true, s, &t, compact));
            SFNTT_TRY(monty_twist_table(ctx, f, plo[i], pcnt[i], false, s, &t, compact));
          }
        }
      }
    }
  } else {
    if (ext > 30) return {SFNTT_INVALID_SIZE, "log_n + added_bits must be <= 30"};
    if (it.log_n) {
      SFNTT_TRY(m31_twiddles(ctx, true, it.log_n, s, &t));
      SFNTT_TRY(m31_twiddles(ctx, false, ext, s, &t));
    }
  }
  return {};
}

}  // namespace sfntt

using sfntt::Status;

namespace {

struct Guard {
  sfntt_ctx* ctx;
  int prev = -1;
  std::lock_guard<std::recursive_mutex> lk;
  explicit Guard(sfntt_ctx* c) : ctx(c), lk(c->mu) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != ctx->device) cudaSetDevice(ctx->device);
  }
  ~Guard() {
    if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
  }
};

int done(sfntt_ctx* ctx, const Status& s) {
  ctx->last_error = s.ok() ? std::string() : s.msg;
  return s.code;
}

}  // namespace

extern "C" {

int sfntt_batch_prepare(sfntt_ctx* ctx, const sfntt_lde_item* items, size_t count) {
  if (!ctx || (count && !items)) return SFNTT_INVALID_ARGUMENT;
  Guard g(ctx);
  for (size_t i = 0; i < count; ++i) {
    Status s = sfntt::prepare_item(ctx, items[i], ctx->stream);
    if (!s.ok()) return done(ctx, s);
  }
  return done(ctx, {});
}

int sfntt_batch_run(sfntt_ctx* ctx, const sfntt_lde_item* items, size_t count, void* stream) {
  if (!ctx || (count && !items)) return SFNTT_INVALID_ARGUMENT;
  Guard g(ctx);
  for (size_t i = 0; i < count; ++i) {
    Status s = sfntt::run_item(ctx, items[i], static_cast<cudaStream_t>(stream));
    if (!s.ok()) return done(ctx, s);
  }
  return done(ctx, {});
}

int sfntt_batch_graph_create(sfntt_ctx* ctx, const sfntt_lde_item* items, size_t count, int lanes, sfntt_graph** out) {
  if (!ctx || !out || (count && !items)) return SFNTT_INVALID_ARGUMENT;
  Guard g(ctx);
  *out = nullptr;
  if (lanes < 1) lanes = 1;
  if (lanes > 32) lanes = 32;
  std::vector<cudaStream_t> lane(lanes, nullptr);
  std::vector<cudaEvent_t> join(lanes, nullptr);
  cudaEvent_t fork = nullptr;
  cudaStream_t origin = nullptr;
  auto* gr = new sfntt_graph();
  gr->device = ctx->device;
  auto build = [&]() -> Status {
    for (size_t i = 0; i < count; ++i) SFNTT_TRY(sfntt::prepare_item(ctx, items[i], ctx->stream));
    SFNTT_CU(cudaStreamSynchronize(ctx->stream));
    SFNTT_CU(cudaStreamCreateWithFlags(&origin, cudaStreamNonBlocking));
    SFNTT_CU(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    for (int l = 0; l < lanes; ++l) {
      SFNTT_CU(cudaStreamCreateWithFlags(&lane[l], cudaStreamNonBlocking));
      SFNTT_CU(cudaEventCreateWithFlags(&join[l], cudaEventDisableTiming));
    }
    const uint64_t k0 = ctx->launches.load();
    SFNTT_CU(cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal));
    Status st;
    st = [&]() -> Status {
      SFNTT_CU(cudaEventRecord(fork, origin));
      for (int l = 0; l < lanes; ++l) SFNTT_CU(cudaStreamWaitEvent(lane[l], fork, 0));
      // largest items first, each to the lane with the least work so far
      std::vector<size_t> order(count);
      for (size_t i = 0; i < count; ++i) order[i] = i;
      auto work = [&](size_t i) {
        return (double)items[i].batch * (double)(1ull << items[i].log_n) * (1.0 + (double)(1u << items[i].added_bits));
      };
      std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return work(a) > work(b); });
      std::vector<double> load(lanes, 0.0);
      for (size_t i : order) {
        int best = 0;
        for (int l = 1; l < lanes; ++l)
          if (load[l] < load[best]) best = l;
        load[best] += work(i);
        SFNTT_TRY(sfntt::run_item(ctx, items[i], lane[best]));
      }
      for (int l = 0; l < lanes; ++l) {
        SFNTT_CU(cudaEventRecord(join[l], lane[l]));
        SFNTT_CU(cudaStreamWaitEvent(origin, join[l], 0));
      }
      return {};
    }();
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(origin, &graph);
    if (!st.ok()) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    SFNTT_CU(e);
    gr->graph = graph;
    gr->kernels = ctx->launches.load() - k0;
    SFNTT_CU(cudaGraphInstantiate(&gr->exec, graph, 0));
    return {};
  };
  Status s = build();
  for (int l = 0; l < lanes; ++l) {
    if (lane[l]) cudaStreamDestroy(lane[l]);
    if (join[l]) cudaEventDestroy(join[l]);
  }
  if (fork) cudaEventDestroy(fork);
  if (origin) cudaStreamDestroy(origin);
  if (!s.ok()) {
    sfntt_graph_destroy(gr);
    cudaGetLastError();
    return done(ctx, s);
  }
  *out = gr;
  return done(ctx, {});
}

int sfntt_batch_persistent_create(sfntt_ctx* ctx, const sfntt_lde_item* items, size_t count, int lanes,
                                  sfntt_graph** out) {
  if (!ctx || !out || (count && !items)) return SFNTT_INVALID_ARGUMENT;
  Guard g(ctx);
  *out = nullptr;
  if (lanes < 1) lanes = 1;
  if (lanes > 32) lanes = 32;
  std::vector<cudaStream_t> lane(lanes + 1, nullptr);  // lane[0]: the persistent phases
  std::vector<cudaEvent_t> join(lanes + 1, nullptr);
  cudaEvent_t fork = nullptr;
  cudaStream_t origin = nullptr;
  auto* gr = new sfntt_graph();
  gr->device = ctx->device;
  auto build = [&]() -> Status {
    for (size_t i = 0; i < count; ++i) SFNTT_TRY(sfntt::prepare_item(ctx, items[i], ctx->stream));
    SFNTT_CU(cudaStreamSynchronize(ctx->stream));
    // the work lists of the three phases (tables are final: every item is prepared)
    sfntt::WorkPhase ph[sfntt::kWorkPhases];
    std::vector<size_t> rest;
    for (size_t i = 0; i < count; ++i) {
      if (!sfntt::worklist_eligible(ctx, items[i])) {
        rest.push_back(i);
        continue;
      }
      for (int p = 0; p < sfntt::kWorkPhases; ++p) SFNTT_TRY(sfntt::worklist_add(ctx, ph[p], p, items[i], ctx->stream));
    }
    // one device block: counters, then per phase its items (128-byte aligned) and units
    size_t off = 256, item_off[sfntt::kWorkPhases], unit_off[sfntt::kWorkPhases];
    for (int p = 0; p < sfntt::kWorkPhases; ++p) {
      item_off[p] = off;
      off += (ph[p].items.size() * sizeof(sfntt::WorkItem) + 255) & ~size_t(255);
      unit_off[p] = off;
      off += (ph[p].units.size() * sizeof(sfntt::WorkUnit) + 255) & ~size_t(255);
    }
    SFNTT_CU(cudaMalloc(&gr->work, off));
    uint8_t* base = static_cast<uint8_t*>(gr->work);
    SFNTT_CU(cudaMemset(base, 0, 256));
    for (int p = 0; p < sfntt::kWorkPhases; ++p) {
      if (!ph[p].items.empty())
        SFNTT_CU(cudaMemcpy(base + item_off[p], ph[p].items.data(), ph[p].items.size() * sizeof(sfntt::WorkItem),
                            cudaMemcpyHostToDevice));
      if (!ph[p].units.empty())
        SFNTT_CU(cudaMemcpy(base + unit_off[p], ph[p].units.data(), ph[p].units.size() * sizeof(sfntt::WorkUnit),
                            cudaMemcpyHostToDevice));
    }
    uint32_t* counters = reinterpret_cast<uint32_t*>(base);
    SFNTT_CU(cudaStreamCreateWithFlags(&origin, cudaStreamNonBlocking));
    SFNTT_CU(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    for (int l = 0; l <= lanes; ++l) {
      SFNTT_CU(cudaStreamCreateWithFlags(&lane[l], cudaStreamNonBlocking));
      SFNTT_CU(cudaEventCreateWithFlags(&join[l], cudaEventDisableTiming));
    }
    const uint64_t k0 = ctx->launches.load();
    SFNTT_CU(cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal));
    Status st = [&]() -> Status {
      SFNTT_CU(cudaEventRecord(fork, origin));
      for (int l = 0; l <= lanes; ++l) SFNTT_CU(cudaStreamWaitEvent(lane[l], fork, 0));
      // lane 0: the three persistent phases, each one launch over every eligible item
      SFNTT_CU(cudaMemsetAsync(counters, 0, sfntt::kWorkPhases * sizeof(uint32_t), lane[0]));
      for (int p = 0; p < sfntt::kWorkPhases; ++p)
        SFNTT_TRY(sfntt::worklist_launch(ctx, p, ph[p], reinterpret_cast<const sfntt::WorkItem*>(base + item_off[p]),
                                         reinterpret_cast<const sfntt::WorkUnit*>(base + unit_off[p]), counters + p,
                                         lane[0]));
      // the other items: per-item launches, largest first to the least-loaded lane
      auto work = [&](size_t i) {
        return (double)items[i].batch * (double)(1ull << items[i].log_n) * (1.0 + (double)(1u << items[i].added_bits));
      };
      std::stable_sort(rest.begin(), rest.end(), [&](size_t a, size_t b) { return work(a) > work(b); });
      std::vector<double> load(lanes, 0.0);
      for (size_t i : rest) {
        int best = 0;
        for (int l = 1; l < lanes; ++l)
          if (load[l] < load[best]) best = l;
        load[best] += work(i);
        SFNTT_TRY(sfntt::run_item(ctx, items[i], lane[1 + best]));
      }
      for (int l = 0; l <= lanes; ++l) {
        SFNTT_CU(cudaEventRecord(join[l], lane[l]));
        SFNTT_CU(cudaStreamWaitEvent(origin, join[l], 0));
      }
      return {};
    }();
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(origin, &graph);
    if (!st.ok()) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    SFNTT_CU(e);
    gr->graph = graph;
    gr->kernels = ctx->launches.load() - k0;
    SFNTT_CU(cudaGraphInstantiate(&gr->exec, graph, 0));
    return {};
  };
  Status s = build();
  for (int l = 0; l <= lanes; ++l) {
    if (lane[l]) cudaStreamDestroy(lane[l]);
    if (join[l]) cudaEventDestroy(join[l]);
  }
  if (fork) cudaEventDestroy(fork);
  if (origin) cudaStreamDestroy(origin);
  if (!s.ok()) {
    sfntt_graph_destroy(gr);
    cudaGetLastError();
    return done(ctx, s);
  }
  *out = gr;
  return done(ctx, {});
}

int sfntt_graph_launch(sfntt_graph* g, void* stream) {
  if (!g || !g->exec) return SFNTT_INVALID_ARGUMENT;
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != g->device) cudaSetDevice(g->device);
  cudaError_t e = cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream));
  if (prev >= 0 && prev != g->device) cudaSetDevice(prev);
  return e == cudaSuccess ? SFNTT_OK : sfntt::map_cuda_error(e);
}

uint64_t sfntt_graph_kernel_count(const sfntt_graph* g) { return g ? g->kernels : 0; }

void sfntt_graph_destroy(sfntt_graph* g) {
  if (!g) return;
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != g->device) cudaSetDevice(g->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->work) cudaFree(g->work);
  if (prev >= 0 && prev != g->device) cudaSetDevice(prev);
  delete g;
}

int sfntt_autotune(sfntt_ctx* ctx, const sfntt_lde_item* items, size_t count, int reps) {
  if (!ctx || (count && !items)) return SFNTT_INVALID_ARGUMENT;
  Guard g(ctx);
  if (reps < 1) reps = 1;
  auto tune = [&]() -> Status {
    std::map<std::string, size_t> first;
    for (size_t i = 0; i < count; ++i) first.emplace(sfntt::key_of(items[i]), i);
    cudaStream_t s = ctx->stream;
    for (auto& kv : first) {
      if (ctx->tuned.count(kv.first)) continue;
      sfntt_lde_item it = items[kv.second];
      SFNTT_TRY(sfntt::prepare_item(ctx, it, s));
      float best_ms = 1e30f;
      int best = SFNTT_PLAN_TMA;
      std::vector<int> plans;
      for (int e : {(int)SFNTT_PLAN_TMA, (int)SFNTT_PLAN_TMA_FOUR_STEP}) {
        if (it.field == SFNTT_M31 && e == SFNTT_PLAN_TMA_FOUR_STEP) continue;  // M31 has no four-step form
        for (int split : {0, (int)SFNTT_PLAN_SPLIT12}) {
          // the split changes nothing unless a layer range exceeds 12 layers
          if (split && it.log_n + it.added_bits < 21) continue;
          for (int one : {0, (int)SFNTT_PLAN_ONE_CTA}) plans.push_back(e | split | one);
        }
      }
      plans.push_back(SFNTT_PLAN_TILE);
      for (int p : plans) {
        it.plan = p;
        SFNTT_TRY(sfntt::run_item(ctx, it, s));  // warm
        SFNTT_CU(cudaEventRecord(ctx->ev_start, s));
        for (int r = 0; r < reps; ++r) SFNTT_TRY(sfntt::run_item(ctx, it, s));
        SFNTT_CU(cudaEventRecord(ctx->ev_stop, s));
        SFNTT_CU(cudaEventSynchronize(ctx->ev_stop));
        float ms = 0.f;
        SFNTT_CU(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
        if (ms < best_ms) {
          best_ms = ms;
          best = p;
        }
      }
      ctx->tuned[kv.first] = best;
    }
    return {};
  };
  return done(ctx, tune());
}

int sfntt_tune_save(sfntt_ctx* ctx, const char* path) {
  if (!ctx || !path) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  std::ofstream f(path);
  if (!f) return done(ctx, {SFNTT_INVALID_ARGUMENT, std::string("cannot write ") + path});
  f << "# sfntt autotune table: field/log_n/columns(pow2)/added_bits plan\n";
  for (auto& kv : ctx->tuned) f << kv.first << " " << kv.second << "\n";
  return done(ctx, {});
}

int sfntt_tune_load(sfntt_ctx* ctx, const char* path) {
  if (!ctx || !path) return SFNTT_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  std::ifstream f(path);
  if (!f) return done(ctx, {SFNTT_INVALID_ARGUMENT, std::string("cannot read ") + path});
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream is(line);
    std::string key;
    int plan = 0;
    if (is >> key >> plan && plan != SFNTT_PLAN_AUTO && sfntt::valid_plan(plan)) ctx->tuned[key] = plan;
  }
  return done(ctx, {});
}

int sfntt_tune_lookup(sfntt_ctx* ctx, const sfntt_lde_item* item) {
  if (!ctx || !item) return -1;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  auto f = ctx->tuned.find(sfntt::key_of(*item));
  return f == ctx->tuned.end() ? 0 : f->second;
}

}  // extern "C"
