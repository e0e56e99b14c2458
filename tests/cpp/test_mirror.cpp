// Parity tests of the C++ host mirror (small-field-metal-ntt_b200/cpp/sfntt.hpp)
// against the oracle (oracle/oracle.h, the CPU restatement of the reference).
// Test infrastructure: links liboracle.so as the checker.
//
//   test_mirror --no-device   host-only checks (no GPU): the mirror compiles,
//                             links and maps a missing device to
//                             NttError::DeviceNotFound
//   test_mirror               parity on cuda:0 (every backend, LDE, server)
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <string>
#include <vector>

#include "../../oracle/oracle.h"
#include "../../small-field-metal-ntt_b200/cpp/sfntt.hpp"

namespace {

int g_checks = 0, g_fail = 0;

// the reference's type names resolve to the CUDA backends
static_assert(std::is_same_v<sfntt::BbMetalCtGsR4, sfntt::BbCudaCtGsR4>);
static_assert(std::is_same_v<sfntt::MetalStockhamR2, sfntt::CudaBackend<sfntt::M31, sfntt::Variant::StockhamR2>>);
static_assert(std::is_base_of_v<sfntt::NttBackend<sfntt::BabyBear>, sfntt::BbMetalR2>);

#define CHECK(cond, ...)                                      \
  do {                                                        \
    ++g_checks;                                               \
    if (!(cond)) {                                            \
      ++g_fail;                                               \
      std::fprintf(stderr, "FAIL %s:%d: ", __FILE__, __LINE__); \
      std::fprintf(stderr, __VA_ARGS__);                      \
      std::fprintf(stderr, "\n");                             \
    }                                                         \
  } while (0)

std::vector<uint32_t> lcg(size_t n, uint64_t seed, bool bb) {
  std::vector<uint32_t> v(n);
  orc_lcg_fill(v.data(), n, seed, bb ? ORC_BB_P : ORC_M31_P, bb ? 1 : 0);
  return v;
}

template <class F>
std::vector<F> as_field(const std::vector<uint32_t>& w) {
  std::vector<F> out(w.size());
  for (size_t i = 0; i < w.size(); ++i) out[i].v = w[i];
  return out;
}

template <class F>
bool same(const std::vector<F>& a, const std::vector<uint32_t>& b) {
  if (a.size() != b.size()) return false;
  for (size_t i = 0; i < a.size(); ++i)
    if (a[i].v != b[i]) return false;
  return true;
}

template <class F, sfntt::Variant V>
void check_backend(const sfntt::Context& ctx) {
  sfntt::CudaBackend<F, V> b(ctx);
  constexpr bool bb = F::kField == SFNTT_BABYBEAR;
  const std::string name(b.name());
  for (uint32_t log_n : {1u, 5u, 10u, 14u, 16u}) {  // 14, 16: cluster launches (V4)
    const size_t n = size_t(1) << log_n;
    auto x = lcg(n, 1000 + log_n, bb);
    auto ref = x;
    if (bb) orc_bb_forward(ref.data(), n);
    else orc_m31_forward(ref.data(), n);
    auto data = as_field<F>(x);
    b.forward_ntt(std::span<F>(data));
    CHECK(same(data, ref), "%s forward log_n %u", name.c_str(), log_n);
    auto [out, ns] = b.forward_ntt_gpu(x, log_n);
    CHECK(out == ref, "%s forward_ntt_gpu log_n %u", name.c_str(), log_n);
    if (V == sfntt::Variant::CtDitR2) {
      bool unsupported = false;
      try {
        b.inverse_ntt(std::span<F>(data));
      } catch (const sfntt::NttError& e) {
        unsupported = e.kind() == sfntt::NttError::Kind::Unsupported;
      }
      CHECK(unsupported, "%s inverse must be Unsupported (the reference panics)", name.c_str());
      continue;
    }
    b.inverse_ntt(std::span<F>(data));
    CHECK(same(data, x), "%s inverse(forward(x)) == x, log_n %u", name.c_str(), log_n);
    auto iref = x;
    if (bb) orc_bb_inverse(iref.data(), n);
    else orc_m31_inverse(iref.data(), n);
    auto [iout, ins] = b.inverse_ntt_gpu(x, log_n);
    CHECK(iout == iref, "%s inverse_ntt_gpu log_n %u", name.c_str(), log_n);
  }
  // InvalidSize carries the offending length (src/ntt/mod.rs:54)
  std::vector<F> bad(12);
  size_t got = 0;
  try {
    b.forward_ntt(std::span<F>(bad));
  } catch (const sfntt::NttError& e) {
    if (e.kind() == sfntt::NttError::Kind::InvalidSize) got = e.size();
  }
  CHECK(got == 12, "%s InvalidSize(12), got %zu", name.c_str(), got);
}

void check_pointwise_and_batch(const sfntt::Context& ctx) {
  sfntt::BbCudaCtGsR4 bb(ctx);
  const size_t n = 1 << 12;
  auto a = lcg(n, 7, true), b = lcg(n, 8, true);
  auto fa = as_field<sfntt::BabyBear>(a), fb = as_field<sfntt::BabyBear>(b);
  std::vector<sfntt::BabyBear> out(n);
  bb.pointwise_mul(fa, fb, out);
  bool ok = true;
  for (size_t i = 0; i < n; ++i) ok &= out[i].v == orc_bb_mul(a[i], b[i]);
  CHECK(ok, "BabyBear pointwise_mul");
  sfntt::CudaCtGsR4 m31(ctx);
  auto c = lcg(n, 9, false), d = lcg(n, 10, false);
  auto fc = as_field<sfntt::M31>(c), fd = as_field<sfntt::M31>(d);
  std::vector<sfntt::M31> mo(n);
  m31.pointwise_mul(fc, fd, mo);
  ok = true;
  for (size_t i = 0; i < n; ++i) ok &= mo[i].v == orc_m31_mul(c[i], d[i]);
  CHECK(ok, "M31 pointwise_mul");
  // BbBatchNtt::forward_ntt_batch_gpu (src/ntt/babybear/batch.rs:76-127)
  const uint32_t log_n = 11, batch = 5;
  auto x = lcg(size_t(batch) << log_n, 11, true);
  auto ref = x;
  orc_bb_forward_batch(ref.data(), log_n, batch, 1);
  sfntt::BbBatchNtt bn(ctx);
  auto [y, ns] = bn.forward_ntt_batch_gpu(x, log_n, batch);
  CHECK(y == ref, "BbBatchNtt forward_ntt_batch_gpu");
  auto [z, ns2] = bn.inverse_ntt_batch_gpu(y, log_n, batch);
  CHECK(z == x, "BbBatchNtt inverse(forward) batch");
}

void check_lde(const sfntt::Context& ctx) {
  struct Case { uint32_t log_n, batch, added; uint32_t shift; };
  for (const Case& c : {Case{10, 3, 1, 0}, Case{14, 2, 2, 0}, Case{13, 4, 1, orc_bb_to_monty(31)}, Case{6, 3, 5, 0}}) {
    auto x = lcg(size_t(c.batch) << c.log_n, 40 + c.log_n, true);
    std::vector<uint32_t> ref(size_t(c.batch) << (c.log_n + c.added));
    orc_bb_coset_lde(x.data(), ref.data(), c.log_n, c.batch, c.added, c.shift, 4);
    for (bool fused : {true, false}) {
      sfntt::CosetLdeBatch lde(ctx, fused);
      auto r = lde.execute(x, c.log_n, c.batch, c.added, c.shift);
      CHECK(r.data == ref, "CosetLdeBatch %s log_n %u batch %u added %u shift %u", fused ? "fused" : "unfused",
            c.log_n, c.batch, c.added, c.shift);
    }
  }
  auto m = lcg(size_t(3) << 12, 77, false);
  std::vector<uint32_t> mref(size_t(3) << 13);
  orc_m31_lde(m.data(), mref.data(), 12, 3, 1, 4);
  sfntt::M31Lde ml(ctx);
  CHECK(ml.execute(m, 12, 3, 1).data == mref, "M31Lde log_n 12 batch 3 added 1");
  // the reference's size check (src/lde/mod.rs:52-54)
  bool invalid = false;
  try {
    sfntt::CosetLdeBatch(ctx).execute(std::span<const uint32_t>(m.data(), 5), 10, 3, 1);
  } catch (const sfntt::NttError& e) {
    invalid = e.kind() == sfntt::NttError::Kind::InvalidSize && e.size() == 5;
  }
  CHECK(invalid, "CosetLdeBatch InvalidSize(input.len())");
}

std::vector<uint32_t> bitrev_cols(const std::vector<uint32_t>& x, uint32_t log_n, uint32_t batch) {
  std::vector<uint32_t> y(x.size());
  const size_t n = size_t(1) << log_n;
  for (size_t c = 0; c < batch; ++c)
    for (size_t r = 0; r < n; ++r) {
      size_t rr = 0;
      for (uint32_t b = 0; b < log_n; ++b) rr |= ((r >> b) & 1) << (log_n - 1 - b);
      y[c * n + rr] = x[c * n + r];
    }
  return y;
}

void check_layout(const sfntt::Context& ctx) {
  const uint32_t log_n = 11, batch = 5;
  const size_t n = size_t(1) << log_n;
  auto x = lcg(size_t(batch) << log_n, 61, false);
  auto [nat, ns] = sfntt::layout(ctx, x, log_n, batch, SFNTT_LAYOUT_NATURAL);
  CHECK(nat == bitrev_cols(x, log_n, batch), "layout natural");
  auto [rows, ns2] = sfntt::layout(ctx, x, log_n, batch, SFNTT_LAYOUT_ROW_MAJOR);
  bool ok = true;
  for (size_t c = 0; c < batch; ++c)
    for (size_t r = 0; r < n; ++r) ok &= rows[r * batch + c] == x[c * n + r];
  CHECK(ok, "layout row-major");
  // Plonky3 convention: natural-order input and output rows
  const uint32_t lb = 12, cols = 3, added = 1;
  auto xn = lcg(size_t(cols) << lb, 62, true);
  std::vector<uint32_t> ref(size_t(cols) << (lb + added));
  orc_bb_coset_lde(bitrev_cols(xn, lb, cols).data(), ref.data(), lb, cols, added, orc_bb_to_monty(31), 4);
  auto r = sfntt::CosetLdeBatch(ctx, true, true).execute(xn, lb, cols, added, orc_bb_to_monty(31));
  CHECK(r.data == bitrev_cols(ref, lb + added, cols), "CosetLdeBatch natural (Plonky3 convention)");
}

void check_server(const sfntt::Context& ctx) {
  // host requests of both fields and uneven sizes, admitted as slots and
  // arena space free up; each must equal the oracle (= the request alone)
  sfntt::Server srv(ctx, size_t(8) << 20, 3);
  struct Req { sfntt_lde_item it; std::vector<uint32_t> in, out, ref; uint64_t ticket = 0; };
  std::vector<Req> reqs;
  const uint32_t shapes[][4] = {{SFNTT_BABYBEAR, 12, 3, 1}, {SFNTT_M31, 11, 2, 2}, {SFNTT_BABYBEAR, 14, 2, 2},
                                {SFNTT_M31, 13, 4, 1}, {SFNTT_BABYBEAR, 9, 7, 0}, {SFNTT_BABYBEAR, 15, 1, 1}};
  for (size_t i = 0; i < sizeof shapes / sizeof shapes[0]; ++i) {
    Req r;
    r.it = sfntt::lde_item((int)shapes[i][0], shapes[i][1], shapes[i][2], shapes[i][3], nullptr, nullptr);
    const bool bb = r.it.field == SFNTT_BABYBEAR;
    r.in = lcg(size_t(r.it.batch) << r.it.log_n, 300 + i, bb);
    r.out.assign(size_t(r.it.batch) << (r.it.log_n + r.it.added_bits), 0);
    r.ref.assign(r.out.size(), 0);
    if (bb) orc_bb_coset_lde(r.in.data(), r.ref.data(), r.it.log_n, r.it.batch, r.it.added_bits, 0, 4);
    else orc_m31_lde(r.in.data(), r.ref.data(), r.it.log_n, r.it.batch, r.it.added_bits, 4);
    reqs.push_back(std::move(r));
  }
  for (auto& r : reqs) r.ticket = srv.submit_host(r.it, r.in, r.out);
  size_t done = 0;
  while (done < reqs.size())
    for (uint64_t t : srv.poll()) {
      srv.release(t);
      ++done;
    }
  CHECK(srv.pending() == 0, "server drained");
  for (size_t i = 0; i < reqs.size(); ++i) CHECK(reqs[i].out == reqs[i].ref, "served request %zu", i);
}

}  // namespace

// KoalaBear (no reference implementation): every variant and the coset LDE
// against the oracle's KoalaBear restatement.
void check_koalabear(const sfntt::Context& ctx) {
  for (uint32_t log_n : {5u, 13u, 17u}) {
    const size_t n = size_t(1) << log_n;
    std::vector<uint32_t> x(n);
    orc_lcg_fill(x.data(), n, 60 + log_n, ORC_KB_P, 2);
    std::vector<uint32_t> ref = x;
    orc_kb_forward(ref.data(), n);
    sfntt::KbCudaCtGsR4 kb(ctx);
    auto [y, ns] = kb.forward_ntt_gpu(x, log_n);
    CHECK(y == ref, "KbCudaCtGsR4 forward log_n %u", log_n);
    auto [z, ns2] = kb.inverse_ntt_gpu(y, log_n);
    CHECK(z == x, "KbCudaCtGsR4 inverse(forward) log_n %u", log_n);
    sfntt::KbCudaStockhamR2 st(ctx);
    CHECK(st.forward_ntt_gpu(x, log_n).first == ref, "KbCudaStockhamR2 forward log_n %u", log_n);
  }
  const uint32_t log_n = 14, batch = 3, added = 2;
  std::vector<uint32_t> x(size_t(batch) << log_n), ref(size_t(batch) << (log_n + added));
  orc_lcg_fill(x.data(), x.size(), 91, ORC_KB_P, 2);
  orc_kb_coset_lde(x.data(), ref.data(), log_n, batch, added, 0, 4);
  for (bool fused : {true, false})
    CHECK(sfntt::KbCosetLdeBatch(ctx, fused).execute(x, log_n, batch, added).data == ref,
          "KbCosetLdeBatch %s log_n 14 batch 3 added 2", fused ? "fused" : "unfused");
}

// Circle LDE and CM31 transforms (no reference counterpart) against the oracle.
void check_circle_and_cm31(const sfntt::Context& ctx) {
  const uint32_t log_n = 14, batch = 3, added = 1;
  std::vector<uint32_t> x(size_t(batch) << log_n), ref(size_t(batch) << (log_n + added));
  orc_lcg_fill(x.data(), x.size(), 5, ORC_M31_P, 0);
  orc_circle_lde(x.data(), ref.data(), log_n, batch, added, 4);
  sfntt::CircleLde circle(ctx);
  CHECK(circle.execute(x, log_n, batch, added).data == ref, "CircleLde log_n 14 batch 3 added 1");
  std::vector<uint32_t> ev = x;
  orc_circle_ntt(ev.data(), log_n, batch, 0);
  auto [got, ns] = circle.ntt(x, log_n, batch, false);
  CHECK(got == ev, "CircleLde::ntt evaluate");
  CHECK(circle.ntt(got, log_n, batch, true).first == x, "CircleLde::ntt interpolate(evaluate)");
  std::vector<uint32_t> p(2 * (size_t(batch) << 10));
  orc_lcg_fill(p.data(), p.size(), 6, ORC_M31_P, 0);
  std::vector<uint32_t> pref = p;
  orc_cm31_ntt(pref.data(), 10, batch, 0);
  sfntt::Cm31Ntt cm(ctx);
  auto [cf, ns2] = cm.ntt(p, 10, batch, false);
  CHECK(cf == pref, "Cm31Ntt forward log_n 10 batch 3");
  CHECK(cm.ntt(cf, 10, batch, true).first == p, "Cm31Ntt inverse(forward)");
}

int main(int argc, char** argv) {
  const bool no_device = argc > 1 && std::strcmp(argv[1], "--no-device") == 0;
  if (no_device) {
    bool not_found = false;
    try {
      sfntt::Context ctx(0);
    } catch (const sfntt::NttError& e) {
      not_found = e.kind() == sfntt::NttError::Kind::DeviceNotFound;
    }
    CHECK(not_found, "Context without a GPU must raise NttError::DeviceNotFound");
    // every status code maps to its NttError variant; InvalidSize keeps the length
    for (int st = SFNTT_INVALID_SIZE; st <= SFNTT_INVALID_ARGUMENT; ++st) {
      int kind = 0;
      size_t size = 0;
      try {
        sfntt::detail::check(nullptr, st, 7);
      } catch (const sfntt::NttError& e) {
        kind = (int)e.kind();
        size = e.size();
      }
      CHECK(kind == st && size == 7, "status %d -> NttError kind %d", st, kind);
    }
  } else {
    sfntt::Context ctx(0);
    std::printf("%s\n", ctx.device_info().c_str());
    check_backend<sfntt::M31, sfntt::Variant::CtDitR2>(ctx);
    check_backend<sfntt::M31, sfntt::Variant::CtGsR2>(ctx);
    check_backend<sfntt::M31, sfntt::Variant::StockhamR2>(ctx);
    check_backend<sfntt::M31, sfntt::Variant::CtGsR4>(ctx);
    check_backend<sfntt::BabyBear, sfntt::Variant::CtDitR2>(ctx);
    check_backend<sfntt::BabyBear, sfntt::Variant::CtGsR2>(ctx);
    check_backend<sfntt::BabyBear, sfntt::Variant::StockhamR2>(ctx);
    check_backend<sfntt::BabyBear, sfntt::Variant::CtGsR4>(ctx);
    check_pointwise_and_batch(ctx);
    check_lde(ctx);
    check_koalabear(ctx);
    check_circle_and_cm31(ctx);
    check_layout(ctx);
    check_server(ctx);
  }
  std::printf("%d checks, %d failed\n", g_checks, g_fail);
  return g_fail ? 1 : 0;
}
