// host_field.hpp -- host-side field constants used to parameterise device
// kernels (generators, inverses, circle points).  Canonical-form arithmetic
// with 64-bit products; only a few hundred operations per call.
#pragma once
#include <cstdint>

#include "../../include/sfntt.h"

namespace sfntt {
namespace host {

constexpr uint32_t BB_P = 0x78000001u;
constexpr uint32_t M31_P = 0x7FFFFFFFu;
constexpr uint32_t BB_TWO_ADICITY = 27;
constexpr uint32_t BB_ROOT = 440564289u;  // primitive 2^27-th root (src/field/babybear.rs:35-37)

inline uint32_t mulmod(uint32_t a, uint32_t b, uint32_t p) { return (uint32_t)((uint64_t)a * b % p); }
inline uint32_t addmod(uint32_t a, uint32_t b, uint32_t p) { uint64_t s = (uint64_t)a + b; return (uint32_t)(s >= p ? s - p : s); }
inline uint32_t submod(uint32_t a, uint32_t b, uint32_t p) { return a >= b ? a - b : p - (b - a); }

inline uint32_t powmod(uint32_t b, uint64_t e, uint32_t p) {
  uint32_t r = 1 % p;
  while (e) {
    if (e & 1) r = mulmod(r, b, p);
    b = mulmod(b, b, p);
    e >>= 1;
  }
  return r;
}
inline uint32_t invmod(uint32_t a, uint32_t p) { return powmod(a, (uint64_t)p - 2, p); }

// BabyBear Montgomery form (R = 2^32): W = w * 2^32 mod p and back.
inline uint32_t bb_to_monty(uint32_t w) { return (uint32_t)(((uint64_t)w << 32) % BB_P); }
inline uint32_t bb_from_monty(uint32_t W) { return mulmod(W, invmod((uint32_t)((1ull << 32) % BB_P), BB_P), BB_P); }

// Canonical two_adic_generator(k) (src/field/babybear.rs:69-76).
inline uint32_t bb_two_adic_generator(uint32_t k) { return powmod(BB_ROOT, 1ull << (BB_TWO_ADICITY - k), BB_P); }

// KoalaBear, p = 2^31 - 2^24 + 1 (planned in the reference, README.md:20):
// p - 1 = 2^24 * 127, smallest multiplicative generator 3, and the primitive
// 2^24-th root 3^((p-1)/2^24) -- the same construction as BabyBear's root,
// which is 31^((p-1)/2^27) for its generator 31.
constexpr uint32_t KB_P = 0x7F000001u;
constexpr uint32_t KB_TWO_ADICITY = 24;
constexpr uint32_t KB_ROOT = 1791270792u;

// The two Montgomery-form (R = 2^32) two-adic fields behind one descriptor.
struct MontyField {
  uint32_t p;
  uint32_t two_adicity;
  uint32_t root;       // canonical primitive 2^two_adicity-th root of unity
  uint32_t generator;  // multiplicative generator (the Plonky3-style coset shift)
  const char* name;
};
constexpr MontyField kBabyBear{BB_P, BB_TWO_ADICITY, BB_ROOT, 31u, "BabyBear"};
constexpr MontyField kKoalaBear{KB_P, KB_TWO_ADICITY, KB_ROOT, 3u, "KoalaBear"};
inline const MontyField& monty_field(int field) { return field == SFNTT_KOALABEAR ? kKoalaBear : kBabyBear; }

inline uint32_t field_p(int field) { return field == SFNTT_M31 ? M31_P : monty_field(field).p; }

inline uint32_t to_monty(const MontyField& f, uint32_t w) { return (uint32_t)(((uint64_t)w << 32) % f.p); }
inline uint32_t from_monty(const MontyField& f, uint32_t W) {
  return mulmod(W, invmod((uint32_t)((1ull << 32) % f.p), f.p), f.p);
}
inline uint32_t two_adic_generator(const MontyField& f, uint32_t k) {
  return powmod(f.root, 1ull << (f.two_adicity - k), f.p);
}

inline uint32_t shoup(uint32_t w, uint32_t p) { return (uint32_t)(((uint64_t)w << 32) / p); }

// ---- circle group over M31 (src/field/circle.rs) ----
struct CPoint { uint32_t x, y; };
inline CPoint cadd(CPoint a, CPoint b) {
  return {submod(mulmod(a.x, b.x, M31_P), mulmod(a.y, b.y, M31_P), M31_P),
          addmod(mulmod(a.x, b.y, M31_P), mulmod(a.y, b.x, M31_P), M31_P)};
}
inline CPoint cdouble(CPoint a) {
  return {submod(mulmod(2, mulmod(a.x, a.x, M31_P), M31_P), 1, M31_P), mulmod(2, mulmod(a.x, a.y, M31_P), M31_P)};
}
// CIRCLE_GEN = (2, 1268011823) has order 2^31 (src/field/circle.rs:17-20).
inline CPoint subgroup_gen(uint32_t log_size) {
  CPoint p{2u, 1268011823u};
  for (uint32_t i = 0; i < 31 - log_size; ++i) p = cdouble(p);
  return p;
}

}  // namespace host
}  // namespace sfntt
