// field.cuh -- exact 32-bit modular arithmetic for BabyBear, KoalaBear and M31 on sm_100a.
//
// Value conventions follow the reference:
//   BabyBear (p = 2^31 - 2^27 + 1) elements are Montgomery u32 in [0, p)
//     (src/field/babybear.rs:14-65; R = 2^32, REDC with MONTY_CONST = -p^-1).
//   KoalaBear (p = 2^31 - 2^24 + 1; listed as planned in the reference's
//     README.md:20) uses the same Montgomery form and REDC with its own
//     constants; every BabyBear kernel is a template over the two.
//   M31 (p = 2^31 - 1) elements are canonical u32 in [0, p)
//     (src/field/m31.rs:18-67; Mersenne fold (v >> 31) + (v & p)).
//
// Multiplication by a *constant* (twiddles, shift powers, n^-1) uses Shoup's
// precomputed quotient: for w < p and ws = floor(w * 2^32 / p),
//     q = mulhi(x, ws);  r = x*w - q*p  (mod 2^32)   is in [0, 2p) for x < 2^32.
// For BabyBear the constant w is the *canonical* value of the Montgomery-form
// twiddle W (w = W * R^-1), so  x * w  ==  montmul(x, W)  bit for bit: the
// Montgomery representation of the product is unchanged.  All three primes are
// below 2^31, so [0, 2p) fits a u32 and one conditional subtract (written as
// an unsigned min) returns to [0, p).  Variable x variable products use the
// reference's reductions: Montgomery REDC (BabyBear) and the Mersenne fold.
#pragma once
#include <cstdint>

#include "../../include/sfntt.h"

namespace sfntt {

struct BabyBear {
  static constexpr uint32_t P = 0x78000001u;
  static constexpr uint32_t MONTY_CONST = 0x77FFFFFFu;  // -p^-1 mod 2^32
  static constexpr uint32_t R2 = 1172168163u;           // R^2 mod p
  static constexpr uint32_t ONE = 0x0FFFFFFEu;          // R mod p
  static constexpr bool kMontgomery = true;
  static constexpr const char* kTag = "bb";
  static constexpr int kId = SFNTT_BABYBEAR;
};

struct KoalaBear {
  static constexpr uint32_t P = 0x7F000001u;
  static constexpr uint32_t MONTY_CONST = 0x7EFFFFFFu;  // -p^-1 mod 2^32
  static constexpr uint32_t R2 = 402124772u;            // R^2 mod p
  static constexpr uint32_t ONE = 0x01FFFFFEu;          // R mod p
  static constexpr bool kMontgomery = true;
  static constexpr const char* kTag = "kb";
  static constexpr int kId = SFNTT_KOALABEAR;
};

struct M31 {
  static constexpr uint32_t P = 0x7FFFFFFFu;
  static constexpr uint32_t ONE = 1u;
  static constexpr bool kMontgomery = false;
  static constexpr const char* kTag = "m31";
  static constexpr int kId = SFNTT_M31;
};

// Host-side dispatch from a runtime field id (sfntt_field) to its type:
// fn(BabyBear{}), fn(KoalaBear{}) or fn(M31{}).
template <class Fn>
inline decltype(auto) with_field(int field, Fn&& fn) {
  if (field == SFNTT_KOALABEAR) return fn(KoalaBear{});
  if (field == SFNTT_BABYBEAR) return fn(BabyBear{});
  return fn(M31{});
}
// The same over the Montgomery-form fields only (BabyBear unless KoalaBear).
template <class Fn>
inline decltype(auto) with_monty(int field, Fn&& fn) {
  if (field == SFNTT_KOALABEAR) return fn(KoalaBear{});
  return fn(BabyBear{});
}

// x in [0, 2p) -> [0, p)
template <class F>
__device__ __forceinline__ uint32_t reduce2p(uint32_t x) {
  return min(x, x - F::P);
}

// a, b in [0, p) -> (a + b) mod p
template <class F>
__device__ __forceinline__ uint32_t add_mod(uint32_t a, uint32_t b) {
  uint32_t s = a + b;
  return min(s, s - F::P);
}

// a, b in [0, p) -> (a - b) mod p
template <class F>
__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b) {
  uint32_t d = a - b;
  return min(d, d + F::P);
}

// x < 2^32, (w, ws) a Shoup pair -> x*w mod p in [0, 2p)
template <class F>
__device__ __forceinline__ uint32_t mul_shoup_lazy(uint32_t x, uint32_t w, uint32_t ws) {
  uint32_t q = __umulhi(x, ws);
  return x * w - q * F::P;
}

template <class F>
__device__ __forceinline__ uint32_t mul_shoup(uint32_t x, uint32_t w, uint32_t ws) {
  return reduce2p<F>(mul_shoup_lazy<F>(x, w, ws));
}

// Montgomery REDC of t = a*b (src/field/babybear.rs:41-51), for any odd
// p < 2^31 with R = 2^32:
//   m = t_lo * (-p^-1);  (t + m p) >> 32  = hi(t) + hi(m p) + carry(t_lo != 0)
// (t_lo + lo(m p) is 0 mod 2^32, so it carries exactly when t_lo != 0); the
// sum is below 2p.
template <class F>
__device__ __forceinline__ uint32_t monty_mul(uint32_t a, uint32_t b) {
  uint32_t lo = a * b;
  uint32_t hi = __umulhi(a, b);
  uint32_t m = lo * F::MONTY_CONST;
  uint32_t r = hi + __umulhi(m, F::P) + (lo != 0u ? 1u : 0u);
  return min(r, r - F::P);
}

// Variable x variable product in the field's own representation.
__device__ __forceinline__ uint32_t mul_var(BabyBear, uint32_t a, uint32_t b) { return monty_mul<BabyBear>(a, b); }
__device__ __forceinline__ uint32_t mul_var(KoalaBear, uint32_t a, uint32_t b) { return monty_mul<KoalaBear>(a, b); }

__device__ __forceinline__ uint32_t mul_var(M31, uint32_t a, uint32_t b) {
  // Mersenne fold (src/field/m31.rs:54-67): t = (t >> 31) + (t & p)
  uint64_t t = (uint64_t)a * b;
  uint32_t s = (uint32_t)(t & 0x7FFFFFFFu) + (uint32_t)(t >> 31);
  return min(s, s - M31::P);
}

template <class F>
__device__ __forceinline__ uint32_t mul_var(uint32_t a, uint32_t b) {
  return mul_var(F{}, a, b);
}

template <class F>
__device__ __forceinline__ uint32_t pow_var(uint32_t base, uint32_t e) {
  uint32_t r = F::ONE;
  while (e) {
    if (e & 1u) r = mul_var<F>(r, base);
    base = mul_var<F>(base, base);
    e >>= 1;
  }
  return r;
}

// Canonical value of a field element in the field's representation
// (BabyBear, KoalaBear: REDC(x * 1); M31: identity).
__device__ __forceinline__ uint32_t to_canonical(BabyBear, uint32_t x) { return monty_mul<BabyBear>(x, 1u); }
__device__ __forceinline__ uint32_t to_canonical(KoalaBear, uint32_t x) { return monty_mul<KoalaBear>(x, 1u); }
__device__ __forceinline__ uint32_t to_canonical(M31, uint32_t x) { return x; }

// Shoup quotient floor(w * 2^32 / p) for a canonical w < p.
template <class F>
__device__ __forceinline__ uint32_t shoup_of(uint32_t w) {
  return (uint32_t)(((uint64_t)w << 32) / F::P);
}

}  // namespace sfntt
