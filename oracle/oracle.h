/*
 * oracle.h -- CPU restatement of the reference's NTT / coset-LDE path.
 *
 * TEST INFRASTRUCTURE ONLY.  This code is the parity checker for the CUDA
 * library (tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference legs are its only users).  It is never linked into, called by or
 * shipped with the product library.
 *
 * It restates, in plain C, the pure-Rust CPU modules of
 * moven0831/small-field-metal-ntt (a Rust crate that cannot be compiled here:
 * no cargo/rustc in the image and it needs the macOS `metal` crate):
 *
 *   src/field/m31.rs:18-94            M31 (p = 2^31-1), canonical form
 *   src/field/babybear.rs:14-172      BabyBear (p = 2^31-2^27+1), Montgomery form
 *   src/field/circle.rs:10-151        circle group over M31, cosets
 *   src/ntt/m31/twiddles.rs:19-79     Circle-NTT twiddles (x / y coordinates)
 *   src/ntt/babybear/twiddles.rs:13-19 + babybear.rs:83-97  BabyBear twiddles
 *   src/ntt/m31/cpu_reference.rs:50-153       DCCT forward / inverse
 *   src/ntt/babybear/cpu_reference.rs:34-103  GS-DIF forward / CT-DIT inverse
 *   src/lde/mod.rs:116-176            coset_lde_batch_cpu
 *
 * KoalaBear (p = 2^31 - 2^24 + 1) is listed as planned in the reference's
 * README.md:20 and not implemented there: the orc_kb_* functions run the
 * BabyBear code above over KoalaBear's constants (generator 3, primitive
 * 2^24-th root 3^((p-1)/2^24)).  They are pinned by the same code path's
 * BabyBear golden vectors and by a direct O(n^2) DFT in the tests, not by
 * any reference output.
 *
 * Every function keeps the reference's loop structure (layer -> block -> j)
 * so that it can also serve as the timed CPU baseline.
 */
#ifndef SFNTT_ORACLE_H
#define SFNTT_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_BB_P 2013265921u          /* 0x78000001 */
#define ORC_M31_P 2147483647u         /* 2^31 - 1   */
#define ORC_KB_P 2130706433u          /* 0x7F000001: KoalaBear, 2^31 - 2^24 + 1 */

/* ---- BabyBear field (src/field/babybear.rs) ---------------------------- */
uint32_t orc_bb_monty_reduce(uint64_t t);        /* babybear.rs:41-51 */
uint32_t orc_bb_to_monty(uint32_t v);            /* babybear.rs:54-59 */
uint32_t orc_bb_from_monty(uint32_t m);          /* babybear.rs:62-65 */
uint32_t orc_bb_add(uint32_t a, uint32_t b);     /* babybear.rs:113-121 */
uint32_t orc_bb_sub(uint32_t a, uint32_t b);     /* babybear.rs:124-130 */
uint32_t orc_bb_mul(uint32_t a, uint32_t b);     /* babybear.rs:133-137 */
uint32_t orc_bb_reduce(uint64_t v);              /* babybear.rs:140-145 */
uint32_t orc_bb_inv(uint32_t a);                 /* babybear.rs:147-161 */
uint32_t orc_bb_two_adic_generator(uint32_t log_n); /* babybear.rs:69-76 */

/* ---- M31 field (src/field/m31.rs) -------------------------------------- */
uint32_t orc_m31_reduce(uint64_t v);             /* m31.rs:54-67 */
uint32_t orc_m31_add(uint32_t a, uint32_t b);    /* m31.rs:32-35 */
uint32_t orc_m31_sub(uint32_t a, uint32_t b);    /* m31.rs:38-45 */
uint32_t orc_m31_mul(uint32_t a, uint32_t b);    /* m31.rs:48-51 */
uint32_t orc_m31_inv(uint32_t a);                /* m31.rs:69-83 */

/* ---- Circle group (src/field/circle.rs) -------------------------------- */
typedef struct { uint32_t x, y; } orc_cpoint;
orc_cpoint orc_circle_add(orc_cpoint a, orc_cpoint b);       /* circle.rs:34-40 */
orc_cpoint orc_circle_double(orc_cpoint a);                  /* circle.rs:53-60 */
orc_cpoint orc_circle_mul_scalar(orc_cpoint a, uint32_t n);  /* circle.rs:63-74 */
orc_cpoint orc_circle_subgroup_gen(uint32_t log_size);       /* circle.rs:78-85 */

/* ---- Twiddle tables ----------------------------------------------------
 * Layers are concatenated: BabyBear layer s (2^s entries) starts at 2^s - 1;
 * M31 layer l (n / 2^(l+1) entries) starts at n - n / 2^l.  Both total n - 1.
 */
void orc_bb_twiddles(uint32_t log_n, int inverse, uint32_t *out);  /* Montgomery form */
void orc_m31_twiddles(uint32_t log_n, int inverse, uint32_t *out);

/* ---- NTTs (in place; return 0, or 1 = InvalidSize) ---------------------- */
int orc_bb_forward(uint32_t *data, size_t n);     /* cpu_reference.rs:34-62 */
int orc_bb_inverse(uint32_t *data, size_t n);     /* cpu_reference.rs:69-103 */
int orc_m31_forward(uint32_t *data, size_t n);    /* m31/cpu_reference.rs:50-79 */
int orc_m31_inverse(uint32_t *data, size_t n);    /* m31/cpu_reference.rs:82-120 */

/* ---- Coset LDE (src/lde/mod.rs:127-176) ---------------------------------
 * in: batch columns of n = 2^log_n Montgomery u32 (SoA, in[col*n+row]).
 * out: batch columns of 2^(log_n+added_bits).  shift_monty = 0 selects the
 * reference default shift two_adic_generator(log_n + added_bits + 1).
 * threads > 1 runs columns in parallel (OpenMP); the arithmetic is the same.
 */
int orc_bb_coset_lde(const uint32_t *in, uint32_t *out, uint32_t log_n,
                     uint32_t batch, uint32_t added_bits, uint32_t shift_monty,
                     int threads);

/* M31 "LDE" used by the mixed-field batch / serving configurations: the
 * reference has no M31 LDE, so it is defined as the composition of reference
 * functions inverse(odds(log_n)) -> zero-pad -> forward(odds(log_n+added)). */
int orc_m31_lde(const uint32_t *in, uint32_t *out, uint32_t log_n,
                uint32_t batch, uint32_t added_bits, int threads);

/* Column-parallel batched NTTs (used for the all-cores CPU baseline). */
int orc_bb_forward_batch(uint32_t *data, uint32_t log_n, uint32_t batch, int threads);
int orc_bb_inverse_batch(uint32_t *data, uint32_t log_n, uint32_t batch, int threads);

/* ---- KoalaBear (same algorithms and conventions as BabyBear) ----------- */
uint32_t orc_kb_to_monty(uint32_t v);
uint32_t orc_kb_from_monty(uint32_t m);
uint32_t orc_kb_mul(uint32_t a, uint32_t b);
uint32_t orc_kb_two_adic_generator(uint32_t log_n);  /* Montgomery form */
void orc_kb_twiddles(uint32_t log_n, int inverse, uint32_t *out);
int orc_kb_forward(uint32_t *data, size_t n);
int orc_kb_inverse(uint32_t *data, size_t n);
int orc_kb_forward_batch(uint32_t *data, uint32_t log_n, uint32_t batch, int threads);
int orc_kb_inverse_batch(uint32_t *data, uint32_t log_n, uint32_t batch, int threads);
int orc_kb_coset_lde(const uint32_t *in, uint32_t *out, uint32_t log_n,
                     uint32_t batch, uint32_t added_bits, uint32_t shift_monty,
                     int threads);

/* ---- Canonic-coset circle FFT and circle LDE (Stwo-style; not in the
 * reference).  Domain odds(log_n) ordered half coset then conjugates, values
 * bit-reversed, coefficient r on the basis y^{r_0} x^{r_1} pi(x)^{r_2} ...;
 * the reference's M31 network with twiddles T_0[b] = y(h_{rev(b)}),
 * T_L[b] = x(2^{L-1} h_{rev(b)}).  Layout of the twiddles as orc_m31_twiddles. */
void orc_circle_twiddles(uint32_t log_n, int inverse, uint32_t *out);
int orc_circle_ntt(uint32_t *data, uint32_t log_n, uint32_t batch, int inverse);
int orc_circle_lde(const uint32_t *in, uint32_t *out, uint32_t log_n, uint32_t batch,
                   uint32_t added_bits, int threads);

/* ---- CM31 = M31[i]/(i^2+1): interleaved (re, im) pairs (not in the
 * reference; TODOS.md:27-31 plans it).  orc_cm31_ntt transforms `batch`
 * columns of 2^log_n pairs in place with the M31 NTT on each coordinate. */
void orc_cm31_mul(const uint32_t *a, const uint32_t *b, uint32_t *out, size_t n);
int orc_cm31_ntt(uint32_t *pairs, uint32_t log_n, uint32_t batch, int inverse);

/* Reference data generator (src/ntt/test_utils.rs:38-46, benches seeds):
 * s = s*6364136223846793005 + 1; v = (s >> 33) % p.  BabyBear to_monty
 * applied when monty == 1, KoalaBear's when monty == 2.  Returns the final
 * state. */
uint64_t orc_lcg_fill(uint32_t *out, size_t n, uint64_t seed, uint32_t p, int monty);

#ifdef __cplusplus
}
#endif
#endif
