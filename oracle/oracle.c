/*
 * oracle.c -- CPU restatement of the reference's NTT / coset-LDE path.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker and the timed CPU baseline.
 * The product library never links or calls this file.  Each function cites
 * the reference file:line it restates (paths inside the reference project).
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ================ Montgomery fields (src/field/babybear.rs) ============== */

/* BabyBear's arithmetic restated over a field descriptor, so that KoalaBear
 * (p = 2^31 - 2^24 + 1, listed as planned in the reference's README.md:20 and
 * not implemented there) runs the very code the BabyBear golden vectors pin,
 * with its own constants. */
typedef struct {
    uint32_t p, r2, monty_const, one, two_adicity, root_monty;
} mfield;

static const mfield MF_BB = {
    ORC_BB_P,
    1172168163u,  /* babybear.rs:25 R^2 mod p            */
    2013265919u,  /* babybear.rs:29 -p^-1 mod 2^32       */
    268435454u,   /* babybear.rs:22 R mod p (Montgomery 1) */
    27u,          /* babybear.rs:33                      */
    1476048622u,  /* babybear.rs:37 (440564289 canonical = 31^((p-1)/2^27)) */
};

/* KoalaBear: p - 1 = 2^24 * 127, generator 3, root 3^((p-1)/2^24) =
 * 1791270792 canonical (the construction of BabyBear's root from its
 * generator 31).  R^2, -p^-1 and R are computed from p by the usual
 * definitions; tests/test_oracle.py recomputes every constant. */
static const mfield MF_KB = {
    ORC_KB_P,
    402124772u,   /* R^2 mod p         */
    2130706431u,  /* -p^-1 mod 2^32    */
    33554430u,    /* R mod p           */
    24u,
    331895189u,   /* 1791270792 * R mod p */
};

static inline uint32_t mf_reduce(const mfield *f, uint64_t t) /* babybear.rs:41-51 */
{
    uint32_t t_lo = (uint32_t)t;
    uint32_t m = t_lo * f->monty_const;
    uint64_t mp = (uint64_t)m * f->p;
    uint32_t r = (uint32_t)((t + mp) >> 32);
    return r >= f->p ? r - f->p : r;
}

static inline uint32_t mf_to_monty(const mfield *f, uint32_t v) { return mf_reduce(f, (uint64_t)v * f->r2); }
static inline uint32_t mf_add(const mfield *f, uint32_t a, uint32_t b) /* babybear.rs:113-121 */
{
    uint32_t s = a + b;
    return s >= f->p ? s - f->p : s;
}
static inline uint32_t mf_sub(const mfield *f, uint32_t a, uint32_t b) /* babybear.rs:124-130 */
{
    return a >= b ? a - b : f->p - (b - a);
}
static inline uint32_t mf_mul(const mfield *f, uint32_t a, uint32_t b) /* babybear.rs:133-137 */
{
    return mf_reduce(f, (uint64_t)a * b);
}
static uint32_t mf_inv(const mfield *f, uint32_t a) /* babybear.rs:147-161, Fermat a^(p-2) */
{
    uint32_t result = f->one, base = a, e = f->p - 2;
    while (e > 0) {
        if (e & 1) result = mf_mul(f, result, base);
        base = mf_mul(f, base, base);
        e >>= 1;
    }
    return result;
}
static uint32_t mf_two_adic_generator(const mfield *f, uint32_t log_n) /* babybear.rs:69-76 */
{
    uint32_t g = f->root_monty;
    for (uint32_t i = 0; i < f->two_adicity - log_n; i++) g = mf_mul(f, g, g);
    return g;
}

uint32_t orc_bb_monty_reduce(uint64_t t) { return mf_reduce(&MF_BB, t); }
uint32_t orc_bb_to_monty(uint32_t v) { return mf_to_monty(&MF_BB, v); }
uint32_t orc_bb_from_monty(uint32_t m) { return mf_reduce(&MF_BB, (uint64_t)m); }
uint32_t orc_bb_add(uint32_t a, uint32_t b) { return mf_add(&MF_BB, a, b); }
uint32_t orc_bb_sub(uint32_t a, uint32_t b) { return mf_sub(&MF_BB, a, b); }
uint32_t orc_bb_mul(uint32_t a, uint32_t b) { return mf_mul(&MF_BB, a, b); }
uint32_t orc_bb_reduce(uint64_t v) /* babybear.rs:140-145 */
{
    return orc_bb_to_monty((uint32_t)(v % ORC_BB_P));
}
uint32_t orc_bb_inv(uint32_t a) { return mf_inv(&MF_BB, a); }
uint32_t orc_bb_two_adic_generator(uint32_t log_n) { return mf_two_adic_generator(&MF_BB, log_n); }

uint32_t orc_kb_to_monty(uint32_t v) { return mf_to_monty(&MF_KB, v); }
uint32_t orc_kb_from_monty(uint32_t m) { return mf_reduce(&MF_KB, (uint64_t)m); }
uint32_t orc_kb_mul(uint32_t a, uint32_t b) { return mf_mul(&MF_KB, a, b); }
uint32_t orc_kb_two_adic_generator(uint32_t log_n) { return mf_two_adic_generator(&MF_KB, log_n); }

/* ========================= M31 (src/field/m31.rs) ======================== */

#define M31_P ORC_M31_P

/* The hot helpers are static inline so the NTT loops inline them (the
 * exported orc_* functions below are thin wrappers): calls to exported
 * functions of a shared library would otherwise stay out of line. */
static inline uint32_t m31_reduce_i(uint64_t v) /* m31.rs:54-67 */
{
    uint32_t lo = (uint32_t)(v & 0x7FFFFFFFu);
    uint32_t hi = (uint32_t)(v >> 31);
    uint32_t s = lo + hi;
    return s >= M31_P ? s - M31_P : s;
}
static inline uint32_t m31_add_i(uint32_t a, uint32_t b) { return m31_reduce_i((uint64_t)a + b); } /* m31.rs:32-35 */
static inline uint32_t m31_sub_i(uint32_t a, uint32_t b) /* m31.rs:38-45 */
{
    return a >= b ? a - b : M31_P - (b - a);
}
static inline uint32_t m31_mul_i(uint32_t a, uint32_t b) { return m31_reduce_i((uint64_t)a * b); } /* m31.rs:48-51 */

uint32_t orc_m31_reduce(uint64_t v) { return m31_reduce_i(v); }
uint32_t orc_m31_add(uint32_t a, uint32_t b) { return m31_add_i(a, b); }
uint32_t orc_m31_sub(uint32_t a, uint32_t b) { return m31_sub_i(a, b); }
uint32_t orc_m31_mul(uint32_t a, uint32_t b) { return m31_mul_i(a, b); }

uint32_t orc_m31_inv(uint32_t a) /* m31.rs:69-83 */
{
    uint32_t result = 1, base = a, e = M31_P - 2;
    while (e > 0) {
        if (e & 1) result = m31_mul_i(result, base);
        base = m31_mul_i(base, base);
        e >>= 1;
    }
    return result;
}

/* ===================== Circle group (src/field/circle.rs) ================ */

static const orc_cpoint CIRCLE_GEN = {2u, 1268011823u};   /* circle.rs:17-20 */
static const orc_cpoint CIRCLE_IDENTITY = {1u, 0u};       /* circle.rs:26-29 */

orc_cpoint orc_circle_add(orc_cpoint a, orc_cpoint b) /* circle.rs:34-40 */
{
    orc_cpoint r;
    r.x = orc_m31_sub(orc_m31_mul(a.x, b.x), orc_m31_mul(a.y, b.y));
    r.y = orc_m31_add(orc_m31_mul(a.x, b.y), orc_m31_mul(a.y, b.x));
    return r;
}

orc_cpoint orc_circle_double(orc_cpoint a) /* circle.rs:53-60 */
{
    orc_cpoint r;
    r.x = orc_m31_sub(orc_m31_mul(2u, orc_m31_mul(a.x, a.x)), 1u);
    r.y = orc_m31_mul(2u, orc_m31_mul(a.x, a.y));
    return r;
}

orc_cpoint orc_circle_mul_scalar(orc_cpoint a, uint32_t n) /* circle.rs:63-74 */
{
    orc_cpoint result = CIRCLE_IDENTITY, base = a;
    while (n > 0) {
        if (n & 1) result = orc_circle_add(result, base);
        base = orc_circle_add(base, base);
        n >>= 1;
    }
    return result;
}

orc_cpoint orc_circle_subgroup_gen(uint32_t log_size) /* circle.rs:78-85 */
{
    orc_cpoint p = CIRCLE_GEN;
    for (uint32_t i = 0; i < 31u - log_size; i++) p = orc_circle_double(p);
    return p;
}

typedef struct { orc_cpoint initial, step; uint32_t log_size; } coset_t;

static coset_t coset_odds(uint32_t log_size) /* circle.rs:108-117 */
{
    coset_t c;
    c.step = orc_circle_subgroup_gen(log_size);
    c.initial = orc_circle_subgroup_gen(log_size + 1);
    c.log_size = log_size;
    return c;
}

static orc_cpoint coset_at(const coset_t *c, size_t i) /* circle.rs:136-138 */
{
    return orc_circle_add(c->initial, orc_circle_mul_scalar(c->step, (uint32_t)i));
}

static coset_t coset_double(const coset_t *c) /* circle.rs:143-150 */
{
    coset_t d;
    d.initial = orc_circle_double(c->initial);
    d.step = orc_circle_double(c->step);
    d.log_size = c->log_size - 1;
    return d;
}

static size_t bit_reverse_idx(size_t index, uint32_t log_size) /* m31/twiddles.rs:71-79 */
{
    uint32_t v = (uint32_t)index, r = 0;
    for (uint32_t i = 0; i < log_size; i++) {
        r = (r << 1) | (v & 1);
        v >>= 1;
    }
    return r;
}

/* ============================ Twiddles =================================== */

/* BabyBear::generate_twiddles (babybear.rs:83-97): layer s holds g_{s+1}^j,
 * j < 2^s; generate_inverse_twiddles (babybear/twiddles.rs:13-19) inverts
 * every entry. */
static void mf_twiddles(const mfield *f, uint32_t log_n, int inverse, uint32_t *out)
{
    for (uint32_t s = 0; s < log_n; s++) {
        size_t half = (size_t)1 << s;
        uint32_t g = mf_two_adic_generator(f, s + 1);
        uint32_t w = f->one;
        uint32_t *layer = out + (half - 1);
        for (size_t j = 0; j < half; j++) {
            layer[j] = inverse ? mf_inv(f, w) : w;
            w = mf_mul(f, w, g);
        }
    }
}

void orc_bb_twiddles(uint32_t log_n, int inverse, uint32_t *out) { mf_twiddles(&MF_BB, log_n, inverse, out); }
void orc_kb_twiddles(uint32_t log_n, int inverse, uint32_t *out) { mf_twiddles(&MF_KB, log_n, inverse, out); }

/* generate_twiddles / generate_itwiddles (m31/twiddles.rs:19-68) on
 * Coset::odds(log_n): layer l holds the x coordinate (y on the last layer)
 * of the l-times-doubled coset at bit-reversed positions. */
void orc_m31_twiddles(uint32_t log_n, int inverse, uint32_t *out)
{
    size_t n = (size_t)1 << log_n;
    coset_t cur = coset_odds(log_n);
    for (uint32_t layer = 0; layer < log_n; layer++) {
        size_t half = ((size_t)1 << cur.log_size) / 2;
        int last = (layer == log_n - 1);
        uint32_t *dst = out + (n - (n >> layer));
        for (size_t i = 0; i < half; i++) {
            orc_cpoint p = coset_at(&cur, bit_reverse_idx(i, cur.log_size - 1));
            uint32_t t = last ? p.y : p.x;
            dst[i] = inverse ? orc_m31_inv(t) : t;
        }
        cur = coset_double(&cur);
    }
}

/* TwiddleCache (src/ntt/twiddle_cache.rs): one cached table per
 * (field, direction, log_n).  Tables are filled before any parallel region. */
enum { TW_BB = 0, TW_M31 = 1, TW_KB = 2 };
static uint32_t *g_tw_cache[3][2][32];

static const uint32_t *tw_get(int field, int inverse, uint32_t log_n)
{
    uint32_t **slot = &g_tw_cache[field][inverse][log_n];
    if (*slot == NULL) {
        size_t n = (size_t)1 << log_n;
        uint32_t *t = (uint32_t *)malloc(n * sizeof(uint32_t));
        if (field == TW_M31) orc_m31_twiddles(log_n, inverse, t);
        else if (field == TW_KB) orc_kb_twiddles(log_n, inverse, t);
        else orc_bb_twiddles(log_n, inverse, t);
        *slot = t;
    }
    return *slot;
}

static int mf_tw_id(const mfield *f) { return f == &MF_KB ? TW_KB : TW_BB; }

static int is_pow2(size_t n) { return n != 0 && (n & (n - 1)) == 0; }
static uint32_t ilog2(size_t n) { uint32_t l = 0; while (((size_t)1 << l) < n) l++; return l; }

/* ====================== BabyBear NTT (cpu_reference.rs) ================== */

static void mf_forward_tw(const mfield *f, uint32_t *data, size_t n, uint32_t log_n, const uint32_t *tw)
{
    for (int layer = (int)log_n - 1; layer >= 0; layer--) { /* cpu_reference.rs:45-60 */
        size_t half = (size_t)1 << layer, full = half << 1;
        const uint32_t *t = tw + (half - 1);
        for (size_t block = 0; block < n / full; block++) {
            for (size_t j = 0; j < half; j++) {
                size_t i0 = block * full + j, i1 = i0 + half;
                uint32_t v0 = data[i0], v1 = data[i1];
                data[i0] = mf_add(f, v0, v1);
                data[i1] = mf_mul(f, mf_sub(f, v0, v1), t[j]);
            }
        }
    }
}

static void mf_inverse_tw(const mfield *f, uint32_t *data, size_t n, uint32_t log_n, const uint32_t *itw,
                          int normalize)
{
    for (uint32_t layer = 0; layer < log_n; layer++) { /* cpu_reference.rs:80-95 */
        size_t half = (size_t)1 << layer, full = half << 1;
        const uint32_t *t = itw + (half - 1);
        for (size_t block = 0; block < n / full; block++) {
            for (size_t j = 0; j < half; j++) {
                size_t i0 = block * full + j, i1 = i0 + half;
                uint32_t tmp = mf_mul(f, data[i1], t[j]);
                uint32_t v0 = data[i0];
                data[i0] = mf_add(f, v0, tmp);
                data[i1] = mf_sub(f, v0, tmp);
            }
        }
    }
    if (normalize) { /* cpu_reference.rs:97-101 */
        uint32_t inv_n = mf_inv(f, mf_to_monty(f, (uint32_t)(n % f->p)));
        for (size_t i = 0; i < n; i++) data[i] = mf_mul(f, data[i], inv_n);
    }
}

static int mf_forward(const mfield *f, uint32_t *data, size_t n)
{
    if (!is_pow2(n)) return 1;
    if (n == 1) return 0;
    uint32_t log_n = ilog2(n);
    if (log_n > f->two_adicity) return 1;
    mf_forward_tw(f, data, n, log_n, tw_get(mf_tw_id(f), 0, log_n));
    return 0;
}

static int mf_inverse(const mfield *f, uint32_t *data, size_t n)
{
    if (!is_pow2(n)) return 1;
    if (n == 1) return 0;
    uint32_t log_n = ilog2(n);
    if (log_n > f->two_adicity) return 1;
    mf_inverse_tw(f, data, n, log_n, tw_get(mf_tw_id(f), 1, log_n), 1);
    return 0;
}

int orc_bb_forward(uint32_t *data, size_t n) { return mf_forward(&MF_BB, data, n); }
int orc_bb_inverse(uint32_t *data, size_t n) { return mf_inverse(&MF_BB, data, n); }
int orc_kb_forward(uint32_t *data, size_t n) { return mf_forward(&MF_KB, data, n); }
int orc_kb_inverse(uint32_t *data, size_t n) { return mf_inverse(&MF_KB, data, n); }

/* ======================== M31 NTT (m31/cpu_reference.rs) ================= */

static void m31_forward_tw(uint32_t *data, size_t n, uint32_t log_n, const uint32_t *tw)
{
    for (int layer = (int)log_n - 1; layer >= 0; layer--) { /* cpu_reference.rs:61-74 */
        size_t half = (size_t)1 << layer, full = half << 1;
        const uint32_t *t = tw + (n - (n >> layer));
        for (size_t block = 0; block < n / full; block++) {
            uint32_t w = t[block];
            for (size_t j = 0; j < half; j++) {
                size_t i0 = block * full + j, i1 = i0 + half;
                uint32_t tmp = m31_mul_i(data[i1], w); /* butterfly_forward :137-142 */
                uint32_t v0 = data[i0];
                data[i0] = m31_add_i(v0, tmp);
                data[i1] = m31_sub_i(v0, tmp);
            }
        }
    }
}

static void m31_inverse_tw(uint32_t *data, size_t n, uint32_t log_n, const uint32_t *itw)
{
    for (uint32_t layer = 0; layer < log_n; layer++) { /* cpu_reference.rs:93-107 */
        size_t half = (size_t)1 << layer, full = half << 1;
        const uint32_t *t = itw + (n - (n >> layer));
        for (size_t block = 0; block < n / full; block++) {
            uint32_t w = t[block];
            for (size_t j = 0; j < half; j++) {
                size_t i0 = block * full + j, i1 = i0 + half;
                uint32_t v0 = data[i0], v1 = data[i1]; /* butterfly_inverse :148-153 */
                data[i0] = m31_add_i(v0, v1);
                data[i1] = m31_mul_i(m31_sub_i(v0, v1), w);
            }
        }
    }
    uint32_t inv_n = orc_m31_inv(m31_reduce_i(n)); /* cpu_reference.rs:113-117 */
    for (size_t i = 0; i < n; i++) data[i] = m31_mul_i(data[i], inv_n);
}

int orc_m31_forward(uint32_t *data, size_t n)
{
    if (!is_pow2(n)) return 1;
    if (n == 1) return 0;
    uint32_t log_n = ilog2(n);
    if (log_n > 30) return 1;
    m31_forward_tw(data, n, log_n, tw_get(TW_M31, 0, log_n));
    return 0;
}

int orc_m31_inverse(uint32_t *data, size_t n)
{
    if (!is_pow2(n)) return 1;
    if (n == 1) return 0;
    uint32_t log_n = ilog2(n);
    if (log_n > 30) return 1;
    m31_inverse_tw(data, n, log_n, tw_get(TW_M31, 1, log_n));
    return 0;
}

/* ============================ Batches ===================================== */

static int clamp_threads(int threads) { return threads < 1 ? 1 : threads; }

static int mf_forward_batch(const mfield *f, uint32_t *data, uint32_t log_n, uint32_t batch, int threads)
{
    if (log_n > f->two_adicity) return 1;
    if (log_n == 0) return 0;
    size_t n = (size_t)1 << log_n;
    const uint32_t *tw = tw_get(mf_tw_id(f), 0, log_n);
    long c;
    (void)threads;
#pragma omp parallel for schedule(dynamic, 1) num_threads(clamp_threads(threads))
    for (c = 0; c < (long)batch; c++) mf_forward_tw(f, data + (size_t)c * n, n, log_n, tw);
    return 0;
}

static int mf_inverse_batch(const mfield *f, uint32_t *data, uint32_t log_n, uint32_t batch, int threads)
{
    if (log_n > f->two_adicity) return 1;
    if (log_n == 0) return 0;
    size_t n = (size_t)1 << log_n;
    const uint32_t *itw = tw_get(mf_tw_id(f), 1, log_n);
    long c;
    (void)threads;
#pragma omp parallel for schedule(dynamic, 1) num_threads(clamp_threads(threads))
    for (c = 0; c < (long)batch; c++) mf_inverse_tw(f, data + (size_t)c * n, n, log_n, itw, 1);
    return 0;
}

int orc_bb_forward_batch(uint32_t *data, uint32_t log_n, uint32_t batch, int threads)
{
    return mf_forward_batch(&MF_BB, data, log_n, batch, threads);
}
int orc_bb_inverse_batch(uint32_t *data, uint32_t log_n, uint32_t batch, int threads)
{
    return mf_inverse_batch(&MF_BB, data, log_n, batch, threads);
}
int orc_kb_forward_batch(uint32_t *data, uint32_t log_n, uint32_t batch, int threads)
{
    return mf_forward_batch(&MF_KB, data, log_n, batch, threads);
}
int orc_kb_inverse_batch(uint32_t *data, uint32_t log_n, uint32_t batch, int threads)
{
    return mf_inverse_batch(&MF_KB, data, log_n, batch, threads);
}

/* ========================= Coset LDE (src/lde/mod.rs) ==================== */

/* coset_lde_batch_cpu (lde/mod.rs:127-176): per-column inverse, zero-pad
 * copy, coset shift over rows-then-columns with shift =
 * two_adic_generator(log_n_ext + 1) (lde/mod.rs:158), per-column forward. */
static int mf_coset_lde(const mfield *f, const uint32_t *in, uint32_t *out, uint32_t log_n, uint32_t batch,
                        uint32_t added_bits, uint32_t shift_monty, int threads)
{
    uint32_t log_n_ext = log_n + added_bits;
    if (log_n_ext + 1 > f->two_adicity) return 1;
    size_t n = (size_t)1 << log_n, n_ext = (size_t)1 << log_n_ext;
    uint32_t shift = shift_monty ? shift_monty : mf_two_adic_generator(f, log_n_ext + 1);
    const uint32_t *itw = log_n ? tw_get(mf_tw_id(f), 1, log_n) : NULL;
    const uint32_t *tw = log_n_ext ? tw_get(mf_tw_id(f), 0, log_n_ext) : NULL;
    long c;
    (void)threads;

    /* shift powers, shared by every column (the reference recomputes the
     * running power in its row loop; the values are identical) */
    uint32_t *pw = (uint32_t *)malloc(n_ext * sizeof(uint32_t));
    uint32_t p = f->one;
    for (size_t i = 0; i < n_ext; i++) { pw[i] = p; p = mf_mul(f, p, shift); }

#pragma omp parallel for schedule(dynamic, 1) num_threads(clamp_threads(threads))
    for (c = 0; c < (long)batch; c++) {
        uint32_t *dst = out + (size_t)c * n_ext;
        memcpy(dst, in + (size_t)c * n, n * sizeof(uint32_t));          /* step 1+2 */
        if (log_n) mf_inverse_tw(f, dst, n, log_n, itw, 1);
        memset(dst + n, 0, (n_ext - n) * sizeof(uint32_t));
        for (size_t i = 0; i < n_ext; i++) dst[i] = mf_mul(f, dst[i], pw[i]); /* step 3 */
        if (log_n_ext) mf_forward_tw(f, dst, n_ext, log_n_ext, tw);     /* step 4 */
    }
    free(pw);
    return 0;
}

int orc_bb_coset_lde(const uint32_t *in, uint32_t *out, uint32_t log_n, uint32_t batch,
                     uint32_t added_bits, uint32_t shift_monty, int threads)
{
    return mf_coset_lde(&MF_BB, in, out, log_n, batch, added_bits, shift_monty, threads);
}

int orc_kb_coset_lde(const uint32_t *in, uint32_t *out, uint32_t log_n, uint32_t batch,
                     uint32_t added_bits, uint32_t shift_monty, int threads)
{
    return mf_coset_lde(&MF_KB, in, out, log_n, batch, added_bits, shift_monty, threads);
}

int orc_m31_lde(const uint32_t *in, uint32_t *out, uint32_t log_n, uint32_t batch,
                uint32_t added_bits, int threads)
{
    uint32_t log_n_ext = log_n + added_bits;
    if (log_n_ext > 30) return 1;
    size_t n = (size_t)1 << log_n, n_ext = (size_t)1 << log_n_ext;
    const uint32_t *itw = log_n ? tw_get(TW_M31, 1, log_n) : NULL;
    const uint32_t *tw = log_n_ext ? tw_get(TW_M31, 0, log_n_ext) : NULL;
    long c;
    (void)threads;
#pragma omp parallel for schedule(dynamic, 1) num_threads(clamp_threads(threads))
    for (c = 0; c < (long)batch; c++) {
        uint32_t *dst = out + (size_t)c * n_ext;
        memcpy(dst, in + (size_t)c * n, n * sizeof(uint32_t));
        if (log_n) m31_inverse_tw(dst, n, log_n, itw);
        memset(dst + n, 0, (n_ext - n) * sizeof(uint32_t));
        if (log_n_ext) m31_forward_tw(dst, n_ext, log_n_ext, tw);
    }
    return 0;
}

/* ============ Canonic-coset circle FFT and circle LDE (Stwo-style) ======== */

/* Not in the reference, which lists "M31 Circle LDE proper" only as a goal
 * and comments Stwo out (tests/ntt_cross_validation.rs:281-298).  Definition
 * (the circle FFT of the Circle STARKs construction, restated here):
 *   domain D_k = odds(k) in the order D[i] = h_i (i < n/2), D[n/2 + i] =
 *   conj(h_i), h_i = G_{2^(k+1)} + i G_{2^(k-1)}; values in bit-reversed order
 *   (storage r holds f(D[bitrev_k(r)])); coefficient r multiplies the basis
 *   y^{r_0} x^{r_1} pi(x)^{r_2} pi^2(x)^{r_3} ... (pi(x) = 2x^2 - 1), so
 *   padding coefficients with zeros keeps the function.
 * The network is the reference's M31 network (m31/cpu_reference.rs:61-107:
 * per-block twiddles, layer L stride 2^L) with these twiddles:
 *   T_0[b] = y(h_{bitrev_{k-1}(b)}),  T_L[b] = x(2^{L-1} h_{bitrev_{k-1-L}(b)}) (L >= 1).
 * Every twiddle is a coordinate of m G_{2^(k+1)}: h_i = (1 + 4i) G_{2^(k+1)}. */
static orc_cpoint gpow(uint32_t k, uint64_t m) /* m G_{2^(k+1)}, m mod 2^(k+1) */
{
    return orc_circle_mul_scalar(orc_circle_subgroup_gen(k + 1), (uint32_t)(m & (((uint64_t)1 << (k + 1)) - 1)));
}

void orc_circle_twiddles(uint32_t log_n, int inverse, uint32_t *out)
{
    size_t n = (size_t)1 << log_n;
    for (uint32_t L = 0; L < log_n; L++) {
        size_t cnt = n >> (L + 1);
        uint32_t *dst = out + (n - (n >> L));
        uint32_t bits = log_n - 1 - L;
        for (size_t b = 0; b < cnt; b++) {
            uint64_t i = bit_reverse_idx(b, bits);
            uint64_t m = (1 + 4 * i) << (L ? L - 1 : 0);
            orc_cpoint p = gpow(log_n, m);
            uint32_t t = L == 0 ? p.y : p.x;
            dst[b] = inverse ? orc_m31_inv(t) : t;
        }
    }
}

static uint32_t *g_ctw_cache[2][32];

static const uint32_t *ctw_get(int inverse, uint32_t log_n)
{
    uint32_t **slot = &g_ctw_cache[inverse][log_n];
    if (*slot == NULL) {
        uint32_t *t = (uint32_t *)malloc(((size_t)1 << log_n) * sizeof(uint32_t));
        orc_circle_twiddles(log_n, inverse, t);
        *slot = t;
    }
    return *slot;
}

int orc_circle_ntt(uint32_t *data, uint32_t log_n, uint32_t batch, int inverse)
{
    if (log_n > 30) return 1;
    if (log_n == 0) return 0;
    size_t n = (size_t)1 << log_n;
    const uint32_t *tw = ctw_get(inverse, log_n);
    for (uint32_t c = 0; c < batch; c++) {
        if (inverse) m31_inverse_tw(data + (size_t)c * n, n, log_n, tw);
        else m31_forward_tw(data + (size_t)c * n, n, log_n, tw);
    }
    return 0;
}

/* Interpolate on D_{log_n} (values bit-reversed), zero-pad the coefficients,
 * evaluate on D_{log_n + added_bits}. */
int orc_circle_lde(const uint32_t *in, uint32_t *out, uint32_t log_n, uint32_t batch,
                   uint32_t added_bits, int threads)
{
    uint32_t log_n_ext = log_n + added_bits;
    if (log_n_ext > 30) return 1;
    size_t n = (size_t)1 << log_n, n_ext = (size_t)1 << log_n_ext;
    const uint32_t *itw = log_n ? ctw_get(1, log_n) : NULL;
    const uint32_t *tw = log_n_ext ? ctw_get(0, log_n_ext) : NULL;
    long c;
    (void)threads;
#pragma omp parallel for schedule(dynamic, 1) num_threads(clamp_threads(threads))
    for (c = 0; c < (long)batch; c++) {
        uint32_t *dst = out + (size_t)c * n_ext;
        memcpy(dst, in + (size_t)c * n, n * sizeof(uint32_t));
        if (log_n) m31_inverse_tw(dst, n, log_n, itw);
        memset(dst + n, 0, (n_ext - n) * sizeof(uint32_t));
        if (log_n_ext) m31_forward_tw(dst, n_ext, log_n_ext, tw);
    }
    return 0;
}

/* ================= CM31 = M31[i] / (i^2 + 1) (TODOS.md:27-31) ============ */

/* Not implemented in the reference (planned).  (a + bi)(c + di) =
 * (ac - bd) + (ad + bc) i over M31; a transform of CM31 columns with M31
 * twiddles is the M31 transform of each coordinate. */
void orc_cm31_mul(const uint32_t *a, const uint32_t *b, uint32_t *out, size_t n)
{
    for (size_t k = 0; k < n; k++) {
        uint32_t ar = a[2 * k], ai = a[2 * k + 1], br = b[2 * k], bi = b[2 * k + 1];
        uint32_t re = m31_sub_i(m31_mul_i(ar, br), m31_mul_i(ai, bi));
        uint32_t im = m31_add_i(m31_mul_i(ar, bi), m31_mul_i(ai, br));
        out[2 * k] = re;
        out[2 * k + 1] = im;
    }
}

int orc_cm31_ntt(uint32_t *pairs, uint32_t log_n, uint32_t batch, int inverse)
{
    if (log_n > 30) return 1;
    if (log_n == 0) return 0;
    size_t n = (size_t)1 << log_n;
    uint32_t *col = (uint32_t *)malloc(n * sizeof(uint32_t));
    for (uint32_t c = 0; c < batch; c++) {
        uint32_t *p = pairs + 2 * (size_t)c * n;
        for (int part = 0; part < 2; part++) {
            for (size_t j = 0; j < n; j++) col[j] = p[2 * j + part];
            if (inverse) orc_m31_inverse(col, n);
            else orc_m31_forward(col, n);
            for (size_t j = 0; j < n; j++) p[2 * j + part] = col[j];
        }
    }
    free(col);
    return 0;
}

/* ============================ Data generator ============================= */

uint64_t orc_lcg_fill(uint32_t *out, size_t n, uint64_t seed, uint32_t p, int monty)
{
    uint64_t s = seed;
    for (size_t i = 0; i < n; i++) {
        s = s * 6364136223846793005ull + 1ull;
        uint32_t v = (uint32_t)(s >> 33) % p;
        out[i] = monty == 2 ? orc_kb_to_monty(v) : (monty ? orc_bb_to_monty(v) : v);
    }
    return s;
}
