/*
 * sfntt.h -- C ABI of the B200 (sm_100a) small-field NTT / coset-LDE library.
 *
 * Drop-in boundary for the NTT hot path of moven0831/small-field-metal-ntt.
 * The reference is a Rust crate; a Rust FFI crate (sfntt-sys) binds these
 * symbols one to one.  All functions are plain C:
 * pointers, sizes and integer status codes, no C++ or torch types.
 *
 * Conventions (same as the reference):
 *   - BabyBear values are Montgomery-form u32 in [0, p), p = 2^31 - 2^27 + 1
 *     (src/field/babybear.rs:14-65).  M31 values are canonical u32 in [0, p),
 *     p = 2^31 - 1 (src/field/m31.rs:18-67).
 *   - Forward NTT: natural-order input, bit-reversed-order output.  Inverse:
 *     bit-reversed input, natural output, multiplied by n^-1
 *     (src/ntt/babybear/cpu_reference.rs:29-103, src/ntt/m31/cpu_reference.rs:50-120).
 *   - Batches are SoA / column-major: data[col * n + row] (src/lde/mod.rs:21).
 *   - Results are bit-exact with the reference CPU path for every element.
 *
 * Threading: a context serialises its host-memory calls with an internal
 * mutex; use one context per thread for concurrency.  Device-pointer (_dev)
 * calls are asynchronous on the caller's stream; their device-resident tables
 * must already be cached (sfntt_prepare) before a CUDA graph capture.
 */
#ifndef SFNTT_H
#define SFNTT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: one per NttError variant (src/ntt/mod.rs:52-69) plus three. */
typedef enum sfntt_status {
    SFNTT_OK = 0,
    SFNTT_INVALID_SIZE = 1,      /* NttError::InvalidSize(usize)               */
    SFNTT_DEVICE_NOT_FOUND = 2,  /* NttError::DeviceNotFound                   */
    SFNTT_ALLOC_FAILED = 3,      /* NttError::BufferAllocFailed{requested_bytes} */
    SFNTT_KERNEL_LOAD = 4,       /* NttError::ShaderCompileError: no sm_100a image for this GPU */
    SFNTT_GPU_EXECUTION = 5,     /* NttError::GpuExecutionError(String)        */
    SFNTT_MISMATCH = 6,          /* NttError::CorrectnessMismatch{..}          */
    SFNTT_UNSUPPORTED = 7,       /* V1 inverse: the reference panics (todo!()) */
    SFNTT_TIMEOUT = 8,           /* a bounded device-side wait ran out         */
    SFNTT_INVALID_ARGUMENT = 9   /* null pointer, bad enum, cold cache during capture */
} sfntt_status;

typedef enum sfntt_field {
    SFNTT_M31 = 0,       /* Circle NTT (DCCT) over M31       */
    SFNTT_BABYBEAR = 1,  /* radix-2 NTT over BabyBear        */
    SFNTT_KOALABEAR = 2  /* radix-2 NTT over KoalaBear, p = 2^31 - 2^24 + 1: planned in the reference
                            (README.md:20), no implementation there.  Montgomery u32 like BabyBear;
                            two_adic_generator(k) = 3^((p-1)/2^k), log_n <= 24 */
} sfntt_field;

/* Algorithm variants of the reference shootout (src/ntt/mod.rs:17-25). */
typedef enum sfntt_variant {
    SFNTT_BEST = 0,
    SFNTT_V1_CT_DIT_R2 = 1,    /* one kernel per layer (metal_ct_dit_r2.rs)            */
    SFNTT_V2_CT_GS_R2 = 2,     /* per-layer large strides + one smem tile (metal_r2.rs) */
    SFNTT_V3_STOCKHAM_R2 = 3,  /* out-of-place ping-pong (metal_stockham_r2.rs)        */
    SFNTT_V4_CT_GS_R4 = 4      /* fused multi-layer smem passes (metal_ct_gs_r4.rs)     */
} sfntt_variant;

/* Coset-LDE forms (src/lde/mod.rs:43-107). */
typedef enum sfntt_lde_mode {
    SFNTT_LDE_FUSED = 0,   /* normalize+shift+zero-pad folded into the adjacent NTT passes */
    SFNTT_LDE_UNFUSED = 1, /* iDFT -> normalize -> zero-pad -> shift -> DFT, one kernel each */
    SFNTT_LDE_NATURAL = 2  /* flag, OR'ed into either form: natural-order output rows (Plonky3's
                              convention, with shift_monty = to_monty(31)); no reference counterpart */
} sfntt_lde_mode;

typedef struct sfntt_ctx sfntt_ctx;

/* ---- context: replaces MetalContext::new / backend ::new(shader_dir)
 *      (src/gpu.rs:26-64, src/ntt/babybear/metal_ct_gs_r4.rs:44-85). */
/* Read once at creation, for comparisons: SFNTT_NO_TMA=1 routes every pass
 * through the first (non-TMA) tile engine; SFNTT_NO_CLUSTER=1 runs columns of
 * 2^13 .. 2^16 points as two passes instead of one cluster launch. */
int sfntt_ctx_create(int device, sfntt_ctx **out);
void sfntt_ctx_destroy(sfntt_ctx *ctx);
const char *sfntt_status_string(int status);
const char *sfntt_last_error(const sfntt_ctx *ctx);
/* MetalContext::device_info (src/gpu.rs:132-150): "name, SMs, memory". */
int sfntt_device_info(sfntt_ctx *ctx, char *buf, size_t len);

/* ---- NttBackend<F>::forward_ntt / inverse_ntt (src/ntt/mod.rs:37-44):
 * in place on host memory of len elements (power of two; len == 1 is the
 * identity).  *gpu_ns (optional) receives the device time of the transform. */
int sfntt_forward(sfntt_ctx *ctx, int field, int variant, uint32_t *data, size_t len,
                  uint64_t *gpu_ns);
int sfntt_inverse(sfntt_ctx *ctx, int field, int variant, uint32_t *data, size_t len,
                  uint64_t *gpu_ns);

/* ---- NttBackend<F>::pointwise_mul (src/ntt/mod.rs:46-48). */
int sfntt_pointwise_mul(sfntt_ctx *ctx, int field, const uint32_t *a, size_t len_a,
                        const uint32_t *b, size_t len_b, uint32_t *out, size_t len_out);

/* ---- forward_ntt_gpu / inverse_ntt_gpu(input, log_n) -> (Vec<u32>, ns)
 * (src/ntt/babybear/metal_ct_gs_r4.rs:87-172, src/ntt/m31/metal_ct_gs_r4.rs:61-99):
 * out-of-place; len must equal 2^log_n. */
int sfntt_forward_gpu(sfntt_ctx *ctx, int field, int variant, const uint32_t *in, size_t len,
                      uint32_t log_n, uint32_t *out, uint64_t *gpu_ns);
int sfntt_inverse_gpu(sfntt_ctx *ctx, int field, int variant, const uint32_t *in, size_t len,
                      uint32_t log_n, uint32_t *out, uint64_t *gpu_ns);

/* ---- BbBatchNtt::forward_ntt_batch_gpu / inverse_ntt_batch_gpu
 * (src/ntt/babybear/batch.rs:76-180): batch SoA columns of 2^log_n; len must
 * equal batch << log_n.  field = SFNTT_M31 batches the Circle NTT the same way. */
int sfntt_forward_batch(sfntt_ctx *ctx, int field, const uint32_t *in, size_t len,
                        uint32_t log_n, uint32_t batch, uint32_t *out, uint64_t *gpu_ns);
int sfntt_inverse_batch(sfntt_ctx *ctx, int field, const uint32_t *in, size_t len,
                        uint32_t log_n, uint32_t batch, uint32_t *out, uint64_t *gpu_ns);

/* ---- CosetLdeBatch::execute(input, log_n, batch_size, added_bits)
 * (src/lde/mod.rs:43-107).  in: batch columns of 2^log_n Montgomery u32
 * (len must equal batch << log_n); out: batch columns of 2^(log_n+added_bits),
 * bit-reversed rows.  shift_monty == 0 selects the reference shift
 * two_adic_generator(log_n + added_bits + 1) (src/lde/mod.rs:59); any other
 * value is a Montgomery-form shift (e.g. to_monty(31), the Plonky3 coset).
 * Host buffers; copies are pipelined by column chunks with the compute. */
int sfntt_bb_coset_lde(sfntt_ctx *ctx, const uint32_t *in, size_t len, uint32_t log_n,
                       uint32_t batch, uint32_t added_bits, uint32_t shift_monty, int mode,
                       uint32_t *out, uint64_t *gpu_ns);

/* The same coset LDE for either Montgomery field: field = SFNTT_BABYBEAR
 * (identical to sfntt_bb_coset_lde) or SFNTT_KOALABEAR (no reference
 * implementation; the BabyBear algorithm with KoalaBear's constants, shift_monty
 * == 0 selecting two_adic_generator(log_n + added_bits + 1), log_n + added_bits
 * <= 23). */
int sfntt_coset_lde(sfntt_ctx *ctx, int field, const uint32_t *in, size_t len, uint32_t log_n,
                    uint32_t batch, uint32_t added_bits, uint32_t shift_monty, int mode,
                    uint32_t *out, uint64_t *gpu_ns);

/* M31 blow-up (no reference counterpart: the composition of the reference's
 * inverse on odds(log_n), zero-pad, forward on odds(log_n + added_bits)). */
int sfntt_m31_lde(sfntt_ctx *ctx, const uint32_t *in, size_t len, uint32_t log_n,
                  uint32_t batch, uint32_t added_bits, uint32_t *out, uint64_t *gpu_ns);

/* ---- Canonic-coset circle FFT and circle LDE over M31 (Stwo-style; the
 * reference lists an M31 circle LDE as a goal without code).  Domain
 * odds(log_n) = G_{2^(log_n+1)} + <G_{2^log_n}> ordered as the half coset
 * h_i = (1 + 4i) G_{2^(log_n+1)}, i < n/2, then its conjugates; values in
 * bit-reversed order of that domain; coefficient r multiplies
 * y^{r_0} x^{r_1} pi(x)^{r_2} pi^2(x)^{r_3} ... with pi(x) = 2x^2 - 1, so the
 * LDE (interpolate -> zero-pad -> evaluate on odds(log_n + added_bits)) is a
 * genuine low-degree extension.  The butterfly network and data conventions
 * are the reference's M31 ones (src/ntt/m31/cpu_reference.rs:50-120); only
 * the twiddles differ: layer 0 uses y(h), layer L >= 1 x(2^(L-1) h).
 * sfntt_circle_ntt: inverse = 0 evaluates coefficients, 1 interpolates
 * (times n^-1); len = batch << log_n. */
int sfntt_circle_ntt(sfntt_ctx *ctx, int inverse, const uint32_t *in, size_t len, uint32_t log_n,
                     uint32_t batch, uint32_t *out, uint64_t *gpu_ns);
int sfntt_circle_lde(sfntt_ctx *ctx, const uint32_t *in, size_t len, uint32_t log_n, uint32_t batch,
                     uint32_t added_bits, uint32_t *out, uint64_t *gpu_ns);
int sfntt_prepare_circle(sfntt_ctx *ctx, uint32_t log_n, uint32_t added_bits);
int sfntt_circle_ntt_dev(sfntt_ctx *ctx, int inverse, uint32_t *d_data, uint32_t log_n, uint32_t batch,
                         void *stream);
int sfntt_circle_lde_dev(sfntt_ctx *ctx, const uint32_t *d_in, uint32_t *d_out, uint32_t log_n,
                         uint32_t batch, uint32_t added_bits, void *stream);

/* ---- device-pointer twins (stream = cudaStream_t; NULL = legacy default).
 * Asynchronous; no host synchronisation and no allocation when the tables
 * for (field, log_n) are cached. */
int sfntt_prepare(sfntt_ctx *ctx, int field, uint32_t log_n);
int sfntt_prepare_lde(sfntt_ctx *ctx, int field, uint32_t log_n, uint32_t added_bits,
                      uint32_t shift_monty);
int sfntt_forward_dev(sfntt_ctx *ctx, int field, int variant, uint32_t *d_data, uint32_t log_n,
                      uint32_t batch, void *stream);
int sfntt_inverse_dev(sfntt_ctx *ctx, int field, int variant, uint32_t *d_data, uint32_t log_n,
                      uint32_t batch, void *stream);
/* d_in is read only; d_out holds batch << (log_n + added_bits) elements. */
int sfntt_bb_coset_lde_dev(sfntt_ctx *ctx, const uint32_t *d_in, uint32_t *d_out, uint32_t log_n,
                           uint32_t batch, uint32_t added_bits, uint32_t shift_monty, int mode,
                           void *stream);
int sfntt_coset_lde_dev(sfntt_ctx *ctx, int field, const uint32_t *d_in, uint32_t *d_out,
                        uint32_t log_n, uint32_t batch, uint32_t added_bits, uint32_t shift_monty,
                        int mode, void *stream);
int sfntt_m31_lde_dev(sfntt_ctx *ctx, const uint32_t *d_in, uint32_t *d_out, uint32_t log_n,
                      uint32_t batch, uint32_t added_bits, void *stream);

/* ---- Output conventions of SoA batches (either field; no reference
 * counterpart beyond its one-word-per-thread bitrev_permute kernel,
 * shaders/m31/m31_ntt_ct_dit_r2.metal:22-41).  Flags:
 *   SFNTT_LAYOUT_NATURAL    rows of every column from bit-reversed to natural
 *                           order: out[c*n + r] = in[c*n + bitrev(r)]
 *   SFNTT_LAYOUT_ROW_MAJOR  transpose to row-major rows (Merkle-commitment
 *                           input, one leaf per row): out[R*batch + c] = in[c*n + r],
 *                           R = bitrev(r) with SFNTT_LAYOUT_NATURAL, else r
 * n = 2^log_n.  d_in == d_out is allowed for SFNTT_LAYOUT_NATURAL alone (in
 * place, no scratch); otherwise the buffers must not overlap. */
typedef enum sfntt_layout_flags {
    SFNTT_LAYOUT_NATURAL = 1,
    SFNTT_LAYOUT_ROW_MAJOR = 2
} sfntt_layout_flags;
int sfntt_layout_dev(sfntt_ctx *ctx, const uint32_t *d_in, uint32_t *d_out, uint32_t log_n, uint32_t batch,
                     int flags, void *stream);
/* Host buffers (len must equal batch << log_n); *gpu_ns = device time. */
int sfntt_layout(sfntt_ctx *ctx, const uint32_t *in, size_t len, uint32_t log_n, uint32_t batch, int flags,
                 uint32_t *out, uint64_t *gpu_ns);

/* BabyBear::to_monty / from_monty (src/field/babybear.rs:54-65) on device. */
int sfntt_bb_to_monty_dev(sfntt_ctx *ctx, uint32_t *d_data, size_t len, void *stream);
int sfntt_bb_from_monty_dev(sfntt_ctx *ctx, uint32_t *d_data, size_t len, void *stream);
/* The same for field = SFNTT_BABYBEAR or SFNTT_KOALABEAR. */
int sfntt_to_monty_dev(sfntt_ctx *ctx, int field, uint32_t *d_data, size_t len, void *stream);
int sfntt_from_monty_dev(sfntt_ctx *ctx, int field, uint32_t *d_data, size_t len, void *stream);

/* ---- M31 quadratic extension CM31 = M31[i]/(i^2 + 1) (planned in the
 * reference, TODOS.md:27-31).  An element is an interleaved pair (re, im) of
 * canonical M31 words; a batch is `batch` columns of 2^log_n pairs
 * (len = 2 * (batch << log_n) words).  The Circle NTT of a CM31 column is the
 * Circle NTT of its real parts plus i times that of its imaginary parts (the
 * twiddles lie in M31), with the M31 conventions (forward: bit-reversed out;
 * inverse: times n^-1).  The device calls use a context scratch of
 * 8 * (batch << log_n) bytes: call sfntt_cm31_prepare before a graph capture. */
int sfntt_cm31_prepare(sfntt_ctx *ctx, uint32_t log_n, uint32_t batch);
int sfntt_cm31_ntt_dev(sfntt_ctx *ctx, int inverse, uint32_t *d_pairs, uint32_t log_n, uint32_t batch,
                       void *stream);
int sfntt_cm31_ntt(sfntt_ctx *ctx, int inverse, const uint32_t *in, size_t len, uint32_t log_n,
                   uint32_t batch, uint32_t *out, uint64_t *gpu_ns);
/* out[k] = a[k] * b[k] in CM31 for n pairs (8-byte aligned device pointers). */
int sfntt_cm31_mul_dev(sfntt_ctx *ctx, const uint32_t *d_a, const uint32_t *d_b, uint32_t *d_out, size_t n,
                       void *stream);

/* ---- Uneven batches in one graph launch (no reference counterpart: many
 * polynomials of uneven sizes per launch).  An item is `batch` SoA columns of 2^log_n
 * points of any field, extended by 2^added_bits: BabyBear items are the
 * coset LDE of CosetLdeBatch::execute (src/lde/mod.rs:43-107, shift_monty 0 =
 * reference shift), KoalaBear items the same LDE over KoalaBear, M31 items the
 * composition inverse(odds(log_n)) -> zero-pad -> forward(odds(log_n +
 * added_bits)).  Device pointers. */
typedef enum sfntt_plan {
    SFNTT_PLAN_AUTO = 0,           /* tuned plan for the item's key, else the context default */
    SFNTT_PLAN_TMA = 1,            /* persistent TMA engine, per-position strided twiddles */
    SFNTT_PLAN_TMA_FOUR_STEP = 2,  /* persistent TMA engine, four-step strided passes */
    SFNTT_PLAN_TILE = 3,           /* first (non-TMA) shared-memory tile engine */
    SFNTT_PLAN_ENGINE_MASK = 3,
    /* flags on the TMA engines: */
    SFNTT_PLAN_SPLIT12 = 4,        /* layer ranges above 12 layers: a 12-layer contiguous pass, the rest
                                      in strided passes (default: 8-layer strided passes, the rest
                                      contiguous) -- the stages per pass */
    SFNTT_PLAN_ONE_CTA = 8         /* one persistent CTA per SM (default: as many as fit) */
} sfntt_plan;

typedef struct sfntt_lde_item {
    int field;
    uint32_t log_n, batch, added_bits, shift_monty;
    const uint32_t *d_in;
    uint32_t *d_out;
    int plan;
} sfntt_lde_item;

typedef struct sfntt_graph sfntt_graph;

/* Make every table the items need resident (required before capture). */
int sfntt_batch_prepare(sfntt_ctx *ctx, const sfntt_lde_item *items, size_t count);
/* The plain per-polynomial loop: one item after another on `stream`. */
int sfntt_batch_run(sfntt_ctx *ctx, const sfntt_lde_item *items, size_t count, void *stream);
/* Capture all items into one CUDA graph; items are spread (largest first, to
 * the least-loaded lane) over `lanes` forked streams so independent items
 * overlap.  Replay with sfntt_graph_launch: one launch for the batch. */
int sfntt_batch_graph_create(sfntt_ctx *ctx, const sfntt_lde_item *items, size_t count, int lanes,
                             sfntt_graph **out);
/* The same batch in persistent form: every BabyBear / M31 item with
 * 2^13..2^21 points, blow-up <= 16, the default plan and at most 16 tiles
 * (2^13 input words each) per SM (SFNTT_WORKLIST_TILES at context creation:
 * another limit, 0 = none) runs its LDE in three
 * phases -- inverse low layers, expansion, forward low layers -- and each
 * phase is ONE persistent launch over all those items: its CTAs pop (item,
 * tile range) units from a work list in device memory (owned by the graph)
 * and keep the next tile's TMA load in flight across item boundaries.  The
 * other items run their own launches on `lanes` forked streams beside the
 * phases.  Outputs are identical to the per-item launches.  (The reference
 * dispatches one grid per layer group per batch, src/ntt/babybear/batch.rs:76-180.) */
int sfntt_batch_persistent_create(sfntt_ctx *ctx, const sfntt_lde_item *items, size_t count, int lanes,
                                  sfntt_graph **out);
int sfntt_graph_launch(sfntt_graph *graph, void *stream);
uint64_t sfntt_graph_kernel_count(const sfntt_graph *graph);
void sfntt_graph_destroy(sfntt_graph *graph);
/* Autotuner: for each distinct key (field, log_n, columns rounded up to a power
 * of two, added_bits) time every plan `reps` times on the first item with that
 * key and keep the fastest for SFNTT_PLAN_AUTO items: the engine (TMA with
 * per-position or four-step strided twiddles, or the non-TMA tile engine),
 * the layer split (SFNTT_PLAN_SPLIT12, where a range exceeds 12 layers) and
 * the CTAs per SM (SFNTT_PLAN_ONE_CTA).  The table is text. */
int sfntt_autotune(sfntt_ctx *ctx, const sfntt_lde_item *items, size_t count, int reps);
int sfntt_tune_save(sfntt_ctx *ctx, const char *path);
int sfntt_tune_load(sfntt_ctx *ctx, const char *path);
int sfntt_tune_lookup(sfntt_ctx *ctx, const sfntt_lde_item *item);

/* Serving (no counterpart in the reference, whose API runs one request per
 * call): a server admits LDE / blow-up requests of any size and either field
 * as they arrive, with continuous batching.  It owns `slots` streams and one
 * device arena of `budget_bytes` (the HBM admission budget, allocated once at
 * creation).  Requests queue in submission order; sfntt_server_poll retires
 * finished ones and admits queued ones, in order, while a slot is free and
 * the arena has room for the request (its output; for host requests its
 * input too), so requests that arrive while others run overlap with them on
 * the device.  Tables stay resident in the context.  Results are exact, so a
 * request gives the same output alone and in any mix.
 *   sfntt_server_submit: input at item->d_in on the device (item->d_out is
 *     ignored; the output lives in the arena until release).
 *   sfntt_server_submit_host: input copied from h_in, output copied to h_out
 *     (pinned memory for asynchronous copies) before the ticket completes.
 * A request larger than the budget fails with SFNTT_ALLOC_FAILED.  BabyBear
 * requests outside the fused LDE (log_n 0 or > 24, added_bits > 4) share the
 * context's scratch and run alone.  A server is driven from one thread. */
typedef struct sfntt_server sfntt_server;
int sfntt_server_create(sfntt_ctx *ctx, size_t budget_bytes, int slots, sfntt_server **out);
void sfntt_server_destroy(sfntt_server *server);
int sfntt_server_submit(sfntt_server *server, const sfntt_lde_item *req, uint64_t *ticket);
int sfntt_server_submit_host(sfntt_server *server, const sfntt_lde_item *req, const uint32_t *h_in,
                             uint32_t *h_out, uint64_t *ticket);
/* Retire finished requests, admit queued ones; writes up to `cap` finished
 * tickets (oldest first; the rest are reported by later polls). */
int sfntt_server_poll(sfntt_server *server, uint64_t *done, size_t cap, size_t *n_done);
/* Device address of a finished request's output (valid until release). */
int sfntt_server_result(sfntt_server *server, uint64_t ticket, uint32_t **d_out);
/* Return a finished request's arena space. */
int sfntt_server_release(sfntt_server *server, uint64_t ticket);
/* Requests queued or running. */
size_t sfntt_server_pending(const sfntt_server *server);
/* Packing (no reference counterpart; the reference encodes many columns of
 * one LDE into one command buffer, src/ntt/babybear/metal_ct_gs_r4.rs:181-246,
 * and this applies it across requests): when the request at the front of the
 * queue launches, up to max_requests - 1 queued requests of the same field,
 * log_n, added_bits, shift and plan that each leave part of the GPU idle join
 * it as further columns of one batch (the front request alone decides
 * admission).  Their inputs are gathered into one arena block (device
 * requests: a device-to-device copy from d_in), one LDE runs over all the
 * columns, and each request's output is its slice of the launch's output.
 * max_requests = 1 (the default) launches every request alone. */
int sfntt_server_set_packing(sfntt_server *server, int max_requests);
/* Launches (alone or packed) the server has admitted. */
uint64_t sfntt_server_launches(const sfntt_server *server);
/* Replay a request trace against the wall clock: request i is submitted
 * arrival_s[i] seconds (sorted) after the start, finished requests are
 * released at once; latency_s[i] = completion seen by the host - arrival.
 * h_in / h_out: per-request host buffers (host requests), or both NULL
 * (device inputs at reqs[i].d_in).  slots = 1 is the plain sequential
 * per-request loop; slots > 1 batches continuously. */
int sfntt_serve_trace(sfntt_ctx *ctx, const sfntt_lde_item *reqs, const uint32_t *const *h_in,
                      uint32_t *const *h_out, const double *arrival_s, size_t count, int slots,
                      size_t budget_bytes, double *latency_s, double *makespan_s);
/* The same with packing (max_pack requests per launch, 1 = none); *launches
 * (optional) receives the number of launches the trace took. */
int sfntt_serve_trace_packed(sfntt_ctx *ctx, const sfntt_lde_item *reqs, const uint32_t *const *h_in,
                             uint32_t *const *h_out, const double *arrival_s, size_t count, int slots,
                             int max_pack, size_t budget_bytes, double *latency_s, double *makespan_s,
                             uint64_t *launches);

/* Allocation-free NTT (no counterpart in the reference).  For callers that
 * cannot allocate device memory when they run a transform (a fixed memory
 * pool, a locked-down allocator, a process that forbids device allocation
 * after start-up): the out-of-place Stockham transform (variant V3), forward
 * or inverse, in place on d_data, with its ping-pong partner in a file-scope
 * device array of 2^20 words (4 MiB, held by every GPU that loads the
 * library).  It calls no cudaMalloc/cudaFree.  Limits: batch << log_n <=
 * 2^20 (else SFNTT_INVALID_SIZE); the twiddles for (field, log_n) must be
 * resident (sfntt_prepare; else SFNTT_INVALID_ARGUMENT).  The first call on a
 * device resolves the array's address (cudaGetSymbolAddress): make it before
 * any stream capture.  The address is cached per device until the process
 * exits, so resetting a device (cudaDeviceReset) while the library is loaded
 * is not supported by this call.  All calls share the array; calls that
 * overlap on the GPU race on it. */
int sfntt_stockham_noalloc(sfntt_ctx *ctx, int field, int inverse, uint32_t *d_data, uint32_t log_n,
                           uint32_t batch, void *stream);

/* Pinned host memory for the host-buffer calls (full-bandwidth copies). */
int sfntt_host_alloc(sfntt_ctx *ctx, size_t bytes, void **out);
int sfntt_host_free(sfntt_ctx *ctx, void *p);

/* Device-side waits (TMA tile arrival) are bounded; a kernel that gives up
 * sets a flag in the context.  Host-memory calls check it and return
 * SFNTT_TIMEOUT; after _dev calls, synchronise the stream and call this. */
int sfntt_check_device_error(sfntt_ctx *ctx);

/* Self-test of the bounded device-side wait (no reference counterpart): runs
 * the tile engine's mbarrier wait on a barrier that nothing arrives on
 * (arrive = 0; returns SFNTT_TIMEOUT after timeout_ns, clamped to 1 us..1 s)
 * or that gets its arrival (arrive = 1; returns SFNTT_OK).  The context stays
 * usable either way. */
int sfntt_selftest_bounded_wait(sfntt_ctx *ctx, uint64_t timeout_ns, int arrive);

/* Number of kernels this library has launched through ctx (for launch counts). */
uint64_t sfntt_launch_count(const sfntt_ctx *ctx);

/* Tracing (the reference only times commit->wait, src/gpu.rs:229-232):
 * sfntt_kernel_timing(ctx, 1) brackets every later launch with CUDA events
 * (and clears earlier records); sfntt_kernel_times synchronises and writes one
 * line per kernel: "<name> <launches> <total_ms> <algorithmic_bytes>\n". */
int sfntt_kernel_timing(sfntt_ctx *ctx, int enable);
int sfntt_kernel_times(sfntt_ctx *ctx, char *buf, size_t len);

/* Measured integer ceiling: radix-2 butterflies per second this GPU sustains
 * with register-resident data (gs = 1: GS on canonical values, the forward
 * butterfly; gs = 0: lazy CT, the inverse one).  The NTT passes are bound by
 * 32-bit integer issue, so the bench reports their fraction of this beside
 * the HBM roofline.  No reference counterpart. */
int sfntt_butterfly_peak(sfntt_ctx *ctx, int gs, double *butterflies_per_s);

#ifdef __cplusplus
}
#endif
#endif /* SFNTT_H */
