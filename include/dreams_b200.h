/*
 * dreams_b200.h -- C ABI of the B200 RNS walk engine (libdreams_b200.so).
 *
 * Plain C types only: pointers, sizes, status codes.  Every function returns
 * an int status (DR_OK = 0, negative = error; see dr_strerror).  Functions
 * named *_device take device pointers and a CUDA stream passed as void*;
 * all others take host pointers and synchronise before returning.
 *
 * The reference has no native ABI for this path (its C++ declarations in
 * include/dreams/walk_kernel.h:51-61 are never defined or exported, and its
 * only working engine is Python: python/dreams_rns/runner.py).  Each entry
 * point below names the reference function whose behaviour it provides.
 */
#ifndef DREAMS_B200_H
#define DREAMS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define DR_OK                 0
#define DR_ERR_CUDA          -1   /* CUDA runtime error (message: dr_last_error) */
#define DR_ERR_ARG           -2   /* bad argument (null pointer, size)        */
#define DR_ERR_BLOB          -3   /* malformed program blob (truncated)       */
#define DR_ERR_OPCODE        -4   /* unknown opcode (reference: ValueError)   */
#define DR_ERR_INDEX         -5   /* register/constant/axis/entry index out of
                                     range (reference: IndexError)            */
#define DR_ERR_UNSUPPORTED   -6   /* outside this engine's limits (m, K, dim)  */
#define DR_ERR_NOMEM         -7   /* device memory exhausted / admission cap   */
#define DR_ERR_NOT_INIT      -8   /* dr_init not called                        */
#define DR_ERR_HANDLE        -9   /* unknown batch / server / request handle   */
#define DR_ERR_TIMEOUT      -10   /* a bounded wait expired                    */
#define DR_ERR_MODULUS      -11   /* CRT modulus outside odd [3, 2^31)         */
#define DR_ERR_BUSY         -12   /* request not finished yet (poll again)     */

/* ---- limits --------------------------------------------------------------- */
#define DR_MAX_M        8        /* matrix size (reference config.h MAX_M)     */
#define DR_MAX_AXES     8        /* axes per program (config.h MAX_AXES)       */
#define DR_MAX_K        8192     /* primes per walk                            */
#define DR_MAX_REGS     512      /* virtual registers (compiler.py MAX_REGS)   */

/* ---- walk descriptor ------------------------------------------------------
 * One walk: P = P0 * M(s0) * ... * M(depth-1), residues mod the first K primes
 * of dr_prime_table.  The step matrix M(s) is the program's bytecode evaluated
 * at 0-based step s, where LOAD_X of axis a yields
 *     (sn_a*td_a + s*tn_a*sd_a) * inv(sd_a*td_a)  (mod p)
 * with (sn, sd, tn, td) = axis_params[axis_offset + 4a .. +3]
 * (reference cmf_walk.py:221-224; the PCF walk is sn = shift, tn = direction,
 * sd = td = 1, runner.py:225-227).
 * Outputs: p = P[p_row][m-1], q = P[q_row][m-1] (PCF: q_row = 1, runner.py:401-402;
 * CMF: q_row = m-1, cmf_walk.py:419-420) written to
 * p_res[res_offset + k], q_res[res_offset + k] for k < K.  With a non-zero
 * checkpoint the same outputs after `checkpoint` steps go to
 * cp_res_offset.  The FP64 shadow (p_float, q_float, log_scale) goes to
 * shadow[3*w], and shadow[3*(n_walks + w)] for the checkpoint.            */
#define DR_WALK_INIT_PCF   0x1u   /* P0 = [[1, a0], [0, 1]], else P0 = I     */
#define DR_WALK_SHADOW     0x2u   /* compute the FP64 shadow                  */
#define DR_WALK_VEC        0x4u   /* state-vector walk (reference cmf_walk.py:445-531):
                                     v(depth) = M(depth-1) ... M(0) v(0); p = v[p_row],
                                     q = v[q_row].  v(0) sits in axis_params at
                                     vec_offset: m*K residues (entry i for prime k at
                                     vec_offset + i*K + k, each in [0, p_k)) then the
                                     m doubles of the float v(0) as int64 bit patterns.
                                     No checkpoint, no DR_WALK_INIT_PCF.          */

typedef struct dr_walk_desc {
    uint32_t program;       /* index into the program blob list              */
    uint32_t K;             /* number of primes, 1..DR_MAX_K                  */
    uint64_t depth;         /* steps                                          */
    uint64_t checkpoint;    /* 0 = none, else 0 < checkpoint < depth          */
    int64_t  a0;            /* PCF initial value a(0)                         */
    uint32_t flags;         /* DR_WALK_*                                      */
    uint32_t q_row;         /* row of q in the last column                    */
    uint64_t axis_offset;   /* index of this walk's first axis parameter     */
    uint64_t res_offset;    /* residue output offset                         */
    uint64_t cp_res_offset; /* checkpoint residue output offset              */
    uint32_t p_row;         /* row of p in the last column (0 for the reference's
                               walks; DR_WALK_VEC: state entry of p)          */
    uint32_t reserved;
    uint64_t vec_offset;    /* DR_WALK_VEC: index of v(0) in axis_params      */
} dr_walk_desc;

/* walk status bits (status_out[w]) */
#define DR_STATUS_INV0        0x1u  /* some INV met 0 (returned 0; reference
                                       config.h:166-169 "dead lane")         */
#define DR_STATUS_SHADOW_NAN  0x2u  /* shadow became non-finite               */
#define DR_STATUS_FALLBACK    0x4u  /* walk ran on the per-step interpreter   */
#define DR_STATUS_CRT_OVERFLOW    0x8u  /* device pipeline: the CRT value of p/q
                                           disagrees with the FP64 shadow's
                                           p_float/q_float by more than 1% (K too
                                           small; reference euler2ai_full_verify.py
                                           :152-167 crt_overflowed)               */
#define DR_STATUS_CP_CRT_OVERFLOW 0x10u /* the same for the checkpoint values      */

/* engine selection for dr_walk_batch */
#define DR_ENGINE_AUTO    0   /* planned fast path (difference tables), else
                                 the per-step interpreter                    */
#define DR_ENGINE_INTERP  1   /* per-step bytecode interpreter, chunked      */
#define DR_ENGINE_PLAIN   2   /* the baseline path: the same per-class step
                                 code as AUTO, but no depth chunks and no
                                 persistent grid -- one single-warp block per
                                 (walk, block of 32 primes) runs the whole
                                 depth; a batch of one walk is one walk per
                                 launch (K/32 warps)                         */

typedef struct dr_tune {
    uint32_t chunk_steps;     /* depth-chunk length; 0 = autotuned           */
    uint32_t warps_per_block; /* 0 = default                                  */
    uint32_t engine;          /* DR_ENGINE_*                                  */
    uint32_t shadow_buffer_mb;/* cap of the interpreted shadow's step-matrix
                                 buffer per launch group; 0 = default
                                 (2048); walks beyond it run their shadow in
                                 rounds with resident state                 */
    uint32_t chain_pack_depth;/* integer-difference shadow launches of
                                 difference depth <= this run two chain warps
                                 per scheduler (8 per SM instead of 4): each
                                 chain is slower, but the walks get their SMs;
                                 0 = the autotuned choice for the workload's
                                 shape, else none                           */
} dr_tune;

/* ---- context ---------------------------------------------------------- */
int dr_init(int device);
const char *dr_strerror(int status);
const char *dr_last_error(void);
int dr_version(void);

/* The first K primes below 2^31 in descending order (reference
 * runner.py:33-52 generate_rns_primes). */
int dr_prime_table(int K, uint32_t *out);

/* Per-stage timers of the calls below, summed since the last reset (no
 * reference counterpart; the reference only prints wall-clock rates):
 * ms_out[0] host batch build (planning, tiles, launch geometry), [1]
 * allocation and upload, [2] run (enqueue; the wait as well in
 * dr_walk_batch), [3] read-back, [4] device milliseconds of the batch runs
 * read back (CUDA events).  calls_out (may be NULL) counts each stage's
 * entries.  Fills min(n, 5) entries; reset != 0 zeroes the sums after
 * reading them.  The stages are also NVTX ranges ("dr.build", "dr.upload",
 * "dr.run", "dr.read", "dr.serve.wave") for a profiler's timeline.          */
#define DR_STAGE_COUNT 5
int dr_stage_times(double *ms_out, uint64_t *calls_out, int32_t n, int32_t reset);

/* Validate a program blob (reference compiler.py:64-89 layout) and report how
 * the engine will run it: *cls_out = 1 companion polynomial, 2 companion
 * rational, 3 dense polynomial, 4 per-step interpreter; *degree_out = degree
 * of the step matrix in the step index (difference-table depth). */
int dr_program_info(const uint8_t *blob, uint64_t size, int32_t *cls_out,
                    int32_t *degree_out, int32_t *n_regs_out);

/* ---- walks ------------------------------------------------------------
 * Batch of walks, host buffers (reference runner.py:338-413 run_pcf_walk and
 * cmf_walk.py:363-431 run_cmf_walk, one dict per walk).  blobs: all program
 * blobs back to back, blob_offsets[n_programs + 1].  tune may be NULL.     */
int dr_walk_batch(const dr_walk_desc *walks, int32_t n_walks,
                  const uint8_t *blobs, const uint64_t *blob_offsets, int32_t n_programs,
                  const int64_t *axis_params, uint64_t n_axis_params,
                  const dr_tune *tune,
                  uint32_t *p_res, uint32_t *q_res, uint64_t n_res,
                  double *shadow, uint32_t *status);

/* ---- prepared batches (inputs resident on the device) -------------------
 * dr_batch_create uploads programs and descriptors once; dr_batch_run runs
 * walk -> CRT -> delta -> top-k entirely on the device (the first run
 * launches directly, the second captures a CUDA graph that later runs
 * replay); dr_batch_read copies results to the host.                        */
int dr_batch_create(const dr_walk_desc *walks, int32_t n_walks,
                    const uint8_t *blobs, const uint64_t *blob_offsets, int32_t n_programs,
                    const int64_t *axis_params, uint64_t n_axis_params,
                    const dr_tune *tune, int32_t *batch_out);
int dr_batch_run(int32_t batch, void *stream);
/* A non-blocking CUDA stream for dr_batch_run, owned by the caller.  No
 * reference counterpart (the reference runs one batch at a time).  Batch
 * builds order their uploads on the engine's own stream and wait for it, so
 * runs of batches built while others are running belong on a stream like this
 * one (dreams_rns.sweep_many). */
int dr_stream_create(void **stream_out);
int dr_stream_destroy(void *stream);
int dr_batch_read(int32_t batch, uint32_t *p_res, uint32_t *q_res, uint64_t n_res,
                  double *shadow, uint32_t *status);
int dr_batch_stats(int32_t batch, uint64_t *prime_steps, uint32_t *n_tiles,
                   uint32_t *n_launches, float *last_ms);

/* Device pipeline after the walk, part of every dr_batch_run once set:
 * CRT of p, q (and the checkpoint's p, q) to centred limbs, the Dreams delta
 * (reference runner.py:103-125) and top-k by delta.  DR_DELTA_FIXED scores the
 * final convergent against one target L = lnum_sign * lnum / lden; DR_DELTA_SELF
 * scores the checkpoint convergent against the walk's own final convergent.   */
#define DR_DELTA_NONE   0
#define DR_DELTA_FIXED  1
#define DR_DELTA_SELF   2

typedef struct dr_pipeline {
    int32_t crt;            /* 1: reconstruct on the device                  */
    int32_t delta_mode;     /* DR_DELTA_* (needs crt)                        */
    int32_t topk;           /* 0 = none, else 1..2048                        */
    int32_t l_limbs;        /* limbs of lnum / lden (DR_DELTA_FIXED)         */
    const uint32_t *lnum;   /* |Lnum| little-endian limbs (host pointer)     */
    const uint32_t *lden;   /* Lden limbs, > 0 (host pointer)                */
    int32_t lnum_sign;
    int32_t reserved;
} dr_pipeline;

int dr_batch_set_pipeline(int32_t batch, const dr_pipeline *pl);
/* Constant bank (reference constants.py:182-207 compute_delta_against_constant
 * for every registry constant): with a device pipeline set, each run also
 * scores the final p/q of every top-k hit (or, with no top-k, of every walk)
 * against n_consts targets C_j = sign_j * num_j / den_j (limbs little-endian,
 * l_limbs each, num and den rows of one array each, den > 0).  n_consts = 0
 * removes it.  dr_batch_read_bank returns delta[hit or walk][constant].      */
int dr_batch_set_bank(int32_t batch, int32_t n_consts, int32_t l_limbs, const uint32_t *num,
                      const int32_t *num_sign, const uint32_t *den);
int dr_batch_read_bank(int32_t batch, double *delta, int32_t max_values);
/* delta[n_walks]; topk_idx/topk_val[k]; limbs[4*n_walks][limb_stride] with rows
 * 4w+0 p, 4w+1 q, 4w+2 checkpoint p, 4w+3 checkpoint q and signs[4*n_walks].
 * Any output may be NULL. */
int dr_batch_read_pipeline(int32_t batch, double *delta, int32_t *topk_idx, double *topk_val,
                           uint32_t *limbs, int32_t *signs, int32_t limb_stride);
int dr_batch_destroy(int32_t batch);

/* Autotuner: builds the given walks with candidate depth-chunk lengths and
 * warps per block around the built-in policy, times each as a graph replay
 * (best of three, CUDA events), and returns the fastest in *best (its engine
 * and shadow_buffer_mb fields are inputs); a candidate replaces the built-in
 * policy only when it is at least 2% faster, since shorter chunks cost host
 * build time on every batch.  With the chosen shape it then tries packing
 * the integer-difference shadow chains of depth <= 1, 2, 3, 4 or 16 two
 * warps per scheduler (chain_pack_depth) and keeps the fastest when it is
 * at least 1% faster than no packing (packing costs the host nothing).
 * The choice is remembered for the workload's shape (per launch class:
 * log2 of the (walk, prime block) count and of their steps, longest walk),
 * so later batches of that shape built with a zero chunk_steps and
 * warps_per_block use it.  No reference counterpart (the reference fixes its
 * launch shape, persistent_kernel.cu:877-888). */
int dr_autotune(const dr_walk_desc *walks, int32_t n_walks, const uint8_t *blobs,
                const uint64_t *blob_offsets, int32_t n_programs, const int64_t *axis_params,
                uint64_t n_axis_params, dr_tune *best, float *best_ms);

/* Where a batch's time goes: runs every launch group of the batch alone, one
 * after another, timing each with CUDA events (walk kernels: kind 0; FP64
 * shadow: kind 1 interpreted, kind 2 integer differences).  ms: the launch
 * (kind 1: its step-matrix evaluation), ms2: kind 1's chain kernel.  degree:
 * the difference depth (kind 1: that of a split shadow's integer-difference
 * head, 0 for a plain interpreted shadow).  No reference counterpart (the
 * reference has no profiling hooks). */
int dr_batch_profile(int32_t batch, int32_t max_launches, int32_t *n_launches, int32_t *kind,
                     int32_t *cls, int32_t *m, int32_t *degree, uint32_t *items, float *ms,
                     float *ms2);

/* ---- CRT (reference runner.py:57-81 crt_reconstruct + centered) --------
 * residues[i*K + k] mod moduli[k] for n values.  Outputs the centred value
 * x - M if x > M/2 else x, where x in [0, M) is the reference's CRT result,
 * as sign (+1, -1 or 0) and magnitude limbs (little-endian u32,
 * limbs[i*limb_stride ..]), nlimbs_out[i] = significant limbs.  The reference
 * result x itself is available as unsigned limbs (unsigned_limbs != NULL).
 * moduli must be odd in [3, 2^31); NULL selects dr_prime_table(K).
 * limb_stride >= ceil(31*K/32) + 1.                                          */
int dr_crt_batch(const uint32_t *residues, int32_t K, int32_t n, const uint32_t *moduli,
                 uint32_t *limbs, int32_t limb_stride, int32_t *sign_out,
                 int32_t *nlimbs_out, uint32_t *unsigned_limbs);
int dr_crt_batch_device(const uint32_t *residues_d, int32_t K, int32_t n,
                        const uint32_t *moduli_d, uint32_t *limbs_d, int32_t limb_stride,
                        int32_t *sign_d, int32_t *nlimbs_d, void *stream);

/* Allocation-free variant of dr_crt_batch_device for callers that cannot call
 * cudaMalloc (code running under an allocator that owns all device memory, or
 * that must avoid the device-wide synchronisation cudaFree implies).  It has
 * no counterpart in the reference.  Moduli are the first K primes of
 * dr_prime_table; outputs are the centred limbs and signs of dr_crt_batch.
 * It allocates nothing: its tables live in a static device array sized for
 * K <= 128 (larger K returns DR_ERR_UNSUPPORTED), which every GPU that loads
 * the library holds until exit.  Every call rebuilds the tables there, so
 * calls that overlap on the GPU race; order them on one stream.  The first
 * call on each device looks up the array's device address (cudaGetSymbolAddress
 * with that device current), so make that first call before any stream
 * capture.  Needs no dr_init.                                                */
int dr_crt_batch_device_noalloc(const uint32_t *residues_d, int32_t K, int32_t n,
                                uint32_t *limbs_d, int32_t limb_stride, int32_t *sign_d,
                                void *stream);

/* ---- delta (reference runner.py:103-125 compute_dreams_delta_exact) -----
 * delta = -(1 + ln|p/q - L| / ln|q|), q = 0 -> -inf, p/q == L -> +inf,
 * |q| <= 1 -> -inf.  p, q: sign + magnitude limbs as produced by dr_crt_batch
 * (stride limb_stride).  L = Lnum / Lden given as sign + limbs (stride
 * l_stride); per_item_target != 0 means item i uses target i, else target 0.  */
int dr_delta_batch(const uint32_t *p_limbs, const int32_t *p_sign, const uint32_t *q_limbs,
                   const int32_t *q_sign, int32_t n, int32_t limb_stride,
                   const uint32_t *lnum_limbs, const int32_t *lnum_sign,
                   const uint32_t *lden_limbs, int32_t l_stride, int32_t per_item_target,
                   double *delta_out);

/* Top-k by delta, highest first, NaN last, ties by lower index (the
 * reference's threshold filter persistent_kernel.cu:796-841 kept no order).
 * k <= 2048.  From 2^18 values on, a threshold taken from a strided sample
 * lets one pass over the values keep only the candidates that can rank, so
 * the values are read once; the result is exact (a count check falls back to
 * sorting every value when the threshold kept too few or too many).       */
int dr_topk(const double *delta, int32_t n, int32_t k, int32_t *idx_out, double *val_out);
/* The same on device memory: delta_d[n] in, idx_d[min(k, n)] and val_d
 * (either may be NULL) out, on `stream` (NULL: the engine's stream); returns
 * after synchronising that stream.  *filtered (may be NULL) = 1 when the
 * threshold filter decided the result.                                     */
int dr_topk_device(const double *delta_d, int32_t n, int32_t k, int32_t *idx_d, double *val_d,
                   void *stream, int32_t *filtered);

/* ---- serving: continuous batching of walk requests ---------------------- */
typedef struct dr_serve_config {
    uint64_t mem_cap_bytes;     /* admission cap on device state (0 = 50% free) */
    uint32_t max_inflight;      /* waves in flight (streams), 0 = 2           */
    uint32_t chunk_steps;       /* yield granularity of long walks, 0 = auto    */
    uint32_t max_wave_tiles;    /* tiles per wave, 0 = auto                      */
    uint32_t reserved[3];
} dr_serve_config;

int dr_serve_open(const dr_serve_config *cfg, int32_t *server_out);
/* Submit one walk (walk->program indexes the single blob given here). */
int dr_serve_submit(int32_t server, const dr_walk_desc *walk, const uint8_t *blob,
                    uint64_t blob_size, const int64_t *axis_params, int64_t *request_out);
/* Non-blocking: DR_OK with results when done, DR_ERR_BUSY otherwise.
 * p_res/q_res hold K entries; shadow 3 doubles; latency in seconds. */
int dr_serve_poll(int32_t server, int64_t request, uint32_t *p_res, uint32_t *q_res,
                  double *shadow, uint32_t *status, double *latency_s);
int dr_serve_cancel(int32_t server, int64_t request);
int dr_serve_stats(int32_t server, uint64_t *completed, uint64_t *prime_steps,
                   uint64_t *admitted_bytes, uint32_t *queue_depth);
int dr_serve_close(int32_t server);

#ifdef __cplusplus
}
#endif
#endif /* DREAMS_B200_H */
