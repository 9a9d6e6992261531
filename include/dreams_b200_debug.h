/*
 * dreams_b200_debug.h -- test hooks of libdreams_b200.so (not a production API).
 *
 * No reference counterpart: these expose host-side re-statements of the
 * device algorithms so the planner can be checked on machines without a GPU.
 */
#ifndef DREAMS_B200_DEBUG_H
#define DREAMS_B200_DEBUG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Run the device walk schedule (depth chunks, difference tables, exceptional
 * steps, ordered combine) on the CPU for the first K primes.  axis_params:
 * 4 int64 per program axis.  chunk_steps = 0 means one chunk.  force_interp
 * runs the per-step interpreter schedule instead of the planned class.      */
int dr_debug_sim_walk(const uint8_t *blob, uint64_t size, int32_t K, uint64_t depth,
                      uint64_t checkpoint, const int64_t *axis_params, int32_t pcf_init,
                      int64_t a0, uint32_t q_row, uint64_t chunk_steps, int32_t force_interp,
                      uint32_t *p_out, uint32_t *q_out, uint32_t *cp_p_out, uint32_t *cp_q_out);

/* Difference-table depth of the compiled kernel the engine uses for a
 * (class, m, degree) program, or -1 when it runs on the interpreter. */
int dr_debug_template_degree(int32_t cls, int32_t m, int32_t degree);

/* Integer-pipe issue peaks on the current device, lane-instructions per
 * second: kind 0 wide multiply-add (mad.wide.u32), 1 add+min, 2 their 1:2
 * mix, 3 low multiply-add (mad.lo.u32), 4 unsigned min.  The denominators of
 * the walk kernels' per-pipe roofline. */
int dr_bench_int_peak(int32_t kind, double *lane_ops_per_s);

/* One uncaptured run of a prepared batch with its launch groups concurrent
 * as in dr_batch_run; the kernels stamp the global timer when their first
 * block starts and their last block ends.  spans: 4 floats per launch group
 * (dr_batch_profile's order): [start, end, start2, end2] in ms after the
 * earliest start; start2/end2 belong to the chain kernel of an interpreted
 * shadow group; -1 where a kernel did not run. */
int dr_debug_batch_timeline(int32_t batch, int32_t max_launches, int32_t *n_launches,
                            float *spans);

/* The chain items of the shadow launches (32 walks on one warp each) from the
 * last dr_debug_batch_timeline of the batch: 6 floats per item, [launch group,
 * start, difference tables built (integer-difference chains) or state loaded
 * (interpreted chains), end, chunks re-run exactly, exact single steps
 * (integer-difference) or exact chunks (interpreted)], times in ms on the
 * timeline's scale. */
int dr_debug_chain_items(int32_t batch, int32_t max_items, int32_t *n_items, float *rows);

/* Exercises the host thread pool the batch build runs on: `repeats` jobs
 * over [0, n) with 1..parts parts each; every index must be visited exactly
 * once per job (else DR_ERR_INDEX).  index_sum and visits receive the
 * totals over all jobs.  Needs no GPU. */
int dr_debug_host_pool(int32_t parts, uint64_t n, int32_t repeats, uint64_t *index_sum,
                       uint64_t *visits);

/* *debug_checks = 1 in a DR_DEBUG build (libdreams_b200_debug.so, built by
 * `python dreams-rns-cuda_b200/build.py --debug`), else 0.  A DR_DEBUG build
 * re-checks on the device every index a walk tile takes from its batch's
 * tables (walk, program, group, chunk slot, prime block, outputs, and each
 * bytecode operand against its register, constant, axis and output rows)
 * before using it; the first failure is recorded, the tile is skipped, and
 * the next read of the batch returns DR_ERR_INDEX naming the site, index
 * and bound.  No reference counterpart (the reference has no checks). */
int dr_debug_build_info(int32_t *debug_checks);

/* Host milliseconds (cumulative from the start) at the end of each phase of
 * the calling thread's last dr_batch_create (13 values): plan lookup, program descriptors,
 * code copy, walk validation, workload shape, tile count, tile fill, tile
 * order, shadow lists, launch geometry, table copy, buffers and events,
 * final synchronisation. */
int dr_debug_build_phases(double *ms, int32_t n);

/* Latency floor of the FP64 shadow chain for m = 2: one warp runs `steps`
 * (>= 8) companion fast steps on step matrices computed in registers, so
 * only the step's own dependency chain is timed (best of three launches,
 * CUDA events).  ns_per_step receives the time per step. */
int dr_bench_chain_step(int32_t steps, double *ns_per_step);

/* The FP64 shadow's rescale division on the device: out[i] = x[i] / b[i]
 * rounded to nearest through the same code path the shadow kernels use
 * (Markstein correction, IEEE fallback).  Host buffers; b[i] > 1e10. */
int dr_debug_rescale(const double *x, const double *b, int32_t n, double *out);

/* The serving scheduler's record of its wave launches (first 65536): 12
 * doubles per launch -- selection, launch issued and harvest times (ms after
 * dr_serve_open), device ms from the first upload to the last output copy,
 * requests, long-request wave (0/1), wave slot, walk tiles, longest shadow
 * segment (steps), then the times (ms after dr_serve_open) at which the
 * wave's host build finished its tables and launch geometry, its buffer
 * allocation and upload, and its kernel launches.  n_waves receives the
 * number recorded. */
int dr_debug_serve_waves(int32_t server, int32_t max_waves, int32_t *n_waves, double *rows);

/* Host-side fault injection in the serving loop (no GPU fault is involved):
 * DR_INJECT_ADMIT_NOMEM makes the next `count` admissions fail as if
 * allocating the request's resident state had failed; DR_INJECT_WAVE_NOMEM
 * makes the next `count` wave launches fail as if growing their device
 * buffers had failed.  Each affected request ends with DR_ERR_NOMEM from
 * dr_serve_poll, keeps no slots or admitted bytes, and the server goes on
 * with the others.  kind 0 changes nothing.  *failed (may be NULL) receives
 * the number of requests that have ended with an error of their own.     */
#define DR_INJECT_ADMIT_NOMEM 1
#define DR_INJECT_WAVE_NOMEM  2
int dr_debug_serve_inject(int32_t server, int32_t kind, int32_t count, uint64_t *failed);

#ifdef __cplusplus
}
#endif
#endif /* DREAMS_B200_DEBUG_H */
