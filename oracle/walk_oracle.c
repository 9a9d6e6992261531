/*
 * Plain-C restatement of the reference RNS walk (TEST INFRASTRUCTURE ONLY).
 *
 * Same per-step semantics as the reference numpy engine, one prime at a time:
 *   - bytecode interpreter: reference python/dreams_rns/runner.py:198-260 and
 *     cmf_walk.py:193-258 (registers reset to 0 every step, INV = a^(p-2),
 *     LOAD_X = (sn*td + s*tn*sd) * inv(sd*td) mod p, LOAD_N = s mod p);
 *   - P <- P * M mod p: runner.py:321-333, cmf_walk.py:174-188;
 *   - float64 shadow: runner.py:263-316 and 394-398 (numpy's m x m matmul
 *     accumulates c = a0*b0 then c = fma(ak, bk, c); max |P| > 1e10 rescale).
 * Only the tests and the benchmark's CPU legs load this file's library.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { NOP, LOAD_X, LOAD_C, LOAD_N, ADD, SUB, MUL, NEG, POW2, POW3, INV, STORE, END };

typedef struct { uint32_t op, a0, a1, a2; } insn_t;

static int64_t mod_i128(__int128 v, int64_t p) {
    __int128 r = v % p;
    return (int64_t)(r < 0 ? r + p : r);
}

static uint64_t powmod(uint64_t b, uint64_t e, uint64_t p) {
    uint64_t r = 1 % p;
    b %= p;
    while (e) {
        if (e & 1) r = (uint64_t)((unsigned __int128)r * b % p);
        b = (uint64_t)((unsigned __int128)b * b % p);
        e >>= 1;
    }
    return r;
}

/* Parsed view of a program blob (reference compiler.py:53-89). */
typedef struct {
    uint32_t m, dim, n_ops, n_consts;
    const insn_t *ops;
    const int64_t *consts;
    const int32_t *dirs;
} prog_t;

static int parse(const uint8_t *blob, size_t len, prog_t *p) {
    if (len < 16) return -1;
    const uint32_t *h = (const uint32_t *)blob;
    p->m = h[0]; p->dim = h[1]; p->n_ops = h[2]; p->n_consts = h[3];
    size_t need = 16 + 16 * (size_t)p->n_ops + 8 * (size_t)p->n_consts + 4 * (size_t)p->dim;
    if (len < need || p->m < 1 || p->m > 16) return -1;
    p->ops = (const insn_t *)(blob + 16);
    p->consts = (const int64_t *)(blob + 16 + 16 * (size_t)p->n_ops);
    p->dirs = (const int32_t *)(blob + 16 + 16 * (size_t)p->n_ops + 8 * (size_t)p->n_consts);
    return 0;
}

#define MAXR 512

/* One past the highest register index the program names (operands the
 * interpreter reads or writes), so a step clears only those registers.
 * Clearing all MAXR registers, as the reference allocates them
 * (runner.py:217), gives the same values.  0 = some index is >= MAXR (the
 * reference's register list raises IndexError there). */
static uint32_t reg_span(const prog_t *pr) {
    uint32_t hi = 1;
    for (uint32_t pc = 0; pc < pr->n_ops; ++pc) {
        const insn_t in = pr->ops[pc];
        uint32_t r[3] = {0, 0, 0};
        switch (in.op) {
        case LOAD_X: case LOAD_C: r[0] = in.a1; break;
        case LOAD_N: r[0] = in.a0; break;
        case ADD: case SUB: case MUL: r[0] = in.a0; r[1] = in.a1; r[2] = in.a2; break;
        case NEG: case POW2: case POW3: case INV: r[0] = in.a0; r[1] = in.a1; break;
        case STORE: r[0] = in.a0; break;
        default: break;
        }
        for (int i = 0; i < 3; ++i) {
            if (r[i] >= MAXR) return 0;   /* out of range: the caller reports it */
            if (r[i] + 1 > hi) hi = r[i] + 1;
        }
    }
    return hi;
}

/* Residue walk for one prime.  axis: 4 int64 per axis (sn, sd, tn, td).
 * init: m*m int64 initial matrix.  Writes the full final P (m*m) into out. */
static int walk_prime(const prog_t *pr, uint64_t p, int64_t depth, const int64_t *axis,
                      const int64_t *init, uint64_t *out) {
    const int m = (int)pr->m;
    uint64_t P[256], M[256], C[256];
    uint64_t regs[MAXR];
    uint64_t inv_cd[64], cst[1024];
    if (pr->dim > 64 || pr->n_consts > 1024) return -2;
    for (uint32_t a = 0; a < pr->dim; ++a) {
        __int128 cd = (__int128)axis[4 * a + 1] * axis[4 * a + 3];
        inv_cd[a] = (cd == 1) ? 1 : powmod((uint64_t)mod_i128(cd, (int64_t)p), p - 2, p);
    }
    for (uint32_t i = 0; i < pr->n_consts; ++i) cst[i] = (uint64_t)mod_i128(pr->consts[i], (int64_t)p);
    for (int i = 0; i < m * m; ++i) P[i] = (uint64_t)mod_i128(init[i], (int64_t)p);
    const uint32_t nr = reg_span(pr);
    if (!nr) return -3;
    for (int64_t s = 0; s < depth; ++s) {
        memset(regs, 0, sizeof(uint64_t) * nr);   /* fresh zero registers every step */
        memset(M, 0, sizeof(uint64_t) * m * m);
        for (uint32_t pc = 0; pc < pr->n_ops; ++pc) {
            const insn_t in = pr->ops[pc];
            if (in.op == END) break;
            switch (in.op) {
            case LOAD_X: {
                if (in.a0 >= pr->dim || in.a1 >= MAXR) return -3;
                const int64_t *ax = axis + 4 * in.a0;
                __int128 k = (__int128)ax[0] * ax[3] + (__int128)s * ax[2] * ax[1];
                regs[in.a1] = (uint64_t)((unsigned __int128)mod_i128(k, (int64_t)p) * inv_cd[in.a0] % p);
                break;
            }
            case LOAD_C:
                if (in.a0 >= pr->n_consts || in.a1 >= MAXR) return -3;
                regs[in.a1] = cst[in.a0];
                break;
            case LOAD_N:
                if (in.a0 >= MAXR) return -3;
                regs[in.a0] = (uint64_t)(s % (int64_t)p);
                break;
            case ADD: regs[in.a2] = (regs[in.a0] + regs[in.a1]) % p; break;
            case SUB: regs[in.a2] = (regs[in.a0] + p - regs[in.a1]) % p; break;
            case MUL: regs[in.a2] = regs[in.a0] * regs[in.a1] % p; break;
            case NEG: regs[in.a1] = (p - regs[in.a0]) % p; break;
            case POW2: regs[in.a1] = regs[in.a0] * regs[in.a0] % p; break;
            case POW3: regs[in.a1] = regs[in.a0] * regs[in.a0] % p * regs[in.a0] % p; break;
            case INV: regs[in.a1] = powmod(regs[in.a0], p - 2, p); break;
            case STORE:
                if (in.a1 >= (uint32_t)m || in.a2 >= (uint32_t)m) return -3;
                M[in.a1 * m + in.a2] = regs[in.a0] % p;
                break;
            default: break;
            }
        }
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) {
                uint64_t acc = 0;
                for (int k = 0; k < m; ++k) acc = (acc + P[i * m + k] * M[k * m + j]) % p;
                C[i * m + j] = acc;
            }
        memcpy(P, C, sizeof(uint64_t) * m * m);
    }
    memcpy(out, P, sizeof(uint64_t) * m * m);
    return 0;
}

/* Float64 shadow for one walk.  out: p_f, q_f, log_scale. */
static int walk_shadow(const prog_t *pr, int64_t depth, const int64_t *axis, const int64_t *init,
                       int prow, int qrow, double *out) {
    const int m = (int)pr->m;
    double P[256], M[256], C[256], regs[MAXR];
    double log_scale = 0.0;
    const uint32_t nr = reg_span(pr);
    if (!nr) return -3;
    for (int i = 0; i < m * m; ++i) P[i] = (double)init[i];
    for (int64_t s = 0; s < depth; ++s) {
        memset(M, 0, sizeof(double) * m * m);
        for (uint32_t r = 0; r < nr; ++r) regs[r] = 0.0;
        for (uint32_t pc = 0; pc < pr->n_ops; ++pc) {
            const insn_t in = pr->ops[pc];
            if (in.op == END) break;
            switch (in.op) {
            case LOAD_X: {
                const int64_t *ax = axis + 4 * in.a0;
                __int128 k = (__int128)ax[0] * ax[3] + (__int128)s * ax[2] * ax[1];
                regs[in.a1] = (double)k / (double)((__int128)ax[1] * ax[3]);
                break;
            }
            case LOAD_C: regs[in.a1] = (double)pr->consts[in.a0]; break;
            case LOAD_N: regs[in.a0] = (double)s; break;
            case ADD: regs[in.a2] = regs[in.a0] + regs[in.a1]; break;
            case SUB: regs[in.a2] = regs[in.a0] - regs[in.a1]; break;
            case MUL: regs[in.a2] = regs[in.a0] * regs[in.a1]; break;
            case NEG: regs[in.a1] = -regs[in.a0]; break;
            case POW2: regs[in.a1] = pow(regs[in.a0], 2.0); break;
            case POW3: regs[in.a1] = pow(regs[in.a0], 3.0); break;
            case INV: regs[in.a1] = fabs(regs[in.a0]) > 1e-300 ? 1.0 / regs[in.a0] : 0.0; break;
            case STORE: M[in.a1 * m + in.a2] = regs[in.a0]; break;
            default: break;
            }
        }
        double mx = 0.0;
        int has_nan = 0;   /* np.max propagates NaN, and NaN > 1e10 is false */
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) {
                double c = P[i * m] * M[j];
                for (int k = 1; k < m; ++k) c = fma(P[i * m + k], M[k * m + j], c);
                C[i * m + j] = c;
                double a = fabs(c);
                if (isnan(a)) has_nan = 1;
                else if (a > mx) mx = a;
            }
        memcpy(P, C, sizeof(double) * m * m);
        if (!has_nan && mx > 1e10) {
            for (int i = 0; i < m * m; ++i) P[i] /= mx;
            log_scale += log(mx);
        }
    }
    out[0] = P[prow * m + m - 1];
    out[1] = P[qrow * m + m - 1];
    out[2] = log_scale;
    return 0;
}

/*
 * oracle_walk: residues of P[prow][m-1] and P[qrow][m-1] after ``depth`` steps
 * for each of the K primes, and optionally the float shadow.
 * Returns 0, or a negative code for a malformed program.
 */
typedef struct {
    const prog_t *pr;
    const uint32_t *primes;
    int K, prow, qrow, first, step;
    int64_t depth;
    const int64_t *axis, *init;
    uint32_t *p_out, *q_out;
    int rc;
} prime_job_t;

static void *prime_worker(void *arg) {
    prime_job_t *j = (prime_job_t *)arg;
    uint64_t P[256];
    const int m = (int)j->pr->m;
    j->rc = 0;
    for (int k = j->first; k < j->K; k += j->step) {
        int rc = walk_prime(j->pr, j->primes[k], j->depth, j->axis, j->init, P);
        if (rc) { j->rc = rc; return NULL; }
        j->p_out[k] = (uint32_t)P[j->prow * m + m - 1];
        j->q_out[k] = (uint32_t)P[j->qrow * m + m - 1];
    }
    return NULL;
}

/*
 * oracle_walk_mt: oracle_walk with the primes spread over `threads` POSIX
 * threads (prime k on thread k mod threads; every prime's walk is
 * independent, so the outputs do not depend on the thread count).
 */
int oracle_walk_mt(const uint8_t *blob, uint64_t blob_len, int K, const uint32_t *primes,
                   int64_t depth, const int64_t *axis, const int64_t *init, int prow, int qrow,
                   uint32_t *p_out, uint32_t *q_out, double *shadow_out, int threads) {
    prog_t pr;
    if (parse(blob, (size_t)blob_len, &pr)) return -1;
    if (threads < 1) threads = 1;
    if (threads > K) threads = K > 0 ? K : 1;
    if (threads > 256) threads = 256;
    prime_job_t jobs[256];
    pthread_t tids[256];
    int started[256];
    for (int t = 0; t < threads; ++t) {
        jobs[t] = (prime_job_t){&pr, primes, K, prow, qrow, t, threads, depth, axis, init,
                                p_out, q_out, 0};
        started[t] = (t > 0) && pthread_create(&tids[t], NULL, prime_worker, &jobs[t]) == 0;
        if (t > 0 && !started[t]) prime_worker(&jobs[t]);   /* no thread: run it here */
    }
    int rc_sh = 0;
    if (shadow_out) rc_sh = walk_shadow(&pr, depth, axis, init, prow, qrow, shadow_out);
    prime_worker(&jobs[0]);
    int rc = 0;
    for (int t = 0; t < threads; ++t) {
        if (started[t]) pthread_join(tids[t], NULL);
        if (!rc && jobs[t].rc) rc = jobs[t].rc;
    }
    return rc ? rc : rc_sh;
}

int oracle_walk(const uint8_t *blob, uint64_t blob_len, int K, const uint32_t *primes,
                int64_t depth, const int64_t *axis, const int64_t *init, int prow, int qrow,
                uint32_t *p_out, uint32_t *q_out, double *shadow_out) {
    return oracle_walk_mt(blob, blob_len, K, primes, depth, axis, init, prow, qrow, p_out, q_out,
                          shadow_out, 1);
}
