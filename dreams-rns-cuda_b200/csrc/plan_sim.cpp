// Host re-statement of the device walk algorithm, for CPU testing.
//
// Runs exactly the schedule the kernels run -- depth chunks starting from the
// initial matrix (chunk 0) or I, forward-difference streams initialised by
// evaluating the derived program at D+1 steps, the companion / rational /
// dense step product, exceptional steps re-evaluated with the original
// program, and the ordered chunk combine with one division by the
// accumulated denominator -- in plain 64-bit modular arithmetic.  Tests
// compare it with the C oracle so the planner is validated without a GPU.
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dreams_b200.h"
#include "program.h"

namespace dr {
namespace {

uint64_t mulm(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)((unsigned __int128)a * b % p); }
uint64_t powm(uint64_t b, uint64_t e, uint64_t p) {
    uint64_t r = 1;
    b %= p;
    while (e) {
        if (e & 1) r = mulm(r, b, p);
        b = mulm(b, b, p);
        e >>= 1;
    }
    return r;
}
uint64_t modi(__int128 v, uint64_t p) {
    __int128 r = v % (__int128)p;
    return (uint64_t)(r < 0 ? r + p : r);
}

struct Lane {
    uint64_t p;
    std::vector<uint64_t> x0, dx, cst;
};

void eval(const Lane& L, const std::vector<Insn>& ops, uint32_t n_regs, uint64_t s,
          std::vector<uint64_t>& out) {
    std::vector<uint64_t> r(n_regs + 1, 0);
    const uint64_t p = L.p;
    const uint64_t sm = s % p;
    for (const Insn& in : ops) {
        switch (in.op) {
            case OP_LOAD_X: r[in.b] = (L.x0[in.a] + mulm(sm, L.dx[in.a], p)) % p; break;
            case OP_LOAD_C: r[in.b] = L.cst[in.a]; break;
            case OP_LOAD_N: r[in.a] = sm; break;
            case OP_ADD: r[in.c] = (r[in.a] + r[in.b]) % p; break;
            case OP_SUB: r[in.c] = (r[in.a] + p - r[in.b]) % p; break;
            case OP_MUL: r[in.c] = mulm(r[in.a], r[in.b], p); break;
            case OP_NEG: r[in.b] = (p - r[in.a]) % p; break;
            case OP_POW2: r[in.b] = mulm(r[in.a], r[in.a], p); break;
            case OP_POW3: r[in.b] = mulm(mulm(r[in.a], r[in.a], p), r[in.a], p); break;
            case OP_INV: r[in.b] = powm(r[in.a], p - 2, p); break;
            case OP_STORE: out[in.b] = r[in.a]; break;
            default: break;
        }
    }
}

void matmul(std::vector<uint64_t>& P, const std::vector<uint64_t>& M, uint32_t m, uint64_t p) {
    std::vector<uint64_t> C(m * m, 0);
    for (uint32_t i = 0; i < m; ++i)
        for (uint32_t j = 0; j < m; ++j) {
            uint64_t acc = 0;
            for (uint32_t k = 0; k < m; ++k) acc = (acc + mulm(P[i * m + k], M[k * m + j], p)) % p;
            C[i * m + j] = acc;
        }
    P.swap(C);
}

}  // namespace

// One prime: p/q residues after `depth` (and `checkpoint`) steps.
int sim_walk_prime(const Plan& pl, uint64_t p, uint64_t depth, uint64_t checkpoint,
                   const int64_t* axis, int pcf_init, int64_t a0, uint32_t q_row,
                   uint64_t chunk_len, uint64_t* out /* p, q, cp_p, cp_q */) {
    const uint32_t m = pl.m;
    Lane L;
    L.p = p;
    for (uint32_t a = 0; a < pl.dim; ++a) {
        const int64_t* ax = axis + 4 * a;
        uint64_t cd = mulm(modi(ax[1], p), modi(ax[3], p), p);
        uint64_t inv = powm(cd, p - 2, p);
        L.x0.push_back(mulm(mulm(modi(ax[0], p), modi(ax[3], p), p), inv, p));
        L.dx.push_back(mulm(mulm(modi(ax[2], p), modi(ax[1], p), p), inv, p));
    }
    for (int64_t c : pl.consts) L.cst.push_back(modi(c, p));
    if (chunk_len == 0) chunk_len = depth ? depth : 1;

    // chunk boundaries (a checkpoint always ends a chunk)
    std::vector<uint64_t> bounds{0};
    for (uint64_t s = 0; s < depth;) {
        uint64_t e = std::min(depth, s + chunk_len);
        if (checkpoint && s < checkpoint && e > checkpoint) e = checkpoint;
        bounds.push_back(e);
        s = e;
    }
    std::vector<uint64_t> init(m * m, 0);
    for (uint32_t i = 0; i < m; ++i) init[i * m + i] = 1;
    if (pcf_init) init[0 * m + 1] = modi(a0, p);

    const bool fd = pl.cls != CLS_INTERP;
    const uint32_t D = pl.degree;
    const uint32_t ns = pl.n_streams;
    std::vector<uint64_t> P_total = init, sig_total{1};
    uint64_t sig_t = 1;
    bool have_cp = false;
    uint64_t cp_p = 0, cp_q = 0;
    for (size_t c = 0; c + 1 < bounds.size(); ++c) {
        const uint64_t s0 = bounds[c], s1 = bounds[c + 1];
        std::vector<uint64_t> P(m * m, 0);
        for (uint32_t i = 0; i < m; ++i) P[i * m + i] = 1;
        uint64_t sig = 1;
        std::vector<std::vector<uint64_t>> tab(ns, std::vector<uint64_t>(D + 1, 0));
        if (fd) {
            std::vector<uint64_t> vals(ns);
            for (uint32_t j = 0; j <= D; ++j) {
                eval(L, pl.dops, pl.dn_regs, s0 + j, vals);
                for (uint32_t k = 0; k < ns; ++k) tab[k][j] = vals[k];
            }
            for (uint32_t k = 0; k < ns; ++k)
                for (uint32_t lvl = 1; lvl <= D; ++lvl)
                    for (uint32_t j = D; j >= lvl; --j) tab[k][j] = (tab[k][j] + p - tab[k][j - 1]) % p;
        }
        std::vector<uint64_t> M(m * m);
        for (uint64_t s = s0; s < s1; ++s) {
            if (!fd) {
                std::fill(M.begin(), M.end(), 0);
                eval(L, pl.ops, pl.n_regs, s, M);
                matmul(P, M, m, p);
            } else {
                if (pl.cls == CLS_RATIONAL && tab[m][0] == 0) {
                    std::fill(M.begin(), M.end(), 0);
                    eval(L, pl.ops, pl.n_regs, s, M);
                    matmul(P, M, m, p);
                } else {
                    std::fill(M.begin(), M.end(), 0);
                    if (pl.cls == CLS_DENSE) {
                        for (uint32_t k = 0; k < m * m; ++k) M[k] = tab[k][0];
                    } else {
                        const uint64_t g = pl.cls == CLS_RATIONAL ? tab[m][0] : 1;
                        for (uint32_t i = 0; i + 1 < m; ++i) M[(i + 1) * m + i] = g;
                        for (uint32_t i = 0; i < m; ++i) M[i * m + m - 1] = tab[i][0];
                        if (pl.cls == CLS_RATIONAL) sig = mulm(sig, g, p);
                    }
                    matmul(P, M, m, p);
                }
                for (uint32_t k = 0; k < ns; ++k)
                    for (uint32_t j = 0; j < D; ++j) tab[k][j] = (tab[k][j] + tab[k][j + 1]) % p;
            }
        }
        if (c == 0) {
            std::vector<uint64_t> A = init;
            matmul(A, P, m, p);
            P_total = A;
        } else {
            matmul(P_total, P, m, p);
        }
        sig_t = mulm(sig_t, sig, p);
        if (checkpoint && s1 == checkpoint) {
            uint64_t iv = powm(sig_t, p - 2, p);
            cp_p = mulm(P_total[0 * m + m - 1], iv, p);
            cp_q = mulm(P_total[q_row * m + m - 1], iv, p);
            have_cp = true;
        }
    }
    uint64_t iv = powm(sig_t, p - 2, p);
    out[0] = mulm(P_total[0 * m + m - 1], iv, p);
    out[1] = mulm(P_total[q_row * m + m - 1], iv, p);
    out[2] = have_cp ? cp_p : 0;
    out[3] = have_cp ? cp_q : 0;
    return DR_OK;
}

}  // namespace dr
