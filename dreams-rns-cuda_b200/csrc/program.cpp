// Program parsing, validation, register compaction and the step-matrix planner.
//
// The planner evaluates the bytecode symbolically once per program.  Every
// register value is tracked as a fraction N / prod(g_k^e_k) whose numerator N
// and "atoms" g_k are INV-free polynomials in the step index s (axis values
// are affine in s).  INV of a step-dependent value creates an atom.  From the
// final matrix it derives polynomial "streams" whose values at every step can
// be advanced by forward differences (D additions per stream and step instead
// of re-running the bytecode), and picks an execution class:
//
//   COMPANION  sub-diagonal exactly 1, other non-last columns exactly 0, no
//              atoms: streams are the last-column entries.
//   RATIONAL   same shape with atoms: with g = prod(atoms^E), the walk uses
//              M' = g*M (polynomial) and accumulates g, dividing once at the
//              end.  Steps where some atom is 0 mod p (the reference's INV(0)
//              -> 0 case) are detected through g == 0 and re-evaluated with the
//              plain interpreter, so results stay bit-identical.
//   DENSE      any shape, no atoms: every entry is a stream.
//   INTERP     everything else: the bytecode is interpreted every step.
#include "program.h"

#include <algorithm>
#include <array>
#include <tuple>
#include <cmath>
#include <cstring>
#include <map>
#include <unordered_map>

#include "../../include/dreams_b200.h"

namespace dr {

int parse_blob(const uint8_t* blob, uint64_t size, RawProgram* out, std::string* err) {
    if (!blob || size < 16) {
        if (err) *err = "program blob shorter than its 16-byte header";
        return DR_ERR_BLOB;
    }
    uint32_t h[4];
    std::memcpy(h, blob, 16);
    const uint64_t need = 16 + 16ull * h[2] + 8ull * h[3] + 4ull * h[1];
    if (size < need) {
        if (err) *err = "program blob truncated";
        return DR_ERR_BLOB;
    }
    out->m = h[0];
    out->dim = h[1];
    out->ops.resize(h[2]);
    std::memcpy(out->ops.data(), blob + 16, 16ull * h[2]);
    out->consts.resize(h[3]);
    std::memcpy(out->consts.data(), blob + 16 + 16ull * h[2], 8ull * h[3]);
    out->dirs.resize(h[1]);
    std::memcpy(out->dirs.data(), blob + 16 + 16ull * h[2] + 8ull * h[3], 4ull * h[1]);
    for (const Insn& in : out->ops) {
        if (in.op > OP_END) {  // reference compiler.py:74 Opcode(op) -> ValueError
            if (err) *err = "unknown opcode " + std::to_string(in.op);
            return DR_ERR_OPCODE;
        }
    }
    return DR_OK;
}

namespace {

// ---- operand roles --------------------------------------------------------
struct Roles {
    int nread = 0;
    uint32_t read[2] = {0, 0};
    bool writes = false;
    uint32_t dest = 0;
};

Roles roles(const Insn& in) {
    Roles r;
    switch (in.op) {
        case OP_LOAD_X: case OP_LOAD_C: r.writes = true; r.dest = in.b; break;
        case OP_LOAD_N: r.writes = true; r.dest = in.a; break;
        case OP_ADD: case OP_SUB: case OP_MUL:
            r.nread = 2; r.read[0] = in.a; r.read[1] = in.b; r.writes = true; r.dest = in.c; break;
        case OP_NEG: case OP_POW2: case OP_POW3: case OP_INV:
            r.nread = 1; r.read[0] = in.a; r.writes = true; r.dest = in.b; break;
        case OP_STORE: r.nread = 1; r.read[0] = in.a; break;
        default: break;
    }
    return r;
}

// ---- symbolic DAG ----------------------------------------------------------
enum NK : uint8_t { NK_CONST, NK_AXIS, NK_STEP, NK_ADD, NK_SUB, NK_MUL, NK_NEG, NK_POW2, NK_POW3, NK_INV };

struct Node {
    NK k;
    int32_t a, b;       // operands (node ids) or pool index / axis for leaves
    uint32_t deg;       // degree bound in s
    bool exact;         // constant with a known exact integer value
    __int128 val;
};

constexpr __int128 kI64Max = (__int128)INT64_MAX;
constexpr __int128 kI64Min = (__int128)INT64_MIN;

bool fits_i64(__int128 v) { return v >= kI64Min && v <= kI64Max; }

struct Dag {
    std::vector<Node> nodes;
    std::map<std::tuple<int, int, int>, int> memo;
    std::vector<int64_t>* pool;
    std::map<int64_t, int> pool_index;

    explicit Dag(std::vector<int64_t>* p) : pool(p) {
        for (size_t i = 0; i < p->size(); ++i) pool_index.emplace((*p)[i], (int)i);
    }

    int intern(NK k, int a, int b, uint32_t deg, bool exact, __int128 val) {
        auto key = std::make_tuple((int)k, a, b);
        auto it = memo.find(key);
        if (it != memo.end()) return it->second;
        nodes.push_back(Node{k, a, b, deg, exact, val});
        int id = (int)nodes.size() - 1;
        memo.emplace(key, id);
        return id;
    }
    int pool_const(int idx) { return intern(NK_CONST, idx, 0, 0, true, (__int128)(*pool)[idx]); }
    int konst(__int128 v) {
        int64_t x = (int64_t)v;
        auto it = pool_index.find(x);
        int idx;
        if (it == pool_index.end()) {
            pool->push_back(x);
            idx = (int)pool->size() - 1;
            pool_index.emplace(x, idx);
        } else {
            idx = it->second;
        }
        return pool_const(idx);
    }
    int axis(int a) { return intern(NK_AXIS, a, 0, 1, false, 0); }
    int step() { return intern(NK_STEP, 0, 0, 1, false, 0); }
    const Node& n(int id) const { return nodes[id]; }
    bool is_val(int id, __int128 v) const { return n(id).exact && n(id).val == v; }

    int add(int x, int y) {
        if (is_val(x, 0)) return y;
        if (is_val(y, 0)) return x;
        if (n(x).exact && n(y).exact && fits_i64(n(x).val + n(y).val)) return konst(n(x).val + n(y).val);
        if (x > y) std::swap(x, y);
        return intern(NK_ADD, x, y, std::max(n(x).deg, n(y).deg), false, 0);
    }
    int sub(int x, int y) {
        if (is_val(y, 0)) return x;
        if (n(x).exact && n(y).exact && fits_i64(n(x).val - n(y).val)) return konst(n(x).val - n(y).val);
        return intern(NK_SUB, x, y, std::max(n(x).deg, n(y).deg), false, 0);
    }
    int mul(int x, int y) {
        if (is_val(x, 0) || is_val(y, 0)) return konst(0);
        if (is_val(x, 1)) return y;
        if (is_val(y, 1)) return x;
        if (n(x).exact && n(y).exact) {
            __int128 a = n(x).val, b = n(y).val;
            // |a|, |b| < 2^63 so the product fits in 127 bits
            if (fits_i64(a * b)) return konst(a * b);
        }
        if (x > y) std::swap(x, y);
        return intern(NK_MUL, x, y, n(x).deg + n(y).deg, false, 0);
    }
    int neg(int x) {
        if (n(x).exact && fits_i64(-n(x).val)) return konst(-n(x).val);
        if (n(x).k == NK_NEG) return n(x).a;
        return intern(NK_NEG, x, 0, n(x).deg, false, 0);
    }
    int pow2(int x) {
        if (n(x).exact && fits_i64(n(x).val * n(x).val)) return konst(n(x).val * n(x).val);
        return intern(NK_POW2, x, 0, 2 * n(x).deg, false, 0);
    }
    int pow3(int x) {
        if (n(x).exact) {
            __int128 v = n(x).val;
            if (fits_i64(v * v) && fits_i64(v * v * v)) return konst(v * v * v);
        }
        return intern(NK_POW3, x, 0, 3 * n(x).deg, false, 0);
    }
    int inv_const(int x) {  // x has degree 0
        if (is_val(x, 1) || is_val(x, -1)) return x;   // +-1 are their own inverses mod p
        return intern(NK_INV, x, 0, 0, false, 0);
    }
    int power(int x, uint32_t e) {
        if (e == 0) return konst(1);
        if (e == 1) return x;
        if (e == 2) return pow2(x);
        if (e == 3) return pow3(x);
        int h = power(x, e / 2);
        int h2 = pow2(h);
        return (e & 1) ? mul(h2, x) : h2;
    }
};

using Den = std::vector<std::pair<int, uint32_t>>;  // sorted (atom node, exponent)

struct Frac {
    int num;
    Den den;
};

Den den_max(const Den& a, const Den& b) {
    Den r;
    size_t i = 0, j = 0;
    while (i < a.size() || j < b.size()) {
        if (j == b.size() || (i < a.size() && a[i].first < b[j].first)) r.push_back(a[i++]);
        else if (i == a.size() || b[j].first < a[i].first) r.push_back(b[j++]);
        else { r.emplace_back(a[i].first, std::max(a[i].second, b[j].second)); ++i; ++j; }
    }
    return r;
}

Den den_add(const Den& a, const Den& b) {
    Den r;
    size_t i = 0, j = 0;
    while (i < a.size() || j < b.size()) {
        if (j == b.size() || (i < a.size() && a[i].first < b[j].first)) r.push_back(a[i++]);
        else if (i == a.size() || b[j].first < a[i].first) r.push_back(b[j++]);
        else { r.emplace_back(a[i].first, a[i].second + b[j].second); ++i; ++j; }
    }
    return r;
}

Den den_scale(const Den& a, uint32_t k) {
    Den r = a;
    for (auto& e : r) e.second *= k;
    return r;
}

uint32_t den_exp(const Den& d, int atom) {
    for (auto& e : d)
        if (e.first == atom) return e.second;
    return 0;
}

// prod over atoms of atom^(E[atom] - have[atom])
int den_product(Dag& g, const Den& E, const Den& have) {
    int acc = g.konst(1);
    for (auto& e : E) {
        uint32_t k = e.second - den_exp(have, e.first);
        if (k) acc = g.mul(acc, g.power(e.first, k));
    }
    return acc;
}

// Linear-scan register assignment of a node list; emits derived bytecode.
struct Emitter {
    Dag& g;
    std::vector<Insn> out;
    uint32_t n_regs = 0;
    explicit Emitter(Dag& d) : g(d) {}

    void emit(const std::vector<int>& roots) {
        // post-order over the DAG reachable from the roots
        std::vector<int> order;
        std::vector<char> seen(g.nodes.size(), 0);
        for (int r : roots) {
            std::vector<std::pair<int, int>> st{{r, 0}};
            while (!st.empty()) {
                auto& [id, state] = st.back();
                if (seen[id] == 2) { st.pop_back(); continue; }
                const Node& nd = g.n(id);
                int nk = 0;
                int kids[2];
                if (nd.k == NK_ADD || nd.k == NK_SUB || nd.k == NK_MUL) { kids[0] = nd.a; kids[1] = nd.b; nk = 2; }
                else if (nd.k == NK_NEG || nd.k == NK_POW2 || nd.k == NK_POW3 || nd.k == NK_INV) { kids[0] = nd.a; nk = 1; }
                if (state < nk) {
                    int kid = kids[state];
                    ++state;
                    if (!seen[kid]) st.emplace_back(kid, 0);
                    continue;
                }
                seen[id] = 2;
                order.push_back(id);
                st.pop_back();
            }
        }
        const int INF = 1 << 30;
        std::vector<int> last(g.nodes.size(), -1);
        for (size_t i = 0; i < order.size(); ++i) {
            const Node& nd = g.n(order[i]);
            if (nd.k == NK_ADD || nd.k == NK_SUB || nd.k == NK_MUL) { last[nd.a] = (int)i; last[nd.b] = (int)i; }
            else if (nd.k == NK_NEG || nd.k == NK_POW2 || nd.k == NK_POW3 || nd.k == NK_INV) last[nd.a] = (int)i;
        }
        for (int r : roots) last[r] = INF;
        std::vector<int> reg(g.nodes.size(), -1);
        std::vector<uint32_t> freelist;
        auto alloc = [&]() -> uint32_t {
            if (!freelist.empty()) { uint32_t r = freelist.back(); freelist.pop_back(); return r; }
            return n_regs++;
        };
        for (size_t i = 0; i < order.size(); ++i) {
            int id = order[i];
            const Node& nd = g.n(id);
            uint32_t ra = 0, rb = 0;
            bool bin = (nd.k == NK_ADD || nd.k == NK_SUB || nd.k == NK_MUL);
            bool un = (nd.k == NK_NEG || nd.k == NK_POW2 || nd.k == NK_POW3 || nd.k == NK_INV);
            if (bin || un) ra = (uint32_t)reg[nd.a];
            if (bin) rb = (uint32_t)reg[nd.b];
            // operands whose last use is here are released before the result is placed
            if (bin || un) {
                if (last[nd.a] == (int)i) { freelist.push_back(ra); last[nd.a] = -2; }
                if (bin && last[nd.b] == (int)i) { freelist.push_back(rb); last[nd.b] = -2; }
            }
            uint32_t rd = alloc();
            reg[id] = (int)rd;
            switch (nd.k) {
                case NK_CONST: out.push_back({OP_LOAD_C, (uint32_t)nd.a, rd, 0}); break;
                case NK_AXIS: out.push_back({OP_LOAD_X, (uint32_t)nd.a, rd, 0}); break;
                case NK_STEP: out.push_back({OP_LOAD_N, rd, 0, 0}); break;
                case NK_ADD: out.push_back({OP_ADD, ra, rb, rd}); break;
                case NK_SUB: out.push_back({OP_SUB, ra, rb, rd}); break;
                case NK_MUL: out.push_back({OP_MUL, ra, rb, rd}); break;
                case NK_NEG: out.push_back({OP_NEG, ra, rd, 0}); break;
                case NK_POW2: out.push_back({OP_POW2, ra, rd, 0}); break;
                case NK_POW3: out.push_back({OP_POW3, ra, rd, 0}); break;
                case NK_INV: out.push_back({OP_INV, ra, rd, 0}); break;
            }
            if (last[id] == -1) freelist.push_back(rd);  // never used (cannot happen for roots)
        }
        for (size_t k = 0; k < roots.size(); ++k)
            out.push_back({OP_STORE, (uint32_t)reg[roots[k]], (uint32_t)k, 0});
        if (n_regs == 0) n_regs = 1;
    }
};

}  // namespace

int plan_program(const RawProgram& raw, Plan* P, std::string* err) {
    Plan& p = *P;
    p = Plan();
    p.m = raw.m;
    p.dim = raw.dim;
    p.dirs = raw.dirs;
    p.consts = raw.consts;
    if (raw.m < 1 || raw.m > (uint32_t)kMaxM) {
        if (err) *err = "matrix size m=" + std::to_string(raw.m) + " outside 1..8";
        return raw.m < 1 ? DR_ERR_INDEX : DR_ERR_UNSUPPORTED;
    }
    if (raw.dim > (uint32_t)kMaxAxes) {
        if (err) *err = "more than 8 axes";
        return DR_ERR_UNSUPPORTED;
    }
    if (raw.consts.size() > (size_t)kMaxConsts - 2) {
        if (err) *err = "more than 510 constants";
        return DR_ERR_UNSUPPORTED;
    }
    const uint32_t m = raw.m;

    // ---- executed prefix and index validation (reference runtime IndexError)
    for (const Insn& in : raw.ops) {
        if (in.op == OP_END) break;
        if (in.op == OP_NOP) continue;
        Roles r = roles(in);
        for (int i = 0; i < r.nread; ++i)
            if (r.read[i] >= (uint32_t)DR_MAX_REGS) { if (err) *err = "register index out of range"; return DR_ERR_INDEX; }
        if (r.writes && r.dest >= (uint32_t)DR_MAX_REGS) { if (err) *err = "register index out of range"; return DR_ERR_INDEX; }
        if (in.op == OP_LOAD_X && in.a >= raw.dim) { if (err) *err = "LOAD_X axis out of range"; return DR_ERR_INDEX; }
        if (in.op == OP_LOAD_C && in.a >= raw.consts.size()) { if (err) *err = "LOAD_C index out of range"; return DR_ERR_INDEX; }
        if (in.op == OP_STORE && (in.b >= m || in.c >= m)) { if (err) *err = "STORE entry out of range"; return DR_ERR_INDEX; }
        if (in.op == OP_INV) p.has_inv = true;
        p.exec.push_back(in);
    }

    // ---- register compaction of the executed prefix
    {
        const size_t n = p.exec.size();
        // value instance = (virtual register, defining op); reads before any write see 0
        std::vector<int> cur_def(DR_MAX_REGS, -1);
        std::vector<int> last_use(n, -1);          // per defining op
        std::vector<std::array<int, 2>> src_def(n, {-1, -1});
        bool need_zero = false;
        for (size_t i = 0; i < n; ++i) {
            Roles r = roles(p.exec[i]);
            for (int k = 0; k < r.nread; ++k) {
                int d = cur_def[r.read[k]];
                src_def[i][k] = d;
                if (d < 0) need_zero = true;
                else last_use[d] = (int)i;
            }
            if (r.writes) cur_def[r.dest] = (int)i;
        }
        uint32_t n_phys = 0;
        std::vector<uint32_t> freelist;
        std::vector<uint32_t> phys(n, 0);
        uint32_t zero_reg = 0;
        if (need_zero) zero_reg = n_phys++;
        for (size_t i = 0; i < n; ++i) {
            Insn in = p.exec[i];
            Roles r = roles(in);
            uint32_t rs[2] = {zero_reg, zero_reg};
            for (int k = 0; k < r.nread; ++k) {
                int d = src_def[i][k];
                rs[k] = d < 0 ? zero_reg : phys[d];
            }
            for (int k = 0; k < r.nread; ++k) {
                int d = src_def[i][k];
                if (d >= 0 && last_use[d] == (int)i) {
                    bool dup = (k == 1 && src_def[i][0] == d);
                    if (!dup) freelist.push_back(phys[d]);
                }
            }
            uint32_t rd = 0;
            if (r.writes) {
                if (!freelist.empty()) { rd = freelist.back(); freelist.pop_back(); }
                else rd = n_phys++;
                phys[i] = rd;
                if (last_use[i] < 0) freelist.push_back(rd);   // dead value: slot reusable at once
            }
            Insn o = in;
            switch (in.op) {
                case OP_LOAD_X: case OP_LOAD_C: o.b = rd; break;
                case OP_LOAD_N: o.a = rd; break;
                case OP_ADD: case OP_SUB: case OP_MUL: o.a = rs[0]; o.b = rs[1]; o.c = rd; break;
                case OP_NEG: case OP_POW2: case OP_POW3: case OP_INV: o.a = rs[0]; o.b = rd; break;
                case OP_STORE: o.a = rs[0]; o.b = in.b * m + in.c; o.c = 0; break;
                default: break;
            }
            p.ops.push_back(o);
        }
        if (n_phys == 0) n_phys = 1;
        p.n_regs = n_phys;
        p.zero_reg = zero_reg;
        if (!need_zero) p.zero_reg = 0xffffffffu;
        if (p.n_regs > (uint32_t)kMaxCompactRegs) {
            if (err) *err = "too many simultaneously live registers";
            return DR_ERR_UNSUPPORTED;
        }
    }

    // ---- symbolic evaluation
    Dag g(&p.consts);
    std::vector<Frac> R(DR_MAX_REGS, Frac{g.konst(0), {}});
    std::vector<Frac> Mx(m * m, Frac{g.konst(0), {}});
    std::vector<int> atoms;
    for (const Insn& in : p.exec) {
        switch (in.op) {
            case OP_LOAD_X: R[in.b] = Frac{g.axis((int)in.a), {}}; break;
            case OP_LOAD_C: R[in.b] = Frac{g.pool_const((int)in.a), {}}; break;
            case OP_LOAD_N: R[in.a] = Frac{g.step(), {}}; break;
            case OP_ADD: case OP_SUB: {
                const Frac x = R[in.a], y = R[in.b];
                Den E = den_max(x.den, y.den);
                int nx = g.mul(x.num, den_product(g, E, x.den));
                int ny = g.mul(y.num, den_product(g, E, y.den));
                R[in.c] = Frac{in.op == OP_ADD ? g.add(nx, ny) : g.sub(nx, ny), E};
                break;
            }
            case OP_MUL: {
                const Frac x = R[in.a], y = R[in.b];
                R[in.c] = Frac{g.mul(x.num, y.num), den_add(x.den, y.den)};
                break;
            }
            case OP_NEG: { const Frac x = R[in.a]; R[in.b] = Frac{g.neg(x.num), x.den}; break; }
            case OP_POW2: { const Frac x = R[in.a]; R[in.b] = Frac{g.pow2(x.num), den_scale(x.den, 2)}; break; }
            case OP_POW3: { const Frac x = R[in.a]; R[in.b] = Frac{g.pow3(x.num), den_scale(x.den, 3)}; break; }
            case OP_INV: {
                const Frac x = R[in.a];
                int dp = den_product(g, x.den, Den{});
                if (g.n(x.num).deg == 0) {
                    // constant numerator: INV(N / D) = D * INV(N), and INV(0) = 0 gives 0
                    // on both sides, so no guard is needed
                    R[in.b] = Frac{g.mul(dp, g.inv_const(x.num)), {}};
                } else {
                    int atom = x.num;
                    if (std::find(atoms.begin(), atoms.end(), atom) == atoms.end()) atoms.push_back(atom);
                    R[in.b] = Frac{dp, Den{{atom, 1u}}};
                }
                break;
            }
            case OP_STORE: Mx[in.b * m + in.c] = R[in.a]; break;
            default: break;
        }
    }

    // ---- classification
    auto exact_is = [&](const Frac& f, __int128 v) { return f.den.empty() && g.is_val(f.num, v); };
    auto zero_num = [&](const Frac& f) { return g.is_val(f.num, 0); };
    bool companion = m >= 2;
    for (uint32_t i = 0; i < m && companion; ++i)
        for (uint32_t j = 0; j + 1 < m && companion; ++j) {
            const Frac& f = Mx[i * m + j];
            companion = (i == j + 1) ? exact_is(f, 1) : zero_num(f);
        }
    Den E;
    for (const Frac& f : Mx) E = den_max(E, f.den);
    bool guards_in_E = true;
    for (int a : atoms)
        if (den_exp(E, a) == 0) guards_in_E = false;

    std::vector<int> roots;
    Class cls = CLS_INTERP;
    if (companion && atoms.empty()) {
        cls = CLS_COMPANION;
        for (uint32_t i = 0; i < m; ++i) roots.push_back(Mx[i * m + m - 1].num);
    } else if (companion && guards_in_E && m <= 4) {
        cls = CLS_RATIONAL;
        for (uint32_t i = 0; i < m; ++i) {
            const Frac& f = Mx[i * m + m - 1];
            roots.push_back(g.mul(f.num, den_product(g, E, f.den)));
        }
        roots.push_back(den_product(g, E, Den{}));
    } else if (atoms.empty() && m >= 2 && m <= 3) {
        cls = CLS_DENSE;
        for (uint32_t k = 0; k < m * m; ++k) roots.push_back(Mx[k].num);
    }
    uint32_t deg = 0;
    for (int r : roots) deg = std::max(deg, g.n(r).deg);
    if (cls != CLS_INTERP && template_degree(cls, m, std::max(deg, 1u)) < 0) cls = CLS_INTERP;
    p.cls = cls;
    if (cls == CLS_INTERP) {
        p.degree = 0;
        p.n_streams = 0;
        p.dn_regs = 0;
        return DR_OK;
    }
    p.degree = std::max(deg, 1u);
    Emitter em(g);
    em.emit(roots);
    p.dops = std::move(em.out);
    p.dn_regs = em.n_regs;
    p.n_streams = (uint32_t)roots.size();
    if (p.dn_regs > (uint32_t)kMaxCompactRegs || p.consts.size() > (size_t)kMaxConsts) {
        p.cls = CLS_INTERP;
        p.dops.clear();
        p.n_streams = 0;
        p.degree = 0;
    }
    return DR_OK;
}

double float_bound_log2(const Plan& plan, const int64_t* axis, uint64_t depth) {
    if (plan.has_inv) return INFINITY;
    // registers start at 0.0; clear only those the prefix can name
    uint32_t hi = 0;
    for (const Insn& in : plan.exec) hi = std::max(hi, std::max(in.a, std::max(in.b, in.c)));
    double b[DR_MAX_REGS];
    std::fill(b, b + std::min<uint32_t>(hi + 1, DR_MAX_REGS), 0.0);
    const double last = depth > 0 ? (double)(depth - 1) : 0.0;
    double worst = 0.0;
    for (const Insn& in : plan.exec) {
        double v = 0.0;
        uint32_t dest = 0;
        switch (in.op) {
            case OP_LOAD_X: {
                const int64_t* ax = axis + 4 * in.a;
                if (ax[1] != 1 || ax[3] != 1) return INFINITY;
                v = std::max(std::fabs((double)ax[0]), std::fabs((double)ax[0] + last * (double)ax[2]));
                dest = in.b;
                break;
            }
            case OP_LOAD_C: v = std::fabs((double)plan.consts[in.a]); dest = in.b; break;
            case OP_LOAD_N: v = last; dest = in.a; break;
            case OP_ADD: case OP_SUB: v = b[in.a] + b[in.b]; dest = in.c; break;
            case OP_MUL: v = b[in.a] * b[in.b]; dest = in.c; break;
            case OP_NEG: v = b[in.a]; dest = in.b; break;
            case OP_POW2: v = b[in.a] * b[in.a]; dest = in.b; break;
            case OP_POW3: v = b[in.a] * b[in.a] * b[in.a]; dest = in.b; break;
            default: continue;
        }
        b[dest] = v;
        worst = std::max(worst, v);
    }
    if (!std::isfinite(worst)) return INFINITY;
    return worst > 0 ? std::log2(worst) : -1.0;
}

bool float_companion_shape(const Plan& p) {
    const uint32_t m = p.m;
    if (m < 2) return false;
    // per register: holds a LOAD_C constant (value), or anything else
    std::vector<uint8_t> is_c(p.n_regs + 1, 0);
    std::vector<int64_t> cv(p.n_regs + 1, 0);
    if (p.zero_reg != 0xffffffffu && p.zero_reg < is_c.size()) is_c[p.zero_reg] = 1;
    std::vector<uint8_t> e_c(m * m, 1);      // never stored: 0.0
    std::vector<int64_t> e_v(m * m, 0);
    auto set = [&](uint32_t r, bool c, int64_t v) {
        if (r < is_c.size()) { is_c[r] = c; cv[r] = v; }
    };
    for (const Insn& in : p.ops) {
        switch (in.op) {
            case OP_LOAD_C: set(in.b, in.a < p.consts.size(), in.a < p.consts.size() ? p.consts[in.a] : 0); break;
            case OP_LOAD_N: set(in.a, false, 0); break;
            case OP_LOAD_X: case OP_NEG: case OP_POW2: case OP_POW3: case OP_INV: set(in.b, false, 0); break;
            case OP_ADD: case OP_SUB: case OP_MUL: set(in.c, false, 0); break;
            case OP_STORE:
                if (in.b < m * m) {
                    const bool c = in.a < is_c.size() && is_c[in.a];
                    e_c[in.b] = c;
                    e_v[in.b] = c ? cv[in.a] : 0;
                }
                break;
            default: break;
        }
    }
    for (uint32_t i = 0; i < m; ++i)
        for (uint32_t j = 0; j + 1 < m; ++j) {
            const uint32_t k = i * m + j;
            if (!e_c[k] || e_v[k] != (i == j + 1 ? 1 : 0)) return false;
        }
    return true;
}

}  // namespace dr
