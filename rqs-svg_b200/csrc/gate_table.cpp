// Unitaries of the reference API's gates and their reduction to the
// sub-indices a gate can change.
//
// Each matrix below is the closed form of the corresponding functor in the
// reference (src/qcs.cu:378-1104): row = output sub-index, column = input
// sub-index, bit i of a sub-index = value of target i (src/qcs.cu:255-259,
// 302-309, 354-371). Scalars are built with the same host-side double cos/sin
// calls as the reference constructors, so the matrix entries agree with the
// coefficients the reference multiplies by.

#include "qcs_internal.h"

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <unordered_map>

namespace qcsb
{

std::string strformat(const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return std::string(buf);
}

namespace
{

constexpr double kRsqrt2 = 0.70710678118654752440; // M_SQRT1_2

inline cplx C(double re, double im = 0.0) { return cplx{re, im}; }
inline cplx cmul(cplx a, cplx b) { return cplx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cplx cscale(double s, cplx a) { return cplx{s * a.re, s * a.im}; }
inline cplx cexpi(double x) { return cplx{std::cos(x), std::sin(x)}; }
inline cplx mul_i(cplx a) { return cplx{-a.im, a.re}; }     // i * a
inline cplx mul_mi(cplx a) { return cplx{a.im, -a.re}; }    // -i * a

struct Builder
{
    GateMatrix g;
    explicit Builder(int nt)
    {
        g.nt = nt;
        const int d = 1 << nt;
        for (int i = 0; i < d * d; ++i)
            g.m[i] = C(0.0);
        for (int i = 0; i < d; ++i)
            g.m[i * d + i] = C(1.0);
    }
    void set(int row, int col, cplx v) { g.m[row * (1 << g.nt) + col] = v; }
};

struct GateInfo
{
    const char *name;
    int nt;
    int np;
};

const GateInfo kGates[] = {
    {"global_phase", 0, 1}, {"h", 1, 0}, {"x", 1, 0}, {"y", 1, 0}, {"z", 1, 0},
    {"s", 1, 0}, {"sdg", 1, 0}, {"t", 1, 0}, {"tdg", 1, 0}, {"sx", 1, 0},
    {"rx", 1, 1}, {"ry", 1, 1}, {"rz", 1, 1}, {"u4", 1, 4}, {"u3", 1, 3},
    {"u2", 1, 2}, {"u1", 1, 1}, {"u", 1, 3}, {"p", 1, 1}, {"swap", 2, 0},
    {"iswap", 2, 0}, {"id", 1, 0}, {"sxdg", 1, 0}, {"r", 1, 2}, {"rxx", 2, 1},
    {"ryy", 2, 1}, {"rzz", 2, 1}, {"rzx", 2, 1}, {"dcx", 2, 0}, {"ecr", 2, 0},
    {"xx_plus_yy", 2, 2}, {"xx_minus_yy", 2, 2}, {"rccx", 3, 0}, {"rcccx", 4, 0},
};

// ids: positions in kGates
enum GateIdx
{
    G_GLOBAL_PHASE, G_H, G_X, G_Y, G_Z, G_S, G_SDG, G_T, G_TDG, G_SX, G_RX, G_RY, G_RZ, G_U4, G_U3, G_U2, G_U1,
    G_U, G_P, G_SWAP, G_ISWAP, G_ID, G_SXDG, G_R, G_RXX, G_RYY, G_RZZ, G_RZX, G_DCX, G_ECR, G_XX_PLUS_YY,
    G_XX_MINUS_YY, G_RCCX, G_RCCCX, G_COUNT
};
static_assert(sizeof(kGates) / sizeof(kGates[0]) == G_COUNT, "gate table and ids");

const GateInfo &info(int id)
{
    if (id < 0 || id >= G_COUNT)
        throw std::runtime_error(strformat("unknown gate id %d", id));
    return kGates[id];
}

} // namespace

int gate_id(const char *name)
{
    static const std::unordered_map<std::string, int> ids = [] {
        std::unordered_map<std::string, int> m;
        for (int i = 0; i < G_COUNT; ++i)
            m.emplace(kGates[i].name, i);
        return m;
    }();
    const auto it = name ? ids.find(name) : ids.end();
    if (it == ids.end())
        throw std::runtime_error(strformat("unknown gate '%s'", name ? name : "(null)"));
    return it->second;
}

int gate_arity(int id) { return info(id).nt; }

int gate_nparams(int id) { return info(id).np; }

const char *gate_name(int id) { return info(id).name; }

GateMatrix gate_matrix(int id, const double *p, int np)
{
    const GateInfo &gi = info(id);
    if (np != gi.np)
        throw std::runtime_error(strformat("gate '%s' takes %d parameters, got %d", gi.name, gi.np, np));
    Builder b(gi.nt);
    const int n = id;

    if (n == G_GLOBAL_PHASE)
    {
        b.set(0, 0, cexpi(p[0]));
    }
    else if (n == G_U4 || n == G_U3 || n == G_U)
    {
        const double theta = p[0], phi = p[1], lambda = p[2];
        const double c = std::cos(0.5 * theta), s = std::sin(0.5 * theta);
        const cplx e_phi = cexpi(phi), e_lambda = cexpi(lambda);
        if (n == G_U4)
        {
            // e^{i gamma} [[c, -s e^{i lambda}], [e^{i phi} s, e^{i phi} e^{i lambda} c]]
            const cplx e_gamma = cexpi(p[3]);
            b.set(0, 0, cscale(c, e_gamma));
            b.set(0, 1, cmul(e_gamma, cscale(-s, e_lambda)));
            b.set(1, 0, cmul(e_gamma, cscale(s, e_phi)));
            b.set(1, 1, cmul(e_gamma, cmul(e_phi, cscale(c, e_lambda))));
        }
        else
        {
            // [[c, -s e^{i lambda}], [e^{i phi} s, e^{i (phi + lambda)} c]]
            b.set(0, 0, C(c));
            b.set(0, 1, cscale(-s, e_lambda));
            b.set(1, 0, cscale(s, e_phi));
            b.set(1, 1, cscale(c, cexpi(phi + lambda)));
        }
    }
    else if (n == G_U2)
    {
        const cplx e_phi = cexpi(p[0]), e_lambda = cexpi(p[1]);
        b.set(0, 0, C(kRsqrt2));
        b.set(0, 1, cscale(-kRsqrt2, e_lambda));
        b.set(1, 0, cscale(kRsqrt2, e_phi));
        b.set(1, 1, cscale(kRsqrt2, cexpi(p[0] + p[1])));
    }
    else if (n == G_U1 || n == G_P)
    {
        b.set(1, 1, cexpi(p[0]));
    }
    else if (n == G_H)
    {
        b.set(0, 0, C(kRsqrt2));
        b.set(0, 1, C(kRsqrt2));
        b.set(1, 0, C(kRsqrt2));
        b.set(1, 1, C(-kRsqrt2));
    }
    else if (n == G_X)
    {
        b.set(0, 0, C(0));
        b.set(0, 1, C(1));
        b.set(1, 0, C(1));
        b.set(1, 1, C(0));
    }
    else if (n == G_Y)
    {
        b.set(0, 0, C(0));
        b.set(0, 1, C(0, -1));
        b.set(1, 0, C(0, 1));
        b.set(1, 1, C(0));
    }
    else if (n == G_Z)
    {
        b.set(1, 1, C(-1));
    }
    else if (n == G_S)
    {
        b.set(1, 1, C(0, 1));
    }
    else if (n == G_SDG)
    {
        b.set(1, 1, C(0, -1));
    }
    else if (n == G_T)
    {
        b.set(1, 1, C(kRsqrt2, kRsqrt2));
    }
    else if (n == G_TDG)
    {
        b.set(1, 1, C(kRsqrt2, -kRsqrt2));
    }
    else if (n == G_SX || n == G_SXDG)
    {
        // sx = 1/2 [[1+i, 1-i], [1-i, 1+i]]; sxdg is its conjugate.
        const double sg = (n == G_SX) ? 1.0 : -1.0;
        b.set(0, 0, C(0.5, 0.5 * sg));
        b.set(0, 1, C(0.5, -0.5 * sg));
        b.set(1, 0, C(0.5, -0.5 * sg));
        b.set(1, 1, C(0.5, 0.5 * sg));
    }
    else if (n == G_RX)
    {
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        b.set(0, 0, C(c));
        b.set(0, 1, C(0, -s));
        b.set(1, 0, C(0, -s));
        b.set(1, 1, C(c));
    }
    else if (n == G_RY)
    {
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        b.set(0, 0, C(c));
        b.set(0, 1, C(-s));
        b.set(1, 0, C(s));
        b.set(1, 1, C(c));
    }
    else if (n == G_RZ)
    {
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        b.set(0, 0, C(c, -s));
        b.set(1, 1, C(c, s));
    }
    else if (n == G_ID)
    {
        // identity
    }
    else if (n == G_R)
    {
        // [[c, -i s e^{-i phi}], [-i s e^{i phi}, c]]
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        const double cp = std::cos(p[1]), sp = std::sin(p[1]);
        b.set(0, 0, C(c));
        b.set(0, 1, cscale(-s, mul_i(C(cp, -sp))));
        b.set(1, 0, cscale(-s, mul_i(C(cp, sp))));
        b.set(1, 1, C(c));
    }
    else if (n == G_SWAP)
    {
        b.set(1, 1, C(0));
        b.set(2, 2, C(0));
        b.set(1, 2, C(1));
        b.set(2, 1, C(1));
    }
    else if (n == G_ISWAP)
    {
        b.set(1, 1, C(0));
        b.set(2, 2, C(0));
        b.set(1, 2, C(0, 1));
        b.set(2, 1, C(0, 1));
    }
    else if (n == G_RZZ)
    {
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        b.set(0, 0, C(c, -s));
        b.set(1, 1, C(c, s));
        b.set(2, 2, C(c, s));
        b.set(3, 3, C(c, -s));
    }
    else if (n == G_RXX || n == G_RYY)
    {
        // diagonal c; anti-diagonal -i s, except ryy's 00<->11 entries (+i s).
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        const double outer = (n == G_RXX) ? -s : s;
        for (int k = 0; k < 4; ++k)
            b.set(k, k, C(c));
        b.set(0, 3, C(0, outer));
        b.set(3, 0, C(0, outer));
        b.set(1, 2, C(0, -s));
        b.set(2, 1, C(0, -s));
    }
    else if (n == G_RZX)
    {
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        for (int k = 0; k < 4; ++k)
            b.set(k, k, C(c));
        b.set(0, 2, C(0, -s));
        b.set(2, 0, C(0, -s));
        b.set(1, 3, C(0, s));
        b.set(3, 1, C(0, s));
    }
    else if (n == G_XX_PLUS_YY || n == G_XX_MINUS_YY)
    {
        // acts on {01, 10} (plus) or {00, 11} (minus):
        // [[c, -i s e^{-i beta}], [-i s e^{i beta}, c]]
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        const double cb = std::cos(p[1]), sb = std::sin(p[1]);
        const int lo = (n == G_XX_PLUS_YY) ? 1 : 0;
        const int hi = (n == G_XX_PLUS_YY) ? 2 : 3;
        b.set(lo, lo, C(c));
        b.set(hi, hi, C(c));
        b.set(lo, hi, cscale(-s, mul_i(C(cb, -sb))));
        b.set(hi, lo, cscale(-s, mul_i(C(cb, sb))));
    }
    else if (n == G_DCX)
    {
        // 01 <- 11, 10 <- 01, 11 <- 10
        for (int k = 1; k < 4; ++k)
            b.set(k, k, C(0));
        b.set(1, 3, C(1));
        b.set(2, 1, C(1));
        b.set(3, 2, C(1));
    }
    else if (n == G_ECR)
    {
        const double r = kRsqrt2;
        for (int k = 0; k < 4; ++k)
            b.set(k, k, C(0));
        b.set(0, 1, C(r));
        b.set(0, 3, mul_i(C(r)));
        b.set(1, 0, C(r));
        b.set(1, 2, mul_mi(C(r)));
        b.set(2, 1, mul_i(C(r)));
        b.set(2, 3, C(r));
        b.set(3, 0, mul_mi(C(r)));
        b.set(3, 2, C(r));
    }
    else if (n == G_RCCX)
    {
        // 011 <- -i 111, 101 <- -101, 111 <- i 011
        b.set(3, 3, C(0));
        b.set(7, 7, C(0));
        b.set(3, 7, C(0, -1));
        b.set(5, 5, C(-1));
        b.set(7, 3, C(0, 1));
    }
    else if (n == G_RCCCX)
    {
        // 0011 <- i 0011, 0111 <- 1111, 1011 <- -i 1011, 1111 <- -0111
        b.set(3, 3, C(0, 1));
        b.set(7, 7, C(0));
        b.set(15, 15, C(0));
        b.set(7, 15, C(1));
        b.set(11, 11, C(0, -1));
        b.set(15, 7, C(-1));
    }
    else
    {
        throw std::runtime_error(strformat("gate '%s' has no matrix", gi.name));
    }
    return b.g;
}

double GateOp::changed_amps(int n) const
{
    const int c = __builtin_popcountll(cmask);
    return static_cast<double>(na) * std::ldexp(1.0, n - nt - c);
}

GateOp make_gate_op(const GateMatrix &g, const int *tq, uint64_t cmask, uint64_t cval)
{
    GateOp op;
    op.nt = g.nt;
    for (int i = 0; i < g.nt; ++i)
        op.tq[i] = tq[i];
    op.cmask = cmask;
    op.cval = cval;
    const int d = 1 << g.nt;
    auto is_id = [&](int r, int c) {
        const cplx v = g.m[r * d + c];
        return (r == c) ? (v.re == 1.0 && v.im == 0.0) : (v.re == 0.0 && v.im == 0.0);
    };
    // Active sub-indices: those whose row or column differs from identity.
    op.na = 0;
    for (int s = 0; s < d; ++s)
    {
        bool active = false;
        for (int k = 0; k < d && !active; ++k)
            active = !is_id(s, k) || !is_id(k, s);
        if (active)
        {
            if (op.na == kMaxActive)
                throw std::runtime_error("gate changes more than four sub-indices");
            op.act[op.na++] = static_cast<uint8_t>(s);
        }
    }
    bool diag = true;
    for (int a = 0; a < op.na && diag; ++a)
        for (int b = 0; b < op.na; ++b)
            if (a != b && !is_id(op.act[a], op.act[b]))
            {
                diag = false;
                break;
            }
    op.diag = diag;
    if (diag)
    {
        for (int a = 0; a < op.na; ++a)
            op.mat[a] = g.m[op.act[a] * d + op.act[a]];
    }
    else
    {
        for (int a = 0; a < op.na; ++a)
            for (int b = 0; b < op.na; ++b)
                op.mat[a * op.na + b] = g.m[op.act[a] * d + op.act[b]];
    }
    return op;
}

} // namespace qcsb
