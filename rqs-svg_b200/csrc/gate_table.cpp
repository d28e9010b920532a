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

const GateInfo &lookup(const char *name)
{
    for (const auto &gi : kGates)
        if (std::strcmp(gi.name, name) == 0)
            return gi;
    throw std::runtime_error(strformat("unknown gate '%s'", name));
}

} // namespace

int gate_arity(const char *name) { return lookup(name).nt; }

int gate_nparams(const char *name) { return lookup(name).np; }

GateMatrix gate_matrix(const char *name, const double *p, int np)
{
    const GateInfo &gi = lookup(name);
    if (np != gi.np)
        throw std::runtime_error(strformat("gate '%s' takes %d parameters, got %d", name, gi.np, np));
    Builder b(gi.nt);
    const std::string n(name);

    if (n == "global_phase")
    {
        b.set(0, 0, cexpi(p[0]));
    }
    else if (n == "u4" || n == "u3" || n == "u")
    {
        const double theta = p[0], phi = p[1], lambda = p[2];
        const double c = std::cos(0.5 * theta), s = std::sin(0.5 * theta);
        const cplx e_phi = cexpi(phi), e_lambda = cexpi(lambda);
        if (n == "u4")
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
    else if (n == "u2")
    {
        const cplx e_phi = cexpi(p[0]), e_lambda = cexpi(p[1]);
        b.set(0, 0, C(kRsqrt2));
        b.set(0, 1, cscale(-kRsqrt2, e_lambda));
        b.set(1, 0, cscale(kRsqrt2, e_phi));
        b.set(1, 1, cscale(kRsqrt2, cexpi(p[0] + p[1])));
    }
    else if (n == "u1" || n == "p")
    {
        b.set(1, 1, cexpi(p[0]));
    }
    else if (n == "h")
    {
        b.set(0, 0, C(kRsqrt2));
        b.set(0, 1, C(kRsqrt2));
        b.set(1, 0, C(kRsqrt2));
        b.set(1, 1, C(-kRsqrt2));
    }
    else if (n == "x")
    {
        b.set(0, 0, C(0));
        b.set(0, 1, C(1));
        b.set(1, 0, C(1));
        b.set(1, 1, C(0));
    }
    else if (n == "y")
    {
        b.set(0, 0, C(0));
        b.set(0, 1, C(0, -1));
        b.set(1, 0, C(0, 1));
        b.set(1, 1, C(0));
    }
    else if (n == "z")
    {
        b.set(1, 1, C(-1));
    }
    else if (n == "s")
    {
        b.set(1, 1, C(0, 1));
    }
    else if (n == "sdg")
    {
        b.set(1, 1, C(0, -1));
    }
    else if (n == "t")
    {
        b.set(1, 1, C(kRsqrt2, kRsqrt2));
    }
    else if (n == "tdg")
    {
        b.set(1, 1, C(kRsqrt2, -kRsqrt2));
    }
    else if (n == "sx" || n == "sxdg")
    {
        // sx = 1/2 [[1+i, 1-i], [1-i, 1+i]]; sxdg is its conjugate.
        const double sg = (n == "sx") ? 1.0 : -1.0;
        b.set(0, 0, C(0.5, 0.5 * sg));
        b.set(0, 1, C(0.5, -0.5 * sg));
        b.set(1, 0, C(0.5, -0.5 * sg));
        b.set(1, 1, C(0.5, 0.5 * sg));
    }
    else if (n == "rx")
    {
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        b.set(0, 0, C(c));
        b.set(0, 1, C(0, -s));
        b.set(1, 0, C(0, -s));
        b.set(1, 1, C(c));
    }
    else if (n == "ry")
    {
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        b.set(0, 0, C(c));
        b.set(0, 1, C(-s));
        b.set(1, 0, C(s));
        b.set(1, 1, C(c));
    }
    else if (n == "rz")
    {
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        b.set(0, 0, C(c, -s));
        b.set(1, 1, C(c, s));
    }
    else if (n == "id")
    {
        // identity
    }
    else if (n == "r")
    {
        // [[c, -i s e^{-i phi}], [-i s e^{i phi}, c]]
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        const double cp = std::cos(p[1]), sp = std::sin(p[1]);
        b.set(0, 0, C(c));
        b.set(0, 1, cscale(-s, mul_i(C(cp, -sp))));
        b.set(1, 0, cscale(-s, mul_i(C(cp, sp))));
        b.set(1, 1, C(c));
    }
    else if (n == "swap")
    {
        b.set(1, 1, C(0));
        b.set(2, 2, C(0));
        b.set(1, 2, C(1));
        b.set(2, 1, C(1));
    }
    else if (n == "iswap")
    {
        b.set(1, 1, C(0));
        b.set(2, 2, C(0));
        b.set(1, 2, C(0, 1));
        b.set(2, 1, C(0, 1));
    }
    else if (n == "rzz")
    {
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        b.set(0, 0, C(c, -s));
        b.set(1, 1, C(c, s));
        b.set(2, 2, C(c, s));
        b.set(3, 3, C(c, -s));
    }
    else if (n == "rxx" || n == "ryy")
    {
        // diagonal c; anti-diagonal -i s, except ryy's 00<->11 entries (+i s).
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        const double outer = (n == "rxx") ? -s : s;
        for (int k = 0; k < 4; ++k)
            b.set(k, k, C(c));
        b.set(0, 3, C(0, outer));
        b.set(3, 0, C(0, outer));
        b.set(1, 2, C(0, -s));
        b.set(2, 1, C(0, -s));
    }
    else if (n == "rzx")
    {
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        for (int k = 0; k < 4; ++k)
            b.set(k, k, C(c));
        b.set(0, 2, C(0, -s));
        b.set(2, 0, C(0, -s));
        b.set(1, 3, C(0, s));
        b.set(3, 1, C(0, s));
    }
    else if (n == "xx_plus_yy" || n == "xx_minus_yy")
    {
        // acts on {01, 10} (plus) or {00, 11} (minus):
        // [[c, -i s e^{-i beta}], [-i s e^{i beta}, c]]
        const double c = std::cos(0.5 * p[0]), s = std::sin(0.5 * p[0]);
        const double cb = std::cos(p[1]), sb = std::sin(p[1]);
        const int lo = (n == "xx_plus_yy") ? 1 : 0;
        const int hi = (n == "xx_plus_yy") ? 2 : 3;
        b.set(lo, lo, C(c));
        b.set(hi, hi, C(c));
        b.set(lo, hi, cscale(-s, mul_i(C(cb, -sb))));
        b.set(hi, lo, cscale(-s, mul_i(C(cb, sb))));
    }
    else if (n == "dcx")
    {
        // 01 <- 11, 10 <- 01, 11 <- 10
        for (int k = 1; k < 4; ++k)
            b.set(k, k, C(0));
        b.set(1, 3, C(1));
        b.set(2, 1, C(1));
        b.set(3, 2, C(1));
    }
    else if (n == "ecr")
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
    else if (n == "rccx")
    {
        // 011 <- -i 111, 101 <- -101, 111 <- i 011
        b.set(3, 3, C(0));
        b.set(7, 7, C(0));
        b.set(3, 7, C(0, -1));
        b.set(5, 5, C(-1));
        b.set(7, 3, C(0, 1));
    }
    else if (n == "rcccx")
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
        throw std::runtime_error(strformat("gate '%s' has no matrix", name));
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
            op.act[op.na++] = static_cast<uint8_t>(s);
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
