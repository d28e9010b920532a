// Fused execution: many gates per read and write of the state.
//
// A pass fixes k "local" physical qubits Q (the lowest L qubits, so global
// accesses come in contiguous runs, plus the targets of the pass's
// non-diagonal gates). The register splits into 2^(n-k) chunks; chunk c is
// the 2^k amplitudes whose non-Q bits spell c. One CTA owns a chunk at a
// time: it stages the chunk in shared memory (cp.async, double-buffered so
// the next chunk streams in while this one is processed), applies the pass's
// gates, and streams the chunk back.
//
// Inside a pass the gates run in stages. A stage picks SB local bits S; each
// of the 2^(k-SB) threads takes the 2^SB amplitudes that differ only in S
// into registers, applies every gate of the stage there, and writes them
// back. A non-diagonal gate must have its targets in S. Diagonal gates and
// controls may sit on any qubit, local or not: every amplitude knows its full
// index (local bits from its position, the rest from the chunk), so they are
// evaluated per amplitude (or once per chunk). The host orders the pass's
// gates into as few stages as their dependencies allow.
//
// Every gate is applied with its own FP64 matrix, in an order that respects
// all dependencies, so the result equals the gate-by-gate result up to the
// rounding of each individual product.

#include "fused_pass.h"
#include "fused_device.cuh"

#include "cost_model.h"
#include "simulator.h"

#include <algorithm>
#include <cmath>

namespace qcsb
{
namespace
{

using namespace fdev;

// The run-time program: every op of the parameter block interpreted in turn.
template <typename Real, bool BATCH>
__global__ void __launch_bounds__(128, sizeof(Real) == 8 ? 3 : 4)
    fused_pass_kernel(const __grid_constant__ FPassParams p)
{
    typedef typename Cx<Real>::T V;
    fused_pass_body<Real, BATCH>(p, [&](const ChunkCtx<V> &cx) { run_stages<V, BATCH>(p, cx); });
}

// The matrices of a tensor pass: thread (matrix, col) applies the ops of the
// matrix's stage, exactly as the register stage above applies them, to the
// unit vector of input slot col, with the stage's condition bits set as the
// matrix index says and every other bit outside the stage zero (no op of the
// stage depends on those). The resulting column M[.][col] is written as the
// B fragments of the tensor pass's m16n8k8 products, for the real part Mr,
// the imaginary part Mi and Mr + Mi: B[u][nu] = M[s(nu)][u] for input slot u
// (tensor layout) and output column nu = 8i + 2t' + e of n-tile i, output
// slot s(nu) = 8i + t' + 4e; lane 4g + t of fragment 4 * part + 2j + i
// holds (B[8j + t][8i + g], B[8j + t + 4][8i + g]).
template <typename Real>
__global__ void __launch_bounds__(64) stage_matrix_kernel(const __grid_constant__ FPassParams p,
                                                          const __grid_constant__ TBuildParams tb)
{
    typedef typename Cx<Real>::T V;
    __shared__ V scratch[64][R];
    const int width = tb.width;   // 4: 16 x 16 matrices, 3: 8 x 8 (one thread per column)
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t mat = gid >> width;
    const int col = static_cast<int>(gid & ((1u << width) - 1u));
    if (mat >= tb.nmats)
        return;
    // batched passes: register reg0 + blockIdx.y, its entries and its matrices
    const uint32_t breg = tb.reg0 + blockIdx.y;
    const void *blk = tb.regs > 0 ? static_cast<const void *>(p.mats + static_cast<size_t>(breg) * p.mat_stride) : nullptr;
    const BuildEntries<V> ent{p, blk, tb.batch_float, 0u};
    const uint32_t omat = tb.regs > 0 ? breg * tb.nmats + mat : mat;   // matrix slot written
    int st = 0;
    while (st + 1 < tb.nstages && tb.stages[st + 1].woff <= mat)
        ++st;
    const TStage &S = tb.stages[st];
    const FStage &FS = p.stages[st];
    const uint32_t v = mat - S.woff;
    const int k = p.k;
    uint32_t j0 = 0;
    for (int i = 0; i < S.nlc; ++i)
        if ((v >> i) & 1)
            j0 |= 1u << S.gpos[kStageBits + i];
    uint64_t local = 0;
    for (int i = 0; i < k; ++i)
        local |= p.qbit[i];
    uint64_t cbase = 0, chunk = 0;
    for (int i = 0; i < S.ngc; ++i)
        if ((v >> (S.nlc + i)) & 1)
        {
            const int q = S.gq[i];
            cbase |= 1ull << q;
            chunk |= 1ull << (q - __popcll(local & ((1ull << q) - 1)));
        }
    // the register pass's thread index of this group: j0 without the stage bits
    uint32_t tidx = 0;
    for (int l = 0, pos = 0; l < k; ++l)
    {
        if (l == FS.sbits[0] || l == FS.sbits[1] || l == FS.sbits[2] || l == FS.sbits[3])
            continue;
        if ((j0 >> l) & 1)
            tidx |= 1u << pos;
        ++pos;
    }
    // slot u of the tensor layout is slot reg(u) of the register layout; for
    // 8 x 8 stages the fourth register bit takes the value this matrix's
    // condition bits give it (it is a group bit of the tensor layout)
    const int pad = width == 3 && ((j0 >> S.sbits[3]) & 1) ? 1 << ((S.perm >> 6) & 3) : 0;
    auto reg = [&](int u) {
        int r = pad;
#pragma unroll
        for (int b = 0; b < kStageBits; ++b)
            if (b < width && ((u >> b) & 1))
                r |= 1 << ((S.perm >> (2 * b)) & 3);
        return r;
    };
    const int r0 = reg(col);
    V a[R];
#pragma unroll
    for (int r = 0; r < R; ++r)
        a[r] = r == r0 ? V{1, 0} : V{0, 0};
    const StageSlots<V> ss{scratch[threadIdx.x], 0u, {1u, 2u, 4u, 8u}};
    const int T = 1 << (k - kStageBits);
    for (int oi = FS.op_begin; oi < FS.op_end; ++oi)
    {
        const FOp &op = p.ops[oi];
        if (op.kind == F_SIGNS)
        {
            uint32_t neg = 0;
            const int nt = static_cast<int>(op.lcmask);
            for (int i = 1; i <= nt; ++i)
            {
                const FOp &t = p.ops[oi + i];
                if ((j0 & t.lcmask) == t.lcval && (cbase & t.gcmask) == t.gcval)
                    neg ^= t.moff;
            }
#pragma unroll
            for (int r = 0; r < R; ++r)
            {
                const uint32_t sgn = ((neg >> r) & 1u) << 31;
                a[r].x = flip_by(a[r].x, sgn);
                a[r].y = flip_by(a[r].y, sgn);
            }
            oi += nt;
            continue;
        }
        if (op.kind == F_PRUN)
        {
            phase_inline<V>(a, op, p.ops + oi + 1, j0, cbase, chunk, static_cast<int>(tidx), T, p.tables,
                            [&](int off) { return ent[off]; });
            oi += op.lcmask;
            continue;
        }
        if ((cbase & op.gcmask) != op.gcval)
            continue;
        apply_op<V>(a, op, BuildEntries<V>{p, blk, tb.batch_float, op.moff}, j0, cbase, ss);
    }
    if (tb.umma)
    {
        // the 32 x 32 real operand W of a tcgen05 pass (outputs n: Re 0-15,
        // Im 16-31; inputs k likewise): column u of M gives
        // W[u][o] = Mr[o][u], W[u][16 + o] = Mi[o][u],
        // W[16 + u][o] = -Mi[o][u], W[16 + u][16 + o] = Mr[o][u]; each as a
        // TF32 high part and the TF32 rounding of the remainder
        unsigned char *hi_base = reinterpret_cast<unsigned char *>(tb.out) + static_cast<size_t>(mat) * kUmmaSlab;
        unsigned char *lo_base = hi_base + static_cast<size_t>(tb.nmats) * kUmmaSlab;
        auto put = [&](int nn, int kk, double w) {
            const size_t off = static_cast<size_t>((nn >> 3) * 1024 + (kk >> 3) * 256 + ((kk >> 2) & 1) * 128 +
                                                   (nn & 7) * 16 + (kk & 3) * 4);
            uint32_t h, l;
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(static_cast<float>(w)));
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(static_cast<float>(w - __uint_as_float(h))));
            *reinterpret_cast<uint32_t *>(hi_base + off) = h;
            *reinterpret_cast<uint32_t *>(lo_base + off) = l;
        };
#pragma unroll
        for (int o = 0; o < R; ++o)
        {
            const V y = a[reg(o)];
            put(o, col, y.x);
            put(16 + o, col, y.y);
            put(o, 16 + col, -y.y);
            put(16 + o, 16 + col, y.x);
        }
        return;
    }
    if (width == 3)
    {
        // B[u][nu] = M[s(nu)][u], output slot s(nu) = (nu >> 1) + 4 (nu & 1);
        // lane 4 nu + t of fragment part holds (B[t][nu], B[t + 4][nu])
        const int b = col >> 2, t = col & 3;
#pragma unroll
        for (int nu = 0; nu < 8; ++nu)
        {
            const V y = a[reg((nu >> 1) + 4 * (nu & 1))];
            const double parts[3] = {y.x, y.y - y.x, -(y.x + y.y)};
            const int lane = nu * 4 + t;
#pragma unroll
            for (int part = 0; part < 3; ++part)
            {
                if (tb.tf32)
                {
                    uint32_t hi, lo;
                    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(static_cast<float>(parts[part])));
                    asm("cvt.rna.tf32.f32 %0, %1;"
                        : "=r"(lo)
                        : "f"(static_cast<float>(parts[part] - __uint_as_float(hi))));
                    uint32_t *f = reinterpret_cast<uint32_t *>(tb.out) +
                                  ((static_cast<size_t>(omat) * kTensor3Fragments + part) * 32 + lane) * 4;
                    f[b] = hi;
                    f[2 + b] = lo;
                }
                else
                {
                    Real *f = reinterpret_cast<Real *>(tb.out) +
                              ((static_cast<size_t>(omat) * kTensor3Fragments + part) * 32 + lane) * 2;
                    f[b] = parts[part];
                }
            }
        }
        return;
    }
    const int j = col >> 3, b = (col >> 2) & 1, t = col & 3;
    if (tb.tf32)
    {
        // TF32 high part and the TF32 rounding of the remainder, per entry
        auto split = [](double v, uint32_t &hi, uint32_t &lo) {
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(static_cast<float>(v)));
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(static_cast<float>(v - __uint_as_float(hi))));
        };
        uint32_t *out = reinterpret_cast<uint32_t *>(tb.out) + static_cast<size_t>(mat) * kTensorFragments * 128;
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int g = 0; g < 8; ++g)
            {
                const V y = a[reg(8 * i + (g >> 1) + 4 * (g & 1))];
                const double parts[3] = {y.x, y.y - y.x, -(y.x + y.y)};
                const int lane = g * 4 + t;
#pragma unroll
                for (int part = 0; part < 3; ++part)
                {
                    uint32_t hi, lo;
                    split(parts[part], hi, lo);
                    uint32_t *f = out + ((part * 4 + j * 2 + i) * 32 + lane) * 4;
                    f[b] = hi;
                    f[2 + b] = lo;
                }
            }
        return;
    }
    Real *out = reinterpret_cast<Real *>(tb.out) + static_cast<size_t>(mat) * kTensorFragments * 64;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int g = 0; g < 8; ++g)
        {
            const V y = a[reg(8 * i + (g >> 1) + 4 * (g & 1))];
            const int lane = g * 4 + t;
            out[((0 * 4 + j * 2 + i) * 32 + lane) * 2 + b] = y.x;
            out[((1 * 4 + j * 2 + i) * 32 + lane) * 2 + b] = y.y - y.x;
            out[((2 * 4 + j * 2 + i) * 32 + lane) * 2 + b] = -(y.x + y.y);
        }
}

} // namespace

template <typename R>
int launch_stage_matrices(const FPassParams &prm, const TBuildParams &tb, cudaStream_t stream)
{
    const unsigned threads = 64;
    const unsigned blocks = static_cast<unsigned>((static_cast<uint64_t>(tb.nmats) * (1u << tb.width) + threads - 1) / threads);
    if (tb.regs == 0)
    {
        stage_matrix_kernel<R><<<blocks, threads, 0, stream>>>(prm, tb);
        QCSB_CUDA(cudaGetLastError());
        return 1;
    }
    if (tb.width != 3 || tb.umma)
        throw std::runtime_error("internal: batched stage matrices need 8 x 8 stages");
    // registers in slices of at most 65535 (the grid's y limit)
    int launches = 0;
    TBuildParams slice = tb;
    for (uint32_t r0 = 0; r0 < tb.regs; r0 += 65535u)
    {
        slice.reg0 = r0;
        const dim3 grid(blocks, std::min<uint32_t>(tb.regs - r0, 65535u));
        stage_matrix_kernel<R><<<grid, threads, 0, stream>>>(prm, slice);
        QCSB_CUDA(cudaGetLastError());
        ++launches;
    }
    return launches;
}
template int launch_stage_matrices<double>(const FPassParams &, const TBuildParams &, cudaStream_t);

// ------------------------------------------------------------ planning

OpClass classify(const GateOp &op)
{
    OpClass c;
    uint64_t t = 0;
    for (int i = 0; i < op.nt; ++i)
        t |= 1ull << op.tq[i];
    if (op.diag)
    {
        c.fusable = op.na == 1 || op.nt <= 2;
        c.dense = 0;
        c.diag = t | op.cmask;
    }
    else
    {
        c.fusable = op.nt >= 1 && op.nt <= 2;
        c.dense = t;
        c.diag = op.cmask;
    }
    return c;
}

// X and Y commute when X's dense qubits avoid all of Y's qubits and X's
// diagonal qubits avoid Y's dense qubits (ops that are diagonal on every
// shared qubit commute).
bool commute(const OpClass &x, const OpClass &y)
{
    return (x.dense & (y.dense | y.diag)) == 0 && (x.diag & y.dense) == 0;
}

bool is_perm(const GateOp &op, int size)
{
    // the na x na block is [[0,1],[1,0]]
    if (op.diag || op.na != 2 || size != 2)
        return false;
    const cplx *m = op.mat;
    return m[0].re == 0 && m[0].im == 0 && m[1].re == 1 && m[1].im == 0 &&
           m[2].re == 1 && m[2].im == 0 && m[3].re == 0 && m[3].im == 0;
}

bool is_x(const GateOp &op) { return op.nt == 1 && is_perm(op, 2); }
bool is_swap(const GateOp &op) { return op.nt == 2 && op.act[0] == 1 && op.act[1] == 2 && is_perm(op, 2); }

bool is_real(const GateOp &op)
{
    const int ne = op.diag ? op.na : op.na * op.na;
    for (int e = 0; e < ne; ++e)
        if (op.mat[e].im != 0.0)
            return false;
    return true;
}

// Uncontrolled X gates move later in the queue, each until an op it cannot
// pass, where it is placed (or until the end): an X on qubit q passes an op
// that does not touch q; a diagonal op or a control on q with that bit of its
// pattern flipped (X D X is D with the pattern bit flipped; likewise a
// control's value); a controlled X on target q unchanged (X commutes with X);
// and an uncontrolled 2x2 on q takes it in as a column swap (M X), where it
// ends. Two X on one qubit cancel. Every change is exact (no arithmetic), and
// X gates on scattered qubits (the basis-state input of a QFT) no longer hold
// local bits of a pass that the gates after them need.
std::vector<GateOp> defer_x(const std::vector<GateOp> &q)
{
    std::vector<GateOp> out;
    out.reserve(q.size());
    uint64_t pending = 0;
    auto x_op = [](int t) {
        GateOp x;
        x.nt = 1;
        x.tq[0] = t;
        x.na = 2;
        x.act[0] = 0;
        x.act[1] = 1;
        x.mat[0] = cplx{0.0, 0.0};
        x.mat[1] = cplx{1.0, 0.0};
        x.mat[2] = cplx{1.0, 0.0};
        x.mat[3] = cplx{0.0, 0.0};
        return x;
    };
    for (const GateOp &in : q)
    {
        if (is_x(in) && in.cmask == 0)
        {
            pending ^= 1ull << in.tq[0];
            continue;
        }
        GateOp op = in;
        op.cval ^= op.cmask & pending;
        for (int i = 0; i < op.nt; ++i)
        {
            const int t = op.tq[i];
            if (!((pending >> t) & 1))
                continue;
            if (op.diag)
            {
                for (int a = 0; a < op.na; ++a)
                    op.act[a] ^= static_cast<uint8_t>(1u << i);
                // keep the active sub-indices ascending, entries alongside
                for (int a = 1; a < op.na; ++a)
                    for (int b = a; b > 0 && op.act[b - 1] > op.act[b]; --b)
                    {
                        std::swap(op.act[b - 1], op.act[b]);
                        std::swap(op.mat[b - 1], op.mat[b]);
                    }
            }
            else if (is_x(op))
            {
                // a controlled X on target t commutes with X on t
            }
            else if (op.nt == 1 && op.cmask == 0 && op.na == 2 && op.act[0] == 0 && op.act[1] == 1)
            {
                std::swap(op.mat[0], op.mat[1]);
                std::swap(op.mat[2], op.mat[3]);
                pending &= ~(1ull << t);
            }
            else
            {
                out.push_back(x_op(t));
                pending &= ~(1ull << t);
            }
        }
        out.push_back(op);
    }
    for (int t = 0; t < 64; ++t)
        if ((pending >> t) & 1)
            out.push_back(x_op(t));
    return out;
}

int op_entry_count(const GateOp &op)
{
    if (op.diag)
        return op.na == 1 ? 1 : 4;
    if (op.nt == 1)
        return is_x(op) ? 0 : 4;
    return is_swap(op) ? 0 : 16;
}

// Full 2^nt x 2^nt matrix of a dense GateOp (row-major).
void expand_dense(const GateOp &op, double2 *out)
{
    const int d = 1 << op.nt;
    for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c)
            out[r * d + c] = make_double2(r == c ? 1.0 : 0.0, 0.0);
    for (int a = 0; a < op.na; ++a)
        for (int b = 0; b < op.na; ++b)
            out[op.act[a] * d + op.act[b]] = make_double2(op.mat[a * op.na + b].re, op.mat[a * op.na + b].im);
}

// Greedy pass construction. Ops are taken in queue order; an op joins the
// current pass when its dense targets fit in Q (k qubits) and it commutes
// with every op left behind so far (an op is left behind when it does not
// fit).
std::vector<Segment> plan_greedy(const std::vector<GateOp> &q, int n, int k, int low, int max_ops)
{
    const size_t N = q.size();
    std::vector<OpClass> cls(N);
    for (size_t i = 0; i < N; ++i)
        cls[i] = classify(q[i]);
    std::vector<bool> done(N, false);
    std::vector<Segment> out;
    const uint64_t low_mask = (1ull << low) - 1;
    const uint64_t all = (n >= 64) ? ~0ull : ((1ull << n) - 1);
    size_t first = 0;
    while (true)
    {
        while (first < N && done[first])
            ++first;
        if (first >= N)
            break;
        if (!cls[first].fusable)
        {
            Segment s;
            s.fused = false;
            s.plain_op = (int)first;
            out.push_back(std::move(s));
            done[first] = true;
            continue;
        }
        Segment s;
        s.fused = true;
        s.plain_op = -1;
        uint64_t local = low_mask;
        uint64_t blocked_all = 0, blocked_dense = 0;
        int entries = 0;
        const size_t window_end = std::min(N, first + kPlanWindow);
        for (size_t i = first; i < window_end; ++i)
        {
            if (done[i])
                continue;
            const OpClass &c = cls[i];
            const uint64_t support = c.dense | c.diag;
            const int ec = c.fusable ? op_entry_count(q[i]) : 0;
            bool take = c.fusable && (int)s.pass.ops.size() < max_ops && entries + ec <= kFusedMaxEntries &&
                        (c.dense & blocked_all) == 0 && (c.diag & blocked_dense) == 0;
            if (take)
            {
                const uint64_t nl = local | c.dense;
                if (__builtin_popcountll(nl) > k)
                    take = false;
                else
                    local = nl;
            }
            if (take)
            {
                s.pass.ops.push_back((int)i);
                done[i] = true;
                entries += ec;
            }
            else
            {
                blocked_all |= support;
                blocked_dense |= c.dense;
                if ((blocked_all & all) == all && (blocked_dense & all) == all)
                    break;
            }
        }
        for (int b = 0; b < n && __builtin_popcountll(local) < k; ++b)
            local |= 1ull << b;
        s.pass.local = local;
        s.pass.k = k;
        out.push_back(std::move(s));
    }
    return out;
}

// Order a pass's ops into stages of at most kStageBits local dense bits:
// repeatedly open a stage and add every op whose dependencies are met and
// whose dense targets fit, in queue order, until none fits.
void schedule_stages(const std::vector<GateOp> &q, const PlannedPass &pp, const int *loc_of,
                     std::vector<std::vector<int>> &stage_ops, std::vector<uint32_t> &stage_bits)
{
    const size_t m = pp.ops.size();
    std::vector<OpClass> cls(m);
    std::vector<uint32_t> need(m, 0);
    for (size_t i = 0; i < m; ++i)
    {
        cls[i] = classify(q[pp.ops[i]]);
        uint64_t d = cls[i].dense;
        while (d)
        {
            const int b = __builtin_ctzll(d);
            need[i] |= 1u << loc_of[b];
            d &= d - 1;
        }
    }
    std::vector<bool> done(m, false);
    size_t left = m;
    while (left > 0)
    {
        uint32_t bits = 0;
        std::vector<int> ops;
        bool progress = true;
        while (progress)
        {
            progress = false;
            for (size_t i = 0; i < m; ++i)
            {
                if (done[i])
                    continue;
                bool ready = true;
                for (size_t j = 0; j < i && ready; ++j)
                    if (!done[j] && !commute(cls[j], cls[i]))
                        ready = false;
                if (!ready)
                    continue;
                const uint32_t nb = bits | need[i];
                if (__builtin_popcount(nb) > pp.stage_width)
                    continue;
                bits = nb;
                ops.push_back((int)i);
                done[i] = true;
                --left;
                progress = true;
            }
        }
        stage_ops.push_back(std::move(ops));
        stage_bits.push_back(bits);
    }
}

// Unitary diagonal gates on at most two targets join phase runs, which run
// inside the register stages: -1 phases as one F_SIGNS, gates on at most one
// stage bit as one F_PRUN (table-fed factors), gates wholly on stage bits as
// its per-slot factors, the rest one by one. A one-entry phase (CP, T, ...)
// weighs 1, a diagonal with two or four entries (RZ, RZZ) 2; phases by -1 or
// +-i (Z, CZ, S) weigh 0: an F_PRUN pays only with some weight in it.
constexpr int kStageSlots = 1 << kStageBits;
constexpr int kInlineRunMin = 2;          // gates an F_PRUN needs to beat single ops (about 200 instructions each)

int phase_weight(const GateOp &op)
{
    if (op.na != 1)
        return 2;
    // -1 and +-i run as sign flips and exchanges: cheaper alone than as terms
    const cplx e = op.mat[0];
    const bool clifford = (e.re == -1.0 && e.im == 0.0) || (e.re == 0.0 && (e.im == 1.0 || e.im == -1.0));
    return clifford ? 0 : 1;
}

// A phase of -1 on one pattern (Z, CZ, CCZ): runs as a sign flip.
bool is_sign_op(const GateOp &op)
{
    return op.diag && op.na == 1 && op.mat[0].re == -1.0 && op.mat[0].im == 0.0;
}

bool phase_run_op(const GateOp &op)
{
    if (!op.diag || op.nt > 2)
        return false;
    // the expansion divides by entries (conjugates them): unit modulus only,
    // which excludes the zeroing ops of collapsed measurements
    for (int a = 0; a < op.na; ++a)
        if (std::fabs(op.mat[a].re * op.mat[a].re + op.mat[a].im * op.mat[a].im - 1.0) > 1e-12)
            return false;
    return true;
}

// Within one stage, gather the diagonal ops into as few runs as their order
// allows. A diagonal may sit in any gap between the stage's other ops from
// after the last earlier op it does not commute with to before the first later
// one: an interval of gaps. The fewest gaps that meet every interval are
// found greedily (by interval end), and each diagonal goes to the LATEST of
// them inside its interval, so that runs sit between whole groups of gates
// (the phases of split one-qubit gates before and after a layer) and those
// that nothing later blocks sink to the end of the stage (a QFT's phases to
// qubits outside the stage). Every non-commuting pair keeps its order;
// diagonal ops commute with one another.
std::vector<int> cluster_diagonals(const std::vector<GateOp> &q, const PlannedPass &pp, const std::vector<int> &ops)
{
    const size_t m = ops.size();
    std::vector<OpClass> cls(m);
    std::vector<bool> diag(m);
    std::vector<size_t> rank(m);   // non-diagonal ops before position i
    size_t nd = 0;
    for (size_t i = 0; i < m; ++i)
    {
        cls[i] = classify(q[pp.ops[ops[i]]]);
        diag[i] = phase_run_op(q[pp.ops[ops[i]]]);
        rank[i] = nd;
        if (!diag[i])
            ++nd;
    }
    // gap g lies before the g-th non-diagonal op (g == nd: the stage's end)
    std::vector<size_t> lo(m, 0), hi(m, nd);
    std::vector<size_t> dg;
    for (size_t i = 0; i < m; ++i)
    {
        if (!diag[i])
            continue;
        dg.push_back(i);
        for (size_t j = i; j-- > 0;)
            if (!diag[j] && !commute(cls[i], cls[j]))
            {
                lo[i] = rank[j] + 1;
                break;
            }
        for (size_t j = i + 1; j < m; ++j)
            if (!diag[j] && !commute(cls[i], cls[j]))
            {
                hi[i] = rank[j];
                break;
            }
    }
    std::vector<size_t> by_end = dg;
    std::stable_sort(by_end.begin(), by_end.end(), [&](size_t a, size_t b) { return hi[a] < hi[b]; });
    std::vector<size_t> points;   // ascending
    for (size_t d : by_end)
        if (points.empty() || points.back() < lo[d])
            points.push_back(hi[d]);
    std::vector<std::vector<int>> at(nd + 1);
    for (size_t d : dg)
    {
        // the latest chosen gap inside [lo, hi]
        const auto it = std::upper_bound(points.begin(), points.end(), hi[d]);
        at[*(it - 1)].push_back(ops[d]);
    }
    std::vector<int> out;
    out.reserve(m);
    for (size_t i = 0; i < m; ++i)
    {
        if (diag[i])
            continue;
        out.insert(out.end(), at[rank[i]].begin(), at[rank[i]].end());
        out.push_back(ops[i]);
    }
    out.insert(out.end(), at[nd].begin(), at[nd].end());
    return out;
}

int fop_entries(const GateOp &op, const FOp &f, bool swapped, double2 *m)
{
    switch (f.kind)
    {
    case F_TERM:
        // the entry of active sub-index phys[0]
        m[0] = make_double2(op.mat[f.phys[0]].re, op.mat[f.phys[0]].im);
        return 1;
    case F_PHASE:
        m[0] = make_double2(op.mat[0].re, op.mat[0].im);
        return 1;
    case F_DIAG:
        for (int s = 0; s < 4; ++s)
            m[s] = make_double2(1.0, 0.0);
        for (int a = 0; a < op.na; ++a)
            m[op.act[a]] = make_double2(op.mat[a].re, op.mat[a].im);
        if (op.nt < 2)
        {
            // second target absent: entries 2, 3 repeat 0, 1
            m[2] = m[0];
            m[3] = m[1];
        }
        return 4;
    case F_DENSE1:
    case F_DENSE1R:
    {
        double2 full[4];
        expand_dense(op, full);
        for (int i = 0; i < 4; ++i)
            m[i] = full[i];
        return 4;
    }
    case F_DENSE2:
    {
        double2 full[16];
        expand_dense(op, full);
        // exchanged targets: the two sub-index bits swap roles
        auto sw = [&](int v) { return swapped ? (((v & 1) << 1) | ((v >> 1) & 1)) : v; };
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c)
                m[r * 4 + c] = full[sw(r) * 4 + sw(c)];
        return 16;
    }
    default:
        return 0;
    }
}

int layer_entries(const std::vector<GateOp> &q, const FOpSource &src, uint8_t kind, double2 *m)
{
    if (kind == F_DENSE1X2)
    {
        int off = 0;
        for (int b = 0; b < kStageBits; ++b)
            if (src.layer[b] >= 0)
            {
                expand_dense(q[src.layer[b]], m + off);
                off += 4;
            }
        return off;
    }
    for (int b = 0; b < kStageBits; ++b)
    {
        if (src.layer[b] >= 0)
            expand_dense(q[src.layer[b]], m + 4 * b);
        else
        {
            m[4 * b] = m[4 * b + 3] = make_double2(1.0, 0.0);
            m[4 * b + 1] = m[4 * b + 2] = make_double2(0.0, 0.0);
        }
    }
    return 4 * kStageBits;
}

namespace
{

double2 cmul_host(double2 x, double2 y)
{
    return make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
}

// One inclusion-exclusion member of a phase-run gate: the factor (entry a of
// gate qi, conjugated when conj) on the slots whose stage bits include mono,
// under a condition on the thread's other local bits and on the chunk.
struct TermRec
{
    int qi;
    int a;
    uint8_t mono;
    uint8_t conj;
    uint32_t lcm, lcv;
    uint64_t gcm, gcv;
};

constexpr size_t kPassTableBudget = size_t(1) << 16;   // table entries of one pass (1 MiB)

// Fill the kernel parameters of a pass. Returns false when the pass does not
// fit the parameter block limits.
bool build_params_body(const std::vector<GateOp> &q, const PlannedPass &pp, int n, int k, FPassParams &prm,
                       std::vector<FOpSource> *src, std::vector<double2> *tables, std::vector<StageCond> *conds)
{
    std::memset(&prm, 0, sizeof(prm));
    prm.n = n;
    prm.k = k;
    prm.chunks = 1ull << (n - k);
    int loc_of[kMaxQubits];
    for (int b = 0; b < kMaxQubits; ++b)
        loc_of[b] = -1;
    int nl = 0;
    for (int b = 0; b < n; ++b)
        if ((pp.local >> b) & 1)
        {
            loc_of[b] = nl;
            prm.qmasks[nl] = (1ull << b) - 1;
            prm.qbit[nl] = 1ull << b;
            ++nl;
        }
    if (nl != k)
        throw std::runtime_error("internal: pass locality size mismatch");
    // bit of the chunk index that holds each non-local qubit
    int cpos[kMaxQubits];
    for (int b = 0, c = 0; b < n; ++b)
        cpos[b] = loc_of[b] >= 0 ? -1 : c++;
    const size_t table_start = tables ? tables->size() : 0;
    if (pp.ops.size() > (size_t)kFusedMaxOps)
        return false;

    std::vector<std::vector<int>> stage_ops;
    std::vector<uint32_t> stage_bits;
    schedule_stages(q, pp, loc_of, stage_ops, stage_bits);
    if (stage_ops.size() > (size_t)kFusedMaxStages)
        return false;
    int nops = 0, nentries = 0, ns = 0;
    for (size_t si = 0; si < stage_ops.size(); ++si)
    {
        // stage bits: the needed ones, padded with the lowest other local bits
        // (three-bit stages: with bits no op of the stage involves first, so
        // that the fourth bit is no condition of an 8 x 8 tensor stage)
        uint32_t bits = stage_bits[si];
        if (pp.stage_width < kStageBits)
        {
            uint32_t touched = 0;
            for (int oi : stage_ops[si])
            {
                const GateOp &op = q[pp.ops[oi]];
                uint64_t pattern = op.cmask;
                for (int i = 0; i < op.nt; ++i)
                    pattern |= 1ull << op.tq[i];
                for (int b = 0; b < n; ++b)
                    if (((pattern >> b) & 1) && loc_of[b] >= 0)
                        touched |= 1u << loc_of[b];
            }
            for (int l = 0; l < k && __builtin_popcount(bits) < kStageBits; ++l)
                if (!((touched >> l) & 1))
                    bits |= 1u << l;
        }
        for (int l = 0; l < k && __builtin_popcount(bits) < kStageBits; ++l)
            bits |= 1u << l;
        uint8_t sbits[kStageBits];
        int pos_in_stage[kMaxLocal];
        int nb = 0;
        for (int l = 0; l < k; ++l)
            if ((bits >> l) & 1)
            {
                pos_in_stage[l] = nb;
                sbits[nb++] = static_cast<uint8_t>(l);
            }
        // the bits outside the stage that its ops depend on
        StageCond cond;
        cond.dense = stage_bits[si];
        for (int oi : stage_ops[si])
        {
            const GateOp &op = q[pp.ops[oi]];
            uint64_t pattern = op.cmask;
            for (int i = 0; i < op.nt; ++i)
                pattern |= 1ull << op.tq[i];
            for (int b = 0; b < n; ++b)
            {
                if (!((pattern >> b) & 1))
                    continue;
                const int l = loc_of[b];
                if (l < 0)
                    cond.gmask |= 1ull << b;
                else if (!((bits >> l) & 1))
                    cond.lmask |= 1u << l;
                else
                    cond.touch |= 1u << l;
            }
        }
        // the scheduled stage becomes one register stage, opened at its first op
        auto open_stage = [&]() -> FStage * {
            if (ns >= kFusedMaxStages)
                return nullptr;
            FStage &S = prm.stages[ns++];
            std::memset(&S, 0, sizeof(S));
            std::memcpy(S.sbits, sbits, sizeof(sbits));
            S.op_begin = static_cast<uint16_t>(nops);
            if (conds)
                conds->push_back(cond);
            return &S;
        };
        // the stage bits a diagonal op's pattern (controls and targets) involves
        auto pattern_stage_bits = [&](const GateOp &op) {
            uint64_t cm = op.cmask;
            for (int i = 0; i < op.nt; ++i)
                cm |= 1ull << op.tq[i];
            int c = 0;
            for (int b = 0; b < n; ++b)
                if (((cm >> b) & 1) && loc_of[b] >= 0 && ((bits >> loc_of[b]) & 1))
                    ++c;
            return c;
        };
        auto pattern_bits = [&](const GateOp &op) {
            uint64_t cm = op.cmask;
            for (int i = 0; i < op.nt; ++i)
                cm |= 1ull << op.tq[i];
            return __builtin_popcountll(cm);
        };
        // the terms of a phase-run op: one per inclusion-exclusion member
        auto term_records = [&](int qi, std::vector<TermRec> &out) {
            const GateOp &op = q[qi];
            for (int a = 0; a < op.na; ++a)
            {
                uint64_t cm = op.cmask, cv = op.cval;
                for (int i = 0; i < op.nt; ++i)
                {
                    cm |= 1ull << op.tq[i];
                    if ((op.act[a] >> i) & 1)
                        cv |= 1ull << op.tq[i];
                }
                uint32_t s1 = 0, s0 = 0, lcm = 0, lcv = 0;
                uint64_t gcm = 0, gcv = 0;
                for (int b = 0; b < n; ++b)
                {
                    if (!((cm >> b) & 1))
                        continue;
                    const bool v = (cv >> b) & 1;
                    const int l = loc_of[b];
                    if (l >= 0 && ((bits >> l) & 1))
                        (v ? s1 : s0) |= 1u << pos_in_stage[l];
                    else if (l >= 0)
                    {
                        lcm |= 1u << l;
                        lcv |= v ? 1u << l : 0u;
                    }
                    else
                    {
                        gcm |= 1ull << b;
                        gcv |= v ? 1ull << b : 0ull;
                    }
                }
                for (uint32_t A = s0;; A = (A - 1) & s0)
                {
                    out.push_back(TermRec{qi, a, static_cast<uint8_t>(s1 | A),
                                          static_cast<uint8_t>(__builtin_popcount(A) & 1), lcm, lcv, gcm, gcv});
                    if (A == 0)
                        break;
                }
            }
        };
        auto push_term = [&](const TermRec &r) -> bool {
            if (nops >= kFusedMaxOps || nentries + 1 > kFusedMaxEntries)
                return false;
            FOp &t = prm.ops[nops++];
            std::memset(&t, 0, sizeof(t));
            t.kind = F_TERM;
            t.b0 = r.mono;
            t.b1 = r.conj;
            t.phys[0] = static_cast<uint8_t>(r.a);
            t.lcmask = r.lcm;
            t.lcval = r.lcv;
            t.gcmask = r.gcm;
            t.gcval = r.gcv;
            t.moff = static_cast<uint16_t>(nentries);
            fop_entries(q[r.qi], t, false, prm.entries + nentries);
            ++nentries;
            if (src)
                src->push_back({r.qi, false});
            return true;
        };
        FStage *cur = nullptr;
        std::vector<int> sops = cluster_diagonals(q, pp, stage_ops[si]);
        size_t idx = 0;
        size_t singles_end = 0;   // ops [idx, singles_end) run one by one
        while (idx < sops.size())
        {
            size_t run_end = idx;
            int weight = 0;
            while (idx >= singles_end && run_end < sops.size() && phase_run_op(q[pp.ops[sops[run_end]]]))
                weight += phase_weight(q[pp.ops[sops[run_end++]]]);
            // Ops of the run whose patterns hold at most one stage bit run as
            // one F_PRUN (table entries or one complex product per term and
            // thread, at most 48 per thread to apply), ops wholly on stage bits
            // as its per-slot factors, the others one by one (a phase on
            // 2^(4 - p) of the 16 slots). Clifford phases (S, Sdg) join a run
            // that has other phases, but a run of them alone stays single ops
            // (exchanges and sign flips on the integer pipe, where the run
            // would take FP64 products, the busier pipe on passes of dense
            // gates; measured).
            // -1 phases of the run (Z, CZ, CCZ) become one F_SIGNS; the rest of
            // the run is looked at again without them
            if (run_end > idx)
            {
                std::vector<int> signs, keep;
                for (size_t ri = idx; ri < run_end; ++ri)
                    (is_sign_op(q[pp.ops[sops[ri]]]) ? signs : keep).push_back(sops[ri]);
                if (!signs.empty())
                {
                    if (nops + 1 + (int)signs.size() > kFusedMaxOps)
                        return false;
                    if (cur == nullptr && (cur = open_stage()) == nullptr)
                        return false;
                    FOp &h = prm.ops[nops++];
                    std::memset(&h, 0, sizeof(h));
                    h.kind = F_SIGNS;
                    h.lcmask = static_cast<uint32_t>(signs.size());
                    if (src)
                        src->push_back({pp.ops[signs[0]], false});
                    for (int oi : signs)
                    {
                        const GateOp &op = q[pp.ops[oi]];
                        uint64_t cm = op.cmask, cv = op.cval;
                        for (int i = 0; i < op.nt; ++i)
                        {
                            cm |= 1ull << op.tq[i];
                            if ((op.act[0] >> i) & 1)
                                cv |= 1ull << op.tq[i];
                        }
                        FOp &t = prm.ops[nops++];
                        std::memset(&t, 0, sizeof(t));
                        t.kind = F_SIGNT;
                        uint32_t slots = 0;
                        for (int r = 0; r < kStageSlots; ++r)
                        {
                            bool match = true;
                            for (int b = 0; b < n && match; ++b)
                                if (((cm >> b) & 1) && loc_of[b] >= 0 && ((bits >> loc_of[b]) & 1))
                                    match = ((r >> pos_in_stage[loc_of[b]]) & 1) == ((cv >> b) & 1);
                            if (match)
                                slots |= 1u << r;
                        }
                        for (int b = 0; b < n; ++b)
                        {
                            if (!((cm >> b) & 1))
                                continue;
                            const int l = loc_of[b];
                            const bool v = (cv >> b) & 1;
                            if (l >= 0 && ((bits >> l) & 1))
                                continue;
                            if (l >= 0)
                            {
                                t.lcmask |= 1u << l;
                                t.lcval |= v ? 1u << l : 0u;
                            }
                            else
                            {
                                t.gcmask |= 1ull << b;
                                t.gcval |= v ? 1ull << b : 0ull;
                            }
                        }
                        t.moff = static_cast<uint16_t>(slots);
                        if (src)
                            src->push_back({pp.ops[oi], false});
                    }
                    std::copy(keep.begin(), keep.end(), sops.begin() + idx);
                    sops.erase(sops.begin() + idx + keep.size(), sops.begin() + run_end);
                    continue;
                }
            }
            // (a run of one gate wholly on stage bits also goes in: 16 per-slot
            // factors cost less than a predicated phase on all 16 slots)
            const bool lone_slot_op = run_end - idx == 1 && tables != nullptr && weight > 0 &&
                                      pattern_stage_bits(q[pp.ops[sops[idx]]]) == pattern_bits(q[pp.ops[sops[idx]]]) &&
                                      pattern_bits(q[pp.ops[sops[idx]]]) >= 2;
            if ((run_end - idx >= static_cast<size_t>(kInlineRunMin) || lone_slot_op) && weight > 0)
            {
                // lin: at most one stage bit in the pattern; slot: the whole
                // pattern on stage bits (a fixed factor per slot, folded into
                // 16 per-slot entries; not in batched passes, whose entries
                // are per register); other: single ops
                std::vector<int> lin, slot, other;
                int wlin = 0;
                for (size_t ri = idx; ri < run_end; ++ri)
                {
                    const GateOp &op = q[pp.ops[sops[ri]]];
                    const int sbc = pattern_stage_bits(op);
                    if (sbc <= 1)
                    {
                        lin.push_back(sops[ri]);
                        wlin += phase_weight(op);
                    }
                    else if (tables && sbc == pattern_bits(op))
                        slot.push_back(sops[ri]);
                    else
                        other.push_back(sops[ri]);
                }
                {
                    const bool use_lin = lin.size() >= static_cast<size_t>(kInlineRunMin) && wlin > 0;
                    const bool use_slot = !slot.empty();
                    if (!use_slot)
                        other.insert(other.end(), slot.begin(), slot.end());
                    if (use_lin || use_slot)
                    {
                        if (nops >= kFusedMaxOps)
                            return false;
                        if (cur == nullptr && (cur = open_stage()) == nullptr)
                            return false;
                        const int head = nops++;
                        std::memset(&prm.ops[head], 0, sizeof(FOp));
                        if (src)
                            src->push_back({pp.ops[use_lin ? lin[0] : slot[0]], false});
                        std::vector<TermRec> recs;
                        if (use_lin)
                            for (int oi : lin)
                                term_records(pp.ops[oi], recs);
                        uint64_t packed = 0;
                        uint32_t table_off = 0, used = 0;
                        std::vector<int> where(recs.size(), -1);   // -1 explicit, 0 thread table, 1 + g group g
                        auto factor = [](uint8_t mono) { return mono == 0 ? 0 : 1 + __builtin_ctz(mono); };
                        if (tables)
                        {
                            uint32_t lmask = 0, gmask[kMaxChunkGroups] = {0, 0, 0, 0};
                            std::vector<uint32_t> ccm(recs.size(), 0), ccv(recs.size(), 0);
                            for (size_t i = 0; i < recs.size(); ++i)
                            {
                                const TermRec &r = recs[i];
                                const int e = factor(r.mono);
                                if (r.gcm == 0)
                                {
                                    where[i] = 0;
                                    lmask |= 1u << e;
                                    continue;
                                }
                                if (r.lcm != 0)
                                    continue;
                                // chunk-index bits of the condition, all in one group?
                                uint64_t cm = 0, cv = 0;
                                for (int b = 0; b < n; ++b)
                                    if ((r.gcm >> b) & 1)
                                    {
                                        cm |= 1ull << cpos[b];
                                        cv |= ((r.gcv >> b) & 1) << cpos[b];
                                    }
                                const int g = __builtin_ctzll(cm) / kChunkGroupBits;
                                if (g >= kMaxChunkGroups || (cm >> (g * kChunkGroupBits)) >> kChunkGroupBits)
                                    continue;
                                where[i] = 1 + g;
                                gmask[g] |= 1u << e;
                                ccm[i] = static_cast<uint32_t>(cm >> (g * kChunkGroupBits));
                                ccv[i] = static_cast<uint32_t>(cv >> (g * kChunkGroupBits));
                            }
                            const size_t T = size_t(1) << (k - kStageBits);
                            size_t entries = __builtin_popcount(lmask) * T;
                            for (int g = 0; g < kMaxChunkGroups; ++g)
                                entries += __builtin_popcount(gmask[g]) * (size_t(1) << kChunkGroupBits);
                            if (tables->size() - table_start + entries > kPassTableBudget)
                            {
                                std::fill(where.begin(), where.end(), -1);
                            }
                            else
                            {
                                table_off = static_cast<uint32_t>(tables->size());
                                auto entry = [&](const TermRec &r) {
                                    const cplx m = q[r.qi].mat[r.a];
                                    return make_double2(m.re, r.conj ? -m.im : m.im);
                                };
                                for (int e = 0; e <= kStageBits; ++e)
                                {
                                    if (!((lmask >> e) & 1))
                                        continue;
                                    for (size_t t = 0; t < T; ++t)
                                    {
                                        // local index of thread t's slot 0: zeros at the stage bits
                                        uint32_t j0 = static_cast<uint32_t>(t);
                                        for (int sb = 0; sb < kStageBits; ++sb)
                                        {
                                            const uint32_t lo = j0 & ((1u << sbits[sb]) - 1u);
                                            j0 = lo | ((j0 ^ lo) << 1);
                                        }
                                        double2 v = make_double2(1.0, 0.0);
                                        for (size_t i = 0; i < recs.size(); ++i)
                                            if (where[i] == 0 && factor(recs[i].mono) == e &&
                                                (j0 & recs[i].lcm) == recs[i].lcv)
                                                v = cmul_host(entry(recs[i]), v);
                                        tables->push_back(v);
                                    }
                                }
                                for (int g = 0; g < kMaxChunkGroups; ++g)
                                    for (int e = 0; e <= kStageBits; ++e)
                                    {
                                        if (!((gmask[g] >> e) & 1))
                                            continue;
                                        for (uint32_t c = 0; c < (1u << kChunkGroupBits); ++c)
                                        {
                                            double2 v = make_double2(1.0, 0.0);
                                            for (size_t i = 0; i < recs.size(); ++i)
                                                if (where[i] == 1 + g && factor(recs[i].mono) == e &&
                                                    (c & ccm[i]) == ccv[i])
                                                    v = cmul_host(entry(recs[i]), v);
                                            tables->push_back(v);
                                        }
                                    }
                                packed = lmask;
                                for (int g = 0; g < kMaxChunkGroups; ++g)
                                    packed |= static_cast<uint64_t>(gmask[g]) << (kChunkGroupBits * (g + 1));
                                used = lmask | gmask[0] | gmask[1] | gmask[2] | gmask[3];
                            }
                        }
                        for (size_t i = 0; i < recs.size(); ++i)
                            if (where[i] < 0)
                            {
                                if (!push_term(recs[i]))
                                    return false;
                                used |= 1u << factor(recs[i].mono);
                            }
                        FOp &h = prm.ops[head];
                        h.kind = F_PRUN;
                        h.lcmask = static_cast<uint32_t>(nops - head - 1);
                        h.lcval = table_off;
                        h.gcmask = packed;
                        h.b0 = static_cast<uint8_t>(used);
                        if (use_slot)
                        {
                            if (nentries + kStageSlots > kFusedMaxEntries)
                                return false;
                            h.b1 = 1;
                            h.moff = static_cast<uint16_t>(nentries);
                            for (int r = 0; r < kStageSlots; ++r)
                            {
                                double2 v = make_double2(1.0, 0.0);
                                for (int oi : slot)
                                {
                                    const GateOp &op = q[pp.ops[oi]];
                                    for (int a = 0; a < op.na; ++a)
                                    {
                                        uint64_t cm = op.cmask, cv = op.cval;
                                        for (int i = 0; i < op.nt; ++i)
                                        {
                                            cm |= 1ull << op.tq[i];
                                            if ((op.act[a] >> i) & 1)
                                                cv |= 1ull << op.tq[i];
                                        }
                                        bool match = true;
                                        for (int b = 0; b < n && match; ++b)
                                            if ((cm >> b) & 1)
                                                match = ((r >> pos_in_stage[loc_of[b]]) & 1) == ((cv >> b) & 1);
                                        if (match)
                                            v = cmul_host(make_double2(op.mat[a].re, op.mat[a].im), v);
                                    }
                                }
                                prm.entries[nentries + r] = v;
                            }
                            nentries += kStageSlots;
                        }
                        if (use_lin)
                            lin.clear();
                    }
                    // what is left of the run follows as single ops
                    other.insert(other.end(), lin.begin(), lin.end());
                    std::copy(other.begin(), other.end(), sops.begin() + idx);
                    sops.erase(sops.begin() + idx + other.size(), sops.begin() + run_end);
                    singles_end = idx + other.size();
                    continue;
                }
            }
            // uncontrolled 1-target dense gates on distinct stage bits run as one
            // F_DENSE1X4 / F_DENSE1RX4: gather them from the ops ahead that
            // commute with everything they are moved past
            {
                auto single = [&](const GateOp &g) {
                    if (g.diag || g.nt != 1 || g.cmask != 0 || g.na != 2 || is_x(g))
                        return -1;
                    const int l = loc_of[g.tq[0]];
                    return (l >= 0 && ((bits >> l) & 1)) ? pos_in_stage[l] : -1;
                };
                int pick[kStageBits] = {-1, -1, -1, -1};
                uint32_t seen = 0;
                std::vector<size_t> skipped;
                for (size_t j = idx; j < sops.size() && seen != (1u << kStageBits) - 1; ++j)
                {
                    const GateOp &g = q[pp.ops[sops[j]]];
                    const int b = single(g);
                    bool take = b >= 0 && !((seen >> b) & 1);
                    if (take)
                    {
                        // it moves before the skipped ops: it must commute with them
                        const OpClass cg = classify(g);
                        for (size_t sk : skipped)
                            if (!commute(classify(q[pp.ops[sops[sk]]]), cg))
                            {
                                take = false;
                                break;
                            }
                    }
                    if (take)
                    {
                        pick[b] = static_cast<int>(j);
                        seen |= 1u << b;
                    }
                    else
                        skipped.push_back(j);
                    if (j == idx && !take)
                        break;   // the group must start at the current op
                }
                bool all_real = true;
                for (int b = 0; b < kStageBits; ++b)
                    if (pick[b] >= 0 && !is_real(q[pp.ops[sops[pick[b]]]]))
                        all_real = false;
                // two complex gates: an x2 op; two real ones or three or four:
                // an x4 op, padded with identities on the missing bits (an op
                // dispatch costs about as much as a padded real bit; measured)
                const int count = __builtin_popcount(seen);
                if (count >= 2)
                {
                    const bool pair = count == 2 && !all_real;
                    const int ne = pair ? 8 : 4 * kStageBits;
                    if (nops >= kFusedMaxOps || nentries + ne > kFusedMaxEntries)
                        return false;
                    if (cur == nullptr && (cur = open_stage()) == nullptr)
                        return false;
                    FOp &f = prm.ops[nops++];
                    std::memset(&f, 0, sizeof(f));
                    FOpSource ls{pp.ops[sops[idx]], false, {-1, -1, -1, -1}};
                    for (int b = 0; b < kStageBits; ++b)
                        if (pick[b] >= 0)
                            ls.layer[b] = pp.ops[sops[pick[b]]];
                    if (pair)
                    {
                        f.kind = F_DENSE1X2;
                        int nb = 0;
                        for (int b = 0; b < kStageBits; ++b)
                            if (pick[b] >= 0)
                                (nb++ == 0 ? f.b0 : f.b1) = static_cast<uint8_t>(b);
                    }
                    else
                        f.kind = all_real ? F_DENSE1RX4 : F_DENSE1X4;
                    f.moff = static_cast<uint16_t>(nentries);
                    layer_entries(q, ls, f.kind, prm.entries + nentries);
                    nentries += ne;
                    if (src)
                        src->push_back(ls);
                    // drop the gathered ops from the remaining sequence
                    std::vector<int> rest;
                    for (size_t j = idx; j < sops.size(); ++j)
                    {
                        bool picked = false;
                        for (int b = 0; b < kStageBits; ++b)
                            picked |= pick[b] == static_cast<int>(j);
                        if (!picked)
                            rest.push_back(sops[j]);
                    }
                    sops.resize(idx);
                    sops.insert(sops.end(), rest.begin(), rest.end());
                    continue;
                }
            }
            const int oi = sops[idx++];
            const GateOp &op = q[pp.ops[oi]];
            if (nops >= kFusedMaxOps)
                return false;
            if (cur == nullptr && (cur = open_stage()) == nullptr)
                return false;
            FOp &f = prm.ops[nops++];
            std::memset(&f, 0, sizeof(f));
            f.nt = static_cast<uint8_t>(op.nt);
            uint64_t cm = op.cmask, cv = op.cval;
            bool swapped = false;
            if (op.diag && op.na == 1)
            {
                // one changed sub-index: a phase on the amplitudes whose
                // control and target bits all match
                const cplx e = op.mat[0];
                if (e.re == 0.0 && (e.im == 1.0 || e.im == -1.0))
                {
                    f.kind = F_MULI;
                    f.b1 = e.im < 0.0 ? 1 : 0;
                }
                else
                    f.kind = F_PHASE;
                for (int i = 0; i < op.nt; ++i)
                {
                    cm |= 1ull << op.tq[i];
                    if ((op.act[0] >> i) & 1)
                        cv |= 1ull << op.tq[i];
                }
            }
            else if (op.diag)
            {
                f.kind = F_DIAG;
                for (int i = 0; i < 2; ++i)
                {
                    f.loc[i] = -1;
                    f.spos[i] = -1;
                    f.phys[i] = 0;
                    if (i >= op.nt)
                        continue;
                    const int l = loc_of[op.tq[i]];
                    f.phys[i] = static_cast<uint8_t>(op.tq[i]);
                    if (l >= 0 && ((bits >> l) & 1))
                        f.spos[i] = static_cast<int8_t>(pos_in_stage[l]);
                    else
                        f.loc[i] = static_cast<int8_t>(l);
                }
            }
            else if (op.nt == 1)
            {
                f.kind = is_x(op) ? F_SWAP1 : (is_real(op) ? F_DENSE1R : F_DENSE1);
                f.b0 = static_cast<uint8_t>(pos_in_stage[loc_of[op.tq[0]]]);
            }
            else
            {
                f.kind = is_swap(op) ? F_SWAP2 : F_DENSE2;
                int p0 = pos_in_stage[loc_of[op.tq[0]]];
                int p1 = pos_in_stage[loc_of[op.tq[1]]];
                if (p0 > p1)
                {
                    std::swap(p0, p1);
                    swapped = true;
                }
                f.b0 = static_cast<uint8_t>(p0);
                f.b1 = static_cast<uint8_t>(p1);
            }
            double2 m[16];
            const int ne = fop_entries(op, f, swapped, m);
            if (nentries + ne > kFusedMaxEntries)
                return false;
            f.moff = static_cast<uint16_t>(nentries);
            for (int e = 0; e < ne; ++e)
                prm.entries[nentries + e] = m[e];
            nentries += ne;
            if (src)
                src->push_back({pp.ops[oi], swapped});
            uint32_t lcm = 0, lcv = 0, sm = 0, sv = 0;
            uint64_t gcm = 0, gcv = 0;
            for (int b = 0; b < n; ++b)
                if ((cm >> b) & 1)
                {
                    const bool v = (cv >> b) & 1;
                    const int l = loc_of[b];
                    if (l >= 0 && ((bits >> l) & 1))
                    {
                        sm |= 1u << pos_in_stage[l];
                        if (v)
                            sv |= 1u << pos_in_stage[l];
                    }
                    else if (l >= 0)
                    {
                        lcm |= 1u << l;
                        if (v)
                            lcv |= 1u << l;
                    }
                    else
                    {
                        gcm |= 1ull << b;
                        if (v)
                            gcv |= 1ull << b;
                    }
                }
            f.lcmask = lcm;
            f.lcval = lcv;
            f.smask = static_cast<uint8_t>(sm);
            f.sval = static_cast<uint8_t>(sv);
            f.gcmask = gcm;
            f.gcval = gcv;
            if (f.kind == F_DENSE2 || f.kind == F_SWAP2)
            {
                // the kernel runs it with slot bits b0, b1 moved to 0, 1 and the
                // other two after them: its stage-bit condition in that order
                const uint32_t rest = 15u & ~((1u << f.b0) | (1u << f.b1));
                const int c0 = __builtin_ctz(rest), c1 = 31 - __builtin_clz(rest);
                auto remap = [&](uint32_t m) { return (((m >> c0) & 1u) << 2) | (((m >> c1) & 1u) << 3); };
                f.smask = static_cast<uint8_t>(remap(sm));
                f.sval = static_cast<uint8_t>(remap(sv));
            }
                }
        if (cur)
            cur->op_end = static_cast<uint16_t>(nops);
    }
    prm.nstages = ns;
    prm.nops = nops;
    prm.nentries = nentries;
    return true;
}

} // namespace

bool build_params(const std::vector<GateOp> &q, const PlannedPass &pp, int n, int k, FPassParams &prm,
                  std::vector<FOpSource> *src, std::vector<double2> *tables, std::vector<StageCond> *conds)
{
    const size_t start = tables ? tables->size() : 0;
    if (conds)
        conds->clear();
    const bool ok = build_params_body(q, pp, n, k, prm, src, tables, conds);
    if (!ok && tables)
        tables->resize(start);
    return ok;
}

bool build_pieces(const std::vector<GateOp> &q, const PlannedPass &pp, int n, std::vector<FPassParams> &params,
                  std::vector<std::vector<FOpSource>> *srcs, std::vector<PlannedPass> *pieces,
                  std::vector<double2> *tables, std::vector<std::vector<StageCond>> *conds)
{
    params.emplace_back();
    std::vector<FOpSource> src;
    std::vector<StageCond> cond;
    if (build_params(q, pp, n, pp.k, params.back(), srcs ? &src : nullptr, tables, conds ? &cond : nullptr))
    {
        if (srcs)
            srcs->push_back(std::move(src));
        if (pieces)
            pieces->push_back(pp);
        if (conds)
            conds->push_back(std::move(cond));
        return true;
    }
    params.pop_back();
    if (pp.ops.size() <= 1)
        return false;
    const size_t half = pp.ops.size() / 2;
    PlannedPass a = pp, b = pp;
    a.ops.assign(pp.ops.begin(), pp.ops.begin() + half);
    b.ops.assign(pp.ops.begin() + half, pp.ops.end());
    return build_pieces(q, a, n, params, srcs, pieces, tables, conds) &&
           build_pieces(q, b, n, params, srcs, pieces, tables, conds);
}

// How a planned pass runs: its pieces (built by build_pieces and already
// appended to params / pieces / conds from index `before` on) on the
// register path or as 16 x 16 tensor stages, per piece whichever the cost
// estimate favours (tensor mode 1) or 16 x 16 wherever allowed (2); or the
// same gates replanned with three dense bits per stage as 8 x 8 tensor
// stages, which then replace those pieces: when the estimate favours them
// (1) or wherever every piece allows them (3).
void choose_execution(const std::vector<GateOp> &q, const PlannedPass &pp, int n, int amp_bytes, int tensor_mode,
                      std::vector<FPassParams> &params, std::vector<PlannedPass> &pieces,
                      std::vector<std::vector<StageCond>> &conds, std::vector<double2> *tables, PassChoice &out,
                      size_t before, int engine)
{
    out = PassChoice();
    // automatic mode: below tensor_min_qubits a register pass's chunks fit
    // one wave of CTAs, and a tensor pass's extra launch (the matrix build)
    // costs more than its stages save
    if (tensor_mode == 1 && n < tensor_min_qubits(amp_bytes))
        tensor_mode = 0;
    double cost4 = 0.0;
    for (size_t i = before; i < params.size(); ++i)
    {
        out.tensor.push_back(-1);
        const double creg = register_pass_cost(params[i], amp_bytes);
        double cost = creg;
        if (tensor_mode == 1 || tensor_mode == 2)
        {
            TPassParams tp;
            TBuildParams tb;
            // complex64 16 x 16 stages on tcgen05 where the pass allows it
            bool ok = engine == 1 && amp_bytes == 8 &&
                      make_tensor_params(params[i], conds[i], amp_bytes, tp, tb, kStageBits, true);
            if (!ok)
                ok = make_tensor_params(params[i], conds[i], amp_bytes, tp, tb);
            const double ct = ok ? tensor_pass_cost(tp, amp_bytes) : 0.0;
            if (ok && (tensor_mode == 2 || ct < creg))
            {
                out.tparams.push_back(tp);
                out.tbuild.push_back(tb);
                out.tensor.back() = static_cast<int>(out.tparams.size()) - 1;
                cost = ct;
            }
        }
        cost4 += cost;
    }
    out.cost = cost4;
    if ((tensor_mode != 1 && tensor_mode != 3) || pp.k != kTensorLocal)
        return;
    PlannedPass p3 = pp;
    p3.stage_width = 3;
    std::vector<FPassParams> params3;
    std::vector<PlannedPass> pieces3;
    std::vector<std::vector<StageCond>> conds3;
    const size_t tables_before = tables ? tables->size() : 0;
    bool ok = build_pieces(q, p3, n, params3, nullptr, &pieces3, tables, &conds3);
    std::vector<TPassParams> tp3(ok ? params3.size() : 0);
    std::vector<TBuildParams> tb3(tp3.size());
    double cost3 = 0.0;
    for (size_t j = 0; ok && j < params3.size(); ++j)
    {
        ok = make_tensor_params(params3[j], conds3[j], amp_bytes, tp3[j], tb3[j], 3);
        cost3 += ok ? tensor_pass_cost(tp3[j], amp_bytes) : 0.0;
    }
    if (!ok || (tensor_mode == 1 && cost3 >= cost4))
    {
        if (tables)
            tables->resize(tables_before);
        return;
    }
    params.resize(before);
    pieces.resize(before);
    conds.resize(before);
    out = PassChoice();
    out.cost = cost3;
    for (size_t j = 0; j < params3.size(); ++j)
    {
        params.push_back(params3[j]);
        pieces.push_back(pieces3[j]);
        conds.push_back(std::move(conds3[j]));
        out.tparams.push_back(tp3[j]);
        out.tbuild.push_back(tb3[j]);
        out.tensor.push_back(static_cast<int>(j));
    }
}

namespace
{

template <typename R, bool BATCH>
int launch_pass_impl(void *state, int k, const FPassParams &prm, cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    const int threads = 1 << (k - kStageBits);
    const size_t smem = 2 * sizeof(V) * (size_t(1) << k);
    static bool configured[64] = {};
    int dev = 0;
    QCSB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !configured[dev])
    {
        QCSB_CUDA(cudaFuncSetAttribute(fused_pass_kernel<R, BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       2 * (int)sizeof(V) * (1 << kMaxLocal)));
        if (dev >= 0 && dev < 64)
            configured[dev] = true;
    }
    int per_sm = 0;
    QCSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fused_pass_kernel<R, BATCH>, threads, smem));
    int sms = 148;
    QCSB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    uint64_t grid = prm.chunks;
    const uint64_t cap = (uint64_t)sms * (per_sm > 0 ? per_sm : 1);
    if (grid > cap)
        grid = cap;
    FPassParams &p = const_cast<FPassParams &>(prm);
    p.state = state;
    fused_pass_kernel<R, BATCH><<<static_cast<unsigned>(grid), threads, smem, stream>>>(p);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

} // namespace

template <typename R>
int launch_fused_pass(void *state, int k, const FPassParams &prm, cudaStream_t stream)
{
    return launch_pass_impl<R, false>(state, k, prm, stream);
}

template <typename R>
int launch_fused_batch(void *state, int k, const FPassParams &prm, cudaStream_t stream)
{
    return launch_pass_impl<R, true>(state, k, prm, stream);
}

template int launch_fused_pass<double>(void *, int, const FPassParams &, cudaStream_t);
template int launch_fused_pass<float>(void *, int, const FPassParams &, cudaStream_t);
template int launch_fused_batch<double>(void *, int, const FPassParams &, cudaStream_t);
template int launch_fused_batch<float>(void *, int, const FPassParams &, cudaStream_t);

int clamp_local_bits(int k, int n)
{
    if (k > kMaxLocal)
        k = kMaxLocal;
    if (k > kStageBits + 7)   // at most 128 threads per CTA (launch bounds)
        k = kStageBits + 7;
    if (k < kStageBits + 5)   // at least one warp
        k = kStageBits + 5;
    if (k > n)
        k = n;
    return k;
}

int choose_local_bits(int n, int option)
{
    int k = kDefaultLocal;
    const char *e = std::getenv("QCS_FUSED_LOCAL_BITS");
    if (e && e[0])
        k = std::atoi(e);
    if (option > 0)
        k = option;
    return clamp_local_bits(k, n);
}

// Permutations (X, SWAP and their controlled forms) and diagonal ops cost a
// few instructions per amplitude; every other op runs complex multiply-adds.
bool light_op(const GateOp &op) { return op.diag || is_x(op) || is_swap(op); }

// Cost-model inputs of a pass as it runs (PassFeatures): block width (1 on
// the register path, 3 or 4 for 8 x 8 or 16 x 16 tensor stages), blocks
// (stages), arithmetic (non-light) gates, light ops, the target-qubit stride
// (log2 of the largest stride among the local qubits: the highest local
// qubit) and log2 of the number of chunks (n - k) capped at
// kChunkFeatureCap. The chunk count decides how well a pass fills the GPU
// (waves of CTAs, L2 residency of small registers); past 2^16 chunks a pass
// streams and its time per amplitude no longer depends on it, which lets
// timings from 24-27-qubit registers stand for 30-33-qubit ones. A model is
// trained on registers of one amplitude type (the dtype).
constexpr float kChunkFeatureCap = 16.0f;

PassFeatures pass_features(const std::vector<GateOp> &q, const PlannedPass &pp, int n, int width, int stages)
{
    int light = 0;
    for (int oi : pp.ops)
        light += light_op(q[oi]) ? 1 : 0;
    PassFeatures f;
    f.f[0] = static_cast<float>(width);
    f.f[1] = static_cast<float>(stages);
    f.f[2] = static_cast<float>((int)pp.ops.size() - light);
    f.f[3] = static_cast<float>(light);
    f.f[4] = pp.local ? static_cast<float>(63 - __builtin_clzll(pp.local)) : 0.0f;
    f.f[5] = std::min(static_cast<float>(n - pp.k), kChunkFeatureCap);
    return f;
}

uint64_t fill_local(uint64_t local, int n, int k)
{
    for (int b = 0; b < n && __builtin_popcountll(local) < k; ++b)
        local |= 1ull << b;
    return local;
}

// Dynamic-programming re-cut of the greedy schedule under the cost model.
// The greedy passes, concatenated in execution order, form a valid gate
// order; the planner chooses where to cut it into passes (each cut within
// kLearnedShift gates of a greedy cut) and, per pass, the block width its
// stages run with: gate by gate on the register path, or 8 x 8 or 16 x 16
// tensor stages (the pass is scheduled with three or four dense qubits per
// stage). Every candidate pass is built as the executor would build it, its
// features under each width it allows go through the model in one batch,
// and the cover of the gate order with the least predicted time wins. The
// arithmetic of every gate is the same under any cut; only the grouping
// changes. Passes keep the greedy plan's number of local qubits.
constexpr int kLearnedShift = 3;
// relative margin by which the model must predict a block width other than
// the executor's own choice to be faster before the planner takes it (the
// model's median error on its training timings is about 6%)
constexpr double kLearnedMargin = 0.10;

std::vector<Segment> plan_learned(const std::vector<GateOp> &q, const std::vector<Segment> &greedy, int n,
                                  int amp_bytes, int max_ops, int tensor_mode, CostModel &model,
                                  double *predicted_greedy, double *predicted_learned)
{
    std::vector<Segment> out;
    *predicted_greedy = *predicted_learned = 0.0;
    const double amps_ns = std::ldexp(1.0, n);
    const bool tensor_ok = tensor_mode != 0 && !(tensor_mode == 1 && n < tensor_min_qubits(amp_bytes));
    size_t gi = 0;
    while (gi < greedy.size())
    {
        if (!greedy[gi].fused)
        {
            out.push_back(greedy[gi++]);
            continue;
        }
        const int K = greedy[gi].pass.k;
        const int low = std::min(kLowBits, K);
        const uint64_t low_mask = (1ull << low) - 1;
        std::vector<int> seq, bounds{0};
        size_t gend = gi;
        while (gend < greedy.size() && greedy[gend].fused && greedy[gend].pass.k == K)
        {
            seq.insert(seq.end(), greedy[gend].pass.ops.begin(), greedy[gend].pass.ops.end());
            bounds.push_back(static_cast<int>(seq.size()));
            ++gend;
        }
        const int L = static_cast<int>(seq.size());
        std::vector<uint64_t> dense(L);
        for (int t = 0; t < L; ++t)
        {
            const GateOp &op = q[seq[t]];
            uint64_t d = 0;
            if (!op.diag)
                for (int i = 0; i < op.nt; ++i)
                    d |= 1ull << op.tq[i];
            dense[t] = d;
        }
        std::vector<int> cuts;
        for (int b : bounds)
            for (int d = -kLearnedShift; d <= kLearnedShift; ++d)
                if (b + d >= 0 && b + d <= L)
                    cuts.push_back(b + d);
        std::sort(cuts.begin(), cuts.end());
        cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
        const int C = static_cast<int>(cuts.size());

        // candidates (ci, cj): ops [cuts[ci], cuts[cj]) in one pass, priced
        // under each block width they allow (feature rows [row0, row1) are
        // the pieces of one option)
        struct Option
        {
            int ci, cj, width, row0, row1;
            double factor;   // 1 for the executor's own choice, 1 + kLearnedMargin for the others
        };
        std::vector<Option> opts;
        std::vector<float> feats;
        std::vector<double2> scratch_tables;
        auto add_rows = [&](const std::vector<PlannedPass> &pieces, const std::vector<int> &widths,
                            const std::vector<int> &stages, int ci, int cj, int width, double factor) {
            Option o{ci, cj, width, static_cast<int>(feats.size() / CostModel::kInputs), 0, factor};
            for (size_t i = 0; i < pieces.size(); ++i)
            {
                const PassFeatures f = pass_features(q, pieces[i], n, widths[i], stages[i]);
                feats.insert(feats.end(), f.f, f.f + CostModel::kInputs);
            }
            o.row1 = static_cast<int>(feats.size() / CostModel::kInputs);
            opts.push_back(o);
        };
        for (int ci = 0; ci < C; ++ci)
        {
            uint64_t d = low_mask;
            for (int cj = ci + 1; cj < C; ++cj)
            {
                const int i = cuts[ci], j = cuts[cj];
                if (j - i > max_ops)
                    break;
                for (int t = cuts[cj - 1]; t < j; ++t)
                    if (t >= i)
                        d |= dense[t];
                if (__builtin_popcountll(d) > K)
                    break;
                PlannedPass cp;
                cp.k = K;
                cp.local = fill_local(d, n, K);
                cp.ops.assign(seq.begin() + i, seq.begin() + j);
                std::vector<FPassParams> params;
                std::vector<PlannedPass> pieces;
                std::vector<std::vector<StageCond>> conds;
                scratch_tables.clear();
                if (!build_pieces(q, cp, n, params, nullptr, &pieces, &scratch_tables, &conds))
                    continue;
                std::vector<int> widths(params.size(), 1), stages(params.size());
                double creg = 0.0, c16 = 0.0, c8 = 0.0;
                for (size_t pi = 0; pi < params.size(); ++pi)
                {
                    stages[pi] = params[pi].nstages;
                    creg += register_pass_cost(params[pi], amp_bytes);
                }
                bool ok16 = false, ok8 = false;
                std::vector<PlannedPass> pieces3;
                std::vector<int> stages3;
                if (tensor_ok)
                {
                    ok16 = true;
                    for (size_t pi = 0; pi < params.size() && ok16; ++pi)
                    {
                        TPassParams tp;
                        TBuildParams tb;
                        ok16 = make_tensor_params(params[pi], conds[pi], amp_bytes, tp, tb);
                        c16 += ok16 ? tensor_pass_cost(tp, amp_bytes) : 0.0;
                    }
                    PlannedPass p3 = cp;
                    p3.stage_width = 3;
                    std::vector<FPassParams> params3;
                    std::vector<std::vector<StageCond>> conds3;
                    ok8 = build_pieces(q, p3, n, params3, nullptr, &pieces3, &scratch_tables, &conds3);
                    stages3.resize(params3.size());
                    for (size_t pi = 0; pi < params3.size() && ok8; ++pi)
                    {
                        TPassParams tp;
                        TBuildParams tb;
                        ok8 = make_tensor_params(params3[pi], conds3[pi], amp_bytes, tp, tb, 3);
                        stages3[pi] = params3[pi].nstages;
                        c8 += ok8 ? tensor_pass_cost(tp, amp_bytes) : 0.0;
                    }
                }
                // the executor's own choice for this pass (its cost estimate);
                // the model must predict the others faster by more than its
                // error to take them
                int own = 1;
                double best = creg;
                if (ok16 && c16 < best)
                {
                    own = 4;
                    best = c16;
                }
                if (ok8 && c8 < best)
                    own = 3;
                const double other = 1.0 + kLearnedMargin;
                add_rows(pieces, widths, stages, ci, cj, 1, own == 1 ? 1.0 : other);
                if (ok16)
                    add_rows(pieces, std::vector<int>(params.size(), 4), stages, ci, cj, 4, own == 4 ? 1.0 : other);
                if (ok8)
                    add_rows(pieces3, std::vector<int>(pieces3.size(), 3), stages3, ci, cj, 3, own == 3 ? 1.0 : other);
            }
        }
        const int rows = static_cast<int>(feats.size() / CostModel::kInputs);
        std::vector<float> pred(rows);
        if (rows > 0)
            model.predict(feats.data(), rows, pred.data());
        // cheapest option per candidate, then the cheapest cover
        const double inf = 1e300;
        std::vector<double> best(C, inf);
        std::vector<int> from(C, -1);
        best[0] = 0.0;
        std::vector<double> cost(opts.size(), 0.0);
        for (size_t o = 0; o < opts.size(); ++o)
        {
            for (int r = opts[o].row0; r < opts[o].row1; ++r)
                cost[o] += std::exp(double(pred[r])) * amps_ns;
            cost[o] *= opts[o].factor;
        }
        // options are grouped by ci ascending, so best[ci] is final when read
        for (size_t o = 0; o < opts.size(); ++o)
        {
            const Option &op = opts[o];
            if (best[op.ci] >= inf)
                continue;
            const double c = best[op.ci] + cost[o];
            if (c < best[op.cj])
            {
                best[op.cj] = c;
                from[op.cj] = static_cast<int>(o);
            }
        }
        // the greedy cut's predicted time (each pass at its cheapest width)
        for (size_t p = 0; p + 1 < bounds.size(); ++p)
        {
            double g = inf;
            for (size_t o = 0; o < opts.size(); ++o)
                if (cuts[opts[o].ci] == bounds[p] && cuts[opts[o].cj] == bounds[p + 1])
                    g = std::min(g, cost[o]);
            *predicted_greedy += g < inf ? g : 0.0;
        }
        if (from[C - 1] < 0)
        {
            // no cover (a candidate failed to build): keep the greedy passes
            for (size_t p = gi; p < gend; ++p)
                out.push_back(greedy[p]);
            gi = gend;
            continue;
        }
        *predicted_learned += best[C - 1];
        std::vector<Segment> run;
        for (int c = C - 1; c > 0;)
        {
            const Option &op = opts[from[c]];
            Segment sg;
            sg.fused = true;
            sg.plain_op = -1;
            sg.width = op.width;
            sg.pass.k = K;
            uint64_t d = low_mask;
            for (int t = cuts[op.ci]; t < cuts[op.cj]; ++t)
                d |= dense[t];
            sg.pass.local = fill_local(d, n, K);
            sg.pass.ops.assign(seq.begin() + cuts[op.ci], seq.begin() + cuts[op.cj]);
            run.push_back(std::move(sg));
            c = op.ci;
        }
        out.insert(out.end(), run.rbegin(), run.rend());
        gi = gend;
    }
    return out;
}

uint64_t queue_signature(const std::vector<GateOp> &ops)
{
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        h ^= v;
        h *= 1099511628211ull;
    };
    for (const GateOp &op : ops)
    {
        mix((uint64_t)op.nt | ((uint64_t)op.na << 8) | ((uint64_t)op.diag << 16));
        for (int i = 0; i < op.nt; ++i)
            mix((uint64_t)op.tq[i]);
        mix(op.cmask);
        mix(op.cval);
    }
    mix(ops.size());
    return h;
}

int fused_min_qubits() { return kStageBits + 5; }

void entries_to_float(double2 *entries, size_t count)
{
    // in place, front to back: float2 i ends where double2 i starts or earlier
    float2 *f = reinterpret_cast<float2 *>(entries);
    for (size_t i = 0; i < count; ++i)
    {
        const double2 d = entries[i];
        f[i] = make_float2(static_cast<float>(d.x), static_cast<float>(d.y));
    }
}

FusedExecutor::FusedExecutor(cudaStream_t stream) : stream_(stream)
{
    QCSB_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&err_host_), sizeof(int), cudaHostAllocMapped));
    *err_host_ = 0;
    const cudaError_t e = cudaHostGetDevicePointer(reinterpret_cast<void **>(&err_dev_), err_host_, 0);
    if (e != cudaSuccess)
    {
        // a throwing constructor runs no destructor: free the flag here
        cudaFreeHost(err_host_);
        err_host_ = nullptr;
        throw std::runtime_error(strformat("cudaHostGetDevicePointer: %s", cudaGetErrorString(e)));
    }
}

void FusedExecutor::check_device_error()
{
    if (err_host_ != nullptr && *const_cast<volatile int *>(err_host_) != 0)
    {
        *err_host_ = 0;
        throw std::runtime_error("a tensor-memory pass gave up waiting for its tensor cores; the register is invalid");
    }
}

FusedExecutor::~FusedExecutor()
{
    if (err_host_)
        cudaFreeHost(err_host_);
    if (judge_a_)
        cudaEventDestroy(judge_a_);
    if (judge_b_)
        cudaEventDestroy(judge_b_);
    if (tables_copied_)
    {
        cudaEventSynchronize(tables_copied_);
        cudaEventDestroy(tables_copied_);
    }
    cudaFree(tables_dev_);
    cudaFreeHost(tables_host_);
    cudaFree(mats_dev_);
}

// Copy the flush's phase-run tables to the device, behind the previous
// flush's passes on the stream (which may still read the device buffer; the
// copy is ordered after them). The pinned staging buffer is reused once the
// previous copy has completed. Returns null when there are no tables.
const double2 *FusedExecutor::upload_tables(const std::vector<double2> &tables)
{
    if (tables.empty())
        return nullptr;
    const size_t count = tables.size();
    if (tables_copied_)
        QCSB_CUDA(cudaEventSynchronize(tables_copied_));
    else
        QCSB_CUDA(cudaEventCreateWithFlags(&tables_copied_, cudaEventDisableTiming));
    if (count > tables_cap_)
    {
        // the old device buffer may still be read by queued passes
        QCSB_CUDA(cudaStreamSynchronize(stream_));
        cudaFree(tables_dev_);
        cudaFreeHost(tables_host_);
        tables_dev_ = nullptr;
        tables_host_ = nullptr;
        tables_cap_ = 0;
        const size_t cap = std::max(count + count / 2, size_t(1) << 16);
        QCSB_CUDA(cudaMalloc(&tables_dev_, cap * sizeof(double2)));
        QCSB_CUDA(cudaMallocHost(&tables_host_, cap * sizeof(double2)));
        tables_cap_ = cap;
    }
    std::memcpy(tables_host_, tables.data(), count * sizeof(double2));
    QCSB_CUDA(cudaMemcpyAsync(tables_dev_, tables_host_, count * sizeof(double2), cudaMemcpyHostToDevice, stream_));
    QCSB_CUDA(cudaEventRecord(tables_copied_, stream_));
    return tables_dev_;
}

// Record the device time of the previous learned-mode flush in the judge.
void FusedExecutor::settle_judge()
{
    if (pending_learned_ < 0)
        return;
    QCSB_CUDA(cudaEventSynchronize(judge_b_));
    float ms = 0.0f;
    QCSB_CUDA(cudaEventElapsedTime(&ms, judge_a_, judge_b_));
    for (auto &e : judge_)
        if (e.first == pending_sig_)
        {
            (pending_learned_ ? e.second.learned_ms : e.second.greedy_ms) = ms;
            last_greedy_ms = e.second.greedy_ms;
            last_learned_ms = e.second.learned_ms;
        }
    pending_learned_ = -1;
}

// Hash of everything a queue's plan depends on: every field of every op,
// matrix entries bit for bit.
static uint64_t queue_content_hash(const std::vector<GateOp> &ops)
{
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        h ^= v;
        h *= 1099511628211ull;
    };
    for (const GateOp &op : ops)
    {
        mix((uint64_t)op.nt | ((uint64_t)op.na << 8) | ((uint64_t)op.diag << 16));
        for (int i = 0; i < op.nt; ++i)
            mix((uint64_t)op.tq[i]);
        mix(op.cmask);
        mix(op.cval);
        for (int i = 0; i < op.na; ++i)
            mix(op.act[i]);
        const int nm = op.diag ? op.na : op.na * op.na;
        for (int i = 0; i < nm; ++i)
        {
            uint64_t re, im;
            std::memcpy(&re, &op.mat[i].re, sizeof(re));
            std::memcpy(&im, &op.mat[i].im, sizeof(im));
            mix(re);
            mix(im);
        }
    }
    mix(ops.size());
    return h;
}

static bool same_op(const GateOp &a, const GateOp &b)
{
    if (a.nt != b.nt || a.na != b.na || a.diag != b.diag || a.cmask != b.cmask || a.cval != b.cval)
        return false;
    for (int i = 0; i < a.nt; ++i)
        if (a.tq[i] != b.tq[i])
            return false;
    for (int i = 0; i < a.na; ++i)
        if (a.act[i] != b.act[i])
            return false;
    const int nm = a.diag ? a.na : a.na * a.na;
    return std::memcmp(a.mat, b.mat, sizeof(a.mat[0]) * nm) == 0;
}

FusedExecutor::FlushPlan *FusedExecutor::find_plan(const std::vector<GateOp> &queued, uint64_t hash, int n,
                                                   int amp_bytes, int k, int max_ops, int tag)
{
    for (auto &p : plans_)
    {
        if (p->hash != hash || p->n != n || p->amp_bytes != amp_bytes || p->k != k || p->max_ops != max_ops ||
            p->tensor_mode != tensor_mode_ || p->tensor_engine != tensor_engine_ || p->tag != tag ||
            p->queued.size() != queued.size())
            continue;
        bool same = true;
        for (size_t i = 0; i < queued.size() && same; ++i)
            same = same_op(p->queued[i], queued[i]);
        if (same)
            return p.get();
    }
    return nullptr;
}

// One launch of a plan: a plain gate kernel, a register pass, or a tensor
// pass (its stage-matrix builder, then the pass).
int FusedExecutor::launch_plan_step(FlushPlan &plan, long st, void *state, const double2 *tables_dev,
                                    qcs_b200_stats &stats, KernelTimer &timer, const PassFeatures *features)
{
    const bool c64 = plan.amp_bytes == (int)sizeof(float2);
    const int n = plan.n;
    int launches = 0;
    if (st < 0)
    {
        const GateOp &op = plan.ops[-1 - st];
        if (timer.enabled)
            timer.begin(stream_, KernelTimer::kPlain, 2.0 * plan.amp_bytes * op.changed_amps(n));
        const int k = c64 ? launch_gate_plain<float>(static_cast<float2 *>(state), n, op, stream_)
                          : launch_gate_plain<double>(static_cast<double2 *>(state), n, op, stream_);
        if (timer.enabled)
            timer.end(stream_);
        stats.plain_gate_kernels += k;
        return k;
    }
    FPassParams &prm = plan.params[st];
    prm.tables = tables_dev;
    if (timer.enabled)
        timer.begin(stream_, KernelTimer::kFused, 2.0 * plan.amp_bytes * std::ldexp(1.0, n), features);
    const int t = plan.tensor_of[st];
    if (t >= 0)
    {
        TPassParams &tp = plan.tparams[t];
        TBuildParams &tb = plan.tbuild[t];
        double2 *mats = nullptr;
        bool build = true;
        if (plan.mats != nullptr)
        {
            // the plan's own matrices: built on its first replay, reused after
            mats = reinterpret_cast<double2 *>(static_cast<char *>(plan.mats) + plan.mat_off[t]);
            build = !plan.mats_built;
        }
        else
        {
            if (tb.nmats > mats_cap_)
            {
                // the old buffer may still be read by queued passes
                QCSB_CUDA(cudaStreamSynchronize(stream_));
                cudaFree(mats_dev_);
                mats_dev_ = nullptr;
                mats_cap_ = 0;
                const size_t cap = std::max<size_t>(tb.nmats, 256);
                QCSB_CUDA(cudaMalloc(&mats_dev_, cap * kTensorMatrixBytes));
                mats_cap_ = cap;
            }
            mats = mats_dev_;
        }
        prm.state = state;
        tb.out = mats;
        tp.mats = mats;
        tp.state = state;
        tp.err = err_dev_;
        if (build)
            launches += launch_stage_matrices<double>(prm, tb, stream_);
        if (tp.umma)
            launches += launch_tc_pass(tp, stream_);
        else
            launches += c64 ? launch_tensor_pass<float>(tp, stream_) : launch_tensor_pass<double>(tp, stream_);
        ++stats.tensor_passes;
        stats.tensor8_passes += tp.width == 3 ? 1 : 0;
        stats.tcgen05_passes += tp.umma ? 1 : 0;
    }
    else
    {
        launches += c64 ? launch_fused_pass<float>(state, plan.ks[st], prm, stream_)
                        : launch_fused_pass<double>(state, plan.ks[st], prm, stream_);
    }
    if (timer.enabled)
        timer.end(stream_);
    ++stats.fused_passes;
    return launches;
}

// Bytes of one matrix of a tensor pass in its format: 8 x 8 mma.sync
// fragments, 16 x 16 mma.sync fragments, or tcgen05 slabs (high and low).
static size_t tensor_matrix_bytes(const TPassParams &tp)
{
    if (tp.umma)
        return 2 * static_cast<size_t>(kUmmaSlab);
    return static_cast<size_t>(tp.width == 3 ? kTensor3Fragments : kTensorFragments) * 32 * 16;
}

int FusedExecutor::replay(FlushPlan &plan, void *state, qcs_b200_stats &stats, KernelTimer &timer)
{
    if (plan.mats == nullptr && !plan.tparams.empty())
    {
        // first replay: give the plan its own matrices (256-byte aligned per
        // pass) if they fit the budget; the builds below fill them
        size_t total = 0;
        plan.mat_off.assign(plan.tparams.size(), 0);
        for (size_t t = 0; t < plan.tparams.size(); ++t)
        {
            plan.mat_off[t] = total;
            total += (plan.tparams[t].nmats * tensor_matrix_bytes(plan.tparams[t]) + 255) & ~size_t(255);
        }
        // kept matrices are a cache: they are made only while 256 MiB stay
        // free beside them, so that they never take the memory the
        // register's own scratch (sampler, staging) would need later
        size_t free_b = 0, total_b = 0;
        const bool room = total <= kKeptMatsBytes && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess &&
                          free_b >= total + kKeptMatsFreeReserve;
        if (!room || cudaMalloc(&plan.mats, total) != cudaSuccess)
        {
            plan.mats = nullptr;
            (void)cudaGetLastError();   // no room: keep building into the shared buffer
        }
    }
    const double2 *tables_dev = upload_tables(plan.tables);
    int launches = 0;
    for (long st : plan.steps)
        launches += launch_plan_step(plan, st, state, tables_dev, stats, timer, nullptr);
    if (plan.mats != nullptr)
        plan.mats_built = true;
    ++stats.replayed_flushes;
    return launches;
}

int FusedExecutor::run(void *state, int n, int amp_bytes, const std::vector<GateOp> &queued, int mode,
                       qcs_b200_stats &stats, KernelTimer &timer)
{
    const bool c64 = amp_bytes == (int)sizeof(float2);
    // Small registers: a pass would not fill a warp; run gate by gate.
    if (n < fused_min_qubits())
    {
        int launches = 0;
        for (const GateOp &op : queued)
        {
            if (timer.enabled)
                timer.begin(stream_, KernelTimer::kPlain, 2.0 * amp_bytes * op.changed_amps(n));
            const int k = c64 ? launch_gate_plain<float>(static_cast<float2 *>(state), n, op, stream_)
                              : launch_gate_plain<double>(static_cast<double2 *>(state), n, op, stream_);
            if (timer.enabled)
                timer.end(stream_);
            stats.plain_gate_kernels += k;
            launches += k;
        }
        return launches;
    }
    const int k = choose_local_bits(n, local_bits_);
    const int low = std::min(kLowBits, k);
    const int max_ops = (max_ops_ > 0 && max_ops_ < kFusedMaxOps) ? max_ops_ : kFusedMaxOps;
    // Kept plans are used and made only when no pass timing is recorded (the
    // timings carry features of the planning) and the judge is not timing
    // this flush.
    const uint64_t hash = timer.enabled ? 0 : queue_content_hash(queued);
    const bool learned = mode == QCS_FUSION_LEARNED && model_ != nullptr && model_->trained();
    int tag = 0;
    if (!learned && !timer.enabled)
        if (FlushPlan *kept = find_plan(queued, hash, n, amp_bytes, k, max_ops, 0))
        {
            last_plan_learned = 0;
            return replay(*kept, state, stats, timer);
        }

    auto plan = std::make_unique<FlushPlan>();
    plan->n = n;
    plan->amp_bytes = amp_bytes;
    plan->k = k;
    plan->max_ops = max_ops;
    plan->tensor_mode = tensor_mode_;
    plan->tensor_engine = tensor_engine_;
    plan->ops = defer_x(queued);
    const std::vector<GateOp> &ops = plan->ops;
    std::vector<Segment> segs;
    bool timed_flush = false;
    if (learned)
    {
        settle_judge();
        const uint64_t sig = queue_signature(ops);
        JudgeEntry *entry = nullptr;
        for (auto &e : judge_)
            if (e.first == sig)
                entry = &e.second;
        if (entry == nullptr)
        {
            judge_.push_back({sig, JudgeEntry{}});
            entry = &judge_.back().second;
        }
        // learned plan first; then the greedy one once, for comparison; then
        // whichever measured faster
        bool use_learned;
        if (entry->learned_ms < 0.0)
            use_learned = true;
        else if (entry->greedy_ms < 0.0)
            use_learned = false;
        else
            use_learned = entry->learned_ms <= entry->greedy_ms;
        last_greedy_ms = entry->greedy_ms;
        last_learned_ms = entry->learned_ms;
        last_plan_learned = use_learned ? 1 : 0;
        tag = use_learned ? 1 : 2;
        timed_flush = entry->learned_ms < 0.0 || entry->greedy_ms < 0.0;
        if (!timed_flush && !timer.enabled)
            if (FlushPlan *kept = find_plan(queued, hash, n, amp_bytes, k, max_ops, tag))
                return replay(*kept, state, stats, timer);
        segs = plan_greedy(ops, n, k, low, max_ops);
        if (use_learned)
        {
            // the learned plan of a queue is computed once (building and
            // pricing every candidate pass takes host time) and reused
            const uint64_t key = sig ^ (static_cast<uint64_t>(n) << 56) ^ (static_cast<uint64_t>(amp_bytes) << 48) ^
                                 (static_cast<uint64_t>(tensor_mode_) << 44) ^ static_cast<uint64_t>(max_ops);
            const std::vector<Segment> *cached = nullptr;
            for (const auto &e : learned_plans_)
                if (e.first == key)
                    cached = &e.second;
            if (cached != nullptr)
            {
                segs = *cached;
            }
            else
            {
                double pg = 0.0, pl = 0.0;
                segs = plan_learned(ops, segs, n, amp_bytes, max_ops, tensor_mode_, *model_, &pg, &pl);
                learned_plans_.push_back({key, segs});
            }
        }
        if (timed_flush)
        {
            if (!judge_a_)
            {
                QCSB_CUDA(cudaEventCreate(&judge_a_));
                QCSB_CUDA(cudaEventCreate(&judge_b_));
            }
            QCSB_CUDA(cudaEventRecord(judge_a_, stream_));
            pending_sig_ = sig;
            pending_learned_ = use_learned ? 1 : 0;
        }
    }
    else
    {
        last_plan_learned = 0;
        segs = plan_greedy(ops, n, k, low, max_ops);
    }

    // Passes launch as soon as they are built, so that the GPU runs while the
    // host plans the rest, until the first pass that needs phase-run tables:
    // from there on, passes are built first and launched after the tables of
    // all of them have gone to the device in one copy (order is kept).
    std::vector<PlannedPass> pieces;
    std::vector<std::vector<StageCond>> conds;
    size_t launched = 0;   // steps launched while planning
    int launches = 0;
    auto step_features = [&](long st, PassFeatures &f) -> const PassFeatures * {
        if (!timer.enabled || st < 0)
            return nullptr;
        const int t = plan->tensor_of[st];
        const int width = t >= 0 ? plan->tparams[t].width : 1;
        f = pass_features(ops, pieces[st], n, width, plan->params[st].nstages);
        return &f;
    };
    auto add_step = [&](long st) {
        plan->steps.push_back(st);
        if (plan->tables.empty())
        {
            PassFeatures f;
            launches += launch_plan_step(*plan, st, state, nullptr, stats, timer, step_features(st, f));
            launched = plan->steps.size();
        }
    };
    for (const Segment &s : segs)
    {
        if (!s.fused)
        {
            add_step(-1 - (long)s.plain_op);
            continue;
        }
        std::vector<FPassParams> &params = plan->params;
        const size_t before = params.size();
        if (!build_pieces(ops, s.pass, n, params, nullptr, &pieces, &plan->tables, &conds))
        {
            params.resize(before);
            pieces.resize(before);
            conds.resize(before);
            for (int oi : s.pass.ops)
                add_step(-1 - (long)oi);
            continue;
        }
        // a width the learned planner chose fixes the path (where the pass
        // allows it; else the register path)
        int tmode = tensor_mode_;
        if (s.width == 1)
            tmode = 0;
        else if (s.width == 4 && tensor_mode_ != 0)
            tmode = 2;
        else if (s.width == 3 && tensor_mode_ != 0)
            tmode = 3;
        PassChoice choice;
        choose_execution(ops, s.pass, n, amp_bytes, tmode, params, pieces, conds, &plan->tables, choice, before,
                         tensor_engine_);
        for (size_t i = before; i < params.size(); ++i)
        {
            plan->ks.push_back(pieces[i].k);
            const int t = choice.tensor[i - before];
            if (t >= 0)
            {
                plan->tparams.push_back(choice.tparams[t]);
                plan->tbuild.push_back(choice.tbuild[t]);
                plan->tensor_of.push_back(static_cast<int>(plan->tparams.size()) - 1);
            }
            else
            {
                plan->tensor_of.push_back(-1);
            }
        }
        // complex64 register passes read their entries as float2; tensor
        // passes build their matrices from the double2 entries
        for (size_t i = before; i < params.size(); ++i)
            if (c64 && plan->tensor_of[i] < 0)
                entries_to_float(params[i].entries, params[i].nentries);
        for (size_t i = before; i < params.size(); ++i)
            add_step((long)i);
    }
    if (launched < plan->steps.size())
    {
        const double2 *tables_dev = upload_tables(plan->tables);
        for (size_t i = launched; i < plan->steps.size(); ++i)
        {
            PassFeatures f;
            const long st = plan->steps[i];
            launches += launch_plan_step(*plan, st, state, tables_dev, stats, timer, step_features(st, f));
        }
    }
    if (timed_flush)
        QCSB_CUDA(cudaEventRecord(judge_b_, stream_));
    // plans whose parameter blocks would take much host memory (a flush of
    // thousands of passes) are not kept
    const size_t plan_bytes = plan->params.size() * sizeof(FPassParams) + plan->tparams.size() * sizeof(TPassParams) +
                              plan->tbuild.size() * sizeof(TBuildParams) + plan->tables.size() * sizeof(double2);
    if (!timer.enabled && !timed_flush && plan_bytes <= kKeptPlanBytes)
    {
        plan->queued = queued;
        plan->hash = hash;
        plan->tag = tag;
        if (plans_.size() < kKeptPlans)
            plans_.push_back(std::move(plan));
        else
        {
            plans_[plans_next_] = std::move(plan);
            plans_next_ = (plans_next_ + 1) % kKeptPlans;
        }
    }
    return launches;
}

} // namespace qcsb
