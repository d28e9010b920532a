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
// evaluated per amplitude (or once per chunk).
//
// Every gate is applied with its own FP64 matrix, in an order that respects
// all dependencies, so the result equals the gate-by-gate result up to the
// rounding of each individual product.

#include "simulator.h"

#include <algorithm>
#include <cmath>

namespace qcsb
{
namespace
{

constexpr int kFusedMaxOps = 48;
constexpr int kFusedMaxStages = 24;
constexpr int kLowBits = 3;      // qubits 0..2 are always local: 128-byte runs
constexpr int kMaxLocal = 12;
constexpr size_t kPlanWindow = 4096;   // ops scanned past the first pending one

enum FKind : uint8_t
{
    F_DENSE1 = 0,  // 2x2 on one stage bit
    F_SWAP1 = 1,   // X: exchange the pair
    F_DENSE2 = 2,  // 4x4 on two stage bits
    F_SWAP2 = 3,   // exchange sub-indices 01 and 10
    F_DIAG = 4,    // diagonal on up to 4 targets anywhere
};

struct FOp
{
    uint8_t kind;
    uint8_t nt;
    uint8_t b0, b1;        // stage-bit positions (dense kinds)
    int8_t loc[4];         // local bit of target i, -1 when outside Q (diag)
    uint8_t phys[4];       // physical qubit of target i
    uint32_t lcmask, lcval; // controls on local bits
    uint64_t gcmask, gcval; // controls on non-local physical bits
    double2 m[16];
};

struct FStage
{
    uint8_t sbits[4];      // local bit positions of the stage, ascending
    uint16_t op_begin, op_end;
};

struct FPassParams
{
    double2 *state;
    int n;
    int k;
    uint64_t chunks;
    uint64_t qmasks[kMaxLocal];  // (1 << qphys[i]) - 1, ascending: chunk deposit
    uint64_t qbit[kMaxLocal];    // 1 << qphys[i]
    int nstages;
    FStage stages[kFusedMaxStages];
    FOp ops[kFusedMaxOps];
};

__device__ __forceinline__ int swz(int j) { return j ^ (((j >> 3) ^ (j >> 6) ^ (j >> 9)) & 7); }

__device__ __forceinline__ double2 cmul(double2 m, double2 v)
{
    double2 r;
    r.x = fma(m.x, v.x, -m.y * v.y);
    r.y = fma(m.x, v.y, m.y * v.x);
    return r;
}

__device__ __forceinline__ double2 cmad2(double2 m0, double2 v0, double2 m1, double2 v1)
{
    double2 r;
    r.x = fma(m0.x, v0.x, fma(-m0.y, v0.y, fma(m1.x, v1.x, -m1.y * v1.y)));
    r.y = fma(m0.x, v0.y, fma(m0.y, v0.x, fma(m1.x, v1.y, m1.y * v1.x)));
    return r;
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <int SB, int B>
__device__ __forceinline__ void apply_dense1(double2 (&a)[1 << SB], const FOp &op, const uint32_t (&jr)[1 << SB])
{
    const double2 m00 = op.m[0], m01 = op.m[1], m10 = op.m[2], m11 = op.m[3];
#pragma unroll
    for (int r = 0; r < (1 << SB); ++r)
    {
        if (r & (1 << B))
            continue;
        if ((jr[r] & op.lcmask) != op.lcval)
            continue;
        const int r1 = r | (1 << B);
        const double2 x0 = a[r], x1 = a[r1];
        a[r] = cmad2(m00, x0, m01, x1);
        a[r1] = cmad2(m10, x0, m11, x1);
    }
}

template <int SB, int B>
__device__ __forceinline__ void apply_swap1(double2 (&a)[1 << SB], const FOp &op, const uint32_t (&jr)[1 << SB])
{
#pragma unroll
    for (int r = 0; r < (1 << SB); ++r)
    {
        if (r & (1 << B))
            continue;
        if ((jr[r] & op.lcmask) != op.lcval)
            continue;
        const int r1 = r | (1 << B);
        const double2 t = a[r];
        a[r] = a[r1];
        a[r1] = t;
    }
}

template <int SB, int B0, int B1>
__device__ __forceinline__ void apply_dense2(double2 (&a)[1 << SB], const FOp &op, const uint32_t (&jr)[1 << SB])
{
#pragma unroll
    for (int r = 0; r < (1 << SB); ++r)
    {
        if (r & ((1 << B0) | (1 << B1)))
            continue;
        if ((jr[r] & op.lcmask) != op.lcval)
            continue;
        const int i1 = r | (1 << B0), i2 = r | (1 << B1), i3 = r | (1 << B0) | (1 << B1);
        const double2 x0 = a[r], x1 = a[i1], x2 = a[i2], x3 = a[i3];
        const double2 *m = op.m;
        double2 y0 = cmad2(m[0], x0, m[1], x1), t0 = cmad2(m[2], x2, m[3], x3);
        double2 y1 = cmad2(m[4], x0, m[5], x1), t1 = cmad2(m[6], x2, m[7], x3);
        double2 y2 = cmad2(m[8], x0, m[9], x1), t2 = cmad2(m[10], x2, m[11], x3);
        double2 y3 = cmad2(m[12], x0, m[13], x1), t3 = cmad2(m[14], x2, m[15], x3);
        a[r] = make_double2(y0.x + t0.x, y0.y + t0.y);
        a[i1] = make_double2(y1.x + t1.x, y1.y + t1.y);
        a[i2] = make_double2(y2.x + t2.x, y2.y + t2.y);
        a[i3] = make_double2(y3.x + t3.x, y3.y + t3.y);
    }
}

template <int SB, int B0, int B1>
__device__ __forceinline__ void apply_swap2(double2 (&a)[1 << SB], const FOp &op, const uint32_t (&jr)[1 << SB])
{
#pragma unroll
    for (int r = 0; r < (1 << SB); ++r)
    {
        if (r & ((1 << B0) | (1 << B1)))
            continue;
        if ((jr[r] & op.lcmask) != op.lcval)
            continue;
        const int i1 = r | (1 << B0), i2 = r | (1 << B1);
        const double2 t = a[i1];
        a[i1] = a[i2];
        a[i2] = t;
    }
}

template <int SB>
__device__ __forceinline__ void apply_diag(double2 (&a)[1 << SB], const FOp &op, const uint32_t (&jr)[1 << SB], uint64_t cbase)
{
    uint32_t s_chunk = 0;
    for (int i = 0; i < op.nt; ++i)
        if (op.loc[i] < 0)
            s_chunk |= static_cast<uint32_t>((cbase >> op.phys[i]) & 1ull) << i;
#pragma unroll
    for (int r = 0; r < (1 << SB); ++r)
    {
        const uint32_t j = jr[r];
        if ((j & op.lcmask) != op.lcval)
            continue;
        uint32_t s = s_chunk;
        for (int i = 0; i < op.nt; ++i)
            if (op.loc[i] >= 0)
                s |= ((j >> op.loc[i]) & 1u) << i;
        a[r] = cmul(op.m[s], a[r]);
    }
}

template <int SB>
__device__ __forceinline__ void dispatch_dense1(double2 (&a)[1 << SB], const FOp &op, const uint32_t (&jr)[1 << SB], bool swap)
{
    switch (op.b0)
    {
    case 0: swap ? apply_swap1<SB, 0>(a, op, jr) : apply_dense1<SB, 0>(a, op, jr); break;
    case 1: swap ? apply_swap1<SB, 1>(a, op, jr) : apply_dense1<SB, 1>(a, op, jr); break;
    case 2: swap ? apply_swap1<SB, 2>(a, op, jr) : apply_dense1<SB, 2>(a, op, jr); break;
    default:
        if constexpr (SB > 3)
            swap ? apply_swap1<SB, 3>(a, op, jr) : apply_dense1<SB, 3>(a, op, jr);
        break;
    }
}

template <int SB, int B0>
__device__ __forceinline__ void dispatch_dense2_b1(double2 (&a)[1 << SB], const FOp &op, const uint32_t (&jr)[1 << SB], bool swap)
{
    switch (op.b1)
    {
    case 0: if constexpr (B0 != 0) { swap ? apply_swap2<SB, B0, 0>(a, op, jr) : apply_dense2<SB, B0, 0>(a, op, jr); } break;
    case 1: if constexpr (B0 != 1) { swap ? apply_swap2<SB, B0, 1>(a, op, jr) : apply_dense2<SB, B0, 1>(a, op, jr); } break;
    case 2: if constexpr (B0 != 2) { swap ? apply_swap2<SB, B0, 2>(a, op, jr) : apply_dense2<SB, B0, 2>(a, op, jr); } break;
    default:
        if constexpr (SB > 3 && B0 != 3)
            swap ? apply_swap2<SB, B0, 3>(a, op, jr) : apply_dense2<SB, B0, 3>(a, op, jr);
        break;
    }
}

template <int SB>
__device__ __forceinline__ void dispatch_dense2(double2 (&a)[1 << SB], const FOp &op, const uint32_t (&jr)[1 << SB], bool swap)
{
    switch (op.b0)
    {
    case 0: dispatch_dense2_b1<SB, 0>(a, op, jr, swap); break;
    case 1: dispatch_dense2_b1<SB, 1>(a, op, jr, swap); break;
    case 2: dispatch_dense2_b1<SB, 2>(a, op, jr, swap); break;
    default:
        if constexpr (SB > 3)
            dispatch_dense2_b1<SB, 3>(a, op, jr, swap);
        break;
    }
}

// One CTA per chunk at a time; blockDim.x == 2^(k - SB).
template <int SB>
__global__ void __launch_bounds__(256) fused_pass_kernel(const __grid_constant__ FPassParams p)
{
    extern __shared__ double2 smem[];
    const int k = p.k;
    const int T = 1 << (k - SB);
    const int tid = threadIdx.x;
    constexpr int R = 1 << SB;
    double2 *buf[2] = {smem, smem + (1 << k)};

    // global offset of this thread's element tid + m*T, m < R
    uint64_t dep_tid = 0;
    for (int i = 0; i < k - SB; ++i)
        if ((tid >> i) & 1)
            dep_tid |= p.qbit[i];
    uint64_t hb[SB];
#pragma unroll
    for (int b = 0; b < SB; ++b)
        hb[b] = p.qbit[k - SB + b];

    auto chunk_base = [&](uint64_t c) -> uint64_t {
        uint64_t g = c;
        for (int i = 0; i < k; ++i)
        {
            const uint64_t lo = g & p.qmasks[i];
            g = lo | ((g ^ lo) << 1);
        }
        return g;
    };
    auto issue_load = [&](uint64_t c, double2 *dst) {
        const uint64_t cb = chunk_base(c) | dep_tid;
#pragma unroll
        for (int m = 0; m < R; ++m)
        {
            uint64_t off = cb;
#pragma unroll
            for (int b = 0; b < SB; ++b)
                if ((m >> b) & 1)
                    off |= hb[b];
            const int e = tid + m * T;
            cp_async16(dst + swz(e), p.state + off);
        }
        cp_async_commit();
    };

    uint64_t c = blockIdx.x;
    if (c >= p.chunks)
        return;
    issue_load(c, buf[0]);
    int cur = 0;
    for (; c < p.chunks; c += gridDim.x)
    {
        const uint64_t next = c + gridDim.x;
        if (next < p.chunks)
        {
            issue_load(next, buf[cur ^ 1]);
            cp_async_wait<1>();
        }
        else
        {
            cp_async_wait<0>();
        }
        __syncthreads();
        double2 *sb = buf[cur];
        const uint64_t cbase = chunk_base(c);

        for (int st = 0; st < p.nstages; ++st)
        {
            const FStage &S = p.stages[st];
            // group base: insert zeros at the stage bits (ascending)
            uint32_t j0 = static_cast<uint32_t>(tid);
#pragma unroll
            for (int b = 0; b < SB; ++b)
            {
                const uint32_t lo = j0 & ((1u << S.sbits[b]) - 1u);
                j0 = lo | ((j0 ^ lo) << 1);
            }
            uint32_t jr[R];
            double2 a[R];
#pragma unroll
            for (int r = 0; r < R; ++r)
            {
                uint32_t j = j0;
#pragma unroll
                for (int b = 0; b < SB; ++b)
                    if ((r >> b) & 1)
                        j |= 1u << S.sbits[b];
                jr[r] = j;
                a[r] = sb[swz(j)];
            }
            for (int oi = S.op_begin; oi < S.op_end; ++oi)
            {
                const FOp &op = p.ops[oi];
                if ((cbase & op.gcmask) != op.gcval)
                    continue;
                switch (op.kind)
                {
                case F_DENSE1: dispatch_dense1<SB>(a, op, jr, false); break;
                case F_SWAP1: dispatch_dense1<SB>(a, op, jr, true); break;
                case F_DENSE2: dispatch_dense2<SB>(a, op, jr, false); break;
                case F_SWAP2: dispatch_dense2<SB>(a, op, jr, true); break;
                default: apply_diag<SB>(a, op, jr, cbase); break;
                }
            }
#pragma unroll
            for (int r = 0; r < R; ++r)
                sb[swz(jr[r])] = a[r];
            __syncthreads();
        }

        // write back
        const uint64_t cb = cbase | dep_tid;
#pragma unroll
        for (int m = 0; m < R; ++m)
        {
            uint64_t off = cb;
#pragma unroll
            for (int b = 0; b < SB; ++b)
                if ((m >> b) & 1)
                    off |= hb[b];
            const int e = tid + m * T;
            __stcs(p.state + off, sb[swz(e)]);
        }
        __syncthreads();
        cur ^= 1;
    }
}

// ------------------------------------------------------------ planning

struct OpClass
{
    bool fusable;
    uint64_t dense;   // qubits the op is non-diagonal on (dense targets)
    uint64_t diag;    // qubits the op is diagonal on (controls, diag targets)
};

OpClass classify(const GateOp &op)
{
    OpClass c;
    uint64_t t = 0;
    for (int i = 0; i < op.nt; ++i)
        t |= 1ull << op.tq[i];
    if (op.diag)
    {
        c.fusable = op.nt <= 4;
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

bool is_x(const GateOp &op)
{
    // 2x2 [[0,1],[1,0]] on both sub-indices
    if (op.nt != 1 || op.na != 2 || op.diag)
        return false;
    const cplx *m = op.mat;
    return m[0].re == 0 && m[0].im == 0 && m[1].re == 1 && m[1].im == 0 &&
           m[2].re == 1 && m[2].im == 0 && m[3].re == 0 && m[3].im == 0;
}

bool is_swap(const GateOp &op)
{
    if (op.nt != 2 || op.na != 2 || op.diag || op.act[0] != 1 || op.act[1] != 2)
        return false;
    const cplx *m = op.mat;
    return m[0].re == 0 && m[0].im == 0 && m[1].re == 1 && m[1].im == 0 &&
           m[2].re == 1 && m[2].im == 0 && m[3].re == 0 && m[3].im == 0;
}

// Full 2^nt x 2^nt matrix (dense) or 2^nt diagonal (diag) of a GateOp.
void expand(const GateOp &op, double2 *out)
{
    const int d = 1 << op.nt;
    if (op.diag)
    {
        for (int s = 0; s < d; ++s)
            out[s] = make_double2(1.0, 0.0);
        for (int a = 0; a < op.na; ++a)
            out[op.act[a]] = make_double2(op.mat[a].re, op.mat[a].im);
        return;
    }
    for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c)
            out[r * d + c] = make_double2(r == c ? 1.0 : 0.0, 0.0);
    for (int a = 0; a < op.na; ++a)
        for (int b = 0; b < op.na; ++b)
            out[op.act[a] * d + op.act[b]] = make_double2(op.mat[a * op.na + b].re, op.mat[a * op.na + b].im);
}

struct PlannedPass
{
    std::vector<int> ops;   // indices into the queue, in execution order
    uint64_t local = 0;     // physical qubits of Q
};

struct Segment
{
    bool fused;
    int plain_op;           // when !fused
    PlannedPass pass;
};

// Greedy pass construction. Ops are taken in queue order; an op joins the
// current pass when its dense targets fit in Q (k qubits) and it commutes
// with every op left behind so far (an op is left behind when it does not
// fit). Commutation test: X and Y commute when X's dense qubits avoid all of
// Y's qubits and X's diagonal qubits avoid Y's dense qubits (ops that are
// diagonal on every shared qubit commute).
std::vector<Segment> plan_greedy(const std::vector<GateOp> &q, int n, int k, int low)
{
    const size_t N = q.size();
    std::vector<OpClass> cls(N);
    for (size_t i = 0; i < N; ++i)
        cls[i] = classify(q[i]);
    std::vector<bool> done(N, false);
    std::vector<Segment> out;
    const uint64_t low_mask = (low >= 64) ? ~0ull : ((1ull << low) - 1);
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
        const size_t window_end = std::min(N, first + kPlanWindow);
        for (size_t i = first; i < window_end; ++i)
        {
            if (done[i])
                continue;
            const OpClass &c = cls[i];
            const uint64_t support = c.dense | c.diag;
            bool take = c.fusable && (int)s.pass.ops.size() < kFusedMaxOps &&
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
            }
            else
            {
                blocked_all |= support;
                blocked_dense |= c.dense;
                if ((blocked_all & all) == all && (blocked_dense & all) == all)
                    break;
            }
        }
        // fill Q up to k qubits with the lowest unused ones
        for (int b = 0; b < n && __builtin_popcountll(local) < k; ++b)
            local |= 1ull << b;
        s.pass.local = local;
        out.push_back(std::move(s));
    }
    return out;
}

// Split a pass into stages of SB bits and fill the kernel parameters.
// Returns false when the pass does not fit the parameter block limits.
template <int SB>
bool build_params(const std::vector<GateOp> &q, const PlannedPass &pp, int n, int k, FPassParams &prm)
{
    std::memset(&prm, 0, sizeof(prm));
    prm.n = n;
    prm.k = k;
    prm.chunks = 1ull << (n - k);
    int qphys[kMaxLocal];
    int nl = 0;
    int loc_of[kMaxQubits];
    for (int b = 0; b < kMaxQubits; ++b)
        loc_of[b] = -1;
    for (int b = 0; b < n; ++b)
        if ((pp.local >> b) & 1)
        {
            loc_of[b] = nl;
            qphys[nl++] = b;
        }
    if (nl != k)
        throw std::runtime_error("internal: pass locality size mismatch");
    for (int i = 0; i < k; ++i)
    {
        prm.qmasks[i] = (1ull << qphys[i]) - 1;
        prm.qbit[i] = 1ull << qphys[i];
    }
    uint64_t all_local_mask = pp.local;
    int nst = 0;
    int cur_bits[4];
    int ncur = 0;
    auto close_stage = [&](int begin, int end) -> bool {
        if (nst >= kFusedMaxStages)
            return false;
        // pad with the lowest local bits not in the stage
        int bits[4];
        int nb = ncur;
        for (int i = 0; i < ncur; ++i)
            bits[i] = cur_bits[i];
        for (int l = 0; l < k && nb < SB; ++l)
        {
            bool used = false;
            for (int i = 0; i < nb; ++i)
                used = used || bits[i] == l;
            if (!used)
                bits[nb++] = l;
        }
        std::sort(bits, bits + SB);
        FStage &S = prm.stages[nst++];
        for (int i = 0; i < SB; ++i)
            S.sbits[i] = static_cast<uint8_t>(bits[i]);
        for (int i = SB; i < 4; ++i)
            S.sbits[i] = 0;
        S.op_begin = static_cast<uint16_t>(begin);
        S.op_end = static_cast<uint16_t>(end);
        return true;
    };
    int stage_begin = 0;
    ncur = 0;
    int nops = 0;
    std::vector<int> stage_of(pp.ops.size());
    // first assign stages (by local bit positions), then encode ops with
    // their stage-relative bit positions
    std::vector<std::vector<int>> stage_bits;
    std::vector<std::pair<int, int>> ranges;
    for (size_t oi = 0; oi < pp.ops.size(); ++oi)
    {
        const GateOp &op = q[pp.ops[oi]];
        const OpClass c = classify(op);
        int need[2];
        int nneed = 0;
        for (int b = 0; b < n; ++b)
            if ((c.dense >> b) & 1)
                need[nneed++] = loc_of[b];
        int add = 0;
        for (int i = 0; i < nneed; ++i)
        {
            bool have = false;
            for (int j = 0; j < ncur; ++j)
                have = have || cur_bits[j] == need[i];
            add += have ? 0 : 1;
        }
        if (ncur + add > SB)
        {
            stage_bits.push_back(std::vector<int>(cur_bits, cur_bits + ncur));
            ranges.push_back({stage_begin, (int)oi});
            stage_begin = (int)oi;
            ncur = 0;
        }
        for (int i = 0; i < nneed; ++i)
        {
            bool have = false;
            for (int j = 0; j < ncur; ++j)
                have = have || cur_bits[j] == need[i];
            if (!have)
                cur_bits[ncur++] = need[i];
        }
        stage_of[oi] = (int)ranges.size();
    }
    stage_bits.push_back(std::vector<int>(cur_bits, cur_bits + ncur));
    ranges.push_back({stage_begin, (int)pp.ops.size()});
    if (ranges.size() > (size_t)kFusedMaxStages || pp.ops.size() > (size_t)kFusedMaxOps)
        return false;
    for (size_t si = 0; si < ranges.size(); ++si)
    {
        ncur = (int)stage_bits[si].size();
        for (int i = 0; i < ncur; ++i)
            cur_bits[i] = stage_bits[si][i];
        if (!close_stage(ranges[si].first, ranges[si].second))
            return false;
    }
    prm.nstages = nst;
    (void)all_local_mask;
    for (size_t oi = 0; oi < pp.ops.size(); ++oi)
    {
        const GateOp &op = q[pp.ops[oi]];
        FOp &f = prm.ops[nops++];
        const FStage &S = prm.stages[stage_of[oi]];
        auto stage_pos = [&](int local_bit) -> int {
            for (int i = 0; i < SB; ++i)
                if (S.sbits[i] == local_bit)
                    return i;
            throw std::runtime_error("internal: target not in stage");
        };
        f.nt = static_cast<uint8_t>(op.nt);
        for (int i = 0; i < 4; ++i)
        {
            f.loc[i] = -1;
            f.phys[i] = 0;
        }
        for (int i = 0; i < op.nt; ++i)
        {
            f.phys[i] = static_cast<uint8_t>(op.tq[i]);
            f.loc[i] = static_cast<int8_t>(loc_of[op.tq[i]]);
        }
        uint32_t lcm = 0, lcv = 0;
        uint64_t gcm = 0, gcv = 0;
        for (int b = 0; b < n; ++b)
            if ((op.cmask >> b) & 1)
            {
                const bool v = (op.cval >> b) & 1;
                if (loc_of[b] >= 0)
                {
                    lcm |= 1u << loc_of[b];
                    if (v)
                        lcv |= 1u << loc_of[b];
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
        f.gcmask = gcm;
        f.gcval = gcv;
        if (op.diag)
        {
            f.kind = F_DIAG;
            expand(op, f.m);
        }
        else if (op.nt == 1)
        {
            f.kind = is_x(op) ? F_SWAP1 : F_DENSE1;
            f.b0 = static_cast<uint8_t>(stage_pos(loc_of[op.tq[0]]));
            expand(op, f.m);
        }
        else
        {
            f.kind = is_swap(op) ? F_SWAP2 : F_DENSE2;
            f.b0 = static_cast<uint8_t>(stage_pos(loc_of[op.tq[0]]));
            f.b1 = static_cast<uint8_t>(stage_pos(loc_of[op.tq[1]]));
            expand(op, f.m);
        }
    }
    return true;
}

constexpr int kStageBits = 3;

int launch_fused_pass(double2 *state, int n, int k, const FPassParams &prm, cudaStream_t stream)
{
    const int threads = 1 << (k - kStageBits);
    const size_t smem = 2 * sizeof(double2) * (size_t(1) << k);
    static bool configured[64] = {};
    int dev = 0;
    QCSB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !configured[dev])
    {
        QCSB_CUDA(cudaFuncSetAttribute(fused_pass_kernel<kStageBits>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       2 * 16 * (1 << kMaxLocal)));
        if (dev >= 0 && dev < 64)
            configured[dev] = true;
    }
    uint64_t grid = prm.chunks;
    const uint64_t cap = 148ull * 4;
    if (grid > cap)
        grid = cap;
    FPassParams p = prm;
    p.state = state;
    fused_pass_kernel<kStageBits><<<static_cast<unsigned>(grid), threads, smem, stream>>>(p);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

int choose_local_bits(int n)
{
    const char *e = std::getenv("QCS_FUSED_LOCAL_BITS");
    int k = 11;
    if (e && e[0])
        k = std::atoi(e);
    if (k > kMaxLocal)
        k = kMaxLocal;
    if (k > kStageBits + 8)   // at most 256 threads per CTA
        k = kStageBits + 8;
    if (k < kStageBits + 5)
        k = kStageBits + 5;
    if (k > n)
        k = n;
    return k;
}

} // namespace

FusedExecutor::FusedExecutor(cudaStream_t stream) : stream_(stream) {}
FusedExecutor::~FusedExecutor() {}

int FusedExecutor::run(double2 *state, int n, const std::vector<GateOp> &ops, int mode, qcs_b200_stats &stats,
                       KernelTimer &timer)
{
    auto plain = [&](const GateOp &op) {
        if (timer.enabled)
            timer.begin(stream_, KernelTimer::kPlain, 2.0 * sizeof(double2) * op.changed_amps(n));
        const int k = launch_gate_plain(state, n, op, stream_);
        if (timer.enabled)
            timer.end(stream_);
        stats.plain_gate_kernels += k;
        return k;
    };
    (void)mode;
    int launches = 0;
    // Small registers: a pass would not fill a warp; run gate by gate.
    if (n < kStageBits + 5)
    {
        for (const GateOp &op : ops)
            launches += plain(op);
        return launches;
    }
    const int k = choose_local_bits(n);
    const int low = std::min(kLowBits, k);
    const std::vector<Segment> segs = plan_greedy(ops, n, k, low);
    FPassParams *prm = new FPassParams;
    for (const Segment &s : segs)
    {
        if (!s.fused)
        {
            launches += plain(ops[s.plain_op]);
            continue;
        }
        if (build_params<kStageBits>(ops, s.pass, n, k, *prm))
        {
            if (timer.enabled)
                timer.begin(stream_, KernelTimer::kFused, 2.0 * sizeof(double2) * std::ldexp(1.0, n));
            launches += launch_fused_pass(state, n, k, *prm, stream_);
            if (timer.enabled)
                timer.end(stream_);
            ++stats.fused_passes;
        }
        else
        {
            for (int oi : s.pass.ops)
                launches += plain(ops[oi]);
        }
    }
    delete prm;
    return launches;
}

} // namespace qcsb
