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

#include "cost_model.h"
#include "simulator.h"

#include <algorithm>
#include <cmath>

namespace qcsb
{
namespace
{

constexpr int kFusedMaxOps = 64;
constexpr int kFusedMaxStages = 64;
constexpr int kLowBits = 3;      // qubits 0..2 are always local: 128-byte runs
constexpr int kStageBits = 4;    // amplitudes per thread in a stage: 2^4
constexpr int kDefaultLocal = 11;
constexpr int kMaxLocal = 12;
constexpr size_t kPlanWindow = 4096;   // ops scanned past the first pending one

enum FKind : uint8_t
{
    F_DENSE1 = 0,  // 2x2 on one stage bit
    F_SWAP1 = 1,   // X: exchange the pair
    F_DENSE2 = 2,  // 4x4 on two stage bits (b0 < b1)
    F_SWAP2 = 3,   // exchange sub-indices 01 and 10
    F_PHASE = 4,   // multiply by m[0] where the condition bits match
    F_DIAG = 5,    // diagonal on one or two targets anywhere
};

// One gate of a pass. Conditions: (local index & lcmask) == lcval and
// (physical chunk bits & gcmask) == gcval. For F_PHASE the condition includes
// the target bits of the single changed sub-index.
struct FOp
{
    uint8_t kind;
    uint8_t nt;
    uint8_t b0, b1;         // stage-bit positions (dense kinds)
    int8_t loc[2];          // F_DIAG: local bit of target i, -1 when outside Q
    uint8_t phys[2];        // F_DIAG: physical qubit of target i
    uint32_t lcmask, lcval;
    uint64_t gcmask, gcval;
    double2 m[16];
};

struct FStage
{
    uint8_t sbits[kStageBits];   // local bit positions of the stage, ascending
    uint16_t op_begin, op_end;
};

struct FPassParams
{
    void *state;
    int n;
    int k;
    uint64_t chunks;
    uint64_t qmasks[kMaxLocal];  // (1 << qphys[i]) - 1, ascending: chunk deposit
    uint64_t qbit[kMaxLocal];    // 1 << qphys[i]
    int nstages;
    FStage stages[kFusedMaxStages];
    FOp ops[kFusedMaxOps];
};

// Shared-memory swizzle, an XOR of higher index bits into the bits that pick
// the bank group: 16-byte amplitudes (8 per 128-byte line) fold 3 bits,
// 8-byte amplitudes (16 per line) fold 4. Both are linear over GF(2).
template <typename V>
__device__ __forceinline__ int swz(int j);
template <>
__device__ __forceinline__ int swz<double2>(int j) { return j ^ (((j >> 3) ^ (j >> 6) ^ (j >> 9)) & 7); }
template <>
__device__ __forceinline__ int swz<float2>(int j) { return j ^ (((j >> 4) ^ (j >> 8)) & 15); }

template <typename V>
__device__ __forceinline__ V cvt(double2 m);
template <>
__device__ __forceinline__ double2 cvt<double2>(double2 m) { return m; }
template <>
__device__ __forceinline__ float2 cvt<float2>(double2 m) { return make_float2(static_cast<float>(m.x), static_cast<float>(m.y)); }

template <typename V>
__device__ __forceinline__ V cmul(V m, V v)
{
    V r;
    r.x = fma(m.x, v.x, -m.y * v.y);
    r.y = fma(m.x, v.y, m.y * v.x);
    return r;
}

template <typename V>
__device__ __forceinline__ V cmad2(V m0, V v0, V m1, V v1)
{
    V r;
    r.x = fma(m0.x, v0.x, fma(-m0.y, v0.y, fma(m1.x, v1.x, -m1.y * v1.y)));
    r.y = fma(m0.x, v0.y, fma(m0.y, v0.x, fma(m1.x, v1.y, m1.y * v1.x)));
    return r;
}

template <typename V>
__device__ __forceinline__ void cp_async_amp(V *smem, const V *gmem);
template <>
__device__ __forceinline__ void cp_async_amp<double2>(double2 *smem, const double2 *gmem)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
template <>
__device__ __forceinline__ void cp_async_amp<float2>(float2 *smem, const float2 *gmem)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

constexpr int R = 1 << kStageBits;

// Gate application on a thread's 2^kStageBits amplitudes a[r] (r = bits of
// the stage's local bits; jr[r] = the amplitude's local index). Gates without
// local controls take the unconditional path; controlled ones predicate each
// pair or amplitude on (jr & lcmask) == lcval.

template <typename V, int B>
__device__ __forceinline__ void apply_dense1(V (&a)[R], const FOp &op, const uint32_t (&jr)[R])
{
    const V m00 = cvt<V>(op.m[0]), m01 = cvt<V>(op.m[1]), m10 = cvt<V>(op.m[2]), m11 = cvt<V>(op.m[3]);
    const uint32_t cm = op.lcmask, cv = op.lcval;
    if (cm == 0)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (r & (1 << B))
                continue;
            const int r1 = r | (1 << B);
            const V x0 = a[r], x1 = a[r1];
            a[r] = cmad2(m00, x0, m01, x1);
            a[r1] = cmad2(m10, x0, m11, x1);
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        if (r & (1 << B))
            continue;
        if ((jr[r] & cm) == cv)
        {
            const int r1 = r | (1 << B);
            const V x0 = a[r], x1 = a[r1];
            a[r] = cmad2(m00, x0, m01, x1);
            a[r1] = cmad2(m10, x0, m11, x1);
        }
    }
}

template <typename V, int B>
__device__ __forceinline__ void apply_swap1(V (&a)[R], const FOp &op, const uint32_t (&jr)[R])
{
    const uint32_t cm = op.lcmask, cv = op.lcval;
    if (cm == 0)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (r & (1 << B))
                continue;
            const int r1 = r | (1 << B);
            const V t = a[r];
            a[r] = a[r1];
            a[r1] = t;
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        if (r & (1 << B))
            continue;
        if ((jr[r] & cm) == cv)
        {
            const int r1 = r | (1 << B);
            const V t = a[r];
            a[r] = a[r1];
            a[r1] = t;
        }
    }
}

template <typename V, int B0, int B1>
__device__ __forceinline__ void apply_dense2(V (&a)[R], const FOp &op, const uint32_t (&jr)[R])
{
    const uint32_t cm = op.lcmask, cv = op.lcval;
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        if (r & ((1 << B0) | (1 << B1)))
            continue;
        if ((jr[r] & cm) != cv)
            continue;
        const int i1 = r | (1 << B0), i2 = r | (1 << B1), i3 = r | (1 << B0) | (1 << B1);
        const V x0 = a[r], x1 = a[i1], x2 = a[i2], x3 = a[i3];
        const double2 *m = op.m;
        const V y0 = cmad2(cvt<V>(m[0]), x0, cvt<V>(m[1]), x1), t0 = cmad2(cvt<V>(m[2]), x2, cvt<V>(m[3]), x3);
        const V y1 = cmad2(cvt<V>(m[4]), x0, cvt<V>(m[5]), x1), t1 = cmad2(cvt<V>(m[6]), x2, cvt<V>(m[7]), x3);
        const V y2 = cmad2(cvt<V>(m[8]), x0, cvt<V>(m[9]), x1), t2 = cmad2(cvt<V>(m[10]), x2, cvt<V>(m[11]), x3);
        const V y3 = cmad2(cvt<V>(m[12]), x0, cvt<V>(m[13]), x1), t3 = cmad2(cvt<V>(m[14]), x2, cvt<V>(m[15]), x3);
        a[r] = V{y0.x + t0.x, y0.y + t0.y};
        a[i1] = V{y1.x + t1.x, y1.y + t1.y};
        a[i2] = V{y2.x + t2.x, y2.y + t2.y};
        a[i3] = V{y3.x + t3.x, y3.y + t3.y};
    }
}

template <typename V, int B0, int B1>
__device__ __forceinline__ void apply_swap2(V (&a)[R], const FOp &op, const uint32_t (&jr)[R])
{
    const uint32_t cm = op.lcmask, cv = op.lcval;
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        if (r & ((1 << B0) | (1 << B1)))
            continue;
        if ((jr[r] & cm) == cv)
        {
            const int i1 = r | (1 << B0), i2 = r | (1 << B1);
            const V t = a[i1];
            a[i1] = a[i2];
            a[i2] = t;
        }
    }
}

template <typename V>
__device__ __forceinline__ void apply_phase(V (&a)[R], const FOp &op, const uint32_t (&jr)[R])
{
    const V e = cvt<V>(op.m[0]);
    const uint32_t cm = op.lcmask, cv = op.lcval;
#pragma unroll
    for (int r = 0; r < R; ++r)
        if ((jr[r] & cm) == cv)
            a[r] = cmul(e, a[r]);
}

template <typename V>
__device__ __forceinline__ void apply_diag(V (&a)[R], const FOp &op, const uint32_t (&jr)[R], uint64_t cbase)
{
    // one or two targets: entries in registers, chosen per amplitude by its
    // target bits (from the local index, or from the chunk when not local)
    const V d0 = cvt<V>(op.m[0]), d1 = cvt<V>(op.m[1]), d2 = cvt<V>(op.m[2]), d3 = cvt<V>(op.m[3]);
    const uint32_t cm = op.lcmask, cv = op.lcval;
    const int l0 = op.loc[0], l1 = op.nt > 1 ? op.loc[1] : -1;
    const uint32_t c0 = l0 < 0 ? static_cast<uint32_t>((cbase >> op.phys[0]) & 1ull) : 0u;
    const uint32_t c1 = (op.nt > 1 && l1 < 0) ? static_cast<uint32_t>((cbase >> op.phys[1]) & 1ull) : 0u;
    const uint32_t sh0 = l0 < 0 ? 0u : static_cast<uint32_t>(l0);
    const uint32_t sh1 = l1 < 0 ? 0u : static_cast<uint32_t>(l1);
    const uint32_t use0 = l0 < 0 ? 0u : 1u, use1 = l1 < 0 ? 0u : 1u;
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        const uint32_t j = jr[r];
        if ((j & cm) != cv)
            continue;
        const uint32_t s0 = use0 ? ((j >> sh0) & 1u) : c0;
        const uint32_t s1 = use1 ? ((j >> sh1) & 1u) : c1;
        const V d = s1 ? (s0 ? d3 : d2) : (s0 ? d1 : d0);
        a[r] = cmul(d, a[r]);
    }
}

template <typename V>
__device__ __forceinline__ void dispatch_dense1(V (&a)[R], const FOp &op, const uint32_t (&jr)[R])
{
    switch (op.b0)
    {
    case 0: apply_dense1<V, 0>(a, op, jr); break;
    case 1: apply_dense1<V, 1>(a, op, jr); break;
    case 2: apply_dense1<V, 2>(a, op, jr); break;
    default: apply_dense1<V, 3>(a, op, jr); break;
    }
}

template <typename V>
__device__ __forceinline__ void dispatch_swap1(V (&a)[R], const FOp &op, const uint32_t (&jr)[R])
{
    switch (op.b0)
    {
    case 0: apply_swap1<V, 0>(a, op, jr); break;
    case 1: apply_swap1<V, 1>(a, op, jr); break;
    case 2: apply_swap1<V, 2>(a, op, jr); break;
    default: apply_swap1<V, 3>(a, op, jr); break;
    }
}

// (b0, b1) with b0 < b1 encoded as b0 * 4 + b1
template <typename V>
__device__ __forceinline__ void dispatch_dense2(V (&a)[R], const FOp &op, const uint32_t (&jr)[R])
{
    switch (op.b0 * 4 + op.b1)
    {
    case 1: apply_dense2<V, 0, 1>(a, op, jr); break;
    case 2: apply_dense2<V, 0, 2>(a, op, jr); break;
    case 3: apply_dense2<V, 0, 3>(a, op, jr); break;
    case 6: apply_dense2<V, 1, 2>(a, op, jr); break;
    case 7: apply_dense2<V, 1, 3>(a, op, jr); break;
    default: apply_dense2<V, 2, 3>(a, op, jr); break;
    }
}

template <typename V>
__device__ __forceinline__ void dispatch_swap2(V (&a)[R], const FOp &op, const uint32_t (&jr)[R])
{
    switch (op.b0 * 4 + op.b1)
    {
    case 1: apply_swap2<V, 0, 1>(a, op, jr); break;
    case 2: apply_swap2<V, 0, 2>(a, op, jr); break;
    case 3: apply_swap2<V, 0, 3>(a, op, jr); break;
    case 6: apply_swap2<V, 1, 2>(a, op, jr); break;
    case 7: apply_swap2<V, 1, 3>(a, op, jr); break;
    default: apply_swap2<V, 2, 3>(a, op, jr); break;
    }
}

// One CTA per chunk at a time; blockDim.x == 2^(k - kStageBits) <= 128, so
// that three CTAs (12 warps, 3 x 64 KB of double-buffered chunks) share an SM.
template <typename Real>
__global__ void __launch_bounds__(128, sizeof(Real) == 8 ? 3 : 4) fused_pass_kernel(const __grid_constant__ FPassParams p)
{
    typedef typename Cx<Real>::T V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *smem = reinterpret_cast<V *>(smem_raw);
    V *state = static_cast<V *>(p.state);
    const int k = p.k;
    const int T = 1 << (k - kStageBits);
    const int tid = threadIdx.x;
    const int chunk_elems = 1 << k;

    // global offset of this thread's element tid + m*T, m < R
    uint64_t dep_tid = 0;
    for (int i = 0; i < k - kStageBits; ++i)
        if ((tid >> i) & 1)
            dep_tid |= p.qbit[i];
    uint64_t hb[kStageBits];
#pragma unroll
    for (int b = 0; b < kStageBits; ++b)
        hb[b] = p.qbit[k - kStageBits + b];

    auto chunk_base = [&](uint64_t c) -> uint64_t {
        uint64_t g = c;
        for (int i = 0; i < k; ++i)
        {
            const uint64_t lo = g & p.qmasks[i];
            g = lo | ((g ^ lo) << 1);
        }
        return g;
    };
    auto elem_offset = [&](int m) -> uint64_t {
        uint64_t off = dep_tid;
#pragma unroll
        for (int b = 0; b < kStageBits; ++b)
            if ((m >> b) & 1)
                off |= hb[b];
        return off;
    };
    auto issue_load = [&](uint64_t c, V *dst) {
        const uint64_t cb = chunk_base(c);
#pragma unroll
        for (int m = 0; m < R; ++m)
            cp_async_amp<V>(dst + swz<V>(tid + m * T), state + (cb | elem_offset(m)));
        cp_async_commit();
    };

    uint64_t c = blockIdx.x;
    if (c >= p.chunks)
        return;
    issue_load(c, smem);
    int cur = 0;
    for (; c < p.chunks; c += gridDim.x)
    {
        V *sb = smem + cur * chunk_elems;
        const uint64_t next = c + gridDim.x;
        if (next < p.chunks)
        {
            issue_load(next, smem + (cur ^ 1) * chunk_elems);
            cp_async_wait<1>();
        }
        else
        {
            cp_async_wait<0>();
        }
        __syncthreads();
        const uint64_t cbase = chunk_base(c);

        for (int st = 0; st < p.nstages; ++st)
        {
            const FStage &S = p.stages[st];
            uint32_t j0 = static_cast<uint32_t>(tid);
#pragma unroll
            for (int b = 0; b < kStageBits; ++b)
            {
                const uint32_t lo = j0 & ((1u << S.sbits[b]) - 1u);
                j0 = lo | ((j0 ^ lo) << 1);
            }
            // swz is linear over GF(2) and j0 shares no bit with a stage
            // offset, so swz(j0 | off) = swz(j0) ^ swz(off)
            uint32_t bit[kStageBits], sbit[kStageBits];
#pragma unroll
            for (int b = 0; b < kStageBits; ++b)
            {
                bit[b] = 1u << S.sbits[b];
                sbit[b] = static_cast<uint32_t>(swz<V>(static_cast<int>(bit[b])));
            }
            const uint32_t p0 = static_cast<uint32_t>(swz<V>(static_cast<int>(j0)));
            uint32_t jr[R], pos[R];
            V a[R];
#pragma unroll
            for (int r = 0; r < R; ++r)
            {
                uint32_t j = j0, q = p0;
#pragma unroll
                for (int b = 0; b < kStageBits; ++b)
                    if ((r >> b) & 1)
                    {
                        j |= bit[b];
                        q ^= sbit[b];
                    }
                jr[r] = j;
                pos[r] = q;
                a[r] = sb[q];
            }
            for (int oi = S.op_begin; oi < S.op_end; ++oi)
            {
                const FOp &op = p.ops[oi];
                if ((cbase & op.gcmask) != op.gcval)
                    continue;
                switch (op.kind)
                {
                case F_DENSE1: dispatch_dense1<V>(a, op, jr); break;
                case F_SWAP1: dispatch_swap1<V>(a, op, jr); break;
                case F_DENSE2: dispatch_dense2<V>(a, op, jr); break;
                case F_SWAP2: dispatch_swap2<V>(a, op, jr); break;
                case F_PHASE: apply_phase<V>(a, op, jr); break;
                default: apply_diag<V>(a, op, jr, cbase); break;
                }
            }
#pragma unroll
            for (int r = 0; r < R; ++r)
                sb[pos[r]] = a[r];
            __syncthreads();
        }

        const uint64_t cb = cbase;
#pragma unroll
        for (int m = 0; m < R; ++m)
            __stcs(state + (cb | elem_offset(m)), sb[swz<V>(tid + m * T)]);
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

struct PlannedPass
{
    std::vector<int> ops;   // indices into the queue, in execution order
    uint64_t local = 0;     // physical qubits of Q
    int k = 0;              // |Q|
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
        const size_t window_end = std::min(N, first + kPlanWindow);
        for (size_t i = first; i < window_end; ++i)
        {
            if (done[i])
                continue;
            const OpClass &c = cls[i];
            const uint64_t support = c.dense | c.diag;
            bool take = c.fusable && (int)s.pass.ops.size() < max_ops &&
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
                if (__builtin_popcount(nb) > kStageBits)
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

// Fill the kernel parameters of a pass. Returns false when the pass does not
// fit the parameter block limits.
bool build_params(const std::vector<GateOp> &q, const PlannedPass &pp, int n, int k, FPassParams &prm)
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
    if (pp.ops.size() > (size_t)kFusedMaxOps)
        return false;

    std::vector<std::vector<int>> stage_ops;
    std::vector<uint32_t> stage_bits;
    schedule_stages(q, pp, loc_of, stage_ops, stage_bits);
    if (stage_ops.size() > (size_t)kFusedMaxStages)
        return false;
    prm.nstages = (int)stage_ops.size();
    int nops = 0;
    for (size_t si = 0; si < stage_ops.size(); ++si)
    {
        // stage bits: the needed ones, padded with the lowest other local bits
        uint32_t bits = stage_bits[si];
        for (int l = 0; l < k && __builtin_popcount(bits) < kStageBits; ++l)
            bits |= 1u << l;
        FStage &S = prm.stages[si];
        int pos_in_stage[kMaxLocal];
        int nb = 0;
        for (int l = 0; l < k; ++l)
            if ((bits >> l) & 1)
            {
                pos_in_stage[l] = nb;
                S.sbits[nb++] = static_cast<uint8_t>(l);
            }
        S.op_begin = static_cast<uint16_t>(nops);
        for (int oi : stage_ops[si])
        {
            const GateOp &op = q[pp.ops[oi]];
            FOp &f = prm.ops[nops++];
            std::memset(&f, 0, sizeof(f));
            f.nt = static_cast<uint8_t>(op.nt);
            uint64_t cm = op.cmask, cv = op.cval;
            if (op.diag && op.na == 1)
            {
                // one changed sub-index: a phase on the amplitudes whose
                // control and target bits all match
                f.kind = F_PHASE;
                for (int i = 0; i < op.nt; ++i)
                {
                    cm |= 1ull << op.tq[i];
                    if ((op.act[0] >> i) & 1)
                        cv |= 1ull << op.tq[i];
                }
                f.m[0] = make_double2(op.mat[0].re, op.mat[0].im);
            }
            else if (op.diag)
            {
                f.kind = F_DIAG;
                for (int s = 0; s < 4; ++s)
                    f.m[s] = make_double2(1.0, 0.0);
                for (int a = 0; a < op.na; ++a)
                    f.m[op.act[a]] = make_double2(op.mat[a].re, op.mat[a].im);
                for (int i = 0; i < op.nt; ++i)
                {
                    f.phys[i] = static_cast<uint8_t>(op.tq[i]);
                    f.loc[i] = static_cast<int8_t>(loc_of[op.tq[i]]);
                }
                if (op.nt < 2)
                {
                    // second target absent: entries 2, 3 repeat 0, 1
                    f.m[2] = f.m[0];
                    f.m[3] = f.m[1];
                    f.loc[1] = -1;
                    f.phys[1] = 0;
                }
            }
            else if (op.nt == 1)
            {
                f.kind = is_x(op) ? F_SWAP1 : F_DENSE1;
                f.b0 = static_cast<uint8_t>(pos_in_stage[loc_of[op.tq[0]]]);
                expand_dense(op, f.m);
            }
            else
            {
                f.kind = is_swap(op) ? F_SWAP2 : F_DENSE2;
                int p0 = pos_in_stage[loc_of[op.tq[0]]];
                int p1 = pos_in_stage[loc_of[op.tq[1]]];
                double2 full[16];
                expand_dense(op, full);
                if (p0 < p1)
                {
                    for (int i = 0; i < 16; ++i)
                        f.m[i] = full[i];
                }
                else
                {
                    // exchange the roles of the two targets: sub-index bits swap
                    auto sw = [](int s) { return ((s & 1) << 1) | ((s >> 1) & 1); };
                    for (int r = 0; r < 4; ++r)
                        for (int c = 0; c < 4; ++c)
                            f.m[r * 4 + c] = full[sw(r) * 4 + sw(c)];
                    std::swap(p0, p1);
                }
                f.b0 = static_cast<uint8_t>(p0);
                f.b1 = static_cast<uint8_t>(p1);
            }
            uint32_t lcm = 0, lcv = 0;
            uint64_t gcm = 0, gcv = 0;
            for (int b = 0; b < n; ++b)
                if ((cm >> b) & 1)
                {
                    const bool v = (cv >> b) & 1;
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
        }
        S.op_end = static_cast<uint16_t>(nops);
    }
    return true;
}

template <typename R>
int launch_fused_pass(void *state, int k, const FPassParams &prm, cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    const int threads = 1 << (k - kStageBits);
    const size_t smem = 2 * sizeof(V) * (size_t(1) << k);
    static bool configured[64] = {};
    int dev = 0;
    QCSB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !configured[dev])
    {
        QCSB_CUDA(cudaFuncSetAttribute(fused_pass_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       2 * (int)sizeof(V) * (1 << kMaxLocal)));
        if (dev >= 0 && dev < 64)
            configured[dev] = true;
    }
    int per_sm = 0;
    QCSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fused_pass_kernel<R>, threads, smem));
    int sms = 148;
    QCSB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    uint64_t grid = prm.chunks;
    const uint64_t cap = (uint64_t)sms * (per_sm > 0 ? per_sm : 1);
    if (grid > cap)
        grid = cap;
    FPassParams &p = const_cast<FPassParams &>(prm);
    p.state = state;
    fused_pass_kernel<R><<<static_cast<unsigned>(grid), threads, smem, stream>>>(p);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

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

PassFeatures pass_features(const PlannedPass &pp, int n, int amp_bytes)
{
    int top = 0;
    for (int b = 0; b < n; ++b)
        if ((pp.local >> b) & 1)
            top = b;
    PassFeatures f;
    f.f[0] = static_cast<float>(pp.k);
    f.f[1] = static_cast<float>(top);
    f.f[2] = static_cast<float>(pp.ops.size());
    f.f[3] = static_cast<float>(amp_bytes);
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
// order; the planner chooses where to cut it into passes, and each pass's
// number of local qubits k, to minimise the sum of predicted pass times.
// A candidate pass [i, j) with local qubits k is feasible when the low
// qubits plus its dense targets fit in k and it holds at most max_ops gates.
std::vector<Segment> plan_learned(const std::vector<GateOp> &q, const std::vector<Segment> &greedy, int n,
                                  int amp_bytes, int max_ops, CostModel &model, double *predicted_greedy,
                                  double *predicted_learned)
{
    const int kmin = clamp_local_bits(kStageBits + 5, n);
    const int kmax = clamp_local_bits(kMaxLocal, n);
    const int low = std::min(kLowBits, kmin);
    const uint64_t low_mask = (1ull << low) - 1;
    std::vector<Segment> out;
    *predicted_greedy = *predicted_learned = 0.0;
    size_t gi = 0;
    while (gi < greedy.size())
    {
        if (!greedy[gi].fused)
        {
            out.push_back(greedy[gi++]);
            continue;
        }
        std::vector<int> seq;
        std::vector<PassFeatures> greedy_feats;
        while (gi < greedy.size() && greedy[gi].fused)
        {
            seq.insert(seq.end(), greedy[gi].pass.ops.begin(), greedy[gi].pass.ops.end());
            greedy_feats.push_back(pass_features(greedy[gi].pass, n, amp_bytes));
            ++gi;
        }
        const int L = (int)seq.size();
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
        struct Cand
        {
            int i, j, k;
            uint64_t local;
        };
        std::vector<Cand> cands;
        std::vector<float> feats;
        for (int j = 1; j <= L; ++j)
        {
            uint64_t d = low_mask;
            for (int i = j - 1; i >= 0 && j - i <= max_ops; --i)
            {
                d |= dense[i];
                const int need = __builtin_popcountll(d);
                if (need > kmax)
                    break;
                for (int k = std::max(need, kmin); k <= kmax; ++k)
                {
                    PlannedPass pp;
                    pp.k = k;
                    pp.local = fill_local(d, n, k);
                    pp.ops.assign(j - i, 0);
                    const PassFeatures f = pass_features(pp, n, amp_bytes);
                    cands.push_back({i, j, k, pp.local});
                    feats.insert(feats.end(), f.f, f.f + 4);
                }
            }
        }
        std::vector<float> pred(cands.size());
        model.predict(feats.data(), (int)cands.size(), pred.data());
        std::vector<float> gpred(greedy_feats.size());
        model.predict(&greedy_feats[0].f[0], (int)greedy_feats.size(), gpred.data());
        const double amps_ns = std::ldexp(1.0, n);
        for (float v : gpred)
            *predicted_greedy += std::exp(double(v)) * amps_ns;
        const double inf = 1e300;
        std::vector<double> best(L + 1, inf);
        std::vector<int> from(L + 1, -1);
        best[0] = 0.0;
        // candidates are grouped by j ascending, so best[i] is final when read
        for (size_t c = 0; c < cands.size(); ++c)
        {
            const Cand &cd = cands[c];
            const double cost = best[cd.i] + std::exp(double(pred[c])) * amps_ns;
            if (cost < best[cd.j])
            {
                best[cd.j] = cost;
                from[cd.j] = (int)c;
            }
        }
        *predicted_learned += best[L];
        std::vector<Segment> run;
        for (int j = L; j > 0;)
        {
            const Cand &cd = cands[from[j]];
            Segment sg;
            sg.fused = true;
            sg.plain_op = -1;
            sg.pass.k = cd.k;
            sg.pass.local = cd.local;
            sg.pass.ops.assign(seq.begin() + cd.i, seq.begin() + cd.j);
            run.push_back(std::move(sg));
            j = cd.i;
        }
        out.insert(out.end(), run.rbegin(), run.rend());
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

} // namespace

int fused_min_qubits() { return kStageBits + 5; }

FusedExecutor::FusedExecutor(cudaStream_t stream) : stream_(stream) {}

FusedExecutor::~FusedExecutor()
{
    if (judge_a_)
        cudaEventDestroy(judge_a_);
    if (judge_b_)
        cudaEventDestroy(judge_b_);
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

int FusedExecutor::run(void *state, int n, int amp_bytes, const std::vector<GateOp> &ops, int mode,
                       qcs_b200_stats &stats, KernelTimer &timer)
{
    const bool c64 = amp_bytes == (int)sizeof(float2);
    auto plain = [&](const GateOp &op) {
        if (timer.enabled)
            timer.begin(stream_, KernelTimer::kPlain, 2.0 * amp_bytes * op.changed_amps(n));
        const int k = c64 ? launch_gate_plain<float>(static_cast<float2 *>(state), n, op, stream_)
                          : launch_gate_plain<double>(static_cast<double2 *>(state), n, op, stream_);
        if (timer.enabled)
            timer.end(stream_);
        stats.plain_gate_kernels += k;
        return k;
    };
    int launches = 0;
    // Small registers: a pass would not fill a warp; run gate by gate.
    if (n < fused_min_qubits())
    {
        for (const GateOp &op : ops)
            launches += plain(op);
        return launches;
    }
    const int k = choose_local_bits(n, local_bits_);
    const int low = std::min(kLowBits, k);
    const int max_ops = (max_ops_ > 0 && max_ops_ < kFusedMaxOps) ? max_ops_ : kFusedMaxOps;
    std::vector<Segment> segs = plan_greedy(ops, n, k, low, max_ops);

    bool timed_flush = false;
    if (mode == QCS_FUSION_LEARNED && model_ != nullptr && model_->trained())
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
        if (use_learned)
        {
            double pg = 0.0, pl = 0.0;
            segs = plan_learned(ops, segs, n, amp_bytes, max_ops, *model_, &pg, &pl);
        }
        if (entry->learned_ms < 0.0 || entry->greedy_ms < 0.0)
        {
            if (!judge_a_)
            {
                QCSB_CUDA(cudaEventCreate(&judge_a_));
                QCSB_CUDA(cudaEventCreate(&judge_b_));
            }
            QCSB_CUDA(cudaEventRecord(judge_a_, stream_));
            pending_sig_ = sig;
            pending_learned_ = use_learned ? 1 : 0;
            timed_flush = true;
        }
    }
    else
    {
        last_plan_learned = 0;
    }

    FPassParams *prm = new FPassParams;
    for (const Segment &s : segs)
    {
        if (!s.fused)
        {
            launches += plain(ops[s.plain_op]);
            continue;
        }
        if (build_params(ops, s.pass, n, s.pass.k, *prm))
        {
            if (timer.enabled)
            {
                const PassFeatures f = pass_features(s.pass, n, amp_bytes);
                timer.begin(stream_, KernelTimer::kFused, 2.0 * amp_bytes * std::ldexp(1.0, n), &f);
            }
            launches += c64 ? launch_fused_pass<float>(state, s.pass.k, *prm, stream_)
                             : launch_fused_pass<double>(state, s.pass.k, *prm, stream_);
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
    if (timed_flush)
        QCSB_CUDA(cudaEventRecord(judge_b_, stream_));
    return launches;
}

} // namespace qcsb
