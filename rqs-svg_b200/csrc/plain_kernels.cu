// Plain-path kernels: one launch per gate, state preparation, measurement
// reductions, collapse, <Z> sums and logical-order transfers.
//
// Layout: the register is one contiguous array of complex amplitudes
// (double2 for complex128, float2 for complex64); physical qubit q is bit q
// of the index. A gate on targets T with controls C visits "groups": the
// 2^(n - |T u C|) indices whose T and C bits are zero, enumerated by
// inserting zero bits at the sorted operand positions (the role of
// thread_num_to_state_index_q*, reference src/qcs.cu:156-376), then ORs in
// the control values and each active target offset.
//
// Consecutive threads take consecutive groups, so every warp reads and writes
// contiguous amplitudes wherever the operand bits are >= 5; loads and stores
// use evict-first hints (each amplitude is touched once per pass over a
// register far larger than L2). Gate arithmetic runs in the amplitude's
// precision; every reduction accumulates in FP64.

#include "qcs_internal.h"

#include <cuda_runtime.h>

#include <cstdlib>

namespace qcsb
{
namespace
{

constexpr int kThreads = 256;
constexpr int kSMs = 148;
constexpr int kMaxOps = kMaxQubits;

template <typename V>
__device__ __forceinline__ V cfma(V m, V v, V acc)
{
    acc.x = fma(m.x, v.x, acc.x);
    acc.x = fma(-m.y, v.y, acc.x);
    acc.y = fma(m.x, v.y, acc.y);
    acc.y = fma(m.y, v.x, acc.y);
    return acc;
}

template <typename V>
__device__ __forceinline__ V cmul(V m, V v)
{
    V r;
    r.x = fma(m.x, v.x, -m.y * v.y);
    r.y = fma(m.x, v.y, m.y * v.x);
    return r;
}

template <typename V>
__device__ __forceinline__ double norm2(V a)
{
    const double x = a.x, y = a.y;
    return fma(x, x, y * y);
}

template <typename V>
__host__ __device__ __forceinline__ V make_cx(double re, double im);
template <>
__host__ __device__ __forceinline__ double2 make_cx<double2>(double re, double im) { return make_double2(re, im); }
template <>
__host__ __device__ __forceinline__ float2 make_cx<float2>(double re, double im)
{
    return make_float2(static_cast<float>(re), static_cast<float>(im));
}

// Insert a zero bit below each mask boundary: masks[i] = (1 << pos_i) - 1
// for operand positions sorted ascending.
template <int MAXOPS>
__device__ __forceinline__ uint64_t insert_zero_bits(uint64_t g, const uint64_t *masks, int nops)
{
#pragma unroll
    for (int i = 0; i < MAXOPS; ++i)
    {
        if (i >= nops)
            break;
        const uint64_t lo = g & masks[i];
        g = lo | ((g ^ lo) << 1);
    }
    return g;
}

template <typename R, int NA, bool DIAG>
struct PlainParams
{
    typedef typename Cx<R>::T V;
    V *state;
    uint64_t ngroups;
    uint64_t cval;
    int nops;
    uint64_t masks[kMaxOps];
    uint64_t off[NA];
    V m[DIAG ? NA : NA * NA];
};

template <bool STREAM, typename V>
__device__ __forceinline__ V ld_amp(const V *p) { return STREAM ? __ldcs(p) : *p; }
template <bool STREAM, typename V>
__device__ __forceinline__ void st_amp(V *p, V v)
{
    if (STREAM)
        __stcs(p, v);
    else
        *p = v;
}

// STREAM selects evict-first cache hints; U groups per thread per iteration.
template <typename R, int NA, bool DIAG, int U, bool STREAM>
__global__ void __launch_bounds__(kThreads) gate_plain_kernel(const __grid_constant__ PlainParams<R, NA, DIAG> p)
{
    typedef typename Cx<R>::T V;
    const uint64_t step = (uint64_t)gridDim.x * kThreads * U;
    for (uint64_t g0 = (uint64_t)blockIdx.x * kThreads * U + threadIdx.x; g0 < p.ngroups; g0 += step)
    {
        uint64_t base[U];
        V v[U][NA];
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const uint64_t g = g0 + (uint64_t)u * kThreads;
            base[u] = insert_zero_bits<kMaxOps>(g, p.masks, p.nops) | p.cval;
            if (g < p.ngroups)
            {
#pragma unroll
                for (int a = 0; a < NA; ++a)
                    v[u][a] = ld_amp<STREAM>(p.state + (base[u] | p.off[a]));
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
        {
            const uint64_t g = g0 + (uint64_t)u * kThreads;
            if (g >= p.ngroups)
                continue;
            if (DIAG)
            {
#pragma unroll
                for (int a = 0; a < NA; ++a)
                    st_amp<STREAM>(p.state + (base[u] | p.off[a]), cmul(p.m[a], v[u][a]));
            }
            else
            {
#pragma unroll
                for (int a = 0; a < NA; ++a)
                {
                    V acc = make_cx<V>(0.0, 0.0);
#pragma unroll
                    for (int b = 0; b < NA; ++b)
                        acc = cfma(p.m[a * NA + b], v[u][b], acc);
                    st_amp<STREAM>(p.state + (base[u] | p.off[a]), acc);
                }
            }
        }
    }
}

// Sorted operand positions (targets and controls) as insertion masks.
int fill_masks(const GateOp &op, uint64_t *masks)
{
    uint64_t bits = op.cmask;
    for (int i = 0; i < op.nt; ++i)
        bits |= 1ull << op.tq[i];
    int nops = 0;
    while (bits)
    {
        const int pos = __builtin_ctzll(bits);
        masks[nops++] = (1ull << pos) - 1;
        bits &= bits - 1;
    }
    return nops;
}

unsigned grid_for(uint64_t work_items, int per_block, uint64_t cap = (uint64_t)kSMs * 16)
{
    uint64_t blocks = (work_items + per_block - 1) / per_block;
    if (blocks > cap)
        blocks = cap;
    if (blocks == 0)
        blocks = 1;
    return static_cast<unsigned>(blocks);
}

// Launch shape of the plain gate kernel (tuning knob QCS_PLAIN_VARIANT):
//   0  grid-stride over 148 x 16 blocks, U groups per thread, evict-first hints
//   1  one thread per group over the whole grid, default cache policy
//   2  one thread per group over the whole grid, evict-first hints (default:
//      measured fastest on B200, 103% of the copy bandwidth at 30 qubits)
//   3  grid-stride, U groups per thread, default cache policy
int plain_variant()
{
    static int v = [] {
        const char *e = std::getenv("QCS_PLAIN_VARIANT");
        const int x = (e && e[0]) ? std::atoi(e) : 2;
        return (x >= 0 && x <= 3) ? x : 2;
    }();
    return v;
}

template <typename R, int NA, bool DIAG>
int launch_plain_na(typename Cx<R>::T *state, int n, const GateOp &op, cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    constexpr int U = NA == 1 ? 4 : (NA == 2 ? 2 : 1);
    PlainParams<R, NA, DIAG> p;
    std::memset(&p, 0, sizeof(p));
    p.state = state;
    p.nops = fill_masks(op, p.masks);
    p.ngroups = 1ull << (n - p.nops);
    p.cval = op.cval;
    for (int a = 0; a < NA; ++a)
    {
        uint64_t off = 0;
        for (int i = 0; i < op.nt; ++i)
            if ((op.act[a] >> i) & 1)
                off |= 1ull << op.tq[i];
        p.off[a] = off;
    }
    const int nm = DIAG ? NA : NA * NA;
    for (int k = 0; k < nm; ++k)
        p.m[k] = make_cx<V>(op.mat[k].re, op.mat[k].im);
    const uint64_t one_shot_cap = 1ull << 31;
    switch (plain_variant())
    {
    case 0:
        gate_plain_kernel<R, NA, DIAG, U, true><<<grid_for(p.ngroups, kThreads * U), kThreads, 0, stream>>>(p);
        break;
    case 2:
        gate_plain_kernel<R, NA, DIAG, 1, true><<<grid_for(p.ngroups, kThreads, one_shot_cap), kThreads, 0, stream>>>(p);
        break;
    case 3:
        gate_plain_kernel<R, NA, DIAG, U, false><<<grid_for(p.ngroups, kThreads * U), kThreads, 0, stream>>>(p);
        break;
    default:
        gate_plain_kernel<R, NA, DIAG, 1, false><<<grid_for(p.ngroups, kThreads, one_shot_cap), kThreads, 0, stream>>>(p);
        break;
    }
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template <typename R, bool DIAG>
int launch_plain_dispatch(typename Cx<R>::T *state, int n, const GateOp &op, cudaStream_t stream)
{
    switch (op.na)
    {
    case 1: return launch_plain_na<R, 1, DIAG>(state, n, op, stream);
    case 2: return launch_plain_na<R, 2, DIAG>(state, n, op, stream);
    case 3: return launch_plain_na<R, 3, DIAG>(state, n, op, stream);
    case 4: return launch_plain_na<R, 4, DIAG>(state, n, op, stream);
    default: throw std::runtime_error(strformat("internal: %d active sub-indices", op.na));
    }
}

// ------------------------------------------------------------ preparation

template <typename V>
__global__ void fill_kernel(V *state, uint64_t count, V value)
{
    for (uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x; i < count; i += (uint64_t)gridDim.x * kThreads)
        __stcs(state + i, value);
}

template <typename V>
__global__ void sequential_kernel(V *state, uint64_t count)
{
    for (uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x; i < count; i += (uint64_t)gridDim.x * kThreads)
        __stcs(state + i, make_cx<V>(static_cast<double>(i), 0.0));
}

template <typename V>
__global__ void set_one_kernel(V *state, uint64_t index, V value) { state[index] = value; }

// a *= sqrt(target / norm), the factor formed in FP64 from the squared norm
// the reduction left in device memory (no host round trip); a zero norm
// leaves the state as it is.
template <typename V>
__global__ void rescale_kernel(V *state, uint64_t count, double target, const double *norm)
{
    const double nrm = *norm;
    if (!(nrm > 0.0))
        return;
    const double f = sqrt(target / nrm);
    for (uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x; i < count; i += (uint64_t)gridDim.x * kThreads)
    {
        const V a = state[i];
        __stcs(state + i, make_cx<V>(a.x * f, a.y * f));
    }
}

// ------------------------------------------------------------ reductions

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename R>
struct ProbParams
{
    const typename Cx<R>::T *state;
    uint64_t ngroups;
    uint64_t cval;
    uint64_t tbit;
    int nops;
    uint64_t masks[kMaxOps];
    double2 *partials;
    double2 *result;      // final (P0, P1); may be mapped host memory
    unsigned *ticket;     // zero between calls
    volatile unsigned *done;   // host-mapped: set to seq once result is written (or null)
    unsigned seq;
};

// Fixed-order sum of count double2 partials by one block of kThreads threads
// (the same order in every call, so repeated measurements agree bit for bit).
__device__ __forceinline__ double2 block_sum_partials(const double2 *partials, int count)
{
    double s0 = 0.0, s1 = 0.0;
    for (int i = threadIdx.x; i < count; i += kThreads)
    {
        const double2 v = __ldcg(partials + i);
        s0 += v.x;
        s1 += v.y;
    }
    __shared__ double sh[2][kThreads / 32];
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0)
    {
        sh[0][w] = s0;
        sh[1][w] = s1;
    }
    __syncthreads();
    double t0 = 0.0, t1 = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < kThreads / 32; ++k)
        {
            t0 += sh[0][k];
            t1 += sh[1][k];
        }
    return make_double2(t0, t1);
}

// Per-block (sum |a0|^2, sum |a1|^2) over the groups; fixed reduction order,
// so repeated calls give identical sums. The last block to finish adds the
// per-block partials and writes (P0, P1) to p.result.
template <typename R>
__global__ void __launch_bounds__(kThreads) measure_probs_kernel(const __grid_constant__ ProbParams<R> p)
{
    double s0 = 0.0, s1 = 0.0;
    for (uint64_t g = (uint64_t)blockIdx.x * kThreads + threadIdx.x; g < p.ngroups; g += (uint64_t)gridDim.x * kThreads)
    {
        const uint64_t i0 = insert_zero_bits<kMaxOps>(g, p.masks, p.nops) | p.cval;
        s0 += norm2(__ldcs(p.state + i0));
        s1 += norm2(__ldcs(p.state + (i0 | p.tbit)));
    }
    __shared__ double sh[2][kThreads / 32];
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0)
    {
        sh[0][w] = s0;
        sh[1][w] = s1;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double t0 = 0.0, t1 = 0.0;
        for (int k = 0; k < kThreads / 32; ++k)
        {
            t0 += sh[0][k];
            t1 += sh[1][k];
        }
        p.partials[blockIdx.x] = make_double2(t0, t1);
        __threadfence();
    }
    __shared__ bool last;
    if (threadIdx.x == 0)
        last = atomicAdd(p.ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last)
        return;
    __threadfence();
    const double2 total = block_sum_partials(p.partials, gridDim.x);
    if (threadIdx.x == 0)
    {
        *p.result = total;
        *p.ticket = 0;
        if (p.done != nullptr)
        {
            // the result reaches host memory before the flag does
            __threadfence_system();
            *p.done = p.seq;
        }
    }
}


template <typename V>
__global__ void collapse_kernel(V *state, uint64_t ngroups, uint64_t lowmask, uint64_t zero_bit)
{
    for (uint64_t g = (uint64_t)blockIdx.x * kThreads + threadIdx.x; g < ngroups; g += (uint64_t)gridDim.x * kThreads)
    {
        const uint64_t lo = g & lowmask;
        const uint64_t i = lo | ((g ^ lo) << 1) | zero_bit;
        __stcs(state + i, make_cx<V>(0.0, 0.0));
    }
}

// Kept amplitudes are not touched (no reads at all).
template <typename V>
__global__ void collapse_mask_kernel(V *state, uint64_t count, uint64_t cmask, uint64_t cval)
{
    for (uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x; i < count; i += (uint64_t)gridDim.x * kThreads)
        if ((i & cmask) != cval)
            __stcs(state + i, make_cx<V>(0.0, 0.0));
}

// <Z> sums. Thread k of the grid (G = gridDim * 256 = 2^gbits threads)
// visits indices i = it * G + k. Bits of i below gbits are fixed per thread;
// bits at or above gbits are the bits of `it`. Per block the kernel writes
// n + 1 partial sums: [0] the block's total, [1 + q] the part with bit q set.
constexpr int kZThreads = 256;
constexpr int kZMinBits = 12;                 // registers below this use one thread
constexpr int kZMaxHi = kMaxQubits - kZMinBits; // "it" bits per thread

template <typename V>
__global__ void zsums_small_kernel(const V *state, int n, double *sums)
{
    double s[kMaxQubits + 1];
    for (int j = 0; j <= n; ++j)
        s[j] = 0.0;
    for (uint64_t i = 0; i < (1ull << n); ++i)
    {
        const double pr = norm2(state[i]);
        s[0] += pr;
        for (int q = 0; q < n; ++q)
            if ((i >> q) & 1)
                s[1 + q] += pr;
    }
    for (int j = 0; j <= n; ++j)
        sums[j] = s[j];
}

template <typename V>
__global__ void __launch_bounds__(kZThreads) zsums_kernel(const V *state, int n, int gbits, double *partials)
{
    const uint64_t gt = (uint64_t)blockIdx.x * kZThreads + threadIdx.x;
    const uint64_t G = 1ull << gbits;
    const uint64_t iters = 1ull << (n - gbits);
    double total = 0.0;
    double hi[kZMaxHi];
    const int nhi = n - gbits;
#pragma unroll
    for (int q = 0; q < kZMaxHi; ++q)
        hi[q] = 0.0;
    if (nhi >= 4)
    {
        // 16 iterations at a time: 16 loads in flight; bits 0..3 of `it` get
        // their partial sums from fixed index sets, higher bits get the
        // block's total once
        for (uint64_t blk = 0; blk < (iters >> 4); ++blk)
        {
            double pr[16];
#pragma unroll
            for (int i = 0; i < 16; ++i)
                pr[i] = norm2(__ldcs(state + ((blk << 4) + i) * G + gt));
            double t = 0.0;
#pragma unroll
            for (int i = 0; i < 16; ++i)
                t += pr[i];
            total += t;
#pragma unroll
            for (int b = 0; b < 4; ++b)
            {
                double s = 0.0;
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if ((i >> b) & 1)
                        s += pr[i];
                hi[b] += s;
            }
#pragma unroll
            for (int q = 4; q < kZMaxHi; ++q)
                if (q < nhi && ((blk >> (q - 4)) & 1))
                    hi[q] += t;
        }
    }
    else
    {
        for (uint64_t it = 0; it < iters; ++it)
        {
            const double pr = norm2(__ldcs(state + it * G + gt));
            total += pr;
#pragma unroll
            for (int q = 0; q < kZMaxHi; ++q)
                if (q < nhi && ((it >> q) & 1))
                    hi[q] += pr;
        }
    }
    __shared__ double sh[kZThreads / 32];
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    auto block_sum = [&](double v) -> double {
        v = warp_sum(v);
        __syncthreads();
        if (l == 0)
            sh[w] = v;
        __syncthreads();
        double t = 0.0;
        if (threadIdx.x == 0)
            for (int k = 0; k < kZThreads / 32; ++k)
                t += sh[k];
        return t;
    };
    double *out = partials + (size_t)blockIdx.x * (n + 1);
    const double btotal = block_sum(total);
    if (threadIdx.x == 0)
        out[0] = btotal;
    // Low bits: q < gbits. Thread bits (q < 8) mask the per-thread totals;
    // block bits (8 <= q < gbits) are uniform in the block.
    const int tbits = gbits < 8 ? gbits : 8;
    for (int q = 0; q < tbits; ++q)
    {
        const double v = block_sum(((threadIdx.x >> q) & 1) ? total : 0.0);
        if (threadIdx.x == 0)
            out[1 + q] = v;
    }
    if (threadIdx.x == 0)
        for (int q = tbits; q < gbits; ++q)
            out[1 + q] = ((gt >> q) & 1) ? btotal : 0.0;
    for (int q = 0; q < nhi; ++q)
    {
        const double v = block_sum(hi[q]);
        if (threadIdx.x == 0)
            out[1 + gbits + q] = v;
    }
}

__global__ void zsums_final_kernel(const double *partials, int nblocks, int nsums, double *sums)
{
    for (int j = threadIdx.x; j < nsums; j += blockDim.x)
    {
        double s = 0.0;
        for (int b = 0; b < nblocks; ++b)
            s += partials[(size_t)b * nsums + j];
        sums[j] = s;
    }
}

// ------------------------------------------------------------ transfers

struct PermParams
{
    int n;
    int l2p[kMaxQubits];
};

__device__ __forceinline__ uint64_t logical_to_physical(uint64_t l, const PermParams &pp)
{
    uint64_t ph = 0;
    for (int j = 0; j < pp.n; ++j)
        ph |= ((l >> j) & 1ull) << pp.l2p[j];
    return ph;
}

template <typename V>
__global__ void gather_logical_kernel(const V *state, PermParams pp, uint64_t begin, uint64_t count, double2 *out)
{
    for (uint64_t k = (uint64_t)blockIdx.x * kThreads + threadIdx.x; k < count; k += (uint64_t)gridDim.x * kThreads)
    {
        const V a = state[logical_to_physical(begin + k, pp)];
        out[k] = make_double2(a.x, a.y);
    }
}

template <typename V>
__global__ void scatter_logical_kernel(V *state, PermParams pp, uint64_t begin, uint64_t count, const double2 *in)
{
    for (uint64_t k = (uint64_t)blockIdx.x * kThreads + threadIdx.x; k < count; k += (uint64_t)gridDim.x * kThreads)
        state[logical_to_physical(begin + k, pp)] = make_cx<V>(in[k].x, in[k].y);
}

template <typename V>
__global__ void widen_kernel(const V *in, uint64_t count, double2 *out)
{
    for (uint64_t k = (uint64_t)blockIdx.x * kThreads + threadIdx.x; k < count; k += (uint64_t)gridDim.x * kThreads)
        out[k] = make_double2(in[k].x, in[k].y);
}

template <typename V>
__global__ void narrow_kernel(const double2 *in, uint64_t count, V *out)
{
    for (uint64_t k = (uint64_t)blockIdx.x * kThreads + threadIdx.x; k < count; k += (uint64_t)gridDim.x * kThreads)
        out[k] = make_cx<V>(in[k].x, in[k].y);
}

template <typename V>
__global__ void gather_indices_kernel(const V *state, const uint64_t *physical, uint64_t count, double2 *out)
{
    for (uint64_t k = (uint64_t)blockIdx.x * kThreads + threadIdx.x; k < count; k += (uint64_t)gridDim.x * kThreads)
    {
        const V a = state[physical[k]];
        out[k] = make_double2(a.x, a.y);
    }
}

// Per block: sum of conj(x_i) * y_i (re, im), max |x_i - y_i|, sum |x_i|^2
// and sum |y_i|^2, written as five doubles; a fixed grid and order make
// repeated calls identical.
__global__ void __launch_bounds__(kThreads) compare_kernel(const double2 *x, const double2 *y, uint64_t count,
                                                           double *partials)
{
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (uint64_t k = (uint64_t)blockIdx.x * kThreads + threadIdx.x; k < count; k += (uint64_t)gridDim.x * kThreads)
    {
        const double2 a = __ldcs(x + k), b = __ldcs(y + k);
        v[0] += a.x * b.x + a.y * b.y;
        v[1] += a.x * b.y - a.y * b.x;
        const double dx = a.x - b.x, dy = a.y - b.y;
        v[2] = fmax(v[2], sqrt(dx * dx + dy * dy));
        v[3] += a.x * a.x + a.y * a.y;
        v[4] += b.x * b.x + b.y * b.y;
    }
    __shared__ double sh[5][kThreads / 32];
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
#pragma unroll
    for (int i = 0; i < 5; ++i)
    {
        double t = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
            const double u = __shfl_xor_sync(0xffffffffu, t, o);
            t = i == 2 ? fmax(t, u) : t + u;
        }
        if (l == 0)
            sh[i][w] = t;
    }
    __syncthreads();
    if (threadIdx.x < 5)
    {
        const int i = threadIdx.x;
        double t = 0.0;
        for (int k = 0; k < kThreads / 32; ++k)
            t = i == 2 ? fmax(t, sh[i][k]) : t + sh[i][k];
        partials[5 * blockIdx.x + i] = t;
    }
}

PermParams make_perm(int n, const int *l2p)
{
    PermParams pp;
    pp.n = n;
    for (int j = 0; j < n; ++j)
        pp.l2p[j] = l2p[j];
    return pp;
}

} // namespace

template <typename R>
int launch_gate_plain(typename Cx<R>::T *state, int n, const GateOp &op, cudaStream_t stream)
{
    if (op.na == 0)
        return 0;
    return op.diag ? launch_plain_dispatch<R, true>(state, n, op, stream)
                   : launch_plain_dispatch<R, false>(state, n, op, stream);
}

template <typename R>
int launch_init_zero(typename Cx<R>::T *state, int n, cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    QCSB_CUDA(cudaMemsetAsync(state, 0, sizeof(V) << n, stream));
    set_one_kernel<V><<<1, 1, 0, stream>>>(state, 0, make_cx<V>(1.0, 0.0));
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template <typename R>
int launch_init_flat(typename Cx<R>::T *state, int n, cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    const uint64_t count = 1ull << n;
    fill_kernel<V><<<grid_for(count, kThreads * 4), kThreads, 0, stream>>>(state, count, make_cx<V>(1.0, 0.0));
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template <typename R>
int launch_init_sequential(typename Cx<R>::T *state, int n, cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    const uint64_t count = 1ull << n;
    sequential_kernel<V><<<grid_for(count, kThreads * 4), kThreads, 0, stream>>>(state, count);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template <typename R>
int launch_rescale(typename Cx<R>::T *state, int n, double target, const double *norm_dev, cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    const uint64_t count = 1ull << n;
    rescale_kernel<V><<<grid_for(count, kThreads * 4), kThreads, 0, stream>>>(state, count, target, norm_dev);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template <typename R>
int launch_set_amplitude(typename Cx<R>::T *state, uint64_t index, double re, double im, cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    set_one_kernel<V><<<1, 1, 0, stream>>>(state, index, make_cx<V>(re, im));
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template <typename R>
int launch_measure_probs(const typename Cx<R>::T *state, int n, int t, uint64_t cmask, uint64_t cval,
                         double2 *partials, double2 *result, unsigned *ticket, unsigned *done, unsigned seq,
                         cudaStream_t stream)
{
    ProbParams<R> p;
    std::memset(&p, 0, sizeof(p));
    p.state = state;
    GateOp op;
    op.nt = 1;
    op.tq[0] = t;
    op.cmask = cmask;
    p.nops = fill_masks(op, p.masks);
    p.ngroups = 1ull << (n - p.nops);
    p.cval = cval;
    p.tbit = 1ull << t;
    p.partials = partials;
    p.result = result;
    p.ticket = ticket;
    p.done = done;
    p.seq = seq;
    // A fixed grid (independent of n) keeps the partial count constant.
    measure_probs_kernel<R><<<kReduceBlocks, kThreads, 0, stream>>>(p);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template <typename R>
int launch_collapse(typename Cx<R>::T *state, int n, int t, int keep_value, cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    const uint64_t ngroups = 1ull << (n - 1);
    const uint64_t zero_bit = keep_value ? 0ull : (1ull << t);
    collapse_kernel<V><<<grid_for(ngroups, kThreads * 4), kThreads, 0, stream>>>(state, ngroups, (1ull << t) - 1, zero_bit);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template <typename R>
int launch_collapse_mask(typename Cx<R>::T *state, int n, uint64_t cmask, uint64_t cval, cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    const uint64_t count = 1ull << n;
    collapse_mask_kernel<V><<<grid_for(count, kThreads * 4), kThreads, 0, stream>>>(state, count, cmask, cval);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template <typename R>
int launch_zsums(const typename Cx<R>::T *state, int n, double *partials, double *sums, cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    const int nsums = n + 1;
    if (n < kZMinBits)
    {
        zsums_small_kernel<V><<<1, 1, 0, stream>>>(state, n, sums);
        QCSB_CUDA(cudaGetLastError());
        return 1;
    }
    // 2^gbits threads in total: at most 512 blocks of 256 threads.
    const int gbits = n < 17 ? n : 17;
    const int blocks = 1 << (gbits - 8);
    zsums_kernel<V><<<blocks, kZThreads, 0, stream>>>(state, n, gbits, partials);
    QCSB_CUDA(cudaGetLastError());
    zsums_final_kernel<<<1, 64, 0, stream>>>(partials, blocks, nsums, sums);
    QCSB_CUDA(cudaGetLastError());
    return 2;
}

template <typename R>
int launch_gather_indices(const typename Cx<R>::T *state, const uint64_t *physical, uint64_t count, double2 *out,
                          cudaStream_t stream)
{
    gather_indices_kernel<typename Cx<R>::T><<<grid_for(count, kThreads), kThreads, 0, stream>>>(state, physical, count, out);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

int launch_compare(const double2 *x, const double2 *y, uint64_t count, double *partials, cudaStream_t stream)
{
    compare_kernel<<<kReduceBlocks, kThreads, 0, stream>>>(x, y, count, partials);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template <typename R>
int launch_gather_logical(const typename Cx<R>::T *state, int n, const int *l2p, uint64_t begin,
                          uint64_t count, double2 *out, cudaStream_t stream)
{
    gather_logical_kernel<typename Cx<R>::T><<<grid_for(count, kThreads * 4), kThreads, 0, stream>>>(state, make_perm(n, l2p), begin, count, out);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template <typename R>
int launch_scatter_logical(typename Cx<R>::T *state, int n, const int *l2p, uint64_t begin,
                           uint64_t count, const double2 *in, cudaStream_t stream)
{
    scatter_logical_kernel<typename Cx<R>::T><<<grid_for(count, kThreads * 4), kThreads, 0, stream>>>(state, make_perm(n, l2p), begin, count, in);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template <typename R>
int launch_widen(const typename Cx<R>::T *in, uint64_t count, double2 *out, cudaStream_t stream)
{
    widen_kernel<typename Cx<R>::T><<<grid_for(count, kThreads * 4), kThreads, 0, stream>>>(in, count, out);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template <typename R>
int launch_narrow(const double2 *in, uint64_t count, typename Cx<R>::T *out, cudaStream_t stream)
{
    narrow_kernel<typename Cx<R>::T><<<grid_for(count, kThreads * 4), kThreads, 0, stream>>>(in, count, out);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

#define QCSB_INSTANTIATE(R)                                                                                         \
    template int launch_gate_plain<R>(Cx<R>::T *, int, const GateOp &, cudaStream_t);                               \
    template int launch_init_zero<R>(Cx<R>::T *, int, cudaStream_t);                                                \
    template int launch_init_flat<R>(Cx<R>::T *, int, cudaStream_t);                                                \
    template int launch_init_sequential<R>(Cx<R>::T *, int, cudaStream_t);                                          \
    template int launch_set_amplitude<R>(Cx<R>::T *, uint64_t, double, double, cudaStream_t);                      \
    template int launch_rescale<R>(Cx<R>::T *, int, double, const double *, cudaStream_t);                          \
    template int launch_measure_probs<R>(const Cx<R>::T *, int, int, uint64_t, uint64_t, double2 *, double2 *,      \
                                         unsigned *, unsigned *, unsigned, cudaStream_t);                           \
    template int launch_collapse<R>(Cx<R>::T *, int, int, int, cudaStream_t);                                       \
    template int launch_collapse_mask<R>(Cx<R>::T *, int, uint64_t, uint64_t, cudaStream_t);                        \
    template int launch_zsums<R>(const Cx<R>::T *, int, double *, double *, cudaStream_t);                          \
    template int launch_gather_logical<R>(const Cx<R>::T *, int, const int *, uint64_t, uint64_t, double2 *,        \
                                          cudaStream_t);                                                            \
    template int launch_scatter_logical<R>(Cx<R>::T *, int, const int *, uint64_t, uint64_t, const double2 *,       \
                                           cudaStream_t);                                                           \
    template int launch_widen<R>(const Cx<R>::T *, uint64_t, double2 *, cudaStream_t);                              \
    template int launch_narrow<R>(const double2 *, uint64_t, Cx<R>::T *, cudaStream_t);                           \
    template int launch_gather_indices<R>(const Cx<R>::T *, const uint64_t *, uint64_t, double2 *, cudaStream_t);

QCSB_INSTANTIATE(double)
QCSB_INSTANTIATE(float)

} // namespace qcsb
