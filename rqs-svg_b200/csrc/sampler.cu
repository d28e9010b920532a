// Shot sampler: draws full bitstrings from the current state without
// modifying it, with the outcome rule of measure_qubit (reference
// src/qcs.cu:2609-2626) applied qubit by qubit in measurement order.
//
// Measuring steps j = 0, 1, ..., n-1 (physical qubit order[j] at step j)
// sequentially is a walk down a binary tree: the node reached after steps
// 0..d-1 holds the squared norm of the amplitudes consistent with those
// outcomes, and step d compares P0 = child(bit = 0) with r = u * (P0 + P1).
//
// Data layout:
//   L[r], r < 2^s:  sum of |a|^2 over amplitudes whose step-0..s-1 bits equal
//                   r (one pass over the register, coalesced for the
//                   identity order since those bits are the low bits);
//   tree level d:   2^d doubles at offset 2^d, T_d[p] = T_{d+1}[p] +
//                   T_{d+1}[p + 2^d]; level s is L itself;
//   steps >= s:     per shot, the 2^(n-s) amplitudes below the chosen leaf
//                   are loaded into shared memory and reduced to a local tree.
// s = max(min(n, 20), n - 11), so the per-shot subtree is at most 2048
// doubles (its tree: 32 KB of shared memory).

#include "qcs_internal.h"

namespace qcsb
{
namespace
{

constexpr int kThreads = 256;
constexpr int kMaxLocalBits = 11;

struct OrderParams
{
    int n;
    int s;
    int order[kMaxQubits];
};

__device__ __forceinline__ uint64_t deposit_steps(uint64_t v, const OrderParams &op, int first, int count)
{
    uint64_t idx = 0;
    for (int k = 0; k < count; ++k)
        idx |= ((v >> k) & 1ull) << op.order[first + k];
    return idx;
}

template <typename V>
__global__ void __launch_bounds__(kThreads) leaf_sums_kernel(const V *state, OrderParams op, double *leaves)
{
    const uint64_t nleaves = 1ull << op.s;
    const uint64_t nh = 1ull << (op.n - op.s);
    bool identity = true;
    for (int j = 0; j < op.n; ++j)
        identity = identity && (op.order[j] == j);
    for (uint64_t r = (uint64_t)blockIdx.x * kThreads + threadIdx.x; r < nleaves; r += (uint64_t)gridDim.x * kThreads)
    {
        const uint64_t base = identity ? r : deposit_steps(r, op, 0, op.s);
        double acc = 0.0;
        for (uint64_t h = 0; h < nh; ++h)
        {
            const uint64_t idx = identity ? (base | (h << op.s)) : (base | deposit_steps(h, op, op.s, op.n - op.s));
            const V a = __ldcs(state + idx);
            const double x = a.x, y = a.y;
            acc = fma(x, x, fma(y, y, acc));
        }
        leaves[r] = acc;
    }
}

// Level d (2^d nodes at tree + 2^d) from level d + 1.
__global__ void tree_level_kernel(double *tree, int d)
{
    const uint64_t size = 1ull << d;
    const double *child = tree + 2 * size;
    double *parent = tree + size;
    for (uint64_t p = (uint64_t)blockIdx.x * kThreads + threadIdx.x; p < size; p += (uint64_t)gridDim.x * kThreads)
        parent[p] = child[p] + child[p + size];
}

template <typename V>
__global__ void __launch_bounds__(kThreads) shots_kernel(const V *state, OrderParams op, const double *tree,
                                                         uint32_t num_shots, const double *uniforms, uint64_t *out_bits)
{
    __shared__ double local[2 << kMaxLocalBits];
    __shared__ uint64_t leaf_sh;
    const int m_bits = op.n - op.s;
    const int m = 1 << m_bits;
    for (uint32_t shot = blockIdx.x; shot < num_shots; shot += gridDim.x)
    {
        const double *u = uniforms + (size_t)shot * op.n;
        if (threadIdx.x == 0)
        {
            uint64_t p = 0;
            for (int d = 0; d < op.s; ++d)
            {
                const double *child = tree + (2ull << d);
                const double p0 = child[p];
                const double p1 = child[p | (1ull << d)];
                const double r = u[d] * (p0 + p1);
                if (p0 < r)
                    p |= 1ull << d;
            }
            leaf_sh = p;
        }
        __syncthreads();
        const uint64_t p = leaf_sh;
        uint64_t bits = p;
        if (m_bits > 0)
        {
            bool identity = true;
            for (int j = 0; j < op.n; ++j)
                identity = identity && (op.order[j] == j);
            const uint64_t base = identity ? p : deposit_steps(p, op, 0, op.s);
            // leaves of the local tree at offset m
            for (int h = threadIdx.x; h < m; h += kThreads)
            {
                const uint64_t idx = identity ? (base | ((uint64_t)h << op.s))
                                              : (base | deposit_steps((uint64_t)h, op, op.s, m_bits));
                const V a = state[idx];
                const double x = a.x, y = a.y;
                local[m + h] = fma(x, x, y * y);
            }
            __syncthreads();
            for (int e = m_bits - 1; e >= 0; --e)
            {
                const int size = 1 << e;
                for (int q = threadIdx.x; q < size; q += kThreads)
                    local[size + q] = local[2 * size + q] + local[2 * size + q + size];
                __syncthreads();
            }
            if (threadIdx.x == 0)
            {
                uint64_t q = 0;
                for (int e = 0; e < m_bits; ++e)
                {
                    const double *child = local + (2 << e);
                    const double p0 = child[q];
                    const double p1 = child[q | (1ull << e)];
                    const double r = u[op.s + e] * (p0 + p1);
                    if (p0 < r)
                        q |= 1ull << e;
                }
                bits |= q << op.s;
            }
        }
        if (threadIdx.x == 0)
            out_bits[shot] = bits;
        __syncthreads();
    }
}

int split_for(int n)
{
    int s = n < 20 ? n : 20;
    if (n - s > kMaxLocalBits)
        s = n - kMaxLocalBits;
    return s;
}

} // namespace

size_t sampler_tree_bytes(int n, int *split_out)
{
    const int s = split_for(n);
    if (split_out)
        *split_out = s;
    return sizeof(double) * (2ull << s);
}

template <typename R>
int launch_sampler(const typename Cx<R>::T *state, int n, const int *order, uint32_t num_shots,
                   const double *uniforms, uint64_t *out_bits, double *tree, int split,
                   cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    OrderParams op;
    op.n = n;
    op.s = split;
    for (int j = 0; j < n; ++j)
        op.order[j] = order[j];
    int launches = 0;
    const uint64_t nleaves = 1ull << split;
    unsigned grid = static_cast<unsigned>((nleaves + kThreads - 1) / kThreads);
    if (grid > 148 * 16)
        grid = 148 * 16;
    leaf_sums_kernel<V><<<grid, kThreads, 0, stream>>>(state, op, tree + nleaves);
    QCSB_CUDA(cudaGetLastError());
    ++launches;
    for (int d = split - 1; d >= 0; --d)
    {
        const uint64_t size = 1ull << d;
        unsigned g = static_cast<unsigned>((size + kThreads - 1) / kThreads);
        if (g > 148 * 16)
            g = 148 * 16;
        tree_level_kernel<<<g, kThreads, 0, stream>>>(tree, d);
        QCSB_CUDA(cudaGetLastError());
        ++launches;
    }
    if (num_shots > 0)
    {
        unsigned g = num_shots < 148u * 8u ? num_shots : 148u * 8u;
        shots_kernel<V><<<g, kThreads, 0, stream>>>(state, op, tree, num_shots, uniforms, out_bits);
        QCSB_CUDA(cudaGetLastError());
        ++launches;
    }
    return launches;
}

template int launch_sampler<double>(const double2 *, int, const int *, uint32_t, const double *, uint64_t *, double *,
                                    int, cudaStream_t);
template int launch_sampler<float>(const float2 *, int, const int *, uint32_t, const double *, uint64_t *, double *,
                                   int, cudaStream_t);

} // namespace qcsb
