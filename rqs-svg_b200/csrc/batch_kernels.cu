// <Z> of every register of a batch in one pass over the arena, and the
// |0..0> preparation of registers that no fused pass initialises.
//
// Work item = a slice of up to 2^16 amplitudes of one register; one CTA of
// 256 threads per item. Thread t reads amplitudes t + 256 j: bits 0..7 of the
// index are t's bits (constant per thread), bits 8.. come from j (at most 8
// bits), bits above the slice from the item. So a thread only needs its total
// and one sum per loop bit; the thread-bit sums and the slice-bit sums follow
// from the totals. Everything accumulates in FP64.

#include "batch.h"

namespace qcsb
{
namespace
{

constexpr int kZThreads = 256;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// partials[item * kBatchZPartials + ...] = total, sums over bits 0..7 (thread
// bits), sums over bits 8..15 (loop bits) of this slice
template <typename V>
__global__ void __launch_bounds__(kZThreads) batch_zsums_kernel(const V *arena, const BatchZItem *items,
                                                                double *partials)
{
    const BatchZItem it = items[blockIdx.x];
    const int sb = it.n < kBatchZSliceBits ? it.n : kBatchZSliceBits;
    const int jbits = sb - 8;
    const V *base = arena + it.amp_off + ((uint64_t)it.slice << sb);
    const int t = threadIdx.x;
    double tot = 0.0, hi[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int nj = 1 << jbits;
    for (int j = 0; j < nj; ++j)
    {
        const V a = __ldcs(base + t + (j << 8));
        const double p = (double)a.x * (double)a.x + (double)a.y * (double)a.y;
        tot += p;
#pragma unroll
        for (int b = 0; b < 8; ++b)
            if (b < jbits && ((j >> b) & 1))
                hi[b] += p;
    }
    double v[kBatchZPartials];
    v[0] = tot;
#pragma unroll
    for (int b = 0; b < 8; ++b)
        v[1 + b] = ((t >> b) & 1) ? tot : 0.0;
#pragma unroll
    for (int b = 0; b < 8; ++b)
        v[9 + b] = hi[b];
    __shared__ double sh[kBatchZPartials][kZThreads / 32];
    const int w = t / 32, l = t % 32;
#pragma unroll
    for (int i = 0; i < kBatchZPartials; ++i)
    {
        const double s = warp_sum(v[i]);
        if (l == 0)
            sh[i][w] = s;
    }
    __syncthreads();
    if (t < kBatchZPartials)
    {
        double s = 0.0;
        for (int k = 0; k < kZThreads / 32; ++k)
            s += sh[t][k];
        partials[(uint64_t)blockIdx.x * kBatchZPartials + t] = s;
    }
}

// One thread per register: <Z_q> = (total - 2 sum_q) / total.
__global__ void batch_zfinal_kernel(const double *partials, const BatchZItem *items, const BatchZReg *regs,
                                    uint32_t num_regs, double *out)
{
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= num_regs)
        return;
    const BatchZReg g = regs[r];
    const int n = g.n;
    const int sb = n < kBatchZSliceBits ? n : kBatchZSliceBits;
    double tot = 0.0, s[kMaxQubits];
    for (int q = 0; q < n; ++q)
        s[q] = 0.0;
    for (uint32_t i = 0; i < g.count; ++i)
    {
        const double *p = partials + (uint64_t)(g.first + i) * kBatchZPartials;
        const uint32_t slice = items[g.first + i].slice;
        tot += p[0];
        for (int q = 0; q < 8 && q < n; ++q)
            s[q] += p[1 + q];
        for (int q = 8; q < sb; ++q)
            s[q] += p[9 + (q - 8)];
        for (int q = sb; q < n; ++q)
            if ((slice >> (q - sb)) & 1)
                s[q] += p[0];
    }
    for (int q = 0; q < n; ++q)
        out[g.out_off + q] = tot > 0.0 ? (tot - 2.0 * s[q]) / tot : 0.0;
}

template <typename V>
__global__ void batch_set_ones_kernel(V *base, uint64_t stride, uint32_t count)
{
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < count)
    {
        V one;
        one.x = 1;
        one.y = 0;
        base[(uint64_t)r * stride] = one;
    }
}

} // namespace

template <typename R>
int launch_batch_zsums(const void *arena, const BatchZItem *items, uint32_t num_items, const BatchZReg *regs,
                       uint32_t num_regs, double *partials, double *out, cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    if (num_items == 0)
        return 0;
    batch_zsums_kernel<V><<<num_items, kZThreads, 0, stream>>>(static_cast<const V *>(arena), items, partials);
    QCSB_CUDA(cudaGetLastError());
    batch_zfinal_kernel<<<(num_regs + 127) / 128, 128, 0, stream>>>(partials, items, regs, num_regs, out);
    QCSB_CUDA(cudaGetLastError());
    return 2;
}

template <typename R>
int launch_batch_set_ones(void *base, uint64_t stride, uint32_t count, cudaStream_t stream)
{
    typedef typename Cx<R>::T V;
    if (count == 0)
        return 0;
    batch_set_ones_kernel<V><<<(count + 127) / 128, 128, 0, stream>>>(static_cast<V *>(base), stride, count);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

template int launch_batch_zsums<double>(const void *, const BatchZItem *, uint32_t, const BatchZReg *, uint32_t,
                                        double *, double *, cudaStream_t);
template int launch_batch_zsums<float>(const void *, const BatchZItem *, uint32_t, const BatchZReg *, uint32_t,
                                       double *, double *, cudaStream_t);
template int launch_batch_set_ones<double>(void *, uint64_t, uint32_t, cudaStream_t);
template int launch_batch_set_ones<float>(void *, uint64_t, uint32_t, cudaStream_t);

} // namespace qcsb
