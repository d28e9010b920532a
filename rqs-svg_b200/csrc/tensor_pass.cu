// Tensor passes: the stages of a fused pass as dense 16 x 16 complex
// matrices on the tensor cores (mma.sync m16n8k8): FP64 (DMMA) for
// complex128 registers, TF32 with a three-term split and FP32 accumulation
// for complex64 registers.
//
// A fused pass (fused_pass.cu) stages a 2^11-amplitude chunk in shared memory
// and runs its gates in stages of 4 local "stage bits". On the register path
// every thread applies the stage's gates one by one to the 16 amplitudes that
// differ in those bits. A tensor pass instead applies the stage's whole
// product as one 16 x 16 matrix M to every 16-amplitude group of the chunk.
// Gates of the stage that depend on bits outside it (controls, diagonal
// targets) make M depend on those bits; the stage then has one matrix per
// assignment of its condition bits (at most 2^8), all built on the GPU in
// FP64 from the pass's ops before the pass (stage_matrix_kernel).
//
// Product layout. A warp takes 16 groups (rows r) at a time: y_r = M x_r for
// all 16 rows, with M = Mr + i Mi, in three real products (a three-
// multiplication form of the complex product): K1 = Mr (Re x + Im x), then
// Re y = K1 + B2 Im x and Im y = K1 + B1 Re x with B1 = Mi - Mr and
// B2 = -(Mr + Mi) (the builder stores B0 = Mr, B1 and B2), the last two
// accumulated onto a copy of K1 by the tensor cores, so no addition follows
// the products: twelve m16n8k8 products per 16 rows (K = 16 input slots in
// two k-steps, N = 16 output slots in two n-tiles) instead of the sixteen of
// the four-product form. Lane (g, t) of
// the warp (g = lane / 4, t = lane % 4) holds rows g and g + 8 at input
// slots t, t + 4, t + 8, t + 12 for the A fragments; output column
// nu = 8i + 2t + e of n-tile i stands for output slot 8i + t + 4e, so the
// accumulators give the lane the same four slots of the same rows: it loads
// and stores the same 8 shared-memory positions, and the stage runs in place
// without barriers between the warp's tiles.
//
// complex128: 48 FP64 multiply-adds per amplitude and stage on the tensor
// pipe plus one addition (Re x + Im x) (the register path: 8 multiply-adds per complex 2x2
// gate), at the FP64 tensor rate, which on B200 equals the FMA rate, but
// with one instruction per 1024 multiply-adds instead of 32.
//
// complex64: every operand is split into a TF32 high part and a TF32 low
// part (the matrices rounded to nearest when they are built, the data by
// masking: within 2^-21 relative); each product is a_lo b_hi + a_hi b_lo +
// a_hi b_hi (the lo x lo term, ~2^-21 relative, is dropped) accumulated in
// FP32, at the TF32 tensor rate (7.3x the FP64 rate on B200).

#include "fused_pass.h"

#include <algorithm>
#include <cstring>

namespace qcsb
{
namespace
{

constexpr int kThreads = 1 << (kTensorLocal - kStageBits);   // 128: 4 warps, two 16-group tiles each
// chunk buffers of a tensor pass's CTA: 2 (double-buffered: the next chunk
// streams in during this one's stages; three CTAs per SM) or 1 (more CTAs
// per SM instead: four for 16 x 16 stages at 128 registers, measured 5.5-5.8%
// faster on the 30-qubit circuits; six or eight for 8 x 8 stages, below)
constexpr int kTensor3Buffers = 1;
constexpr int kTensor4Buffers = 1;
constexpr int kSlots = 1 << kStageBits;
constexpr int kChunk = 1 << kTensorLocal;

// Shared-memory swizzles (linear over GF(2)): 16-byte amplitudes fold 3
// index bits into the 3 bits that pick a 16-byte bank group, 8-byte
// amplitudes fold 4.
__host__ __device__ __forceinline__ int swz16(int j) { return j ^ (((j >> 3) ^ (j >> 6) ^ (j >> 9)) & 7); }
__host__ __device__ __forceinline__ int swz8(int j) { return j ^ (((j >> 4) ^ (j >> 8)) & 15); }

template <typename Real>
struct Tensor;

template <>
struct Tensor<double>
{
    typedef double2 V;
    typedef double2 Frag;   // (b0, b1)
    static __device__ __forceinline__ int swz(int j) { return swz16(j); }
    static __device__ __forceinline__ void cp_async(V *smem, const V *gmem)
    {
        const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
    }
    // A fragment: a0 = A[g][t], a1 = A[g + 8][t], a2 = A[g][t + 4],
    // a3 = A[g + 8][t + 4]
    struct AFrag
    {
        double a0, a1, a2, a3;
    };
    static __device__ __forceinline__ AFrag afrag(double a0, double a1, double a2, double a3)
    {
        return AFrag{a0, a1, a2, a3};
    }
    // D += A B, m16n8k8 FP64: b0 = B[t][g], b1 = B[t + 4][g]; d0 = D[g][2t],
    // d1 = D[g][2t + 1], d2 = D[g + 8][2t], d3 = D[g + 8][2t + 1]
    static __device__ __forceinline__ void mma(double (&d)[4], const AFrag &a, const Frag &b)
    {
        asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
            : "d"(a.a0), "d"(a.a1), "d"(a.a2), "d"(a.a3), "d"(b.x), "d"(b.y));
    }
};

template <>
struct Tensor<float>
{
    typedef float2 V;
    typedef uint4 Frag;   // TF32 (hi b0, hi b1, lo b0, lo b1)
    static __device__ __forceinline__ int swz(int j) { return swz8(j); }
    static __device__ __forceinline__ void cp_async(V *smem, const V *gmem)
    {
        const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
    }
    static __device__ __forceinline__ void tf32mma(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                                   uint32_t b0, uint32_t b1)
    {
        asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
    }
    // A fragment (layout as for FP64) split into TF32 high and low parts,
    // once per tile: both n-tiles use it
    struct AFrag
    {
        uint32_t h0, h1, h2, h3, l0, l1, l2, l3;
    };
    // high part: x's top 10 mantissa bits (masked); low part: the next 11
    // significant bits of the exact remainder (|x - hi - lo| <= 2^-21 |x|);
    // two integer ops and one subtraction per value
    static __device__ __forceinline__ void split(float x, uint32_t &h, uint32_t &l)
    {
        h = __float_as_uint(x) & 0xFFFFE000u;
        l = __float_as_uint(x - __uint_as_float(h)) & 0xFFFFE000u;
    }
    static __device__ __forceinline__ AFrag afrag(float a0, float a1, float a2, float a3)
    {
        AFrag f;
        split(a0, f.h0, f.l0);
        split(a1, f.h1, f.l1);
        split(a2, f.h2, f.l2);
        split(a3, f.h3, f.l3);
        return f;
    }
    // D += A B with A and B split into TF32 high and low parts; the small
    // terms go first
    static __device__ __forceinline__ void mma(float (&d)[4], const AFrag &a, const Frag &b)
    {
        tf32mma(d, a.l0, a.l1, a.l2, a.l3, b.x, b.y);
        tf32mma(d, a.h0, a.h1, a.h2, a.h3, b.z, b.w);
        tf32mma(d, a.h0, a.h1, a.h2, a.h3, b.x, b.y);
    }
};

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// CTAs per SM of the single-buffered 16 x 16 pass
template <typename Real>
constexpr int tensor_ctas_per_sm() { return sizeof(Real) == 8 ? 5 : 5; }

template <typename Real, int NBUF>
__global__ void __launch_bounds__(kThreads, NBUF == 1 ? tensor_ctas_per_sm<Real>() : 3) tensor_pass_kernel(const __grid_constant__ TPassParams p)
{
    typedef Tensor<Real> TT;
    typedef typename TT::V V;
    typedef typename TT::Frag Frag;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *smem = reinterpret_cast<V *>(smem_raw);
    V *const state = static_cast<V *>(p.state);
    const Frag *const mats = reinterpret_cast<const Frag *>(p.mats);
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;

    // chunk staging: element tid + m * kThreads of the chunk, m < 16, is the
    // amplitude at local index tid + m * 128 (its bits deposited at the
    // pass's local qubits)
    uint64_t dep_tid = 0;
    for (int i = 0; i < kTensorLocal - kStageBits; ++i)
        if ((tid >> i) & 1)
            dep_tid |= p.qbit[i];
    uint64_t hb[kStageBits];
#pragma unroll
    for (int b = 0; b < kStageBits; ++b)
        hb[b] = p.qbit[kTensorLocal - kStageBits + b];
    auto chunk_base = [&](uint64_t c) -> uint64_t {
        uint64_t x = c;
        for (int i = 0; i < kTensorLocal; ++i)
        {
            const uint64_t lo = x & p.qmasks[i];
            x = lo | ((x ^ lo) << 1);
        }
        return x;
    };
    auto elem_offset = [&](int m) -> uint64_t {
        uint64_t off = dep_tid;
#pragma unroll
        for (int b = 0; b < kStageBits; ++b)
            if ((m >> b) & 1)
                off |= hb[b];
        return off;
    };
    auto issue_load = [&](uint64_t cb, V *dst) {
        if (p.from_zero)
        {
#pragma unroll
            for (int m = 0; m < kSlots; ++m)
            {
                const bool one = cb == 0 && m == 0 && tid == 0;
                dst[TT::swz(tid + m * kThreads)] = V{one ? Real(1) : Real(0), Real(0)};
            }
        }
        else
        {
#pragma unroll
            for (int m = 0; m < kSlots; ++m)
                TT::cp_async(dst + TT::swz(tid + m * kThreads), state + (cb | elem_offset(m)));
        }
        cp_commit();
    };

    // B fragments of one stage matrix: (Mr, Mi, Mr + Mi) x k-step j x
    // n-tile i, read right before each product (from L1: every tile of a
    // stage with the same condition bits reads the same 6 KiB); holding all
    // 12 in registers would cost 48 registers and two CTAs per SM
    auto matrix_of = [&](int st, uint64_t cb, int mt) -> uint32_t {
        const TStage &S = p.stages[st];
        uint32_t vc = 0;
        for (int i = 0; i < S.ngc; ++i)
            vc |= static_cast<uint32_t>((cb >> S.gq[i]) & 1) << i;
        const uint32_t tile = static_cast<uint32_t>(warp | (mt << 2));
        return (tile & ((1u << S.nlc) - 1u)) | (vc << S.nlc);
    };

    uint64_t c = blockIdx.x;
    if (c >= p.chunks)
        return;
    uint64_t cbase_next = chunk_base(c);
    issue_load(cbase_next, smem);
    int cur = 0;
    for (; c < p.chunks; c += gridDim.x)
    {
        // NBUF as in tensor3_pass_kernel
        V *sb = smem + (NBUF == 2 ? cur * kChunk : 0);
        const uint64_t cbase = cbase_next;
        const uint64_t next = c + gridDim.x;
        if (next < p.chunks)
            cbase_next = chunk_base(next);
        if (NBUF == 2 && next < p.chunks)
        {
            issue_load(cbase_next, smem + (cur ^ 1) * kChunk);
            cp_wait<1>();
        }
        else
        {
            cp_wait<0>();
        }
        __syncthreads();

        for (int st = 0; st < p.nstages; ++st)
        {
            const TStage &S = p.stages[st];
            // swizzled offsets of the group and slot bits (the swizzle is
            // linear over GF(2): positions combine by XOR)
            const uint16_t *sw = p.swz[st];
            uint32_t gbit[7], sbit[kStageBits];
#pragma unroll
            for (int i = 0; i < 7; ++i)
                gbit[i] = sw[i];
#pragma unroll
            for (int b = 0; b < kStageBits; ++b)
                sbit[b] = sw[7 + b];
            const uint32_t lane_pos = ((g & 1) ? gbit[0] : 0u) ^ ((g & 2) ? gbit[1] : 0u) ^
                                      ((g & 4) ? gbit[2] : 0u) ^ ((t & 1) ? sbit[0] : 0u) ^ ((t & 2) ? sbit[1] : 0u);
            const uint32_t hpos = gbit[3];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
            {
                const uint32_t tile = static_cast<uint32_t>(warp | (mt << 2));
                const uint32_t v = matrix_of(st, cbase, mt);
                const Frag *w = mats + (static_cast<size_t>(S.woff + v) * kTensorFragments) * 32 + lane;
                const uint32_t base = lane_pos ^ ((tile & 1) ? gbit[4] : 0u) ^ ((tile & 2) ? gbit[5] : 0u) ^
                                      ((tile & 4) ? gbit[6] : 0u);
                auto pos = [&](int h, int m) {
                    return base ^ (h ? hpos : 0u) ^ ((m & 1) ? sbit[2] : 0u) ^ ((m & 2) ? sbit[3] : 0u);
                };
                // x[h][m]: row g + 8h, input slot t + 4m; A fragments of the
                // real parts, the imaginary parts and their sums per k-step j
                typename TT::AFrag ar[2], ai[2], as[2];
#pragma unroll
                for (int j = 0; j < 2; ++j)
                {
                    const V x00 = sb[pos(0, 2 * j)], x10 = sb[pos(1, 2 * j)];
                    const V x01 = sb[pos(0, 2 * j + 1)], x11 = sb[pos(1, 2 * j + 1)];
                    ar[j] = TT::afrag(x00.x, x10.x, x01.x, x11.x);
                    ai[j] = TT::afrag(x00.y, x10.y, x01.y, x11.y);
                    as[j] = TT::afrag(x00.x + x00.y, x10.x + x10.y, x01.x + x01.y, x11.x + x11.y);
                }
#pragma unroll
                for (int i = 0; i < 2; ++i)
                {
                    // K1 = B0 (Re x + Im x); Re y = K1 + B2 Im x; Im y = K1 + B1 Re x
                    Real k1[4] = {0, 0, 0, 0};
#pragma unroll
                    for (int j = 0; j < 2; ++j)
                        TT::mma(k1, as[j], __ldg(w + (0 * 4 + j * 2 + i) * 32));
                    Real yr[4] = {k1[0], k1[1], k1[2], k1[3]}, yi[4] = {k1[0], k1[1], k1[2], k1[3]};
#pragma unroll
                    for (int j = 0; j < 2; ++j)
                    {
                        TT::mma(yr, ai[j], __ldg(w + (2 * 4 + j * 2 + i) * 32));
                        TT::mma(yi, ar[j], __ldg(w + (1 * 4 + j * 2 + i) * 32));
                    }
                    // e = 0: row g, slot t + 8i; 1: row g, slot t + 8i + 4; 2, 3: row g + 8
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        sb[pos(e >> 1, 2 * i + (e & 1))] = V{yr[e], yi[e]};
                }
            }
            __syncthreads();
        }

#pragma unroll
        for (int m = 0; m < kSlots; ++m)
            __stcs(state + (cbase | elem_offset(m)), sb[TT::swz(tid + m * kThreads)]);
        __syncthreads();
        if (NBUF == 1 && next < p.chunks)
            issue_load(cbase_next, smem);
        cur ^= 1;
    }
}

// 8 x 8 stages (three slot bits; TPassParams::width 3). A warp takes 16
// rows (8-amplitude groups) at a time: lane (g, t) holds rows g and g + 8 at
// input slots t and t + 4 (one k-step), and output column nu = 2t + e of the
// single n-tile stands for output slot t + 4e, so the lane stores to the
// positions it loaded. Three m16n8k8 products per 16 rows (as above):
// 24 multiply-adds per amplitude and stage, half those of a 16 x 16 stage
// for three quarters of its qubits. 256 rows per chunk: 16 tiles, four per
// warp; group bits 4..7 pick the tile, warp + 4 x the warp's tile index (the
// stage's local condition bits are the lowest group bits, so with at most
// two of them a warp runs all its tiles with one matrix, fetched before the
// stage begins).
// CTAs per SM of the single-buffered 8 x 8 pass: six for complex128 (80
// registers; 6 x 32 KiB of chunk), eight for complex64 (64 registers); each
// step from four measured faster (30-qubit layered and matching complex128:
// 0.6998 -> 0.6725 -> 0.6551 s and 1.2803 -> 1.2310 -> 1.1979 s at 4, 5, 6)
template <typename Real>
constexpr int tensor3_ctas_per_sm() { return sizeof(Real) == 8 ? 6 : 8; }

template <typename Real, int NBUF>
__global__ void __launch_bounds__(kThreads, NBUF == 1 ? tensor3_ctas_per_sm<Real>() : 3)
    tensor3_pass_kernel(const __grid_constant__ TPassParams p)
{
    typedef Tensor<Real> TT;
    typedef typename TT::V V;
    typedef typename TT::Frag Frag;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *smem = reinterpret_cast<V *>(smem_raw);
    V *const state = static_cast<V *>(p.state);
    const Frag *const mats = reinterpret_cast<const Frag *>(p.mats);
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;

    uint64_t dep_tid = 0;
    for (int i = 0; i < kTensorLocal - kStageBits; ++i)
        if ((tid >> i) & 1)
            dep_tid |= p.qbit[i];
    uint64_t hb[kStageBits];
#pragma unroll
    for (int b = 0; b < kStageBits; ++b)
        hb[b] = p.qbit[kTensorLocal - kStageBits + b];
    // batched passes: the register's amplitudes start at register << n (the
    // bits above n of the base; matrix choices read bits below n only)
    auto chunk_base = [&](uint64_t c) -> uint64_t {
        uint64_t x = p.reg_mats > 0 ? (c & ((1ull << p.batch_cbits) - 1)) : c;
        for (int i = 0; i < kTensorLocal; ++i)
        {
            const uint64_t lo = x & p.qmasks[i];
            x = lo | ((x ^ lo) << 1);
        }
        if (p.reg_mats > 0)
            x |= (c >> p.batch_cbits) << p.n;
        return x;
    };
    auto elem_offset = [&](int m) -> uint64_t {
        uint64_t off = dep_tid;
#pragma unroll
        for (int b = 0; b < kStageBits; ++b)
            if ((m >> b) & 1)
                off |= hb[b];
        return off;
    };
    auto issue_load = [&](uint64_t cb, V *dst) {
        if (p.from_zero)
        {
#pragma unroll
            for (int m = 0; m < kSlots; ++m)
            {
                const bool one = (cb & ((1ull << p.n) - 1)) == 0 && m == 0 && tid == 0;
                dst[TT::swz(tid + m * kThreads)] = V{one ? Real(1) : Real(0), Real(0)};
            }
        }
        else
        {
#pragma unroll
            for (int m = 0; m < kSlots; ++m)
                TT::cp_async(dst + TT::swz(tid + m * kThreads), state + (cb | elem_offset(m)));
        }
        cp_commit();
    };

    Frag bf[kTensor3Fragments];
    int bf_st = -1;
    uint32_t bf_v = 0;
    uint64_t bf_reg = 0;   // register whose matrices bf holds (batched passes)
    auto matrix_of = [&](int st, uint64_t cb, int mt) -> uint32_t {
        const TStage &S = p.stages[st];
        uint32_t vc = 0;
        for (int i = 0; i < S.ngc; ++i)
            vc |= static_cast<uint32_t>((cb >> S.gq[i]) & 1) << i;
        const uint32_t tile = static_cast<uint32_t>(warp | (mt << 2));
        return (tile & ((1u << S.nlc) - 1u)) | (vc << S.nlc);
    };
    auto fetch = [&](int st, uint32_t v, uint64_t cb) {
        const uint64_t reg = cb >> p.n;
        const Frag *w =
            mats + (static_cast<size_t>(reg * p.reg_mats + p.stages[st].woff + v) * kTensor3Fragments) * 32 + lane;
#pragma unroll
        for (int f = 0; f < kTensor3Fragments; ++f)
            bf[f] = __ldg(w + f * 32);
        bf_st = st;
        bf_v = v;
        bf_reg = reg;
    };

    uint64_t c = blockIdx.x;
    if (c >= p.chunks)
        return;
    uint64_t cbase_next = chunk_base(c);
    issue_load(cbase_next, smem);
    if (p.nstages > 0)
        fetch(0, matrix_of(0, cbase_next, 0), cbase_next);
    int cur = 0;
    for (; c < p.chunks; c += gridDim.x)
    {
        // NBUF 2: the next chunk streams in while this one is processed;
        // NBUF 1: one buffer, loaded after the last one's stores (more CTAs
        // per SM instead)
        V *sb = smem + (NBUF == 2 ? cur * kChunk : 0);
        const uint64_t cbase = cbase_next;
        const uint64_t next = c + gridDim.x;
        if (next < p.chunks)
            cbase_next = chunk_base(next);
        if (NBUF == 2 && next < p.chunks)
        {
            issue_load(cbase_next, smem + (cur ^ 1) * kChunk);
            cp_wait<1>();
        }
        else
        {
            cp_wait<0>();
        }
        __syncthreads();

        for (int st = 0; st < p.nstages; ++st)
        {
            const uint16_t *sw = p.swz[st];
            uint32_t gbit[8], sbit[3];
#pragma unroll
            for (int i = 0; i < 8; ++i)
                gbit[i] = sw[i];
#pragma unroll
            for (int b = 0; b < 3; ++b)
                sbit[b] = sw[8 + b];
            const uint32_t lane_pos = ((g & 1) ? gbit[0] : 0u) ^ ((g & 2) ? gbit[1] : 0u) ^
                                      ((g & 4) ? gbit[2] : 0u) ^ ((t & 1) ? sbit[0] : 0u) ^ ((t & 2) ? sbit[1] : 0u);
            const uint32_t hpos = gbit[3];
            // the stage's matrix of tile mt: local condition bits from the
            // tile, chunk condition bits from the chunk (once per stage)
            const TStage &S = p.stages[st];
            uint32_t vc = 0;
            for (int i = 0; i < S.ngc; ++i)
                vc |= static_cast<uint32_t>((cbase >> S.gq[i]) & 1) << i;
            const uint32_t vlo = (1u << S.nlc) - 1u, vhi = vc << S.nlc;
            const uint64_t creg = cbase >> p.n;
#pragma unroll
            for (int mt = 0; mt < 4; ++mt)
            {
                const uint32_t tile = static_cast<uint32_t>(warp | (mt << 2));
                const uint32_t v = (tile & vlo) | vhi;
                if (bf_st != st || bf_v != v || bf_reg != creg)
                    fetch(st, v, cbase);
                const uint32_t base = lane_pos ^ ((tile & 1) ? gbit[4] : 0u) ^ ((tile & 2) ? gbit[5] : 0u) ^
                                      ((tile & 4) ? gbit[6] : 0u) ^ ((tile & 8) ? gbit[7] : 0u);
                auto pos = [&](int h, int m) { return base ^ (h ? hpos : 0u) ^ (m ? sbit[2] : 0u); };
                const V x00 = sb[pos(0, 0)], x10 = sb[pos(1, 0)], x01 = sb[pos(0, 1)], x11 = sb[pos(1, 1)];
                const typename TT::AFrag ar = TT::afrag(x00.x, x10.x, x01.x, x11.x);
                const typename TT::AFrag ai = TT::afrag(x00.y, x10.y, x01.y, x11.y);
                const typename TT::AFrag as =
                    TT::afrag(x00.x + x00.y, x10.x + x10.y, x01.x + x01.y, x11.x + x11.y);
                // K1 = B0 (Re x + Im x); Re y = K1 + B2 Im x; Im y = K1 + B1 Re x
                Real k1[4] = {0, 0, 0, 0};
                TT::mma(k1, as, bf[0]);
                Real yr[4] = {k1[0], k1[1], k1[2], k1[3]}, yi[4] = {k1[0], k1[1], k1[2], k1[3]};
                TT::mma(yr, ai, bf[2]);
                TT::mma(yi, ar, bf[1]);
                // e = 0: row g, slot t; 1: row g, slot t + 4; 2, 3: row g + 8
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    sb[pos(e >> 1, e & 1)] = V{yr[e], yi[e]};
            }
            if (st + 1 < p.nstages)
                fetch(st + 1, matrix_of(st + 1, cbase, 0), cbase);
            else if (next < p.chunks)
                fetch(0, matrix_of(0, cbase_next, 0), cbase_next);
            __syncthreads();
        }

#pragma unroll
        for (int m = 0; m < kSlots; ++m)
            __stcs(state + (cbase | elem_offset(m)), sb[TT::swz(tid + m * kThreads)]);
        __syncthreads();
        if (NBUF == 1 && next < p.chunks)
            issue_load(cbase_next, smem);
        cur ^= 1;
    }
}

} // namespace

bool make_tensor_params(const FPassParams &prm, const std::vector<StageCond> &conds, int amp_bytes, TPassParams &tp,
                        TBuildParams &tb, int width, bool umma)
{
    if (prm.k != kTensorLocal || static_cast<int>(conds.size()) != prm.nstages || prm.nstages <= 0)
        return false;
    if (width != 3 && width != kStageBits)
        return false;
    if (umma && (amp_bytes != 8 || width != kStageBits))
        return false;
    std::memset(&tp, 0, sizeof(tp));
    std::memset(&tb, 0, sizeof(tb));
    tp.n = prm.n;
    tp.from_zero = prm.from_zero;
    tp.chunks = prm.chunks;
    tp.width = width;
    std::memcpy(tp.qmasks, prm.qmasks, sizeof(tp.qmasks));
    std::memcpy(tp.qbit, prm.qbit, sizeof(tp.qbit));
    tp.nstages = prm.nstages;
    // A quarter warp's (16-byte amplitudes) or half warp's (8-byte) loads go
    // to distinct bank groups when the lane bits of a stage (slot bits 0 and
    // 1, group bit 0, and for 8-byte amplitudes group bit 1) sit on local
    // positions of distinct residues mod 3 (mod 4): the swizzle sends
    // position l to bank-group bit l mod 3 (mod 4).
    // A tcgen05 pass's rows are threads: a half warp (16 rows, one slot each
    // per load) meets distinct bank pairs when group bits 0-3 (thread bits
    // 0-3) sit on positions of distinct residues mod 4; the slot bits are
    // free.
    const bool c64 = amp_bytes == 8;
    const int mod = c64 ? 4 : 3;
    const int row_bank_bits = umma ? 4 : c64 ? 2 : 1;
    const int tile_bits = umma ? kUmmaMaxLocalCond : width == 3 ? kTensor3TileBits : kTensorTileBits;
    const int ngroup = kTensorLocal - width;   // 7 (4 rows + 3 tile bits) or 8 (4 + 4)
    uint32_t woff = 0;
    for (int s = 0; s < prm.nstages; ++s)
    {
        const FStage &FS = prm.stages[s];
        const StageCond &cond = conds[s];
        // register slots (0..3) that become tensor slots: all four, or for
        // 8 x 8 stages the ones dense ops target, then untouched ones; the
        // remaining register bit (pad) is a group bit of the tensor layout,
        // and a condition bit when an op's pattern involves it
        int slots[kStageBits], nslots = 0, padslot = -1;
        auto taken = [&](int b) {
            for (int i = 0; i < nslots; ++i)
                if (slots[i] == b)
                    return true;
            return false;
        };
        if (width == kStageBits)
        {
            for (int b = 0; b < kStageBits; ++b)
                slots[nslots++] = b;
        }
        else
        {
            if (__builtin_popcount(cond.dense) > width)
                return false;
            for (int b = 0; b < kStageBits; ++b)
                if ((cond.dense >> FS.sbits[b]) & 1)
                    slots[nslots++] = b;
            for (int b = 0; b < kStageBits && nslots < width; ++b)
                if (!taken(b) && !((cond.touch >> FS.sbits[b]) & 1))
                    slots[nslots++] = b;
            for (int b = 0; b < kStageBits && nslots < width; ++b)
                if (!taken(b))
                    slots[nslots++] = b;
            for (int b = 0; b < kStageBits; ++b)
                if (!taken(b))
                    padslot = b;
        }
        const bool pad_cond = padslot >= 0 && ((cond.touch >> FS.sbits[padslot]) & 1);
        const int nlc = __builtin_popcount(cond.lmask) + (pad_cond ? 1 : 0);
        const int ngc = __builtin_popcountll(cond.gmask);
        if (nlc > tile_bits || nlc + ngc > kTensorMaxCond)
            return false;
        const uint32_t nm = 1u << (nlc + ngc);
        if (woff + nm > static_cast<uint32_t>(kTensorMaxMats))
            return false;
        TStage &S = tp.stages[s];
        // slot bits 0 and 1: two of distinct residues where there are
        int order[kStageBits] = {slots[0], slots[1], slots[2], slots[3 % nslots]};
        bool found = false;
        for (int a = 0; a < nslots && !found; ++a)
            for (int b = a + 1; b < nslots && !found; ++b)
                if (FS.sbits[slots[a]] % mod != FS.sbits[slots[b]] % mod)
                {
                    int rest = 0;
                    order[0] = slots[a];
                    order[1] = slots[b];
                    for (int c2 = 0; c2 < nslots; ++c2)
                        if (c2 != a && c2 != b)
                            order[2 + rest++] = slots[c2];
                    found = true;
                }
        uint8_t perm = 0;
        uint32_t tensor_mask = 0;
        for (int b = 0; b < width; ++b)
        {
            S.sbits[b] = FS.sbits[order[b]];
            perm |= static_cast<uint8_t>(order[b] << (2 * b));
            tensor_mask |= 1u << S.sbits[b];
        }
        if (padslot >= 0)
        {
            S.sbits[3] = FS.sbits[padslot];
            perm |= static_cast<uint8_t>(padslot << 6);
        }
        S.perm = perm;
        // group bits: the local condition bits first among the tile bits,
        // the other positions outside the tensor slots after them; the first
        // row bits on the residues the slot bits leave free
        std::vector<int> tile, rows, other;
        for (int l = 0; l < kTensorLocal; ++l)
            if ((cond.lmask >> l) & 1)
                tile.push_back(l);
        if (pad_cond)
            tile.push_back(FS.sbits[padslot]);
        for (int l = 0; l < kTensorLocal; ++l)
            if (!((tensor_mask >> l) & 1) && !((cond.lmask >> l) & 1) && !(pad_cond && l == FS.sbits[padslot]))
                other.push_back(l);
        uint32_t used = umma ? 0u : (1u << (S.sbits[0] % mod)) | (1u << (S.sbits[1] % mod));
        for (int r = 0; r < row_bank_bits; ++r)
            for (size_t i = 0; i < other.size(); ++i)
                if (!((used >> (other[i] % mod)) & 1))
                {
                    used |= 1u << (other[i] % mod);
                    rows.push_back(other[i]);
                    other.erase(other.begin() + static_cast<long>(i));
                    break;
                }
        for (int l : other)
            (rows.size() < 4 ? rows : tile).push_back(l);
        if (rows.size() != 4 || static_cast<int>(tile.size()) != ngroup - 4)
            return false;
        for (int i = 0; i < 4; ++i)
            S.gpos[i] = static_cast<uint8_t>(rows[i]);
        for (int i = 0; i < ngroup - 4; ++i)
            S.gpos[4 + i] = static_cast<uint8_t>(tile[i]);
        S.nlc = static_cast<uint8_t>(nlc);
        S.ngc = static_cast<uint8_t>(ngc);
        int i = 0;
        for (int q = 0; q < 64; ++q)
            if ((cond.gmask >> q) & 1)
                S.gq[i++] = static_cast<uint8_t>(q);
        S.woff = woff;
        woff += nm;
        tb.stages[s] = S;
        for (int gb = 0; gb < ngroup; ++gb)
            tp.swz[s][gb] = static_cast<uint16_t>(c64 ? swz8(1 << S.gpos[gb]) : swz16(1 << S.gpos[gb]));
        for (int b = 0; b < width; ++b)
            tp.swz[s][ngroup + b] = static_cast<uint16_t>(c64 ? swz8(1 << S.sbits[b]) : swz16(1 << S.sbits[b]));
    }
    tb.nstages = prm.nstages;
    tb.nmats = woff;
    tb.tf32 = c64 ? 1 : 0;
    tb.width = width;
    tb.umma = umma ? 1 : 0;
    tp.umma = umma ? 1 : 0;
    tp.nmats = woff;
    return true;
}

// Pass costs in one unit (multiply-adds per amplitude at the register path's
// FP64 rate), calibrated on B200 with the 30-qubit layered and matching
// circuits: register passes keep the FP64 pipe about 45% busy; complex64
// register passes take about 0.75 of the complex128 time; a complex128
// 16 x 16 tensor stage measured like 82 units, a complex64 one like 30.
double register_pass_cost(const FPassParams &prm, int amp_bytes)
{
    double fma = 0.0;
    for (int o = 0; o < prm.nops; ++o)
    {
        const FOp &op = prm.ops[o];
        switch (op.kind)
        {
        case F_DENSE1: fma += 8; break;
        case F_DENSE1R: fma += 4; break;
        case F_DENSE1X4: fma += 32; break;
        case F_DENSE1RX4: fma += 16; break;
        case F_DENSE1X2: fma += 16; break;
        case F_DENSE2: fma += 16; break;
        case F_PHASE: fma += 2; break;
        case F_DIAG: fma += 4; break;
        case F_PRUN: fma += 4.0 * __builtin_popcount(op.b0) + (op.b1 ? 4 : 0); break;
        default: fma += 0.5; break;   // exchanges, sign flips, terms
        }
    }
    return fma / 0.45 * (amp_bytes == 8 ? 0.75 : 1.0);
}

double tensor_pass_cost(const TPassParams &tp, int amp_bytes)
{
    // an 8 x 8 stage: half the tensor-core work of a 16 x 16 one and the
    // same shared-memory round trip; measured on the 30-qubit layered and
    // matching circuits: 0.63 of a 16 x 16 stage for complex128, 0.93 for
    // complex64 (whose stages are not bound by the tensor pipe). complex128
    // stages lost 10% of their time when the additions after the products
    // went into the tensor cores' accumulation (the factors below)
    if (tp.width == 3)
        return (amp_bytes == 8 ? 28.0 : 47.0) * tp.nstages;
    // tcgen05 16 x 16 stages (complex64): measured 1% below mma.sync ones
    if (tp.umma)
        return 29.0 * tp.nstages;
    return (amp_bytes == 8 ? 30.0 : 74.0) * tp.nstages;
}

template <typename R>
int launch_tensor_pass(const TPassParams &tp, cudaStream_t stream)
{
    typedef typename Tensor<R>::V V;
    if (tp.reg_mats > 0 && tp.width != 3)
        throw std::runtime_error("internal: batched tensor passes run 8 x 8 stages only");
    const size_t smem = kTensor4Buffers * sizeof(V) * kChunk;
    const size_t smem3 = kTensor3Buffers * sizeof(V) * kChunk;
    static bool configured[64] = {};
    int dev = 0, sms = 0, per_sm = 0;
    QCSB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !configured[dev])
    {
        QCSB_CUDA(cudaFuncSetAttribute(tensor_pass_kernel<R, kTensor4Buffers>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
        QCSB_CUDA(cudaFuncSetAttribute(tensor3_pass_kernel<R, kTensor3Buffers>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem3)));
        if (dev >= 0 && dev < 64)
            configured[dev] = true;
    }
    QCSB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (tp.width == 3)
        QCSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tensor3_pass_kernel<R, kTensor3Buffers>,
                                                                kThreads, smem3));
    else
        QCSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tensor_pass_kernel<R, kTensor4Buffers>,
                                                                kThreads, smem));
    const uint64_t grid = std::min<uint64_t>(tp.chunks, static_cast<uint64_t>(sms) * std::max(per_sm, 1));
    if (tp.width == 3)
        tensor3_pass_kernel<R, kTensor3Buffers><<<static_cast<unsigned>(grid), kThreads, smem3, stream>>>(tp);
    else
        tensor_pass_kernel<R, kTensor4Buffers><<<static_cast<unsigned>(grid), kThreads, smem, stream>>>(tp);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}
template int launch_tensor_pass<double>(const TPassParams &, cudaStream_t);
template int launch_tensor_pass<float>(const TPassParams &, cudaStream_t);

} // namespace qcsb
