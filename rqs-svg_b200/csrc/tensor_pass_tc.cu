// Complex64 tensor passes on the fifth-generation tensor cores (tcgen05).
//
// The stages of a pass as dense 16 x 16 complex matrices, as in
// tensor_pass.cu, but issued as tcgen05.mma with TF32 operands and FP32
// accumulators in tensor memory (TMEM) instead of warp-level mma.sync.
//
// A CTA of 128 threads owns one 2^11-amplitude chunk at a time (staged in
// shared memory, double-buffered). In a stage, thread t holds one row: the
// 16 amplitudes of its group (the values of the stage's four slot bits, its
// other local bits fixed by t). Each thread splits its row into TF32 high and
// low parts and writes them to TMEM lane t (tcgen05.st): columns 0-31 hold
// the high parts [Re x_0..15 | Im x_0..15], columns 32-63 the low parts. The
// stage matrix M = Mr + i Mi acts on a row as one real product
//     [Re y | Im y] = [Re x | Im x] W,  W = [[Mr^T, Mi^T], [-Mi^T, Mr^T]],
// a 32 x 32 real B operand in shared memory (K-major, no swizzle; built on
// the GPU from the pass's ops, split into TF32 high and low parts). One
// thread issues 12 MMAs per stage: M = 128 rows, N = 32 per matrix variant,
// K = 8 per instruction over the 32 inputs, for the three terms
// lo x hi, hi x lo, hi x hi (the lo x lo term, ~2^-21 relative, is dropped),
// accumulated in FP32 in TMEM columns 64 onwards; tcgen05.commit signals an
// mbarrier when they are done, and every warp reads its rows back with
// tcgen05.ld and stores them to the chunk.
//
// Matrix variants: a stage whose gates depend on one local bit outside the
// stage has two matrices; that bit is thread bit 5 (warp bit 0), both
// matrices sit side by side in B (N = 64), and each warp reads the 32
// columns of its own. Chunk condition bits pick the B tiles per chunk.
//
// TMEM: 128 columns per CTA, allocated once and freed before the CTA exits;
// shared memory keeps at most four CTAs on an SM (4 x 128 = 512 columns), so
// an allocation never waits. Every wait on the mbarrier is bounded: past the
// limit the CTA records an error for the host and leaves its loops.
//
// This kernel is for one GPU: no cluster launch and no multicast.

#include "fused_pass.h"

#include <algorithm>

namespace qcsb
{
namespace
{

constexpr int kThreads = 128;
constexpr int kChunk = 1 << kTensorLocal;
constexpr int kSlots = 1 << kStageBits;
constexpr uint32_t kCols = 128;               // TMEM columns: A high 0-31, A low 32-63, D 64-127
constexpr uint32_t kColD = 64;
constexpr uint32_t kSpinLimit = 1u << 22;     // mbarrier polls before giving up (well under a minute)
constexpr size_t kChunkBytes = sizeof(float2) * kChunk;
constexpr size_t kBBytes = 2 * 2 * kUmmaSlab;  // high and low parts of up to two matrices
constexpr size_t kSmem = 2 * kChunkBytes + kBBytes;

__device__ __forceinline__ int swz8(int j) { return j ^ (((j >> 4) ^ (j >> 8)) & 15); }

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// x = hi + lo + e: hi keeps x's sign, exponent and top 10 mantissa bits (a
// TF32 value, by masking), lo the next 11 significant bits of the exact
// remainder, |e| <= 2^-21 |x|; two integer ops and one subtraction per value
// (the tensor cores read a TF32 operand's top 19 bits)
__device__ __forceinline__ void tf32_split(float x, uint32_t &hi, uint32_t &lo)
{
    hi = __float_as_uint(x) & 0xFFFFE000u;
    lo = __float_as_uint(x - __uint_as_float(hi)) & 0xFFFFE000u;
}

// Shared-memory descriptor of a B operand (K-major, no swizzle): 16-byte
// rows of 4 TF32 inputs, 8 such rows (8 outputs) per 128-byte core matrix;
// the two K halves of a K-step 128 bytes apart (leading byte offset), the
// groups of 8 outputs 1024 bytes apart (stride byte offset); version 1.
__device__ __forceinline__ uint64_t b_descriptor(uint32_t saddr)
{
    uint64_t d = static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>(128u >> 4) << 16;
    d |= static_cast<uint64_t>(1024u >> 4) << 32;
    d |= 1ull << 46;
    return d;
}

// Instruction descriptor: FP32 accumulator, TF32 A and B, both K-major,
// M = 128, N columns.
__device__ __forceinline__ uint32_t instr_descriptor(uint32_t n)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate)
{
    const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile("{\n\t"
                 ".reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t"
                 "}\n" ::"r"(d_tmem),
                 "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2),
                 "r"(mask3));
}

__device__ __forceinline__ void tmem_store32(uint32_t taddr, const uint32_t (&v)[32])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, "
                 "%32};\n" ::"r"(taddr),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
                 "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]),
                 "r"(v[17]), "r"(v[18]), "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]),
                 "r"(v[25]), "r"(v[26]), "r"(v[27]), "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
                 : "memory");
}

__device__ __forceinline__ void tmem_load32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                 "[%32];\n"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                   "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                   "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                   "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                   "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                 : "r"(taddr)
                 : "memory");
}

__device__ __forceinline__ void tmem_wait_store() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_load() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// true when the mbarrier's phase with this parity has completed
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
{
    for (uint32_t i = 0; i < kSpinLimit; ++i)
    {
        uint32_t done;
        asm volatile("{\n\t"
                     ".reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, p;\n\t"
                     "}\n"
                     : "=r"(done)
                     : "r"(mbar), "r"(parity)
                     : "memory");
        if (done)
            return true;
    }
    return false;
}

__device__ __forceinline__ void cp_async8(float2 *smem, const float2 *gmem)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__global__ void __launch_bounds__(kThreads, 4) tc_pass_kernel(const __grid_constant__ TPassParams p)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    float2 *chunks = reinterpret_cast<float2 *>(smem_raw);
    unsigned char *bsm = smem_raw + 2 * kChunkBytes;   // B: high parts (up to 2 slabs), then low parts
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    float2 *const state = static_cast<float2 *>(p.state);
    const unsigned char *const mats = reinterpret_cast<const unsigned char *>(p.mats);
    const int tid = threadIdx.x;
    const int warp = tid >> 5;

    // TMEM columns and the mbarrier; the allocating warp frees them at the end
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(&tmem_slot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(&mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_slot;
    const uint32_t mbar_addr = smem_addr(&mbar);
    const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
    uint32_t phase = 0;
    bool failed = false;

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
    auto issue_load = [&](uint64_t cb, float2 *dst) {
        if (p.from_zero)
        {
#pragma unroll
            for (int m = 0; m < kSlots; ++m)
            {
                const bool one = cb == 0 && m == 0 && tid == 0;
                dst[swz8(tid + m * kThreads)] = make_float2(one ? 1.0f : 0.0f, 0.0f);
            }
        }
        else
        {
#pragma unroll
            for (int m = 0; m < kSlots; ++m)
                cp_async8(dst + swz8(tid + m * kThreads), state + (cb | elem_offset(m)));
        }
        cp_commit();
    };

    // B operands of stage st for the chunk at cb, into registers: nv slabs of
    // high parts, then nv of low parts (loaded one stage ahead, so that
    // their latency hides behind the stage before)
    constexpr int kBPieces = 2 * 2 * kUmmaSlab / 16 / kThreads;
    uint4 breg[kBPieces];
    auto prefetch_b = [&](int st, uint64_t cb) {
        const TStage &S = p.stages[st];
        uint32_t vc = 0;
        for (int i = 0; i < S.ngc; ++i)
            vc |= static_cast<uint32_t>((cb >> S.gq[i]) & 1) << i;
        const uint32_t m0 = S.woff + (vc << S.nlc);
        const int nb16 = (1 << S.nlc) * kUmmaSlab / 16;
#pragma unroll
        for (int i = 0; i < kBPieces; ++i)
        {
            const int piece = tid + i * kThreads;   // over [high part | low part]
            if (piece < 2 * nb16)
            {
                const int part = piece >= nb16 ? 1 : 0;
                const int off = piece - part * nb16;
                const size_t src =
                    (static_cast<size_t>(part) * p.nmats + m0) * kUmmaSlab + static_cast<size_t>(off) * 16;
                breg[i] = __ldg(reinterpret_cast<const uint4 *>(mats + src));
            }
        }
    };

    uint64_t c = blockIdx.x;
    int cur = 0;
    uint64_t cbase_next = c < p.chunks ? chunk_base(c) : 0;
    if (c < p.chunks)
    {
        issue_load(cbase_next, chunks);
        if (p.nstages > 0)
            prefetch_b(0, cbase_next);
    }
    for (; c < p.chunks && !failed; c += gridDim.x)
    {
        float2 *sb = chunks + cur * kChunk;
        const uint64_t cbase = cbase_next;
        const uint64_t next = c + gridDim.x;
        if (next < p.chunks)
        {
            cbase_next = chunk_base(next);
            issue_load(cbase_next, chunks + (cur ^ 1) * kChunk);
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
            const int nv = 1 << S.nlc;   // 1 or 2 matrices side by side
            const int nb16 = nv * kUmmaSlab / 16;   // 16-byte pieces per part
            // this thread's row: thread bits 0-3, 4, 5, 6 are group bits 0-3,
            // 6, 4, 5 (bit 5 = warp bit 0 is the local condition bit)
            const uint16_t *sw = p.swz[st];
            uint32_t p0 = 0;
            {
                const int gb_of[7] = {0, 1, 2, 3, 6, 4, 5};
#pragma unroll
                for (int b = 0; b < 7; ++b)
                    if ((tid >> b) & 1)
                        p0 ^= sw[gb_of[b]];
            }
            uint32_t sbit[kStageBits];
#pragma unroll
            for (int b = 0; b < kStageBits; ++b)
                sbit[b] = sw[7 + b];
            auto pos = [&](int u) {
                uint32_t q = p0;
#pragma unroll
                for (int b = 0; b < kStageBits; ++b)
                    if ((u >> b) & 1)
                        q ^= sbit[b];
                return q;
            };
            {
                uint32_t hi[32], lo[32];
#pragma unroll
                for (int u = 0; u < kSlots; ++u)
                {
                    const float2 x = sb[pos(u)];
                    tf32_split(x.x, hi[u], lo[u]);
                    tf32_split(x.y, hi[16 + u], lo[16 + u]);
                }
                tmem_store32(tmem + lane_base + 0, hi);
                tmem_store32(tmem + lane_base + 32, lo);
            }
            // B to shared memory: nv slabs of high parts at bsm, low parts at
            // bsm + 2 slabs
#pragma unroll
            for (int i = 0; i < kBPieces; ++i)
            {
                const int piece = tid + i * kThreads;
                if (piece < 2 * nb16)
                {
                    const int part = piece >= nb16 ? 1 : 0;
                    const int off = piece - part * nb16;
                    *reinterpret_cast<uint4 *>(bsm + part * 2 * kUmmaSlab + off * 16) = breg[i];
                }
            }
            tmem_wait_store();
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            fence_before_sync();
            __syncthreads();
            if (tid == 0)
            {
                fence_after_sync();
                const uint32_t idesc = instr_descriptor(static_cast<uint32_t>(32 * nv));
                const uint32_t bhi = smem_addr(bsm), blo = smem_addr(bsm + 2 * kUmmaSlab);
                // lo x hi, hi x lo, hi x hi; K-steps of 8 inputs (256 bytes of B)
                uint32_t acc = 0;
#pragma unroll
                for (int term = 0; term < 3; ++term)
                {
                    const uint32_t acol = term == 0 ? 32u : 0u;
                    const uint32_t bbase = term == 1 ? blo : bhi;
#pragma unroll
                    for (int ks = 0; ks < 4; ++ks)
                    {
                        umma_tf32(tmem + kColD, tmem + acol + 8u * ks, b_descriptor(bbase + 256u * ks), idesc, acc);
                        acc = 1;
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                                 mbar_addr)
                             : "memory");
            }
            // the next stage's B (or the next chunk's first) while the MMAs run
            if (st + 1 < p.nstages)
                prefetch_b(st + 1, cbase);
            else if (next < p.chunks)
                prefetch_b(0, cbase_next);
            const bool ok = mbar_wait(mbar_addr, phase);
            phase ^= 1;
            fence_after_sync();
            if (__syncthreads_or(!ok))
            {
                failed = true;
                if (tid == 0 && p.err != nullptr)
                    atomicExch(p.err, 1);
                break;
            }
            {
                const uint32_t v = S.nlc ? static_cast<uint32_t>(warp & 1) : 0u;
                uint32_t y[32];
                tmem_load32(tmem + lane_base + kColD + 32u * v, y);
                tmem_wait_load();
#pragma unroll
                for (int u = 0; u < kSlots; ++u)
                    sb[pos(u)] = make_float2(__uint_as_float(y[u]), __uint_as_float(y[16 + u]));
            }
            fence_before_sync();
            __syncthreads();
        }
        if (failed)
            break;
#pragma unroll
        for (int m = 0; m < kSlots; ++m)
            __stcs(state + (cbase | elem_offset(m)), sb[swz8(tid + m * kThreads)]);
        __syncthreads();
        cur ^= 1;
    }
    cp_wait<0>();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols) : "memory");
}

} // namespace

int launch_tc_pass(const TPassParams &tp, cudaStream_t stream)
{
    if (tp.reg_mats > 0)
        throw std::runtime_error("internal: tcgen05 passes run one register");
    static bool configured[64] = {};
    int dev = 0, sms = 0, per_sm = 0;
    QCSB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !configured[dev])
    {
        QCSB_CUDA(cudaFuncSetAttribute(tc_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(kSmem)));
        if (dev >= 0 && dev < 64)
            configured[dev] = true;
    }
    QCSB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // four CTAs per SM: 128 registers x 128 threads, 49 KiB of dynamic
    // shared memory each, and 4 x 128 = 512 TMEM columns. (The occupancy
    // API answers 0 or 1 for this kernel, which would leave one CTA per SM.)
    per_sm = static_cast<int>(512 / kCols);
    const uint64_t grid = std::min<uint64_t>(tp.chunks, static_cast<uint64_t>(sms) * per_sm);
    tc_pass_kernel<<<static_cast<unsigned>(grid), kThreads, kSmem, stream>>>(tp);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

} // namespace qcsb
