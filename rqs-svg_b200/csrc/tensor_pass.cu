// Tensor passes: the stages of a fused pass as dense 16 x 16 complex
// matrices on the FP64 tensor cores (mma.sync m16n8k8, DMMA).
//
// A fused pass (fused_pass.cu) stages a 2^11-amplitude chunk in shared memory
// and runs its gates in stages of 4 local "stage bits". On the register path
// every thread applies the stage's gates one by one to the 16 amplitudes that
// differ in those bits. A tensor pass instead applies the stage's whole
// product as one 16 x 16 matrix M to every 16-amplitude group of the chunk.
// Gates of the stage that depend on bits outside it (controls, diagonal
// targets) make M depend on those bits; the stage then has one matrix per
// assignment of its condition bits (at most 2^8), all built on the GPU from
// the pass's ops before the pass (stage_matrix_kernel).
//
// Product layout. A warp takes 16 groups (rows r) at a time: y_r = M x_r for
// all 16 rows is D = A B with A (16 x 16 per component) the rows' input
// amplitudes and B[u][nu] = Re or Im of M[u'][u] (nu = output slot u' and
// component). With R = Re(x) B and S = Im(x) B (eight m16n8k8 products each,
// K = 16 input slots, N = 32 output columns), Re y = R_re - S_im and
// Im y = R_im + S_re. Lane (g, t) of the warp (g = lane / 4, t = lane % 4)
// holds rows g and g + 8 at input slots t, t + 4, t + 8, t + 12 for the A
// fragments, and the accumulators give it the same rows at output slots
// 4i + t for n-tiles i: it loads and stores the same 8 shared-memory
// positions, so the stage runs in place without extra barriers.
//
// FP64 work: 64 multiply-adds per amplitude and stage (the register path:
// 8 per complex 2x2 gate), at the FP64 tensor rate, which on B200 equals the
// FMA rate, but with one instruction per 1024 multiply-adds instead of 32.

#include "fused_pass.h"

#include <algorithm>
#include <cstring>

namespace qcsb
{
namespace
{

__device__ __forceinline__ int swz2(int j) { return j ^ (((j >> 3) ^ (j >> 6) ^ (j >> 9)) & 7); }

__device__ __forceinline__ void cp_async16(double2 *smem, const double2 *gmem)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// D += A B for one m16n8k8 FP64 tile (A 16 x 8 row-major fragments a0..a3,
// B 8 x 8 fragments b0, b1, D 16 x 8 fragments d0..d3).
__device__ __forceinline__ void dmma(double (&d)[4], double a0, double a1, double a2, double a3, double b0, double b1)
{
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
                 : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

constexpr int kThreads = 1 << (kTensorLocal - kStageBits);   // 128: 4 warps, two 16-group tiles each
constexpr int kSlots = 1 << kStageBits;
constexpr int kChunk = 1 << kTensorLocal;

__global__ void __launch_bounds__(kThreads, 3) tensor_pass_kernel(const __grid_constant__ TPassParams p)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *smem = reinterpret_cast<double2 *>(smem_raw);
    double2 *const state = static_cast<double2 *>(p.state);
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
    auto issue_load = [&](uint64_t c, double2 *dst) {
        const uint64_t cb = chunk_base(c);
        if (p.from_zero)
        {
#pragma unroll
            for (int m = 0; m < kSlots; ++m)
            {
                const bool one = cb == 0 && m == 0 && tid == 0;
                dst[swz2(tid + m * kThreads)] = make_double2(one ? 1.0 : 0.0, 0.0);
            }
        }
        else
        {
#pragma unroll
            for (int m = 0; m < kSlots; ++m)
                cp_async16(dst + swz2(tid + m * kThreads), state + (cb | elem_offset(m)));
        }
        cp_commit();
    };

    uint64_t c = blockIdx.x;
    if (c >= p.chunks)
        return;
    issue_load(c, smem);
    int cur = 0;
    for (; c < p.chunks; c += gridDim.x)
    {
        double2 *sb = smem + cur * kChunk;
        const uint64_t next = c + gridDim.x;
        if (next < p.chunks)
        {
            issue_load(next, smem + (cur ^ 1) * kChunk);
            cp_wait<1>();
        }
        else
        {
            cp_wait<0>();
        }
        __syncthreads();
        const uint64_t cbase = chunk_base(c);

        for (int st = 0; st < p.nstages; ++st)
        {
            const TStage &S = p.stages[st];
            // swizzled offsets of the group and slot bits (the swizzle is
            // linear over GF(2): positions combine by XOR)
            uint32_t gbit[7], sbit[kStageBits];
#pragma unroll
            for (int i = 0; i < 7; ++i)
                gbit[i] = static_cast<uint32_t>(swz2(1 << S.gpos[i]));
#pragma unroll
            for (int b = 0; b < kStageBits; ++b)
                sbit[b] = static_cast<uint32_t>(swz2(1 << S.sbits[b]));
            uint32_t vc = 0;
            for (int i = 0; i < S.ngc; ++i)
                vc |= static_cast<uint32_t>((cbase >> S.gq[i]) & 1) << i;
            uint32_t lane_pos = ((g & 1) ? gbit[0] : 0u) ^ ((g & 2) ? gbit[1] : 0u) ^ ((g & 4) ? gbit[2] : 0u) ^
                                ((t & 1) ? sbit[0] : 0u) ^ ((t & 2) ? sbit[1] : 0u);
            const uint32_t hpos = gbit[3];
            uint32_t last_v = 0xffffffffu;
            double2 bf[kTensorFragments];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
            {
                const uint32_t tile = static_cast<uint32_t>(mt | (warp << 1));
                const uint32_t v = (tile & ((1u << S.nlc) - 1u)) | (vc << S.nlc);
                if (v != last_v)
                {
                    const double2 *w = p.mats + (static_cast<size_t>(S.woff + v) * kTensorFragments) * 32 + lane;
#pragma unroll
                    for (int f = 0; f < kTensorFragments; ++f)
                        bf[f] = __ldg(w + f * 32);
                    last_v = v;
                }
                const uint32_t base = lane_pos ^ ((tile & 1) ? gbit[4] : 0u) ^ ((tile & 2) ? gbit[5] : 0u) ^
                                      ((tile & 4) ? gbit[6] : 0u);
                auto pos = [&](int h, int m) {
                    return base ^ (h ? hpos : 0u) ^ ((m & 1) ? sbit[2] : 0u) ^ ((m & 2) ? sbit[3] : 0u);
                };
                double2 x[2][4];
#pragma unroll
                for (int h = 0; h < 2; ++h)
#pragma unroll
                    for (int m = 0; m < 4; ++m)
                        x[h][m] = sb[pos(h, m)];
#pragma unroll
                for (int ih = 0; ih < 2; ++ih)
                {
                    double racc[2][4], sacc[2][4];
#pragma unroll
                    for (int ii = 0; ii < 2; ++ii)
#pragma unroll
                        for (int e = 0; e < 4; ++e)
                            racc[ii][e] = sacc[ii][e] = 0.0;
#pragma unroll
                    for (int ii = 0; ii < 2; ++ii)
                    {
                        const int i = 2 * ih + ii;
#pragma unroll
                        for (int j = 0; j < 2; ++j)
                        {
                            const double2 b = bf[j * 4 + i];
                            dmma(racc[ii], x[0][2 * j].x, x[1][2 * j].x, x[0][2 * j + 1].x, x[1][2 * j + 1].x, b.x, b.y);
                            dmma(sacc[ii], x[0][2 * j].y, x[1][2 * j].y, x[0][2 * j + 1].y, x[1][2 * j + 1].y, b.x, b.y);
                        }
                    }
#pragma unroll
                    for (int ii = 0; ii < 2; ++ii)
                    {
                        const int i = 2 * ih + ii;
                        sb[pos(0, i)] = make_double2(racc[ii][0] - sacc[ii][1], racc[ii][1] + sacc[ii][0]);
                        sb[pos(1, i)] = make_double2(racc[ii][2] - sacc[ii][3], racc[ii][3] + sacc[ii][2]);
                    }
                }
            }
            __syncthreads();
        }

#pragma unroll
        for (int m = 0; m < kSlots; ++m)
            __stcs(state + (cbase | elem_offset(m)), sb[swz2(tid + m * kThreads)]);
        __syncthreads();
        cur ^= 1;
    }
}

int residue(int pos) { return pos % 3; }

} // namespace

bool make_tensor_params(const FPassParams &prm, const std::vector<StageCond> &conds, TPassParams &tp,
                        TBuildParams &tb)
{
    if (prm.k != kTensorLocal || static_cast<int>(conds.size()) != prm.nstages || prm.nstages <= 0)
        return false;
    std::memset(&tp, 0, sizeof(tp));
    std::memset(&tb, 0, sizeof(tb));
    tp.n = prm.n;
    tp.from_zero = prm.from_zero;
    tp.chunks = prm.chunks;
    std::memcpy(tp.qmasks, prm.qmasks, sizeof(tp.qmasks));
    std::memcpy(tp.qbit, prm.qbit, sizeof(tp.qbit));
    tp.nstages = prm.nstages;
    uint32_t woff = 0;
    for (int s = 0; s < prm.nstages; ++s)
    {
        const FStage &FS = prm.stages[s];
        const StageCond &cond = conds[s];
        const int nlc = __builtin_popcount(cond.lmask);
        const int ngc = __builtin_popcountll(cond.gmask);
        if (nlc > kTensorTileBits || nlc + ngc > kTensorMaxCond)
            return false;
        const uint32_t nm = 1u << (nlc + ngc);
        if (woff + nm > static_cast<uint32_t>(kTensorMaxMats))
            return false;
        TStage &S = tp.stages[s];
        // slot bits 0 and 1 (the lanes of a quarter warp) and group bit 0 on
        // positions of three different residues mod 3: the swizzle then
        // sends the quarter warp's eight 16-byte accesses to eight bank
        // groups
        int pr[kStageBits] = {0, 1, 2, 3};
        bool found = false;
        for (int a = 0; a < kStageBits && !found; ++a)
            for (int b = a + 1; b < kStageBits && !found; ++b)
                if (residue(FS.sbits[a]) != residue(FS.sbits[b]))
                {
                    int rest = 0;
                    pr[0] = a;
                    pr[1] = b;
                    for (int c2 = 0; c2 < kStageBits; ++c2)
                        if (c2 != a && c2 != b)
                            pr[2 + rest++] = c2;
                    found = true;
                }
        uint8_t perm = 0;
        for (int b = 0; b < kStageBits; ++b)
        {
            S.sbits[b] = FS.sbits[pr[b]];
            perm |= static_cast<uint8_t>(pr[b] << (2 * b));
        }
        S.perm = perm;
        // group bits: the local condition bits first among the tile bits
        // (4..6), the other positions outside the stage after them; group
        // bit 0 on the residue that slot bits 0 and 1 leave free
        uint32_t stage_mask = 0;
        for (int b = 0; b < kStageBits; ++b)
            stage_mask |= 1u << FS.sbits[b];
        std::vector<int> tile, rows;
        for (int l = 0; l < kTensorLocal; ++l)
            if ((cond.lmask >> l) & 1)
                tile.push_back(l);
        std::vector<int> other;
        for (int l = 0; l < kTensorLocal; ++l)
            if (!((stage_mask >> l) & 1) && !((cond.lmask >> l) & 1))
                other.push_back(l);
        const int want = 3 - residue(S.sbits[0]) - residue(S.sbits[1]);
        std::stable_partition(other.begin(), other.end(), [&](int l) { return residue(l) == want; });
        // rows take the first four (the free residue first), tiles the rest
        for (int l : other)
            (rows.size() < 4 ? rows : tile).push_back(l);
        if (rows.size() != 4 || tile.size() != 3)
            return false;
        for (int i = 0; i < 4; ++i)
            S.gpos[i] = static_cast<uint8_t>(rows[i]);
        for (int i = 0; i < 3; ++i)
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
    }
    tb.nstages = prm.nstages;
    tb.nmats = woff;
    return true;
}

double register_pass_cost(const FPassParams &prm)
{
    // multiply-adds per amplitude of each op on the register path
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
    // the register path keeps the FP64 pipe about 45% busy (measured)
    return fma / 0.45;
}

double tensor_pass_cost(const TPassParams &tp)
{
    return 64.0 * tp.nstages / 0.85;
}

template <>
int launch_tensor_pass<double>(const TPassParams &tp, cudaStream_t stream)
{
    const size_t smem = 2 * sizeof(double2) * kChunk;
    static bool configured[64] = {};
    int dev = 0, sms = 0, per_sm = 0;
    QCSB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !configured[dev])
    {
        QCSB_CUDA(cudaFuncSetAttribute(tensor_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem)));
        if (dev >= 0 && dev < 64)
            configured[dev] = true;
    }
    QCSB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    QCSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tensor_pass_kernel, kThreads, smem));
    const uint64_t grid = std::min<uint64_t>(tp.chunks, static_cast<uint64_t>(sms) * std::max(per_sm, 1));
    tensor_pass_kernel<<<static_cast<unsigned>(grid), kThreads, smem, stream>>>(tp);
    QCSB_CUDA(cudaGetLastError());
    return 1;
}

} // namespace qcsb
