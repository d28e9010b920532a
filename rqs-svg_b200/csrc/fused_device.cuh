// Device code of the fused passes: the gate applications on a thread's 16
// amplitudes, the stage and op helpers, and the chunk loop of a pass
// (fused_pass_body), which takes the stage program as a parameter;
// fused_pass.cu instantiates it with the run-time program (run_stages: the
// parameter block's ops interpreted one by one). See fused_pass.cu for the
// execution model.
#pragma once

#include "fused_types.h"

namespace qcsb
{
namespace fdev
{


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
// entries already stored in the amplitude type
template <typename V>
__device__ __forceinline__ V cvt(float2 m) { return m; }

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


// Gate application on a thread's 2^kStageBits amplitudes a[r] (r = the values
// of the stage's local bits; j0 = the thread's local index with the stage
// bits zero). A condition splits into the other local bits (checked once
// against j0: when it fails the op does nothing for this thread) and the
// stage bits (smask/sval, checked per slot r). Ops without a condition take
// the unconditional path.

// Where an op's matrix entries come from: the pass parameters (one register)
// or the register's block of the entry buffer (batched passes). Entries are
// stored in the amplitude type: complex64 passes hold float2 entries (the
// host rounds them once), so the kernel neither converts nor loads 64-bit
// values per use.
template <typename V>
__device__ __forceinline__ V pool_entry(const FPassParams &p, int i)
{
    return reinterpret_cast<const V *>(p.entries)[i];
}
template <typename V>
struct PoolEntries
{
    const FPassParams &p;
    uint32_t off;
    __device__ __forceinline__ V operator[](int i) const { return pool_entry<V>(p, off + i); }
};
// Entries of the stage-matrix builder (FP64): the pass parameters (one
// register, blk null) or a register's block of a batch's entry buffer
// (float2 entries for complex64 batches, double2 otherwise).
template <typename V>
struct BuildEntries
{
    const FPassParams &p;
    const void *blk;
    int flt;
    uint32_t off;
    __device__ __forceinline__ V operator[](int i) const
    {
        if (blk == nullptr)
            return pool_entry<V>(p, off + i);
        if (flt)
        {
            const float2 e = __ldg(static_cast<const float2 *>(blk) + off + i);
            return V{e.x, e.y};
        }
        const double2 e = __ldg(static_cast<const double2 *>(blk) + off + i);
        return V{e.x, e.y};
    }
};
template <typename V>
struct BufferEntries
{
    const V *m;
    __device__ __forceinline__ V operator[](int i) const { return __ldg(m + i); }
};

// A real 2x2 on one amplitude pair: each output component is a real
// combination of the same component of the two inputs. Complex64 runs it on
// the packed FP32 pipe (fma.rn.f32x2: both components per instruction), with
// the same operation order and rounding as the scalar form.
__device__ __forceinline__ unsigned long long pack2(float lo, float hi)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}

template <typename V>
struct RealGate;

template <>
struct RealGate<double2>
{
    double m00, m01, m10, m11;
    __device__ __forceinline__ RealGate(double a, double b, double c, double d) : m00(a), m01(b), m10(c), m11(d) {}
    __device__ __forceinline__ void pair(double2 &y0, double2 &y1) const
    {
        const double2 x0 = y0, x1 = y1;
        y0.x = fma(m00, x0.x, m01 * x1.x);
        y0.y = fma(m00, x0.y, m01 * x1.y);
        y1.x = fma(m11, x1.x, m10 * x0.x);
        y1.y = fma(m11, x1.y, m10 * x0.y);
    }
};

template <>
struct RealGate<float2>
{
    unsigned long long c00, c01, c10, c11;   // each entry twice, packed
    __device__ __forceinline__ RealGate(float a, float b, float c, float d)
        : c00(pack2(a, a)), c01(pack2(b, b)), c10(pack2(c, c)), c11(pack2(d, d))
    {
    }
    __device__ __forceinline__ void pair(float2 &y0, float2 &y1) const
    {
        const unsigned long long x0 = pack2(y0.x, y0.y), x1 = pack2(y1.x, y1.y);
        unsigned long long t0, t1, r0, r1;
        asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(t0) : "l"(c01), "l"(x1));
        asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(t1) : "l"(c10), "l"(x0));
        asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r0) : "l"(c00), "l"(x0), "l"(t0));
        asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r1) : "l"(c11), "l"(x1), "l"(t1));
        asm("mov.b64 {%0, %1}, %2;" : "=f"(y0.x), "=f"(y0.y) : "l"(r0));
        asm("mov.b64 {%0, %1}, %2;" : "=f"(y1.x), "=f"(y1.y) : "l"(r1));
    }
};

// A complex 2x2 on one amplitude pair (y0, y1) <- (m00 y0 + m01 y1,
// m10 y0 + m11 y1). Complex64 runs each output as one multiply and three
// multiply-adds on the packed FP32 pipe: (re, im) += (m.re, m.re) * (x.re,
// x.im) and (-m.im, m.im) * (x.im, x.re), in cmad2's order, so the results
// are the same bit for bit.
template <typename V>
struct ComplexGate;

template <>
struct ComplexGate<double2>
{
    double2 m00, m01, m10, m11;
    __device__ __forceinline__ ComplexGate(double2 a, double2 b, double2 c, double2 d) : m00(a), m01(b), m10(c), m11(d) {}
    __device__ __forceinline__ void pair(double2 &y0, double2 &y1) const
    {
        const double2 x0 = y0, x1 = y1;
        y0 = cmad2(m00, x0, m01, x1);
        y1 = cmad2(m11, x1, m10, x0);
    }
};

template <>
struct ComplexGate<float2>
{
    // per entry: (re, re) and (-im, im), packed
    unsigned long long r00, i00, r01, i01, r10, i10, r11, i11;
    __device__ __forceinline__ ComplexGate(float2 a, float2 b, float2 c, float2 d)
        : r00(pack2(a.x, a.x)), i00(pack2(-a.y, a.y)), r01(pack2(b.x, b.x)), i01(pack2(-b.y, b.y)),
          r10(pack2(c.x, c.x)), i10(pack2(-c.y, c.y)), r11(pack2(d.x, d.x)), i11(pack2(-d.y, d.y))
    {
    }
    // mr * v + mi * swap(v) + mr2 * w + mi2 * swap(w), in cmad2's order
    static __device__ __forceinline__ unsigned long long mad(unsigned long long mr, unsigned long long mi,
                                                             unsigned long long v, unsigned long long vs,
                                                             unsigned long long mr2, unsigned long long mi2,
                                                             unsigned long long w, unsigned long long ws)
    {
        unsigned long long t;
        asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(t) : "l"(mi2), "l"(ws));
        asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(t) : "l"(mr2), "l"(w));
        asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(t) : "l"(mi), "l"(vs));
        asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(t) : "l"(mr), "l"(v));
        return t;
    }
    __device__ __forceinline__ void pair(float2 &y0, float2 &y1) const
    {
        const unsigned long long x0 = pack2(y0.x, y0.y), x0s = pack2(y0.y, y0.x);
        const unsigned long long x1 = pack2(y1.x, y1.y), x1s = pack2(y1.y, y1.x);
        const unsigned long long o0 = mad(r00, i00, x0, x0s, r01, i01, x1, x1s);
        const unsigned long long o1 = mad(r11, i11, x1, x1s, r10, i10, x0, x0s);
        asm("mov.b64 {%0, %1}, %2;" : "=f"(y0.x), "=f"(y0.y) : "l"(o0));
        asm("mov.b64 {%0, %1}, %2;" : "=f"(y1.x), "=f"(y1.y) : "l"(o1));
    }
};

template <typename V, int B, typename M>
__device__ __forceinline__ void apply_dense1(V (&a)[R], const FOp &op, const M &e, uint32_t j0)
{
    const V m00 = cvt<V>(e[0]), m01 = cvt<V>(e[1]), m10 = cvt<V>(e[2]), m11 = cvt<V>(e[3]);
    const ComplexGate<V> g(m00, m01, m10, m11);
    const bool tok = (j0 & op.lcmask) == op.lcval;
    const uint32_t cm = op.smask, cv = op.sval;
    if (cm == 0 && op.lcmask == 0)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (r & (1 << B))
                continue;
            g.pair(a[r], a[r | (1 << B)]);
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        if (r & (1 << B))
            continue;
        if (tok && (r & cm) == cv)
        {
            g.pair(a[r], a[r | (1 << B)]);
        }
    }
}

// Real 2x2: each output component is a real combination of the same
// component of the two inputs (half the multiply-adds of the complex case).
template <typename V, int B, typename M>
__device__ __forceinline__ void apply_dense1r(V (&a)[R], const FOp &op, const M &e, uint32_t j0)
{
    typedef decltype(V::x) S;
    const S m00 = static_cast<S>(e[0].x), m01 = static_cast<S>(e[1].x);
    const S m10 = static_cast<S>(e[2].x), m11 = static_cast<S>(e[3].x);
    const bool tok = (j0 & op.lcmask) == op.lcval;
    const uint32_t cm = op.smask, cv = op.sval;
    const RealGate<V> g(m00, m01, m10, m11);
    auto pair = [&](int r) { g.pair(a[r], a[r | (1 << B)]); };
    if (cm == 0 && op.lcmask == 0)
    {
        // no condition: straight-line code without per-slot predicates
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (!(r & (1 << B)))
                pair(r);
        return;
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        if (r & (1 << B))
            continue;
        if (tok && (r & cm) == cv)
            pair(r);
    }
}

// One uncontrolled 2x2 gate on each of the four stage bits, in bit order:
// one dispatch, and the compiler keeps the amplitudes in place between them.
template <typename V, typename M>
__device__ __forceinline__ void apply_dense1rx4(V (&a)[R], const M &e)
{
    typedef decltype(V::x) S;
#pragma unroll
    for (int b = 0; b < kStageBits; ++b)
    {
        const S m00 = static_cast<S>(e[4 * b].x), m01 = static_cast<S>(e[4 * b + 1].x);
        const S m10 = static_cast<S>(e[4 * b + 2].x), m11 = static_cast<S>(e[4 * b + 3].x);
        const RealGate<V> g(m00, m01, m10, m11);
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (r & (1 << b))
                continue;
            g.pair(a[r], a[r | (1 << b)]);
        }
    }
}

template <typename V, typename M>
__device__ __forceinline__ void apply_dense1x4(V (&a)[R], const M &e)
{
#pragma unroll
    for (int b = 0; b < kStageBits; ++b)
    {
        const V m00 = cvt<V>(e[4 * b]), m01 = cvt<V>(e[4 * b + 1]);
        const V m10 = cvt<V>(e[4 * b + 2]), m11 = cvt<V>(e[4 * b + 3]);
        const ComplexGate<V> g(m00, m01, m10, m11);
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (r & (1 << b))
                continue;
            g.pair(a[r], a[r | (1 << b)]);
        }
    }
}

// F_DENSE1X2: uncontrolled complex 2x2 gates on stage bits B0 < B1.
template <typename V, int B0, int B1, typename M>
__device__ __forceinline__ void apply_dense1x2(V (&a)[R], const M &e)
{
#pragma unroll
    for (int i = 0; i < 2; ++i)
    {
        const int b = i ? B1 : B0;
        const V m00 = cvt<V>(e[4 * i]), m01 = cvt<V>(e[4 * i + 1]);
        const V m10 = cvt<V>(e[4 * i + 2]), m11 = cvt<V>(e[4 * i + 3]);
        const ComplexGate<V> g(m00, m01, m10, m11);
#pragma unroll
        for (int r = 0; r < R; ++r)
        {
            if (r & (1 << b))
                continue;
            g.pair(a[r], a[r | (1 << b)]);
        }
    }
}

template <typename V, int B>
__device__ __forceinline__ void apply_swap1(V (&a)[R], const FOp &op, uint32_t j0)
{
    const bool tok = (j0 & op.lcmask) == op.lcval;
    const uint32_t cm = op.smask, cv = op.sval;
    if (cm == 0 && op.lcmask == 0)
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
        if (tok && (r & cm) == cv)
        {
            const int r1 = r | (1 << B);
            const V t = a[r];
            a[r] = a[r1];
            a[r1] = t;
        }
    }
}

template <typename V, int B0, int B1, typename M>
__device__ __forceinline__ void apply_dense2(V (&a)[R], const FOp &op, const M &m, uint32_t j0)
{
    const bool tok = (j0 & op.lcmask) == op.lcval;
    const uint32_t cm = op.smask, cv = op.sval;
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        if (r & ((1 << B0) | (1 << B1)))
            continue;
        if (!tok || (r & cm) != cv)
            continue;
        const int i1 = r | (1 << B0), i2 = r | (1 << B1), i3 = r | (1 << B0) | (1 << B1);
        const V x0 = a[r], x1 = a[i1], x2 = a[i2], x3 = a[i3];
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
__device__ __forceinline__ void apply_swap2(V (&a)[R], const FOp &op, uint32_t j0)
{
    const bool tok = (j0 & op.lcmask) == op.lcval;
    const uint32_t cm = op.smask, cv = op.sval;
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        if (r & ((1 << B0) | (1 << B1)))
            continue;
        if (tok && (r & cm) == cv)
        {
            const int i1 = r | (1 << B0), i2 = r | (1 << B1);
            const V t = a[i1];
            a[i1] = a[i2];
            a[i2] = t;
        }
    }
}

template <typename V, typename M>
__device__ __forceinline__ void apply_phase(V (&a)[R], const FOp &op, const M &m, uint32_t j0)
{
    const V e = cvt<V>(m[0]);
    const bool tok = (j0 & op.lcmask) == op.lcval;
    const uint32_t cm = op.smask, cv = op.sval;
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (tok && (r & cm) == cv)
            a[r] = cmul(e, a[r]);
}

// Sign flips on the integer pipe (the FP64/FP32 pipes are the busy ones).
__device__ __forceinline__ double flip(double x) { return __longlong_as_double(__double_as_longlong(x) ^ (1ll << 63)); }
__device__ __forceinline__ float flip(float x) { return __int_as_float(__float_as_int(x) ^ (1 << 31)); }
// sign bit XORed with bit 31 of s (s is 0 or 1 << 31)
__device__ __forceinline__ double flip_by(double x, uint32_t s)
{
    return __hiloint2double(__double2hiint(x) ^ static_cast<int>(s), __double2loint(x));
}
__device__ __forceinline__ float flip_by(float x, uint32_t s) { return __uint_as_float(__float_as_uint(x) ^ s); }

// times i: (x, y) -> (-y, x); times -i: (x, y) -> (y, -x)
template <typename V>
__device__ __forceinline__ void apply_muli(V (&a)[R], const FOp &op, uint32_t j0)
{
    const bool tok = (j0 & op.lcmask) == op.lcval;
    const uint32_t cm = op.smask, cv = op.sval;
    const bool minus = op.b1 != 0;
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (tok && (r & cm) == cv)
        {
            const auto x = a[r].x, y = a[r].y;
            a[r].x = minus ? y : flip(y);
            a[r].y = minus ? flip(x) : x;
        }
}

template <typename V, typename M>
__device__ __forceinline__ void apply_diag(V (&a)[R], const FOp &op, const M &m, uint32_t j0, uint64_t cbase)
{
    // one or two targets: entries in registers, chosen per amplitude by its
    // target bits (from the slot r for stage bits, the thread's local index
    // for other local bits, or the chunk when not local)
    const bool tok = (j0 & op.lcmask) == op.lcval;
    const V d0 = cvt<V>(m[0]), d1 = cvt<V>(m[1]), d2 = cvt<V>(m[2]), d3 = cvt<V>(m[3]);
    const uint32_t cm = op.smask, cv = op.sval;
    auto fixed_bit = [&](int i) -> uint32_t {
        if (i >= op.nt)
            return 0u;
        if (op.loc[i] >= 0)
            return (j0 >> op.loc[i]) & 1u;
        return static_cast<uint32_t>((cbase >> op.phys[i]) & 1ull);
    };
    const uint32_t c0 = fixed_bit(0), c1 = fixed_bit(1);
    const int p0 = op.spos[0], p1 = op.nt > 1 ? op.spos[1] : -1;
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        if (!tok || (r & cm) != cv)
            continue;
        const uint32_t s0 = p0 >= 0 ? ((r >> p0) & 1u) : c0;
        const uint32_t s1 = p1 >= 0 ? ((r >> p1) & 1u) : c1;
        const V d = s1 ? (s0 ? d3 : d2) : (s0 ? d1 : d0);
        a[r] = cmul(d, a[r]);
    }
}

template <typename V, typename M>
__device__ __forceinline__ void dispatch_dense1(V (&a)[R], const FOp &op, const M &e, uint32_t j0)
{
    switch (op.b0)
    {
    case 0: apply_dense1<V, 0>(a, op, e, j0); break;
    case 1: apply_dense1<V, 1>(a, op, e, j0); break;
    case 2: apply_dense1<V, 2>(a, op, e, j0); break;
    default: apply_dense1<V, 3>(a, op, e, j0); break;
    }
}

template <typename V, typename M>
__device__ __forceinline__ void dispatch_dense1r(V (&a)[R], const FOp &op, const M &e, uint32_t j0)
{
    switch (op.b0)
    {
    case 0: apply_dense1r<V, 0>(a, op, e, j0); break;
    case 1: apply_dense1r<V, 1>(a, op, e, j0); break;
    case 2: apply_dense1r<V, 2>(a, op, e, j0); break;
    default: apply_dense1r<V, 3>(a, op, e, j0); break;
    }
}

template <typename V>
__device__ __forceinline__ void dispatch_swap1(V (&a)[R], const FOp &op, uint32_t j0)
{
    switch (op.b0)
    {
    case 0: apply_swap1<V, 0>(a, op, j0); break;
    case 1: apply_swap1<V, 1>(a, op, j0); break;
    case 2: apply_swap1<V, 2>(a, op, j0); break;
    default: apply_swap1<V, 3>(a, op, j0); break;
    }
}

template <typename V, typename M>
__device__ __forceinline__ void dispatch_x2(V (&a)[R], const FOp &op, const M &e)
{
#define QCSB_X2(b0, b1)                                                                                            \
    case b0 * 4 + b1: apply_dense1x2<V, b0, b1>(a, e); break;
    switch (op.b0 * 4 + op.b1)
    {
        QCSB_X2(0, 1) QCSB_X2(0, 2) QCSB_X2(0, 3) QCSB_X2(1, 2) QCSB_X2(1, 3)
    default: apply_dense1x2<V, 2, 3>(a, e); break;
    }
#undef QCSB_X2
}

// Where a stage's slots live in shared memory: slot s of this thread is at
// p0 ^ (XOR of sbit[b] over the bits b of s).
template <typename V>
struct StageSlots
{
    V *sb;
    uint32_t p0;
    uint32_t sbit[kStageBits];
};

// Two-target ops are compiled for slot bits (0, 1) only: for other stage bits
// (b0, b1) register r holds slot perm(r) (bits b0, b1, then the other two
// ascending) during the op, moved through the thread's own shared-memory
// positions (no other thread reads them: no barrier), and back. The host
// writes the op's stage-bit condition in that order.
template <typename V, typename M>
__device__ __forceinline__ void apply_two_target(V (&a)[R], const FOp &op, const M &e, uint32_t j0,
                                                 const StageSlots<V> &ss)
{
    const bool move = op.b0 != 0 || op.b1 != 1;
    const uint32_t rest = 15u & ~((1u << op.b0) | (1u << op.b1));
    const uint32_t c0 = static_cast<uint32_t>(__ffs(rest) - 1), c1 = static_cast<uint32_t>(31 - __clz(rest));
    auto sbit_of = [&](uint32_t b) {
        return b == 0 ? ss.sbit[0] : b == 1 ? ss.sbit[1] : b == 2 ? ss.sbit[2] : ss.sbit[3];
    };
    const uint32_t q0 = sbit_of(op.b0), q1 = sbit_of(op.b1), q2 = sbit_of(c0), q3 = sbit_of(c1);
    auto pos = [&](int r) {
        return ss.p0 ^ ((r & 1) ? ss.sbit[0] : 0u) ^ ((r & 2) ? ss.sbit[1] : 0u) ^ ((r & 4) ? ss.sbit[2] : 0u) ^
               ((r & 8) ? ss.sbit[3] : 0u);
    };
    auto pos_perm = [&](int r) {
        return ss.p0 ^ ((r & 1) ? q0 : 0u) ^ ((r & 2) ? q1 : 0u) ^ ((r & 4) ? q2 : 0u) ^ ((r & 8) ? q3 : 0u);
    };
    if (move)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
            ss.sb[pos(r)] = a[r];
#pragma unroll
        for (int r = 0; r < R; ++r)
            a[r] = ss.sb[pos_perm(r)];
    }
    if (op.kind == F_SWAP2)
        apply_swap2<V, 0, 1>(a, op, j0);
    else
        apply_dense2<V, 0, 1>(a, op, e, j0);
    if (move)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
            ss.sb[pos_perm(r)] = a[r];
#pragma unroll
        for (int r = 0; r < R; ++r)
            a[r] = ss.sb[pos(r)];
    }
}

template <typename V, typename M>
__device__ __forceinline__ void apply_op(V (&a)[R], const FOp &op, const M &e, uint32_t j0, uint64_t cbase,
                                         const StageSlots<V> &ss)
{
    switch (op.kind)
    {
    case F_DENSE2:
    case F_SWAP2: apply_two_target<V>(a, op, e, j0, ss); break;
    case F_DENSE1: dispatch_dense1<V>(a, op, e, j0); break;
    case F_DENSE1R: dispatch_dense1r<V>(a, op, e, j0); break;
    case F_MULI: apply_muli<V>(a, op, j0); break;
    case F_DENSE1X4: apply_dense1x4<V>(a, e); break;
    case F_DENSE1RX4: apply_dense1rx4<V>(a, e); break;
    case F_DENSE1X2: dispatch_x2<V>(a, op, e); break;
    case F_SWAP1: dispatch_swap1<V>(a, op, j0); break;
    case F_PHASE: apply_phase<V>(a, op, e, j0); break;
    default: apply_diag<V>(a, op, e, j0, cbase); break;
    }
}

// A phase run inside a register stage (F_PRUN), on amplitudes already in
// registers. Every diagonal gate multiplies the amplitudes whose bits match a
// pattern by a unit-modulus entry d. Split the pattern into the stage bits
// (which pick one of the thread's 16 amplitudes r) and the rest (fixed for
// the thread: its other local bits and the chunk). On the stage bits,
// [pattern matches r] expands by inclusion-exclusion into signed monomials
// prod_{b in m} r_b, so d^[match] = prod over terms (d or conj d)^(monomial m
// of r); the host emits one term (m, conjugate?, thread/chunk condition,
// entry) per expansion member. A run holds only gates whose patterns have at
// most one stage bit, so its monomials are 1 or r_b and five factors suffice
// (E[0] on every slot, E[1 + b] on the slots with stage bit b); gates wholly
// on the stage bits add 16 per-slot factors computed on the host. Factors start from the run's tables: the thread's
// entry of its thread tables and, per 8-bit group of the chunk index, the
// chunk's entry of the group tables (both built on the host from the terms
// whose conditions fall entirely on those bits); the other terms follow the
// header and are multiplied in one by one. Each factor in use then
// multiplies its slots directly: 16 products for E[0], 8 for a stage bit (a
// QFT run: one stage-bit factor, 8 products per thread). Forming the 16 slot
// factors first would take 31 products for any mix, but keeps more values
// live next to the amplitudes, which made the kernel spill.
// The run's five factors start at one, then take the thread's and the
// chunk's table entries (phase_tables), then the explicit terms one by one
// (phase_term, in the host's order), and finally multiply the slots
// (phase_apply).
template <typename V>
__device__ __forceinline__ void phase_tables(V (&E)[kStageBits + 1], const FOp &head, uint64_t chunk, int tid, int T,
                                             const double2 *tables)
{
#pragma unroll
    for (int e = 0; e <= kStageBits; ++e)
        E[e] = V{1, 0};
    const uint64_t packed = head.gcmask;
    if (packed)
    {
        const double2 *tb = tables + head.lcval;
#pragma unroll
        for (int e = 0; e <= kStageBits; ++e)
            if ((packed >> e) & 1)
            {
                E[e] = cvt<V>(__ldg(tb + tid));
                tb += T;
            }
#pragma unroll
        for (int g = 0; g < kMaxChunkGroups; ++g)
        {
            const uint32_t gm = static_cast<uint32_t>(packed >> (kChunkGroupBits * (g + 1))) & 31u;
            if (gm == 0)
                continue;
            const uint32_t idx = static_cast<uint32_t>(chunk >> (kChunkGroupBits * g)) & ((1u << kChunkGroupBits) - 1);
#pragma unroll
            for (int e = 0; e <= kStageBits; ++e)
                if ((gm >> e) & 1)
                {
                    E[e] = cmul(cvt<V>(__ldg(tb + idx)), E[e]);
                    tb += 1 << kChunkGroupBits;
                }
        }
    }
}

template <typename V, typename M>
__device__ __forceinline__ void phase_term(V (&E)[kStageBits + 1], const FOp &t, uint32_t j0, uint64_t cbase,
                                           const M &entry_at)
{
    if ((j0 & t.lcmask) != t.lcval || (cbase & t.gcmask) != t.gcval)
        return;
    V d = cvt<V>(entry_at(t.moff));
    if (t.b1)
        d.y = -d.y;
    switch (t.b0)
    {
    case 0: E[0] = cmul(d, E[0]); break;
    case 1: E[1] = cmul(d, E[1]); break;
    case 2: E[2] = cmul(d, E[2]); break;
    case 4: E[3] = cmul(d, E[3]); break;
    default: E[4] = cmul(d, E[4]); break;
    }
}

template <typename V, typename M>
__device__ __forceinline__ void phase_apply(V (&a)[R], const FOp &head, const V (&E)[kStageBits + 1],
                                            const M &entry_at)
{
    if (head.b1)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
            a[r] = cmul(cvt<V>(entry_at(head.moff + r)), a[r]);
    }
    const uint32_t used = head.b0;
    if (used & 1)
    {
#pragma unroll
        for (int r = 0; r < R; ++r)
            a[r] = cmul(E[0], a[r]);
    }
#pragma unroll
    for (int b = 0; b < kStageBits; ++b)
        if ((used >> (1 + b)) & 1)
        {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if ((r >> b) & 1)
                    a[r] = cmul(E[1 + b], a[r]);
        }
}

template <typename V, typename M>
__device__ __forceinline__ void phase_inline(V (&a)[R], const FOp &head, const FOp *terms, uint32_t j0,
                                             uint64_t cbase, uint64_t chunk, int tid, int T,
                                             const double2 *tables, const M &entry_at)
{
    V E[kStageBits + 1];
    phase_tables<V>(E, head, chunk, tid, T, tables);
    const int nterms = static_cast<int>(head.lcmask);
    for (int i = 0; i < nterms; ++i)
        phase_term<V>(E, terms[i], j0, cbase, entry_at);
    phase_apply<V>(a, head, E, entry_at);
}

// A run of -1 phases (F_SIGNS): the XOR of the 16-bit slot masks whose
// conditions hold (sign_term per term), then one sign-bit flip per slot on
// the integer pipe (apply_signs).
__device__ __forceinline__ uint32_t sign_term(uint32_t neg, const FOp &t, uint32_t j0, uint64_t cbase)
{
    return ((j0 & t.lcmask) == t.lcval && (cbase & t.gcmask) == t.gcval) ? neg ^ t.moff : neg;
}

template <typename V>
__device__ __forceinline__ void apply_signs(V (&a)[R], uint32_t neg)
{
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        const uint32_t s = ((neg >> r) & 1u) << 31;
        a[r].x = flip_by(a[r].x, s);
        a[r].y = flip_by(a[r].y, s);
    }
}

// What a pass program sees of the chunk it works on.
template <typename V>
struct ChunkCtx
{
    V *sb;              // the chunk in shared memory (swizzled)
    uint64_t cbase;     // physical index of the chunk's first amplitude (local bits zero)
    uint64_t chunk;     // work item (chunk index; batched passes: register and chunk)
    const V *entries;   // batched passes: the register's gate entries; else null
    int tid;
    int T;              // threads of the CTA: 2^(k - kStageBits)
};

// Entries of an op: the pass parameters (one register) or the register's
// block of the entry buffer (batched passes).
template <typename V, bool BATCH>
struct EntryAt
{
    const FPassParams &p;
    const V *entries;
    __device__ __forceinline__ V operator()(int off) const
    {
        if (BATCH)
            return __ldg(entries + off);
        return pool_entry<V>(p, off);
    }
};

// One stage on stage bits s[0..3] (local positions, ascending): every thread
// loads its 16 amplitudes, body(a, j0, slots) applies the stage's ops, the
// amplitudes go back and the CTA synchronises.
template <typename V, typename Body>
__device__ __forceinline__ void run_stage(const ChunkCtx<V> &cx, int s0, int s1, int s2, int s3, Body body)
{
    const int sbits[kStageBits] = {s0, s1, s2, s3};
    uint32_t j0 = static_cast<uint32_t>(cx.tid);
#pragma unroll
    for (int b = 0; b < kStageBits; ++b)
    {
        const uint32_t lo = j0 & ((1u << sbits[b]) - 1u);
        j0 = lo | ((j0 ^ lo) << 1);
    }
    // swz is linear over GF(2) and j0 shares no bit with a stage offset, so
    // swz(j0 | off) = swz(j0) ^ swz(off)
    uint32_t sbit[kStageBits];
#pragma unroll
    for (int b = 0; b < kStageBits; ++b)
        sbit[b] = static_cast<uint32_t>(swz<V>(static_cast<int>(1u << sbits[b])));
    const uint32_t p0 = static_cast<uint32_t>(swz<V>(static_cast<int>(j0)));
    // shared-memory position of slot r (recomputed where needed, so that the
    // 16 positions do not stay live in registers)
    auto pos_of = [&](int r) -> uint32_t {
        uint32_t q = p0;
#pragma unroll
        for (int b = 0; b < kStageBits; ++b)
            if ((r >> b) & 1)
                q ^= sbit[b];
        return q;
    };
    V a[R];
#pragma unroll
    for (int r = 0; r < R; ++r)
        a[r] = cx.sb[pos_of(r)];
    const StageSlots<V> ss{cx.sb, p0, {sbit[0], sbit[1], sbit[2], sbit[3]}};
    body(a, j0, ss);
#pragma unroll
    for (int r = 0; r < R; ++r)
        cx.sb[pos_of(r)] = a[r];
    __syncthreads();
}

// One op of a stage other than the runs (F_SIGNS, F_PRUN): skipped when its
// chunk condition fails.
template <typename V, bool BATCH>
__device__ __forceinline__ void exec_op(const FPassParams &p, const ChunkCtx<V> &cx, V (&a)[R], const FOp &op,
                                        uint32_t j0, const StageSlots<V> &ss)
{
    if ((cx.cbase & op.gcmask) != op.gcval)
        return;
    if (BATCH)
        apply_op<V>(a, op, BufferEntries<V>{cx.entries + op.moff}, j0, cx.cbase, ss);
    else
        apply_op<V>(a, op, PoolEntries<V>{p, op.moff}, j0, cx.cbase, ss);
}

// The run-time stage program: the stages and ops of the parameter block,
// interpreted op by op.
template <typename V, bool BATCH>
__device__ __forceinline__ void run_stages(const FPassParams &p, const ChunkCtx<V> &cx)
{
    const EntryAt<V, BATCH> entry_at{p, cx.entries};
    for (int st = 0; st < p.nstages; ++st)
    {
        const FStage &S = p.stages[st];
        run_stage<V>(cx, S.sbits[0], S.sbits[1], S.sbits[2], S.sbits[3],
                     [&](V (&a)[R], uint32_t j0, const StageSlots<V> &ss) {
                         for (int oi = S.op_begin; oi < S.op_end; ++oi)
                         {
                             const FOp &op = p.ops[oi];
                             if (op.kind == F_SIGNS)
                             {
                                 uint32_t neg = 0;
                                 const int nt = static_cast<int>(op.lcmask);
                                 for (int i = 1; i <= nt; ++i)
                                     neg = sign_term(neg, p.ops[oi + i], j0, cx.cbase);
                                 apply_signs<V>(a, neg);
                                 oi += nt;
                                 continue;
                             }
                             if (op.kind == F_PRUN)
                             {
                                 phase_inline<V>(a, op, p.ops + oi + 1, j0, cx.cbase, cx.chunk, cx.tid, cx.T,
                                                 p.tables, entry_at);
                                 oi += op.lcmask;
                                 continue;
                             }
                             exec_op<V, BATCH>(p, cx, a, op, j0, ss);
                         }
                     });
    }
}

// The chunk loop of a pass. One CTA per chunk at a time; blockDim.x ==
// 2^(k - kStageBits) <= 128, so that three CTAs (12 warps, 3 x 64 KB of
// double-buffered chunks) share an SM for complex128 (168 registers) and four
// for complex64 (128 registers; the batched complex64 pass measured 8% faster
// at 128 than at 168). BATCH: the work items are the chunks of many
// registers of the same size and plan (see FPassParams), each with its own
// gate entries. program(cx) runs the pass's stages on one staged chunk.
template <typename Real, bool BATCH, typename Program>
__device__ __forceinline__ void fused_pass_body(const FPassParams &p, const Program &program)
{
    typedef typename Cx<Real>::T V;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *smem = reinterpret_cast<V *>(smem_raw);
    V *const state = static_cast<V *>(p.state);
    const int k = p.k;
    const int T = 1 << (k - kStageBits);
    const int tid = threadIdx.x;
    const int chunk_elems = 1 << k;
    const int cbits = p.n - k;   // log2(chunks of one register)

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
        uint64_t g = BATCH ? (c & ((1ull << cbits) - 1)) : c;
        for (int i = 0; i < k; ++i)
        {
            const uint64_t lo = g & p.qmasks[i];
            g = lo | ((g ^ lo) << 1);
        }
        return g;
    };
    auto reg_of = [&](uint64_t c) -> uint64_t { return BATCH ? (c >> cbits) : 0ull; };
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
        if (p.from_zero)
        {
            // |0..0>: the chunk holding index 0 starts with a one
#pragma unroll
            for (int m = 0; m < R; ++m)
            {
                const bool one = cb == 0 && m == 0 && tid == 0;
                dst[swz<V>(tid + m * T)] = one ? V{1, 0} : V{0, 0};
            }
        }
        else
        {
            const V *src = state + (reg_of(c) << p.n);
#pragma unroll
            for (int m = 0; m < R; ++m)
                cp_async_amp<V>(dst + swz<V>(tid + m * T), src + (cb | elem_offset(m)));
        }
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
        const uint64_t reg = reg_of(c);
        const V *entries = BATCH ? reinterpret_cast<const V *>(p.mats + reg * p.mat_stride) : nullptr;
        const ChunkCtx<V> cx{sb, cbase, c, entries, tid, T};
        program(cx);

        V *const dst = state + (reg << p.n);
#pragma unroll
        for (int m = 0; m < R; ++m)
            __stcs(dst + (cbase | elem_offset(m)), sb[swz<V>(tid + m * T)]);
        __syncthreads();
        cur ^= 1;
    }
}

} // namespace fdev
} // namespace qcsb
