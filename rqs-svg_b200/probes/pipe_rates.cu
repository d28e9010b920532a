// Arithmetic pipe rates of the GPU, the denominators of the tensor passes'
// rooflines: FP64 FMA (DFMA), FP64 tensor (DMMA m16n8k8), both at once in
// different warps of one CTA (do they share a datapath?), TF32 mma.sync
// m16n8k8, and packed FP32 (fma.rn.f32x2). Every operand stays in
// registers; fixed trip counts; every result is stored, so nothing is dead
// code. Grid: SMs x {4, 8} CTAs of 128 threads. Prints TFLOP/s per probe.
//
//   make -C rqs-svg_b200 probes && rqs-svg_b200/bin/pipe_rates
#include <cstdio>
#include <cuda_runtime.h>
#define ITERS 4096

__device__ __forceinline__ void dmma(double (&d)[4], double a0, double a1, double a2, double a3, double b0, double b1) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3]) : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}
__device__ __forceinline__ void tmma(float (&d)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0, unsigned b1) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3]) : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// mode 0: all warps DFMA; 1: all warps DMMA; 2: warps 0,1 DMMA + 2,3 DFMA; 3: TF32 mma; 4: FFMA2
__global__ void __launch_bounds__(128) probe(int mode, double *out, float s) {
  const int warp = threadIdx.x >> 5;
  double acc = 0;
  bool do_dmma = mode == 1 || (mode == 2 && warp < 2);
  bool do_dfma = mode == 0 || (mode == 2 && warp >= 2);
  if (do_dmma) {
    double d[4][4] = {};
    double a = threadIdx.x * 1e-3, b = 1.0 + s;
    for (int i = 0; i < ITERS; ++i) {
#pragma unroll
      for (int c = 0; c < 4; ++c) dmma(d[c], a, a + c, a, a, b, b);
    }
    for (int c = 0; c < 4; ++c) acc += d[c][0] + d[c][1] + d[c][2] + d[c][3];
  }
  if (do_dfma) {
    double x[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) x[c] = threadIdx.x + c;
    const double m = 1.0 + s * 1e-9, q = s;
    // 16 chains x 64 = same flops per warp as DMMA mode's 4 chains x 1 mma (16*8*8*2 per mma /32 lanes = 64 fma per lane)
    for (int i = 0; i < ITERS; ++i) {
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 16; ++c) x[c] = fma(x[c], m, q);
    }
    for (int c = 0; c < 16; ++c) acc += x[c];
  }
  if (mode == 3) {
    float d[4][4] = {};
    unsigned a = __float_as_uint(1.0f + threadIdx.x), b = __float_as_uint(s);
    for (int i = 0; i < ITERS; ++i) {
#pragma unroll
      for (int c = 0; c < 4; ++c) tmma(d[c], a, a + c, a, a, b, b);
    }
    for (int c = 0; c < 4; ++c) acc += d[c][0] + d[c][1] + d[c][2] + d[c][3];
  }
  if (mode == 4) {
    unsigned long long x[16];
    unsigned long long m, q;
    asm("mov.b64 %0, {%1, %2};" : "=l"(m) : "f"(1.0f + s * 1e-9f), "f"(1.0f));
    asm("mov.b64 %0, {%1, %2};" : "=l"(q) : "f"(s), "f"(s));
#pragma unroll
    for (int c = 0; c < 16; ++c) asm("mov.b64 %0, {%1, %2};" : "=l"(x[c]) : "f"((float)threadIdx.x), "f"((float)c));
    for (int i = 0; i < ITERS; ++i) {
#pragma unroll
      for (int r = 0; r < 16; ++r)
#pragma unroll
        for (int c = 0; c < 16; ++c) asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(x[c]) : "l"(m), "l"(q));
    }
    for (int c = 0; c < 16; ++c) { float lo, hi; asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(x[c])); acc += lo + hi; }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

int main() {
  int sms; cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  const char *names[] = {"DFMA (all warps)", "DMMA m16n8k8 (all warps)", "DMMA warps 0-1 + DFMA warps 2-3", "TF32 mma.sync m16n8k8", "FFMA2 f32x2"};
  for (int per_sm : {4, 8}) {
    int blocks = sms * per_sm;
    double *out; cudaMalloc(&out, sizeof(double) * blocks * 128);
    for (int mode = 0; mode < 5; ++mode) {
      cudaEvent_t e0, e1; cudaEventCreate(&e0); cudaEventCreate(&e1);
      probe<<<blocks, 128>>>(mode, out, 0.5f);
      cudaEventRecord(e0);
      probe<<<blocks, 128>>>(mode, out, 0.5f);
      cudaEventRecord(e1);
      cudaError_t err = cudaEventSynchronize(e1);
      float ms; cudaEventElapsedTime(&ms, e0, e1);
      // flops per warp per iteration: DMMA 4 chains x 16*8*8*2; DFMA 32 lanes x 256 fma x 2; TF32 same as DMMA; FFMA2 32*256*2*2
      double warps = blocks * 4.0;
      double per_warp_iter = 0;
      if (mode == 0) per_warp_iter = 32 * 128 * 2;
      if (mode == 1 || mode == 3) per_warp_iter = 4 * 16 * 8 * 8 * 2;
      if (mode == 2) per_warp_iter = (4 * 16 * 8 * 8 * 2 + 32 * 128 * 2) / 2.0;
      if (mode == 4) per_warp_iter = 32 * 256 * 2 * 2;
      double tf = warps * per_warp_iter * ITERS / (ms * 1e-3) / 1e12;
      printf("%d CTAs/SM  %-34s %8.3f ms  %8.2f TFLOP/s  (%s)\n", per_sm, names[mode], ms, tf, cudaGetErrorString(err));
    }
    cudaFree(out);
  }
  return 0;
}
