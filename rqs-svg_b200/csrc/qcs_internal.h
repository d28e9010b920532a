// Internal declarations shared by the host core and the sm_100a kernels.
#pragma once

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "fused_types.h"

namespace qcsb
{

// Largest register the library accepts. 2^34 complex128 amplitudes = 256 GiB,
// above any single B200; the allocator rejects what does not fit first.
constexpr int kMaxQubits = 40;
// Most targets one gate operation may carry (API gates use <= 4).
constexpr int kMaxTargets = 4;
constexpr int kMaxSub = 1 << kMaxTargets;
// Most sub-indices one API gate changes: 4 (two-target gates, and rcccx's
// 0011/0111/1011/1111); rccx changes 3, one-target gates 2.
constexpr int kMaxActive = 4;

std::string strformat(const char *fmt, ...);

// Pass a message to the exception callback installed through
// qcs_set_exception_callback (no-op when none is installed).
void report_error(const char *message);

#define QCSB_CUDA(call)                                                                 \
    do                                                                                  \
    {                                                                                   \
        cudaError_t qcsb_err_ = (call);                                                 \
        if (qcsb_err_ != cudaSuccess)                                                   \
            throw std::runtime_error(::qcsb::strformat("%s failed: %s (%s:%d)", #call,  \
                                                       cudaGetErrorString(qcsb_err_),   \
                                                       __FILE__, __LINE__));            \
    } while (0)

struct cplx
{
    double re, im;
};

// A gate on physical qubits, reduced to the sub-indices it changes.
//
// Sub-index s of a target group has bit i equal to the value of physical
// qubit tq[i] (reference ordering: target i is bit i, src/qcs.cu:255-259).
// act[0..na) lists the sub-indices whose amplitude can change; every other
// sub-index has an identity row and column in the gate's matrix, so only the
// na x na block mat (row-major, output x input) is applied (or its diagonal
// when diag is set). Controls: the gate acts where (index & cmask) == cval.
struct GateOp
{
    int nt = 0;
    int tq[kMaxTargets] = {0, 0, 0, 0};
    uint64_t cmask = 0;
    uint64_t cval = 0;
    bool diag = false;
    int na = 0;
    uint8_t act[kMaxActive] = {};
    cplx mat[kMaxActive * kMaxActive];   // na*na (dense) or na (diag) entries used
    // Number of amplitudes this gate can change in a 2^n register: the
    // algorithmic unit of work (2 * bytes_per_amp * changed amps per gate).
    double changed_amps(int n) const;
};

// Dense 2^nt x 2^nt unitary of an API gate (row = output sub-index).
struct GateMatrix
{
    int nt = 0;
    cplx m[kMaxSub * kMaxSub];   // the first 2^nt x 2^nt entries are set
};

// Gates of the reference API by id (index into the gate table); the name
// lookup throws on unknown names.
int gate_id(const char *name);
int gate_arity(int id);
int gate_nparams(int id);
const char *gate_name(int id);
// Builds the matrix of a gate. Throws on a wrong parameter count.
GateMatrix gate_matrix(int id, const double *params, int nparams);
inline GateMatrix gate_matrix(const char *name, const double *params, int nparams)
{
    return gate_matrix(gate_id(name), params, nparams);
}
inline int gate_arity(const char *name) { return gate_arity(gate_id(name)); }
inline int gate_nparams(const char *name) { return gate_nparams(gate_id(name)); }

// Reduce a dense matrix on targets tq to a GateOp (active set + diag flag).
GateOp make_gate_op(const GateMatrix &g, const int *tq, uint64_t cmask, uint64_t cval);

// ---------------------------------------------------------------- kernels
// Amplitudes are complex128 (R = double, the reference's type) or complex64
// (R = float, a B200 extension). Gate arithmetic runs in R; every norm and
// probability reduction accumulates in FP64. Every launch helper below
// enqueues on `stream` and returns the number of kernels launched.

// Plain path: one kernel applying one GateOp to the whole register.
template <typename R>
int launch_gate_plain(typename Cx<R>::T *state, int n, const GateOp &op, cudaStream_t stream);

// |0..0>, flat (all 1), sequential (a[i] = i), and "entangled" (a[0] = 1,
// leaving the rest as is) state preparation.
template <typename R>
int launch_init_zero(typename Cx<R>::T *state, int n, cudaStream_t stream);
template <typename R>
int launch_init_flat(typename Cx<R>::T *state, int n, cudaStream_t stream);
template <typename R>
int launch_init_sequential(typename Cx<R>::T *state, int n, cudaStream_t stream);
template <typename R>
int launch_set_amplitude(typename Cx<R>::T *state, uint64_t index, double re, double im, cudaStream_t stream);
// Scale every amplitude by sqrt(target / *norm_dev) (norm_dev: a squared norm
// in device memory, written earlier on the same stream).
template <typename R>
int launch_rescale(typename Cx<R>::T *state, int n, double target, const double *norm_dev, cudaStream_t stream);

// Squared-norm sums (P0, P1) of target qubit t over the subspace where
// (index & cmask) == cval, in one launch. partials must hold kReduceBlocks
// double2; result receives one double2 (device memory, or pinned host memory
// the device can write); ticket is a device counter that must be zero before
// the call and is zero again after it. done (pinned host memory, or null)
// receives seq after result has been written, so that the host can wait
// for the result without synchronising the stream.
constexpr int kReduceBlocks = 592;   // 4 x 148 SMs
template <typename R>
int launch_measure_probs(const typename Cx<R>::T *state, int n, int t, uint64_t cmask, uint64_t cval,
                         double2 *partials, double2 *result, unsigned *ticket, unsigned *done, unsigned seq,
                         cudaStream_t stream);

// Zero every amplitude whose bit t differs from keep_value.
template <typename R>
int launch_collapse(typename Cx<R>::T *state, int n, int t, int keep_value, cudaStream_t stream);
// Zero every amplitude i with (i & cmask) != cval: the collapses of several
// measurements in one write pass.
template <typename R>
int launch_collapse_mask(typename Cx<R>::T *state, int n, uint64_t cmask, uint64_t cval, cudaStream_t stream);

// sums[0] = sum |a|^2, sums[1 + q] = sum over amplitudes with bit q set of
// |a|^2 (physical qubits q = 0..n-1). partials must hold
// 512 * (n + 1) doubles; sums receives n + 1 doubles.
template <typename R>
int launch_zsums(const typename Cx<R>::T *state, int n, double *partials, double *sums, cudaStream_t stream);
inline int launch_zsums(const double2 *state, int n, double *partials, double *sums, cudaStream_t stream)
{
    return launch_zsums<double>(state, n, partials, sums, stream);
}

// Gather the register into logical order as complex128: out[l] =
// state[phys(l)], where phys(l) deposits logical bit j of l at physical bit
// l2p[j]; for indices [begin, begin + count). Scatter is the inverse.
template <typename R>
int launch_gather_logical(const typename Cx<R>::T *state, int n, const int *l2p, uint64_t begin,
                          uint64_t count, double2 *out, cudaStream_t stream);
template <typename R>
int launch_scatter_logical(typename Cx<R>::T *state, int n, const int *l2p, uint64_t begin,
                           uint64_t count, const double2 *in, cudaStream_t stream);
// Same-precision conversions for identity-mapped transfers.
template <typename R>
int launch_widen(const typename Cx<R>::T *in, uint64_t count, double2 *out, cudaStream_t stream);
template <typename R>
int launch_narrow(const double2 *in, uint64_t count, typename Cx<R>::T *out, cudaStream_t stream);
// out[k] = state[physical[k]] widened to complex128 (physical indices in
// device memory).
template <typename R>
int launch_gather_indices(const typename Cx<R>::T *state, const uint64_t *physical, uint64_t count, double2 *out,
                          cudaStream_t stream);
// kReduceBlocks x 5 partials: sum conj(x) y (re, im), max |x - y|, sum |x|^2,
// sum |y|^2.
int launch_compare(const double2 *x, const double2 *y, uint64_t count, double *partials, cudaStream_t stream);

// Shot sampler (chain rule over physical qubits in the order given by
// order[0..n)). See sampler.cu for the data layout.
template <typename R>
int launch_sampler(const typename Cx<R>::T *state, int n, const int *order, uint32_t num_shots,
                   const double *uniforms, uint64_t *out_bits, double *tree, int split,
                   cudaStream_t stream);
size_t sampler_tree_bytes(int n, int *split_out);

} // namespace qcsb
