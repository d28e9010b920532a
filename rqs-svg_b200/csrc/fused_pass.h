// Fused passes: the data structures shared by the planner (host), the pass
// kernel (device) and the batch executor. See fused_pass.cu for the
// execution model.
#pragma once

#include "fused_types.h"
#include "qcs_internal.h"

#include <vector>

namespace qcsb
{

constexpr size_t kPlanWindow = 4096;   // ops scanned past the first pending one

// The bits outside a stage that its ops depend on (controls, and the
// targets of diagonal ops, that are not stage bits): local positions and
// physical qubits of the chunk index. A tensor pass (tensor_pass.cu) applies
// the stage as one matrix per assignment of these bits.
struct StageCond
{
    uint32_t lmask = 0;   // local positions (bit l: local qubit l of the pass)
    uint64_t gmask = 0;   // physical qubits that are not local
    uint32_t dense = 0;   // local positions of the stage bits that dense ops target
    uint32_t touch = 0;   // local positions of the stage bits that some op's pattern involves
};

// ---------------------------------------------------------------- tensor passes
// A tensor pass runs the stages of a planned pass as dense 16 x 16 complex
// matrices on the tensor cores (tensor_pass.cu). Each stage's ops depend on
// its 4 stage bits and on a few bits outside the stage (StageCond); the
// stage becomes one matrix per assignment of those condition bits, built on
// the GPU from the pass's ops (stage_matrix_kernel) and applied to every
// 16-amplitude group of the stage by warp-level MMAs.
constexpr int kTensorLocal = 11;       // local qubits of a tensor pass (2^11-amplitude chunks)
// Automatic mode: smaller registers stay on the register path. Measured on
// B200 (layered, CZ-layered and matching-CX circuits, complex128, and HEA
// complex64, device time per flush): tensor passes are 20-36% slower at
// 16-19 qubits, where the register pass's chunks fit one wave of CTAs and
// a tensor pass adds the matrix build; 5-7% faster at 20 qubits (16% slower
// for complex64 HEA), 15-52% faster at 21-23.
constexpr int kTensorMinQubits = 20;      // complex128
constexpr int kTensorMinQubitsC64 = 21;   // complex64
inline int tensor_min_qubits(int amp_bytes) { return amp_bytes == 8 ? kTensorMinQubitsC64 : kTensorMinQubits; }
// Group bits that number a chunk's tiles (tile = warp + 4 x the warp's own
// tile index): local condition bits go to the lowest ones, the warp bits,
// so that with at most two of them every tile of a warp uses one matrix.
constexpr int kTensorTileBits = 3;
constexpr int kTensorMaxCond = 8;      // condition bits of a stage: at most 2^8 matrices
constexpr int kTensorMaxMats = 4096;   // matrices of one pass
// Per matrix: the B fragments of the m16n8k8 products, 12 fragments (real
// part, imaginary part, their sum; x 2 k-steps x 2 n-tiles) x 32 lanes x
// 16 bytes: (b0, b1) in FP64 for complex128, (b0, b1) TF32 high parts and
// (b0, b1) TF32 low parts for complex64; 6 KiB either way.
constexpr int kTensorFragments = 12;
// 8 x 8 stages (three slot bits): one k-step and one n-tile, 3 fragments
// (1.5 KiB) per matrix; 256 rows per chunk in 16 tiles, four per warp, so up
// to four local condition bits pick a tile's matrix (the first two from the
// warp, the others from the warp's tile).
constexpr int kTensor3Fragments = 3;
constexpr int kTensor3TileBits = 4;

struct TStage
{
    uint8_t sbits[kStageBits];   // local positions of slot bits 0..3 (8 x 8 stages: slot bits 0..2, then the
                                 // stage's fourth register bit)
    uint8_t gpos[8];             // local positions of group bits (16 x 16: 0..6, 8 x 8: 0..7); bits 4.. pick the tile
    uint8_t nlc;                 // local condition bits: gpos[4 .. 4 + nlc)
    uint8_t ngc;                 // chunk condition bits: physical qubits gq[0 .. ngc)
    uint8_t gq[kTensorMaxCond];
    uint8_t perm;                // sbits[b] is bit (perm >> 2b) & 3 of the register stage's slot index
    uint8_t pad;
    uint32_t woff;               // first matrix of the stage
};
static_assert(sizeof(TStage) == 28, "TStage layout");

// The matrices of a pass: one per (stage, assignment of its condition bits);
// matrix woff + v of a stage has local condition bit i equal to bit i of v
// and chunk condition bit i equal to bit nlc + i of v.
// complex64 16 x 16 stages on tcgen05 (tensor_pass_tc.cu): per matrix a
// 32 x 32 real B operand [[Mr^T, Mi^T], [-Mi^T, Mr^T]] of TF32 values, in
// the tensor cores' shared-memory layout (K-major, no swizzle: output n,
// input k at byte (n / 8) * 1024 + (k / 8) * 256 + ((k % 8) / 4) * 128 +
// (n % 8) * 16 + (k % 4) * 4), one 4 KiB slab per matrix for the high parts
// and one for the low parts (all high slabs first).
constexpr int kUmmaSlab = 4096;
constexpr int kUmmaMaxLocalCond = 1;   // matrices of a stage side by side in N (two at most)

struct TBuildParams
{
    int nstages;
    uint32_t nmats;
    int tf32;                    // fragments as TF32 high/low parts (complex64 passes)
    int width;                   // slot bits of the stages: 4 (16 x 16) or 3 (8 x 8)
    int umma;                    // B operands of tcgen05 passes instead of mma.sync fragments
    double2 *out;                // nmats x kTensorFragments x 32 lanes x 16 bytes (umma: 2 x nmats slabs)
    // batched passes (8 x 8 stages only): registers whose matrices are built
    // (0: one register, entries in the pass parameters); register r reads
    // its entries at prm.mats + r * prm.mat_stride (float2 entries when
    // batch_float) and writes its nmats matrices after those of r - 1
    uint32_t regs;
    int batch_float;
    uint32_t reg0;               // first register of this launch (grid.y covers at most 65535)
    TStage stages[kFusedMaxStages];
};
// bytes of the matrix buffer per matrix, either format
constexpr size_t kTensorMatrixBytes =
    kTensorFragments * 32 * 16 > 2 * kUmmaSlab ? kTensorFragments * 32 * 16 : 2 * kUmmaSlab;

struct TPassParams
{
    void *state;
    const double2 *mats;
    int n;
    int from_zero;
    int width;                   // 4: 16 x 16 stages, 3: 8 x 8 stages
    int umma;                    // complex64 16 x 16 stages on tcgen05 (tensor_pass_tc.cu)
    uint32_t nmats;              // matrices in mats (umma: the low-part slabs follow the high ones)
    int *err;                    // set to 1 when a tcgen05 pass gives up waiting (host-mapped), or null
    // batched passes (8 x 8 stages only; reg_mats 0: one register): chunk c
    // is chunk c mod 2^batch_cbits of register c >> batch_cbits, whose
    // amplitudes start at register << n and whose matrices start at matrix
    // register * reg_mats
    uint32_t reg_mats;
    int batch_cbits;
    uint64_t chunks;
    uint64_t qmasks[kMaxLocal];
    uint64_t qbit[kMaxLocal];
    int nstages;
    TStage stages[kFusedMaxStages];
    // per stage: shared-memory offsets (swizzled) of the group bits, then of
    // the slot bits (16 x 16: 7 + 4, 8 x 8: 8 + 3)
    uint16_t swz[kFusedMaxStages][12];
};

// Tensor-pass layout of a built pass (amp_bytes 16: complex128, 8:
// complex64) with stages of `width` slot bits (4: 16 x 16, 3: 8 x 8; a
// width-3 layout needs a pass planned with stage_width 3): false when a
// stage depends on more condition bits than a tensor pass handles (or k is
// not kTensorLocal). umma: the layout of a tcgen05 pass (complex64, width 4;
// its rows are threads, so the group bits are ordered for its bank pattern
// and a local condition bit lands on warp bit 0). The matrices are built
// from prm's entries in FP64 (complex64 passes keep them as double2).
bool make_tensor_params(const FPassParams &prm, const std::vector<StageCond> &conds, int amp_bytes, TPassParams &tp,
                        TBuildParams &tb, int width = kStageBits, bool umma = false);
// A tcgen05 pass (complex64, 16 x 16 stages, at most kUmmaMaxLocalCond local
// condition bits per stage); returns the number of kernels launched.
int launch_tc_pass(const TPassParams &tp, cudaStream_t stream);
// Estimated time of a pass on the register path and on the tensor path, in
// one unit (multiply-adds per amplitude at the register path's FP64 rate).
double register_pass_cost(const FPassParams &prm, int amp_bytes);
double tensor_pass_cost(const TPassParams &tp, int amp_bytes);
// Builds the pass's matrices (stage_matrix_kernel) and runs the pass;
// returns the number of kernels launched.
template <typename R>
int launch_stage_matrices(const FPassParams &prm, const TBuildParams &tb, cudaStream_t stream);
template <typename R>
int launch_tensor_pass(const TPassParams &tp, cudaStream_t stream);

struct OpClass
{
    bool fusable;
    uint64_t dense;   // qubits the op is non-diagonal on (dense targets)
    uint64_t diag;    // qubits the op is diagonal on (controls, diag targets)
};

struct PlannedPass
{
    std::vector<int> ops;   // indices into the queue, in execution order
    uint64_t local = 0;     // physical qubits of Q
    int k = 0;              // |Q|
    // stage bits that dense ops may occupy: kStageBits (register stages and
    // 16 x 16 tensor stages) or 3 (8 x 8 tensor stages; the fourth bit of
    // each register-format stage then carries no dense op)
    int stage_width = kStageBits;
};

struct Segment
{
    bool fused;
    int plain_op;           // when !fused
    PlannedPass pass;
    // block width the learned planner chose for the pass: 1 the register
    // path, 3 or 4 tensor stages of 8 x 8 or 16 x 16; -1 lets the executor's
    // cost estimate choose
    int width = -1;
};

// Which queued op an FOp came from, and whether its two targets were
// exchanged to put them in stage-bit order (four ops for the x4 kinds).
struct FOpSource
{
    int op;
    bool swapped;
    int layer[4];   // x4 / x2 kinds: the queued op on each stage bit, -1 for none
};

OpClass classify(const GateOp &op);
// The queue with uncontrolled X gates moved later (exact rewrites of the ops
// they pass; see fused_pass.cu).
std::vector<GateOp> defer_x(const std::vector<GateOp> &q);
std::vector<Segment> plan_greedy(const std::vector<GateOp> &q, int n, int k, int low, int max_ops);
// Fill the kernel parameters of a pass (false when it does not fit the
// parameter block); src, when given, receives one FOpSource per FOp.
// tables: where F_PRUN factor tables are appended (offsets in the ops are
// absolute indices into it; the caller uploads it and sets prm.tables); null
// keeps every term explicit, as batched passes need.
// conds, when given, receives one StageCond per stage of prm.
bool build_params(const std::vector<GateOp> &q, const PlannedPass &pp, int n, int k, FPassParams &prm,
                  std::vector<FOpSource> *src = nullptr, std::vector<double2> *tables = nullptr,
                  std::vector<StageCond> *conds = nullptr);
// Entries an FOp of this kind reads (4 dense 1-target, 16 dense 2-target, 1
// phase, 4 diagonal, 0 permutations), written to m from the GateOp. The x4
// kinds take 4 entries from each of their ops: use layer_entries.
int fop_entries(const GateOp &op, const FOp &f, bool swapped, double2 *m);
// x4 kinds: 4 entries per stage bit (identities where no gate); x2 kinds: 4
// entries for each of the two bits present.
int layer_entries(const std::vector<GateOp> &q, const FOpSource &src, uint8_t kind, double2 *m);
inline bool layer_kind(uint8_t kind)
{
    return kind == F_DENSE1X4 || kind == F_DENSE1RX4 || kind == F_DENSE1X2;
}
// Entries a queued op will need in a pass (the same counts, from the GateOp).
int op_entry_count(const GateOp &op);
// Kernel parameters of a planned pass, cut in two (in order, recursively)
// while a piece does not fit one parameter block; every piece keeps the
// pass's local qubits. False when a single op does not fit. tables as for
// build_params.
bool build_pieces(const std::vector<GateOp> &q, const PlannedPass &pp, int n, std::vector<FPassParams> &params,
                  std::vector<std::vector<FOpSource>> *srcs = nullptr, std::vector<PlannedPass> *pieces = nullptr,
                  std::vector<double2> *tables = nullptr, std::vector<std::vector<StageCond>> *conds = nullptr);
// How one planned pass runs (choose_execution, fused_pass.cu): per piece an
// index into tparams / tbuild (a tensor pass) or -1 (the register path), and
// the estimated cost of the whole. engine 1 runs complex64 16 x 16 stages
// on tcgen05 where a pass allows it, 0 keeps every tensor pass on mma.sync.
struct PassChoice
{
    std::vector<int> tensor;
    std::vector<TPassParams> tparams;
    std::vector<TBuildParams> tbuild;
    double cost = 0.0;
};
void choose_execution(const std::vector<GateOp> &q, const PlannedPass &pp, int n, int amp_bytes, int tensor_mode,
                      std::vector<FPassParams> &params, std::vector<PlannedPass> &pieces,
                      std::vector<std::vector<StageCond>> &conds, std::vector<double2> *tables, PassChoice &out,
                      size_t before, int engine = 1);
int clamp_local_bits(int k, int n);
// Complex64 passes read their entries as float2: round count double2 entries
// in place into the first half of the same memory.
void entries_to_float(double2 *entries, size_t count);
int fused_min_qubits();

template <typename R>
int launch_fused_pass(void *state, int k, const FPassParams &prm, cudaStream_t stream);
template <typename R>
int launch_fused_batch(void *state, int k, const FPassParams &prm, cudaStream_t stream);

} // namespace qcsb
