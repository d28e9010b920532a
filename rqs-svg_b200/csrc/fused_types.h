// Fused-pass data types shared by the host planner and the pass kernels.
// Plain data only, so that device code can include it on its own (under
// NVRTC, which has no standard headers, the fixed-width integer types are
// defined here).
#pragma once

#ifdef __CUDACC_RTC__
typedef unsigned long long uint64_t;
typedef unsigned int uint32_t;
typedef unsigned short uint16_t;
typedef unsigned char uint8_t;
typedef signed char int8_t;
#else
#include <cstdint>
#include <vector_types.h>
#endif

namespace qcsb
{

// Amplitude type of each precision: complex128 (R = double, the reference's
// type) or complex64 (R = float, a B200 extension).
template <typename R>
struct Cx;
template <>
struct Cx<double>
{
    typedef double2 T;
};
template <>
struct Cx<float>
{
    typedef float2 T;
};

constexpr int kFusedMaxOps = 256;       // ops of one pass
constexpr int kFusedMaxEntries = 1024;  // gate entries (complex) of one pass
constexpr int kFusedMaxStages = 96;
constexpr int kLowBits = 3;      // qubits 0..2 are always local: 128-byte runs
constexpr int kStageBits = 4;    // amplitudes per thread in a stage: 2^4
constexpr int kDefaultLocal = 11;
constexpr int kMaxLocal = 12;

enum FKind : uint8_t
{
    F_DENSE1 = 0,  // 2x2 on one stage bit
    F_SWAP1 = 1,   // X: exchange the pair
    F_DENSE2 = 2,  // 4x4 on two stage bits (b0 < b1)
    F_SWAP2 = 3,   // exchange sub-indices 01 and 10
    F_PHASE = 4,   // multiply by entry 0 where the condition bits match
    F_DIAG = 5,    // diagonal on one or two targets anywhere
    F_TERM = 6,    // one term of an inline phase run (F_PRUN; see fused_pass.cu)
    F_DENSE1R = 7, // 2x2 with real entries (RY, H, real U3) on one stage bit
    F_MULI = 9,    // F_PHASE by i (b1 = 0) or -i (b1 = 1) (S, Sdg): exchanges and sign flips
    F_DENSE1X4 = 10,  // an uncontrolled 2x2 gate on each stage bit, in bit order (entries 4b..4b+3 for bit b;
                      // identities on bits without a gate)
    F_DENSE1RX4 = 11, // the same with real entries
    F_PRUN = 12,      // a phase run inside a register stage (fields below)
    F_SIGNS = 13,     // a run of -1 phases (Z, CZ, CCZ): the next lcmask ops are its F_SIGNT terms
    F_SIGNT = 14,     // one -1 phase of an F_SIGNS: slots moff (16-bit mask) under the lc/gc condition
    F_DENSE1X2 = 15,  // uncontrolled complex 2x2 gates on stage bits b0 < b1 (entries 0..3 for b0, 4..7 for b1)
};

// F_PRUN: a run of diagonal gates, each on at most one stage bit, applied to
// the amplitudes in registers through five factors E[0] (all slots) and
// E[1 + b] (slots with stage bit b). Factors whose terms depend only on the
// thread's other local bits come from per-thread tables; those whose terms
// depend only on chunk bits inside one 8-bit group of the chunk index come
// from per-group tables; the remaining terms follow the header as F_TERMs.
//   lcmask: number of F_TERMs that follow
//   lcval:  offset of the run's tables in FPassParams::tables
//   gcmask: bits 0-4 which factors have a thread table (2^(k - 4) entries,
//           indexed by thread); bits 8g+8 .. 8g+12 which have a table for
//           chunk-index group g (256 entries, indexed by chunk bits 8g..8g+7);
//           tables are stored in that order, factors ascending
//   b0:     which factors can differ from 1
//   b1:     1 when 16 per-slot factors (gates whose patterns lie entirely on
//           the stage bits) start at moff
constexpr int kChunkGroupBits = 8;
constexpr int kMaxChunkGroups = 4;

// One gate of a pass. Conditions: (local index & lcmask) == lcval and
// (physical chunk bits & gcmask) == gcval. For F_PHASE the condition includes
// the target bits of the single changed sub-index. The op's matrix entries
// start at moff: in the pass's entry pool, or, for a batched pass, in the
// register's block of the entry buffer.
struct FOp
{
    uint64_t gcmask, gcval;
    uint32_t lcmask, lcval;
    uint8_t kind;
    uint8_t nt;
    uint8_t b0, b1;         // stage-bit positions (dense kinds)
    int8_t loc[2];          // F_DIAG: local bit of target i when it is not a stage bit, else -1
    uint8_t phys[2];        // F_DIAG: physical qubit of target i
    uint16_t moff;
    // register stages: the condition's stage bits, as bits of the amplitude
    // slot r (lcmask/lcval then hold only the other local bits)
    uint8_t smask, sval;
    int8_t spos[2];         // F_DIAG: stage position of target i, -1 when not a stage bit
    uint16_t pad;
};
static_assert(sizeof(FOp) == 40, "FOp layout");

// A stage applies ops [op_begin, op_end) on the amplitudes that differ in its
// stage bits: each thread loads its 2^kStageBits amplitudes into registers,
// runs the ops one by one on them and stores them back.
struct FStage
{
    uint8_t sbits[kStageBits];   // local bit positions of the stage, ascending
    uint16_t op_begin, op_end;
};
static_assert(sizeof(FStage) == 8, "FStage layout");

// Kernel parameters of one pass (passed as a __grid_constant__ block, under
// the 32 KiB kernel parameter limit).
struct FPassParams
{
    void *state;
    int n;
    int k;
    uint64_t chunks;             // work items: chunks of one register, or of all registers of a batch
    uint64_t qmasks[kMaxLocal];  // (1 << qphys[i]) - 1, ascending: chunk deposit
    uint64_t qbit[kMaxLocal];    // 1 << qphys[i]
    int nstages;
    int nops;
    int nentries;
    // batched passes: registers of 2^n amplitudes stored back to back; work
    // item w is chunk w mod 2^(n-k) of register w >> (n-k); register r reads
    // its gate entries at mats + r * mat_stride
    const double2 *mats;         // complex64: each register's block holds float2 entries in its first half
    uint32_t mat_stride;
    int from_zero;               // registers start as |0..0>: build chunks instead of loading them
    const double2 *tables;       // F_PRUN factor tables (device memory), null when no run has any
    FStage stages[kFusedMaxStages];
    FOp ops[kFusedMaxOps];
    double2 entries[kFusedMaxEntries];   // complex64 passes: float2 entries in the first half
};
static_assert(sizeof(FPassParams) <= 32764, "kernel parameter limit");

} // namespace qcsb
