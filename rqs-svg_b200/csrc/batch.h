// Batched execution of many independent circuits (qcs_b200_batch_*).
#pragma once

#include "fused_pass.h"
#include "qcs_b200.h"

#include <vector>

namespace qcsb
{

// One <Z> reduction work item: a slice of up to 2^16 amplitudes of one
// register (register at amplitude offset amp_off, n qubits).
struct BatchZItem
{
    uint64_t amp_off;
    int32_t n;
    uint32_t slice;
};

// Per register: its work items [first, first + count) and where its n
// expectations go.
struct BatchZReg
{
    uint32_t first, count;
    int32_t n;
    uint32_t out_off;
};

constexpr int kBatchZSliceBits = 16;
constexpr int kBatchZPartials = 17;   // total, 8 sums of the thread bits, 8 of the loop bits

template <typename R>
int launch_batch_zsums(const void *arena, const BatchZItem *items, uint32_t num_items, const BatchZReg *regs,
                       uint32_t num_regs, double *partials, double *out, cudaStream_t stream);
// a[reg * stride] = 1 for reg < count (after the registers were zeroed)
template <typename R>
int launch_batch_set_ones(void *base, uint64_t stride, uint32_t count, cudaStream_t stream);

class Batch
{
  public:
    explicit Batch(int amplitude_bits);
    ~Batch();

    uint32_t add_circuit(int n, const qcs_b200_gate *gates, uint32_t count);
    void set_parameters(const double *params, uint64_t count);
    void run();
    void expectation_z(double *out, uint64_t count) const;
    void get_statevector(uint32_t index, double *out, uint64_t count);
    void info(qcs_b200_batch_info *out) const;
    // 0: register passes only; 1 (default): the tuner times 8 x 8 tensor
    // passes per group beside the register passes; 2: tensor passes wherever
    // a pass allows them
    void set_tensor_mode(int mode);
    int tensor_mode() const { return tensor_mode_; }

  private:
    struct Gate
    {
        char name[16];
        int id;      // gate table index (looked up once, at add_circuit)
        int np;
        double params[4];
        int tq[kMaxTargets];
        uint64_t cmask, cval;
    };
    struct Circuit
    {
        int n;
        std::vector<Gate> gates;
        int group = -1;
        uint32_t slot = 0;       // position among its group's registers
        uint64_t z_off = 0;      // first expectation of this circuit
    };
    struct Pass
    {
        FPassParams prm;
        std::vector<FOpSource> src;
        // 8 x 8 tensor pass: per-register stage matrices built on the GPU
        // from each register's entries, then the pass (tensor_pass.cu)
        bool tensor = false;
        TPassParams tp{};
        TBuildParams tb{};
    };
    struct Group
    {
        int n = 0;
        uint64_t signature = 0;
        std::vector<uint32_t> members;   // circuit indices, in slot order
        std::vector<GateOp> shape;       // structural ops (generic parameters)
        int k = 0;
        std::vector<Pass> passes;
        uint32_t stride = 0;             // gate entries per register
        uint64_t mats_off = 0;           // first entry of the group's registers
        uint64_t amp_off = 0;            // first amplitude of the group's registers
    };

    void invalidate();
    void build();
    void plan_group(Group &g, int k, bool tensor = false);
    void ensure_tensor_mats();
    void layout_entries();
    void fill_entries(int only_group = -1);
    void fill_group_range(const Group &g, size_t first, size_t last);
    void enqueue_passes(const Group &g, cudaStream_t s, int *launches);
    void enqueue_group(int gi, cudaStream_t s, int *launches);
    void enqueue_results(cudaStream_t s, int *launches);
    cudaGraphExec_t capture(int gi, int *launches);
    void tune();
    void release_device();

    int amp_bytes_;
    std::vector<Circuit> circuits_;
    std::vector<Group> groups_;
    uint64_t num_params_ = 0;
    bool built_ = false;
    bool ran_ = false;
    bool dirty_ = false;   // parameters set since the entries were last filled

    cudaStream_t stream_ = nullptr;
    void *arena_ = nullptr;
    uint64_t total_amps_ = 0;
    double2 *mats_dev_ = nullptr, *mats_host_ = nullptr;
    uint64_t mats_count_ = 0;
    BatchZItem *zitems_dev_ = nullptr;
    BatchZReg *zregs_dev_ = nullptr;
    uint32_t num_zitems_ = 0;
    double *zpartials_dev_ = nullptr, *zout_dev_ = nullptr, *zout_host_ = nullptr;
    uint64_t zout_count_ = 0;
    // one graph per group (its entries in, its passes) and one for the
    // results (<Z> of every register, out to the host)
    std::vector<cudaGraphExec_t> execs_;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    uint32_t launches_per_run_ = 0;
    double last_ms_ = 0.0;
    int tensor_mode_ = 1;
    // stage matrices of the tensor pass being run (every group's passes run
    // in stream order, each builder right before its pass)
    void *tmats_dev_ = nullptr;
    size_t tmats_bytes_ = 0;
};

} // namespace qcsb
