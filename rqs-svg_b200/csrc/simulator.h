// Host side of the simulator: the state behind one qcs_simulator handle.
#pragma once

#include "fused_pass.h"
#include "qcs_internal.h"
#include "qcs_b200.h"

#include <memory>
#include <random>
#include <vector>

namespace qcsb
{

class FusedExecutor;
class CostModel;

// Features of one fused pass as it runs, the cost model's inputs: block
// width (1: the register path, gates one by one; 3 or 4: tensor stages of
// 8 x 8 or 16 x 16 matrices), blocks (stages), arithmetic gates (complex
// multiply-adds on every amplitude), light ops (diagonal phases and
// permutations), target-qubit stride (log2 of the largest stride among the
// local qubits) and log2 of the chunk count (capped at 16).
struct PassFeatures
{
    float f[6];
};

// Optional per-launch timing with CUDA events on the launching stream.
// Fused passes also keep their features, so that their timings can train the
// cost model.
class KernelTimer
{
  public:
    enum Class
    {
        kFused = 0,
        kPlain = 1,
    };
    ~KernelTimer();
    bool enabled = false;
    void begin(cudaStream_t stream, int cls, double bytes, const PassFeatures *features = nullptr);
    void end(cudaStream_t stream);
    void collect(qcs_b200_kernel_times &out);   // synchronizes on the events
    // Fused-pass samples gathered by collect() (and collected now), cleared on read.
    void take_pass_log(std::vector<PassFeatures> &features, std::vector<float> &ms);
    void clear();

  private:
    struct Rec
    {
        int cls;
        double bytes;
        cudaEvent_t a, b;
        PassFeatures feat;
    };
    cudaEvent_t take();
    std::vector<Rec> recs_;
    std::vector<cudaEvent_t> pool_;
    std::vector<PassFeatures> log_feat_;
    std::vector<float> log_ms_;
};

class Simulator
{
  public:
    Simulator();
    ~Simulator();

    // configuration before allocate_memory (reference qcs_simulator fields,
    // src/qcs.cu:2903-2909)
    int num_qubits_cfg = 0;
    int num_clbits = 0;
    std::vector<uint8_t> clbits;

    void allocate_memory();
    void dispose();
    bool disposed() const { return disposed_; }
    bool allocated() const { return state_ != nullptr; }
    int n() const { return n_; }

    void set_mapping(const std::vector<int> &perm_p2l);
    void reinitialize_mapping();

    void set_seed(uint32_t seed);
    void set_precision(int amplitude_bits);
    int precision() const { return amp_bytes_ * 8; }
    void set_fusion(int mode);
    int fusion() const { return fusion_mode_; }

    // A gate call of the C API, on logical qubits.
    void apply_gate(const char *name, const double *params, int nparams, const int *targets, int ntargets,
                    const int *negctrls, int nneg, const int *ctrls, int nctrl);

    int measure(int qubit);
    void reset_qubit(int qubit);

    void set_zero_state();
    void set_flat_state();
    void set_sequential_state();
    void set_entangled_state();
    void set_random_state();
    void clear_measurement_state();

    void save_statevector(const char *path);
    void get_statevector(double *out, uint64_t count);
    void set_statevector(const double *in, uint64_t count);
    void expectation_z(double *out, double *norm);
    void sample(uint32_t num_shots, uint64_t *out);
    // amplitudes at logical indices, as complex128 (re, im interleaved)
    void get_amplitudes(const uint64_t *indices, uint64_t count, double *out);
    // <a|b> over logical indices, max |a_i - b_i|, <a|a> and <b|b>; same
    // register size and device, either precision
    static void compare(Simulator &a, Simulator &b, double *overlap_re, double *overlap_im, double *max_abs_diff,
                        double *norm_a, double *norm_b);

    int event_create();
    void event_record(int event_num);
    double event_elapsed(int start, int stop);

    void flush();
    void synchronize();
    // Physically move the register's amplitudes so that physical qubit q
    // holds logical qubit q (physical SWAPs through the fused passes: the
    // in-HBM qubit permutation), then return the device pointer of the
    // register in logical order, with the stream synchronised.
    void *device_state_in_logical_order();

    void set_planner_options(int max_ops, int local_bits);
    void set_tensor_mode(int mode);
    int tensor_mode() const { return opt_tensor_; }
    void set_tensor_engine(int engine);
    int tensor_engine() const { return opt_engine_; }
    void set_cost_model(CostModel *model);
    FusedExecutor *fused_executor() { return fused_; }

    qcs_b200_stats stats{};
    KernelTimer timer;

  private:
    void require_allocated(const char *what) const;
    void check_qubit(int q, const char *role) const;
    bool identity_mapping() const;
    void ensure_staging();
    void logical_transfer(double *host, uint64_t count, bool to_host);
    const double2 *stage_chunk_out(uint64_t begin, uint64_t cnt);
    void discard_pending()
    {
        pending_.clear();
        pending_gates_ = 0;
    }
    void restore_reference_layout();
    // frees what allocate_memory allocated (after a failure part way)
    void release_allocation();

    bool disposed_ = false;
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    int n_ = 0;
    void *state_ = nullptr;
    int amp_bytes_ = 16;   // 16: complex128 (the reference's), 8: complex64
    bool c64() const { return amp_bytes_ == 8; }

    std::vector<int> perm_p2l_, perm_l2p_, initial_perm_p2l_;
    // logical -> physical map the reference would hold (it differs from ours
    // only through relabelled swaps)
    std::vector<int> ref_l2p_;
    std::vector<int> measured0_, measured1_;   // logical qubits measured as 0 / 1

    uint32_t seed_ = 0;
    std::mt19937_64 engine_;
    std::vector<cudaEvent_t> events_;
    int fusion_mode_ = QCS_FUSION_GREEDY;
    std::vector<GateOp> pending_;
    size_t pending_gates_ = 0;   // queued ops other than deferred collapses
    FusedExecutor *fused_ = nullptr;
    CostModel *model_ = nullptr;
    int opt_max_ops_ = 0, opt_local_bits_ = 0, opt_tensor_ = 1, opt_engine_ = 1;

    // scratch: reduction partials and results, pinned host mirror,
    // chunk staging for logical-order transfers, sampler tree
    double2 *red_partials_ = nullptr;
    unsigned *red_ticket_ = nullptr;   // last-block counter of the measurement reduction
    double *zsum_partials_ = nullptr;
    double *zsum_result_ = nullptr;
    void *host_pinned_ = nullptr;
    size_t host_pinned_bytes_ = 0;
    void *meas_host_ = nullptr;   // pinned: (P0, P1) and the completion flag of a measurement
    unsigned measure_seq_ = 0;    // sequence number of the last measurement's completion flag
    double2 *staging_dev_ = nullptr;
    double2 *staging_host_ = nullptr;
    uint64_t staging_count_ = 0;
    // Squared norm the register should have (complex64 registers; -1 when
    // unknown): 1 after |0..0>, the kept branch's weight after a measurement
    // (the collapse does not renormalise), unchanged by gates. A flush that
    // ran complex64 tensor passes rescales the register back to it (see
    // flush()).
    double norm_target_ = -1.0;
    void restore_norm(uint64_t tensor_passes_before);
    // sampler: marginal tree, uniforms and outcomes, kept between calls and
    // grown when a call needs more (per-call stream-ordered allocations made
    // some calls stall for tenths of a second)
    void *sampler_dev_ = nullptr;
    size_t sampler_bytes_ = 0;
};

// Fused execution of a queue of gate operations (fused_pass.cu). Returns the
// number of kernels launched; updates the pass counter.
class FusedExecutor
{
  public:
    explicit FusedExecutor(cudaStream_t stream);
    ~FusedExecutor();
    int run(void *state, int n, int amp_bytes, const std::vector<GateOp> &ops, int mode, qcs_b200_stats &stats,
            KernelTimer &timer);

    // Planner knobs: 0 keeps the default (256 gates per pass, 11 local qubits).
    void set_options(int max_ops, int local_bits)
    {
        max_ops_ = max_ops;
        local_bits_ = local_bits;
    }
    // a new model plans anew: its plans and the judge's times are dropped
    void set_cost_model(CostModel *model)
    {
        model_ = model;
        learned_plans_.clear();
        judge_.clear();
        plans_.clear();
    }
    // Tensor passes (tensor_pass.cu): 0 never, 1 where the cost estimate
    // favours them (default; 16 x 16 or 8 x 8 stages, whichever it favours),
    // 2 with 16 x 16 stages wherever a pass allows them, 3 with 8 x 8 stages
    // wherever a pass allows them.
    void set_tensor_mode(int mode) { tensor_mode_ = mode; }
    // 1 (default): complex64 16 x 16 stages on tcgen05 where a pass allows
    // it; 0: every tensor pass on warp-level mma.sync
    void set_tensor_engine(int engine) { tensor_engine_ = engine; }
    // Throws when a tcgen05 pass gave up waiting on its tensor cores since
    // the last check (the flag is host-mapped: no copy, read after a sync).
    void check_device_error();

    // Which planner ran the last flush in learned mode (1 = learned,
    // 0 = greedy) and the device times the judge holds for that queue.
    int last_plan_learned = 0;
    double last_greedy_ms = -1.0, last_learned_ms = -1.0;

  private:
    struct JudgeEntry
    {
        double greedy_ms = -1.0;
        double learned_ms = -1.0;
    };
    // The launches of one flush as planned. A plan is kept with the queue it
    // was made for (every field of every op, matrices bit for bit), so that
    // the same queue again -- a circuit re-run for every sample -- launches
    // without planning.
    struct FlushPlan
    {
        std::vector<GateOp> queued;   // the queue as given: the key
        uint64_t hash = 0;
        int n = 0, amp_bytes = 0, k = 0, max_ops = 0, tensor_mode = 0, tensor_engine = 0;
        int tag = 0;                  // 0 greedy planner, 1 learned plan, 2 greedy plan chosen by the judge
        std::vector<GateOp> ops;      // after defer_x: plain steps index into them
        std::vector<FPassParams> params;
        std::vector<int> ks;          // local qubits of each pass
        std::vector<int> tensor_of;   // per pass: index into tparams / tbuild, or -1
        std::vector<TPassParams> tparams;
        std::vector<TBuildParams> tbuild;
        std::vector<long> steps;      // launch order: >= 0 a pass, < 0 plain op -1 - step
        std::vector<double2> tables;  // phase-run tables of the passes
        // The tensor passes' stage matrices, kept on the device from the
        // plan's first replay on (every tensor pass at its own offset), so
        // that later replays launch no matrix builds. Freed with the plan
        // (cudaFree waits for the kernels that may still read it).
        void *mats = nullptr;
        std::vector<size_t> mat_off;  // bytes, per tensor pass
        bool mats_built = false;
        FlushPlan() = default;
        FlushPlan(const FlushPlan &) = delete;
        FlushPlan &operator=(const FlushPlan &) = delete;
        ~FlushPlan()
        {
            if (mats != nullptr)
                cudaFree(mats);
        }
    };
    static constexpr size_t kKeptMatsBytes = size_t(256) << 20;   // device memory of one kept plan's matrices
    static constexpr size_t kKeptMatsFreeReserve = size_t(256) << 20;   // left free beside kept matrices
    void settle_judge();
    const double2 *upload_tables(const std::vector<double2> &tables);
    int launch_plan_step(FlushPlan &plan, long st, void *state, const double2 *tables_dev, qcs_b200_stats &stats,
                         KernelTimer &timer, const PassFeatures *features);
    FlushPlan *find_plan(const std::vector<GateOp> &queued, uint64_t hash, int n, int amp_bytes, int k,
                         int max_ops, int tag);
    int replay(FlushPlan &plan, void *state, qcs_b200_stats &stats, KernelTimer &timer);
    static constexpr size_t kKeptPlans = 8;
    static constexpr size_t kKeptPlanBytes = size_t(64) << 20;   // host memory of one kept plan's launches
    std::vector<std::unique_ptr<FlushPlan>> plans_;
    size_t plans_next_ = 0;   // the slot the next kept plan replaces once all are used

    cudaStream_t stream_;
    // phase-run tables: built on the host with a flush's plan, staged in
    // pinned memory, copied to the device once per flush
    double2 *tables_host_ = nullptr;
    double2 *tables_dev_ = nullptr;
    size_t tables_cap_ = 0;
    cudaEvent_t tables_copied_ = nullptr;
    int max_ops_ = 0;
    int local_bits_ = 0;
    int tensor_mode_ = 1;
    int tensor_engine_ = 1;
    int *err_host_ = nullptr;   // host-mapped error flag of tcgen05 passes
    int *err_dev_ = nullptr;
    // matrices of the tensor pass being run: every pass's builder writes
    // them right before the pass reads them, in stream order
    double2 *mats_dev_ = nullptr;
    size_t mats_cap_ = 0;   // matrices
    CostModel *model_ = nullptr;
    // "measured device time is the judge": per queue signature, the device
    // time of a flush under each planner; once both are known the faster one
    // is used for that queue from then on.
    std::vector<std::pair<uint64_t, JudgeEntry>> judge_;
    // learned plans by queue signature (with size, precision and options)
    std::vector<std::pair<uint64_t, std::vector<Segment>>> learned_plans_;
    cudaEvent_t judge_a_ = nullptr, judge_b_ = nullptr;
    uint64_t pending_sig_ = 0;
    int pending_learned_ = -1;
};

} // namespace qcsb
