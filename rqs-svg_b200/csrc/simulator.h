// Host side of the simulator: the state behind one qcs_simulator handle.
#pragma once

#include "qcs_internal.h"
#include "qcs_b200.h"

#include <random>
#include <vector>

namespace qcsb
{

class FusedExecutor;

// Optional per-launch timing with CUDA events on the launching stream.
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
    void begin(cudaStream_t stream, int cls, double bytes);
    void end(cudaStream_t stream);
    void collect(qcs_b200_kernel_times &out);   // synchronizes on the events
    void clear();

  private:
    struct Rec
    {
        int cls;
        double bytes;
        cudaEvent_t a, b;
    };
    cudaEvent_t take();
    std::vector<Rec> recs_;
    std::vector<cudaEvent_t> pool_;
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
    void set_fusion(int mode);
    int fusion() const { return fusion_mode_; }

    // A gate call of the C API, on logical qubits.
    void apply_gate(const char *name, const double *params, int nparams,
                    const std::vector<int> &targets, const std::vector<int> &negctrls,
                    const std::vector<int> &ctrls);

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

    int event_create();
    void event_record(int event_num);
    double event_elapsed(int start, int stop);

    void flush();
    void synchronize();

    qcs_b200_stats stats{};
    KernelTimer timer;

  private:
    void require_allocated(const char *what) const;
    void check_qubit(int q, const char *role) const;
    bool identity_mapping() const;
    void ensure_staging();
    void logical_transfer(double *host, uint64_t count, bool to_host);
    void discard_pending() { pending_.clear(); }

    bool disposed_ = false;
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    int n_ = 0;
    double2 *state_ = nullptr;

    std::vector<int> perm_p2l_, perm_l2p_, initial_perm_p2l_;
    std::vector<int> measured0_, measured1_;   // logical qubits measured as 0 / 1

    uint32_t seed_ = 0;
    std::mt19937_64 engine_;
    std::vector<cudaEvent_t> events_;
    int fusion_mode_ = QCS_FUSION_GREEDY;
    std::vector<GateOp> pending_;
    FusedExecutor *fused_ = nullptr;

    // scratch: reduction partials and results, pinned host mirror,
    // chunk staging for logical-order transfers, sampler tree
    double2 *red_partials_ = nullptr;
    double2 *red_result_ = nullptr;
    double *zsum_partials_ = nullptr;
    double *zsum_result_ = nullptr;
    void *host_pinned_ = nullptr;
    size_t host_pinned_bytes_ = 0;
    double2 *staging_dev_ = nullptr;
    double2 *staging_host_ = nullptr;
    uint64_t staging_count_ = 0;
};

// Fused execution of a queue of gate operations (fused_pass.cu). Returns the
// number of kernels launched; updates the pass counter.
class FusedExecutor
{
  public:
    explicit FusedExecutor(cudaStream_t stream);
    ~FusedExecutor();
    int run(double2 *state, int n, const std::vector<GateOp> &ops, int mode, qcs_b200_stats &stats, KernelTimer &timer);

  private:
    cudaStream_t stream_;
    void *prog_dev_ = nullptr;
    size_t prog_bytes_ = 0;
    void *prog_host_ = nullptr;
};

} // namespace qcsb
