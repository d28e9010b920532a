// Host orchestration of the simulator.
//
// Semantics follow the reference's simulator_core (src/qcs.cu:1685-2899) at
// one process: logical<->physical qubit mapping, measured qubits acting as
// implicit controls of later gates (and cancelling gates whose explicit
// control contradicts them), cached re-measurement without a random draw,
// measurement by (P0, P1) reduction + host mt19937_64 draw + zeroing of the
// other branch without renormalisation, and the state preparations.
//
// Execution differs: gate calls become GateOps on physical qubits. In plain
// mode each is launched at once (one kernel per gate, like the reference);
// otherwise they are queued and executed by the fused executor when a result
// is needed.

#include "simulator.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <functional>

#include <curand.h>

// Run a templated launch helper on the register in its precision.
#define QCSB_ON_STATE(fn, ...)                                                   \
    (c64() ? fn<float>(static_cast<float2 *>(state_), __VA_ARGS__)             \
           : fn<double>(static_cast<double2 *>(state_), __VA_ARGS__))

namespace qcsb
{
namespace
{

constexpr uint64_t kStagingAmps = 1ull << 22;   // 64 MiB per staging buffer
constexpr size_t kScratchReserve = 256ull << 20;
constexpr size_t kMeasureFlagOffset = 16;   // in the measurement's pinned buffer, after the (P0, P1) result
constexpr size_t kMeasureHostBytes = 64;

bool contains(const std::vector<int> &v, int x) { return std::find(v.begin(), v.end(), x) != v.end(); }

int env_fusion_mode()
{
    const char *e = std::getenv("QCS_FUSION");
    if (e == nullptr || e[0] == '\0')
        return QCS_FUSION_GREEDY;
    const int m = std::atoi(e);
    if (m < QCS_FUSION_PLAIN || m > QCS_FUSION_LEARNED)
        return QCS_FUSION_GREEDY;
    return m;
}

// QCS_TENSOR_PASSES: the tensor-pass mode of new simulators (0-3; unset or
// out of range: 1, automatic)
int env_tensor_mode()
{
    const char *e = std::getenv("QCS_TENSOR_PASSES");
    if (e == nullptr || e[0] == '\0')
        return 1;
    const int m = std::atoi(e);
    return (m >= 0 && m <= 3) ? m : 1;
}

} // namespace

Simulator::Simulator()
{
    // reference setup(), src/qcs.cu:1789-1858, at a single process: the
    // device is the current one, the seed comes from std::random_device.
    QCSB_CUDA(cudaGetDevice(&device_));
    QCSB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    std::random_device rd;
    set_seed(rd());
    fusion_mode_ = env_fusion_mode();
    opt_tensor_ = env_tensor_mode();
}

Simulator::~Simulator()
{
    if (!disposed_)
    {
        try
        {
            dispose();
        }
        catch (...)
        {
        }
    }
}

void Simulator::set_seed(uint32_t seed)
{
    seed_ = seed;
    engine_ = std::mt19937_64(seed);
}

void Simulator::set_precision(int amplitude_bits)
{
    if (amplitude_bits != 128 && amplitude_bits != 64)
        throw std::runtime_error(strformat("precision %d is not 128 (complex128) or 64 (complex64)", amplitude_bits));
    if (allocated())
        throw std::runtime_error("set_precision: memory is already allocated");
    amp_bytes_ = amplitude_bits / 8;
}

void Simulator::set_fusion(int mode)
{
    if (mode < QCS_FUSION_PLAIN || mode > QCS_FUSION_LEARNED)
        throw std::runtime_error(strformat("fusion mode %d is not one of 0 (plain), 1 (greedy), 2 (learned)", mode));
    if (allocated())
        flush();
    fusion_mode_ = mode;
}

void Simulator::require_allocated(const char *what) const
{
    if (disposed_)
        throw std::runtime_error(strformat("%s: the simulator has been disposed", what));
    if (state_ == nullptr)
        throw std::runtime_error(strformat("%s: allocate_memory must be called first", what));
}

void Simulator::check_qubit(int q, const char *role) const
{
    if (q < 0 || q >= n_)
        throw std::runtime_error(strformat("%s qubit %d is out of range [0, %d)", role, q, n_));
}

void Simulator::allocate_memory()
{
    // reference allocate_memory, src/qcs.cu:1887-1998
    if (disposed_)
        throw std::runtime_error("allocate_memory: the simulator has been disposed");
    const int n = num_qubits_cfg;
    if (state_ != nullptr)
        throw std::runtime_error(strformat("num_qubits is already set %d > 0", n_));
    if (n <= 0)
        throw std::runtime_error("allocate_memory: set_num_qubits must be called with a positive count first");
    size_t free_b = 0, total_b = 0;
    QCSB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t usable = free_b > kScratchReserve ? free_b - kScratchReserve : 0;
    int max_n = 0;
    while (max_n < 62 && ((size_t)amp_bytes_ << (max_n + 1)) <= usable)
        ++max_n;
    if (max_n > kMaxQubits)
        max_n = kMaxQubits;
    if (n > max_n)
        throw std::runtime_error(strformat("num_qubits(%d) > max_num_qubits_local_device(%d) + log_num_procs(0)", n, max_n));
    QCSB_CUDA(cudaGetDevice(&device_));
    // A failure part way (device or pinned memory exhausted) releases what
    // this call allocated and leaves the simulator unallocated: a later
    // allocate_memory may retry, and every other call reports that
    // allocate_memory must come first, so no kernel ever sees a missing
    // buffer. QCS_FAIL_ALLOC_AFTER=k makes allocation k (counted from 0) of
    // this call fail as if memory were exhausted, the host-side test hook
    // of this path.
    const char *fail_env = std::getenv("QCS_FAIL_ALLOC_AFTER");
    const int fail_at = (fail_env != nullptr && fail_env[0] != '\0') ? std::atoi(fail_env) : -1;
    int allocation = 0;
    auto injected = [&](const char *what) {
        if (allocation++ == fail_at)
            throw std::runtime_error(strformat("allocate_memory: %s: injected failure of allocation %d (QCS_FAIL_ALLOC_AFTER)",
                                               what, fail_at));
    };
    try
    {
        injected("cudaMalloc of the state");
        QCSB_CUDA(cudaMalloc(&state_, (size_t)amp_bytes_ << n));
        n_ = n;
        perm_p2l_.assign(n, 0);
        perm_l2p_.assign(n, 0);
        ref_l2p_.assign(n, 0);
        for (int q = 0; q < n; ++q)
            perm_p2l_[q] = perm_l2p_[q] = ref_l2p_[q] = q;
        reinitialize_mapping();
        injected("cudaMalloc of the reduction partials");
        QCSB_CUDA(cudaMalloc(&red_partials_, sizeof(double2) * kReduceBlocks));
        injected("cudaMalloc of the reduction ticket");
        QCSB_CUDA(cudaMalloc(&red_ticket_, sizeof(unsigned)));
        QCSB_CUDA(cudaMemset(red_ticket_, 0, sizeof(unsigned)));
        injected("cudaMalloc of the <Z> partials");
        QCSB_CUDA(cudaMalloc(&zsum_partials_, sizeof(double) * 512 * (kMaxQubits + 1)));
        injected("cudaMalloc of the <Z> sums");
        QCSB_CUDA(cudaMalloc(&zsum_result_, sizeof(double) * (kMaxQubits + 1)));
        injected("cudaMallocHost of the host buffer");
        QCSB_CUDA(cudaMallocHost(&host_pinned_, 1 << 16));
        host_pinned_bytes_ = 1 << 16;
        // the measurement's result and completion flag: written only by the
        // measurement kernel
        injected("cudaMallocHost of the measurement result");
        QCSB_CUDA(cudaMallocHost(&meas_host_, kMeasureHostBytes));
        *reinterpret_cast<unsigned *>(static_cast<char *>(meas_host_) + kMeasureFlagOffset) = 0;
        measure_seq_ = 0;
        injected("cudaHostAlloc of the pass error flag");
        fused_ = new FusedExecutor(stream_);
        fused_->set_options(opt_max_ops_, opt_local_bits_);
        fused_->set_tensor_mode(opt_tensor_);
        fused_->set_tensor_engine(opt_engine_);
        fused_->set_cost_model(model_);
        set_zero_state();
    }
    catch (...)
    {
        release_allocation();
        throw;
    }
}

void Simulator::release_allocation()
{
    if (stream_)
        cudaStreamSynchronize(stream_);
    delete fused_;
    fused_ = nullptr;
    cudaFree(state_);
    cudaFree(red_partials_);
    cudaFree(red_ticket_);
    cudaFree(zsum_partials_);
    cudaFree(zsum_result_);
    if (host_pinned_)
        cudaFreeHost(host_pinned_);
    if (meas_host_)
        cudaFreeHost(meas_host_);
    state_ = nullptr;
    red_partials_ = nullptr;
    red_ticket_ = nullptr;
    zsum_partials_ = zsum_result_ = nullptr;
    host_pinned_ = nullptr;
    host_pinned_bytes_ = 0;
    meas_host_ = nullptr;
    n_ = 0;
    // the failure was reported by the exception; an exhausted allocation
    // must not surface again as the error of a later launch check
    (void)cudaGetLastError();
}

void Simulator::set_planner_options(int max_ops, int local_bits)
{
    if (max_ops < 0 || local_bits < 0)
        throw std::runtime_error("planner options must be non-negative (0 keeps the default)");
    if (allocated())
        flush();
    opt_max_ops_ = max_ops;
    opt_local_bits_ = local_bits;
    if (fused_)
        fused_->set_options(max_ops, local_bits);
}

void Simulator::set_tensor_mode(int mode)
{
    if (mode < 0 || mode > 3)
        throw std::runtime_error(strformat(
            "tensor pass mode %d is not 0 (never), 1 (auto), 2 (always, 16 x 16) or 3 (always, 8 x 8)", mode));
    if (allocated())
        flush();
    opt_tensor_ = mode;
    if (fused_)
        fused_->set_tensor_mode(mode);
}

void Simulator::set_tensor_engine(int engine)
{
    if (engine < 0 || engine > 1)
        throw std::runtime_error(strformat("tensor engine %d is not 0 (mma.sync) or 1 (tcgen05 where possible)", engine));
    if (allocated())
        flush();
    opt_engine_ = engine;
    if (fused_)
        fused_->set_tensor_engine(engine);
}

void Simulator::set_cost_model(CostModel *model)
{
    if (allocated())
        flush();
    model_ = model;
    if (fused_)
        fused_->set_cost_model(model);
}

void Simulator::dispose()
{
    // reference dispose, src/qcs.cu:2836-2845 (MPI_Finalize has no
    // counterpart in a single process)
    if (disposed_)
        throw std::runtime_error("dispose: the simulator has already been disposed");
    discard_pending();
    disposed_ = true;
    if (stream_)
        cudaStreamSynchronize(stream_);
    delete fused_;
    fused_ = nullptr;
    cudaFree(state_);
    cudaFree(red_partials_);
    cudaFree(red_ticket_);
    red_ticket_ = nullptr;
    cudaFree(zsum_partials_);
    cudaFree(zsum_result_);
    cudaFree(staging_dev_);
    cudaFree(sampler_dev_);
    sampler_dev_ = nullptr;
    sampler_bytes_ = 0;
    if (host_pinned_)
        cudaFreeHost(host_pinned_);
    if (meas_host_)
        cudaFreeHost(meas_host_);
    meas_host_ = nullptr;
    if (staging_host_)
        cudaFreeHost(staging_host_);
    state_ = nullptr;
    red_partials_ = staging_dev_ = staging_host_ = nullptr;
    zsum_partials_ = zsum_result_ = nullptr;
    host_pinned_ = nullptr;
    for (cudaEvent_t e : events_)
        cudaEventDestroy(e);
    events_.clear();
    if (stream_)
        cudaStreamDestroy(stream_);
    stream_ = nullptr;
    n_ = 0;
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess)
        throw std::runtime_error(strformat("dispose: %s", cudaGetErrorString(err)));
}

void Simulator::set_mapping(const std::vector<int> &perm_p2l)
{
    // reference qcs_simulator_set_mapping_cxx, src/qcs.cu:3045-3062
    if (num_qubits_cfg <= 0)
        throw std::runtime_error("set_num_qubits must be called before set_mapping");
    if ((int)perm_p2l.size() != num_qubits_cfg)
        throw std::runtime_error(strformat("mapping size %d does not match num_qubits %d", (int)perm_p2l.size(), num_qubits_cfg));
    std::vector<bool> used(num_qubits_cfg, false);
    for (int l : perm_p2l)
    {
        if (l < 0 || l >= num_qubits_cfg)
            throw std::runtime_error(strformat("mapping value %d is out of range [0, %d)", l, num_qubits_cfg));
        if (used[l])
            throw std::runtime_error(strformat("mapping value %d appears multiple times", l));
        used[l] = true;
    }
    initial_perm_p2l_ = perm_p2l;
}

void Simulator::reinitialize_mapping()
{
    // reference reinitialize_mapping, src/qcs.cu:1860-1885: the mapping
    // becomes the initial one (identity when none was set) and the data stay
    // where they are. Relabelled swaps (apply_gate) moved logical qubits to
    // other physical bits here but not in the reference; logical qubit q sat
    // at the reference's physical bit ref(q) and sits at ours(q), so the
    // reference's bit v is our bit ours(ref^-1(v)). After the reset the
    // reference holds q at init(q), i.e. at our bit ours(ref^-1(init(q))).
    if (n_ == 0)
        return;
    std::vector<int> init_l2p(n_);
    if (initial_perm_p2l_.empty())
    {
        for (int q = 0; q < n_; ++q)
            init_l2p[q] = q;
    }
    else
    {
        if ((int)initial_perm_p2l_.size() != n_)
            throw std::runtime_error(strformat("mapping size %d does not match num_qubits %d", (int)initial_perm_p2l_.size(), n_));
        for (int p = 0; p < n_; ++p)
            init_l2p[initial_perm_p2l_[p]] = p;
    }
    std::vector<int> ref_p2l(n_);
    for (int q = 0; q < n_; ++q)
        ref_p2l[ref_l2p_[q]] = q;
    std::vector<int> ours(n_);
    for (int q = 0; q < n_; ++q)
        ours[q] = perm_l2p_[ref_p2l[init_l2p[q]]];
    perm_l2p_ = ours;
    for (int q = 0; q < n_; ++q)
        perm_p2l_[perm_l2p_[q]] = q;
    ref_l2p_ = init_l2p;
}

bool Simulator::identity_mapping() const
{
    for (int q = 0; q < n_; ++q)
        if (perm_l2p_[q] != q)
            return false;
    return true;
}

void Simulator::apply_gate(const char *name, const double *params, int nparams, const int *targets, int ntargets,
                           const int *negctrls, int nneg, const int *ctrls, int nctrl)
{
    require_allocated("gate");
    ++stats.gates_received;
    const int id = gate_id(name);
    const int arity = gate_arity(id);
    if (ntargets != arity)
        throw std::runtime_error(strformat("gate %s takes %d target qubits, got %d", name, arity, ntargets));
    uint64_t seen = 0;
    auto claim = [&](const int *qs, int count, const char *role) {
        uint64_t mask = 0;
        for (int i = 0; i < count; ++i)
        {
            const int q = qs[i];
            check_qubit(q, role);
            if ((seen >> q) & 1)
                throw std::runtime_error(
                    strformat("gate %s: qubit %d appears more than once among targets and controls", name, q));
            seen |= 1ull << q;
            mask |= 1ull << q;
        }
        return mask;
    };
    const uint64_t tmask = claim(targets, ntargets, "target");
    uint64_t ctl[2] = {claim(negctrls, nneg, "negative control"), claim(ctrls, nctrl, "control")};
    const GateMatrix gm = gate_matrix(id, params, nparams);

    // Measured qubits that are not targets become controls on their measured
    // value; a contradicting explicit control cancels the gate
    // (reference prepare_control_qubit_num_list, src/qcs.cu:2161-2204).
    std::vector<int> *measured[2] = {&measured0_, &measured1_};
    bool condition = true;
    for (int v = 0; v < 2; ++v)
        for (int q : *measured[v])
        {
            const uint64_t bit = 1ull << q;
            if (tmask & bit)
                continue;   // a gate on a measured qubit makes it unmeasured
            if (ctl[1 - v] & bit)
                condition = false;
            else
                ctl[v] |= bit;
        }
    if (!condition)
        return;   // measured lists are left as they were (src/qcs.cu:2689-2691)
    for (int v = 0; v < 2; ++v)
        measured[v]->erase(std::remove_if(measured[v]->begin(), measured[v]->end(),
                                          [&](int q) { return (tmask >> q) & 1; }),
                           measured[v]->end());

    uint64_t cmask = 0, cval = 0;
    for (int v = 0; v < 2; ++v)
        for (uint64_t m = ctl[v]; m; m &= m - 1)
        {
            const int p = perm_l2p_[__builtin_ctzll(m)];
            cmask |= 1ull << p;
            if (v)
                cval |= 1ull << p;
        }
    int tq[kMaxTargets] = {0, 0, 0, 0};
    for (int i = 0; i < arity; ++i)
        tq[i] = perm_l2p_[targets[i]];
    const GateOp op = make_gate_op(gm, tq, cmask, cval);

    if (op.na == 0)
        return;   // identity on every amplitude
    if (fusion_mode_ != QCS_FUSION_PLAIN && arity == 2 && nneg == 0 && nctrl == 0 && std::strcmp(name, "swap") == 0)
    {
        // An uncontrolled SWAP exchanges which physical bits hold the two
        // logical qubits: exact, and no data moves. Implicit controls from
        // measured qubits do not matter here, since the branch they exclude
        // is all zeros and stays zeros under any qubit permutation.
        std::swap(perm_l2p_[targets[0]], perm_l2p_[targets[1]]);
        perm_p2l_[perm_l2p_[targets[0]]] = targets[0];
        perm_p2l_[perm_l2p_[targets[1]]] = targets[1];
        ++stats.gates_applied;
        return;
    }
    ++stats.gates_applied;
    stats.algorithmic_bytes += 2.0 * amp_bytes_ * op.changed_amps(n_);
    if (fusion_mode_ == QCS_FUSION_PLAIN)
    {
        if (timer.enabled)
            timer.begin(stream_, KernelTimer::kPlain, 2.0 * amp_bytes_ * op.changed_amps(n_));
        const int k = QCSB_ON_STATE(launch_gate_plain, n_, op, stream_);
        if (timer.enabled)
            timer.end(stream_);
        stats.kernel_launches += k;
        stats.plain_gate_kernels += k;
    }
    else
    {
        pending_.push_back(op);
        ++pending_gates_;
    }
}

void Simulator::flush()
{
    if (pending_.empty() || state_ == nullptr)
        return;
    if (pending_gates_ == 0)
    {
        // only collapses of measurements (each on its own qubit, since a
        // re-measurement with no gate between is answered from the cache):
        // one write pass zeroes every branch they exclude
        uint64_t cmask = 0, cval = 0;
        for (const GateOp &z : pending_)
        {
            cmask |= 1ull << z.tq[0];
            if (z.act[0] == 0)
                cval |= 1ull << z.tq[0];
        }
        stats.kernel_launches += QCSB_ON_STATE(launch_collapse_mask, n_, cmask, cval, stream_);
        discard_pending();
        return;
    }
    if (c64() && norm_target_ < 0.0 && opt_tensor_ != 0 && fusion_mode_ != QCS_FUSION_PLAIN)
    {
        // the norm to restore after this flush is the register's norm now
        stats.kernel_launches += launch_zsums<float>(static_cast<const float2 *>(state_), n_, zsum_partials_,
                                                     zsum_result_, stream_);
        double *h = static_cast<double *>(host_pinned_);
        QCSB_CUDA(cudaMemcpyAsync(h, zsum_result_, sizeof(double), cudaMemcpyDeviceToHost, stream_));
        QCSB_CUDA(cudaStreamSynchronize(stream_));
        norm_target_ = h[0];
    }
    const uint64_t tensor_before = stats.tensor_passes;
    const int k = fused_->run(state_, n_, amp_bytes_, pending_, fusion_mode_, stats, timer);
    stats.kernel_launches += k;
    discard_pending();
    restore_norm(tensor_before);
}

// Complex64 tensor passes accumulate in FP32 on the tensor cores, and their
// rounding is biased toward smaller magnitudes: on B200 the 30-qubit
// matching circuit (110 passes) lost 5.5e-5 of its squared norm that way,
// against ~1e-6 on the register path, whose FP32 operations round to
// nearest. The gates of a flush are unitary and its collapses keep a known
// weight, so the flush must end at the target norm: an FP64 reduction and
// one scaling pass, both on the stream (no host round trip), restore it.
void Simulator::restore_norm(uint64_t tensor_passes_before)
{
    if (!c64() || stats.tensor_passes == tensor_passes_before || norm_target_ < 0.0)
        return;
    stats.kernel_launches += launch_zsums<float>(static_cast<const float2 *>(state_), n_, zsum_partials_,
                                                 zsum_result_, stream_);
    stats.kernel_launches += launch_rescale<float>(static_cast<float2 *>(state_), n_, norm_target_, zsum_result_,
                                                   stream_);
}

void Simulator::synchronize()
{
    require_allocated("synchronize");
    flush();
    QCSB_CUDA(cudaStreamSynchronize(stream_));
    fused_->check_device_error();
}

int Simulator::measure(int q)
{
    // reference measure_qubit, src/qcs.cu:2545-2677
    require_allocated("measure");
    check_qubit(q, "measured");
    if (contains(measured0_, q))
        return 0;
    if (contains(measured1_, q))
        return 1;
    // Queued collapses of earlier measurements need not run first: the
    // reduction below only reads the branch those measurements kept.
    if (pending_gates_ > 0)
        flush();
    uint64_t cmask = 0, cval = 0;
    for (int m : measured0_)
        cmask |= 1ull << perm_l2p_[m];
    for (int m : measured1_)
    {
        cmask |= 1ull << perm_l2p_[m];
        cval |= 1ull << perm_l2p_[m];
    }
    const int t = perm_l2p_[q];
    // (P0, P1) lands directly in pinned host memory, followed by a sequence
    // number the host spins on (a stream synchronisation costs a few
    // microseconds more per measurement); past 500 us of spinning it
    // synchronises the stream instead, which also reports any error
    double2 *h = static_cast<double2 *>(meas_host_);
    unsigned *done = reinterpret_cast<unsigned *>(static_cast<char *>(meas_host_) + kMeasureFlagOffset);
    const unsigned seq = ++measure_seq_;
    stats.kernel_launches += QCSB_ON_STATE(launch_measure_probs, n_, t, cmask, cval, red_partials_, h, red_ticket_,
                                           done, seq, stream_);
    const volatile unsigned *flag = done;
    const auto t0 = std::chrono::steady_clock::now();
    for (unsigned i = 0; *flag != seq; ++i)
        if ((i & 255u) == 255u && std::chrono::steady_clock::now() - t0 > std::chrono::microseconds(500))
        {
            QCSB_CUDA(cudaStreamSynchronize(stream_));
            break;
        }
    std::atomic_thread_fence(std::memory_order_acquire);
    fused_->check_device_error();
    const double p0 = h->x, p1 = h->y;
    const double sum = p0 + p1;
    std::uniform_real_distribution<double> dist(0, sum);
    const double r = dist(engine_);
    const int result = p0 < r;
    (result ? measured1_ : measured0_).push_back(q);
    norm_target_ = result ? p1 : p0;
    if (fusion_mode_ == QCS_FUSION_PLAIN)
    {
        stats.kernel_launches += QCSB_ON_STATE(launch_collapse, n_, t, result, stream_);
    }
    else
    {
        // zero the other branch as a queued diagonal op, so that it rides
        // along with the next pass instead of costing a pass of its own
        GateOp z;
        z.nt = 1;
        z.tq[0] = t;
        z.diag = true;
        z.na = 1;
        z.act[0] = static_cast<uint8_t>(result ? 0 : 1);
        z.mat[0] = cplx{0.0, 0.0};
        pending_.push_back(z);
    }
    return result;
}

void *Simulator::device_state_in_logical_order()
{
    require_allocated("get_device_state");
    // Cycle by cycle: logical q, held at physical p, swaps places with
    // whatever physical q holds; every swap puts at least one qubit home, so
    // at most n - 1 swaps, which the fused planner packs into passes (a
    // pass exchanges any of its local qubits in registers and shared memory)
    const GateMatrix swap = gate_matrix("swap", nullptr, 0);
    for (int q = 0; q < n_; ++q)
    {
        const int p = perm_l2p_[q];
        if (p == q)
            continue;
        const int r = perm_p2l_[q];   // the logical qubit physical q holds
        const int tq[kMaxTargets] = {q, p, 0, 0};
        const GateOp op = make_gate_op(swap, tq, 0, 0);
        if (fusion_mode_ == QCS_FUSION_PLAIN)
        {
            const int k = QCSB_ON_STATE(launch_gate_plain, n_, op, stream_);
            stats.kernel_launches += k;
            stats.plain_gate_kernels += k;
        }
        else
        {
            pending_.push_back(op);
            ++pending_gates_;
        }
        perm_l2p_[q] = q;
        perm_p2l_[q] = q;
        perm_l2p_[r] = p;
        perm_p2l_[p] = r;
    }
    synchronize();
    return state_;
}

void Simulator::reset_qubit(int q)
{
    // reference qcs_simulator_reset_cxx, src/qcs.cu:3077-3081
    if (measure(q))
        apply_gate("x", nullptr, 0, &q, 1, nullptr, 0, nullptr, 0);
}

void Simulator::clear_measurement_state()
{
    measured0_.clear();
    measured1_.clear();
}

// |0..0> and the flat state are unchanged by any qubit permutation, and a
// loaded state is written through whatever map is current, so before those
// the layout left by relabelled swaps can return to the reference's map.
void Simulator::restore_reference_layout()
{
    perm_l2p_ = ref_l2p_;
    for (int q = 0; q < n_; ++q)
        perm_p2l_[perm_l2p_[q]] = q;
}

void Simulator::set_zero_state()
{
    require_allocated("set_zero_state");
    discard_pending();
    clear_measurement_state();
    restore_reference_layout();
    stats.kernel_launches += QCSB_ON_STATE(launch_init_zero, n_, stream_);
    norm_target_ = 1.0;
}

void Simulator::set_flat_state()
{
    require_allocated("set_flat_state");
    discard_pending();
    clear_measurement_state();
    restore_reference_layout();
    stats.kernel_launches += QCSB_ON_STATE(launch_init_flat, n_, stream_);
    norm_target_ = -1.0;
}

void Simulator::set_sequential_state()
{
    require_allocated("set_sequential_state");
    discard_pending();
    clear_measurement_state();
    stats.kernel_launches += QCSB_ON_STATE(launch_init_sequential, n_, stream_);
    norm_target_ = -1.0;
}

void Simulator::set_entangled_state()
{
    // reference initialize_entangled at one process, src/qcs.cu:2081-2095:
    // amplitude 0 becomes 1, every other amplitude keeps its value.
    require_allocated("set_entangled_state");
    flush();
    clear_measurement_state();
    stats.kernel_launches += QCSB_ON_STATE(launch_set_amplitude, 0, 1.0, 0.0, stream_);
    norm_target_ = -1.0;
}

void Simulator::set_random_state()
{
    // reference initialize_use_curand, src/qcs.cu:2097-2119: unnormalised
    // N(0, 1) real and imaginary parts from cuRAND's default generator seeded
    // with the simulator seed. The measured lists are kept, as there.
    require_allocated("set_random_state");
    discard_pending();
    curandGenerator_t gen;
    if (curandCreateGenerator(&gen, CURAND_RNG_PSEUDO_DEFAULT) != CURAND_STATUS_SUCCESS)
        throw std::runtime_error("curandCreateGenerator failed");
    curandStatus_t st = curandSetStream(gen, stream_);
    if (st == CURAND_STATUS_SUCCESS)
        st = curandSetPseudoRandomGeneratorSeed(gen, seed_);
    if (st == CURAND_STATUS_SUCCESS)
        st = c64() ? curandGenerateNormal(gen, static_cast<float *>(state_), 2ull << n_, 0.0f, 1.0f)
                   : curandGenerateNormalDouble(gen, static_cast<double *>(state_), 2ull << n_, 0.0, 1.0);
    curandDestroyGenerator(gen);
    if (st != CURAND_STATUS_SUCCESS)
        throw std::runtime_error(strformat("cuRAND failed with status %d", (int)st));
    ++stats.kernel_launches;
    norm_target_ = -1.0;
}

void Simulator::ensure_staging()
{
    if (staging_dev_ != nullptr)
        return;
    // both buffers or neither: a failed pinned allocation frees the device
    // one, so that a later call allocates again instead of copying through
    // a missing host buffer
    const uint64_t count = std::max<uint64_t>(2, std::min<uint64_t>(kStagingAmps, 1ull << n_));
    double2 *dev = nullptr, *host = nullptr;
    QCSB_CUDA(cudaMalloc(&dev, sizeof(double2) * count));
    const cudaError_t err = cudaMallocHost(&host, sizeof(double2) * count);
    if (err != cudaSuccess)
    {
        cudaFree(dev);
        (void)cudaGetLastError();
        throw std::runtime_error(strformat("cudaMallocHost of the staging buffer: %s", cudaGetErrorString(err)));
    }
    staging_dev_ = dev;
    staging_host_ = host;
    staging_count_ = count;
}

// Move the whole register between device (physical order) and host (logical
// order) through the pinned staging buffer, one chunk at a time.
void Simulator::logical_transfer(double *host, uint64_t count, bool to_host)
{
    (void)count;
    ensure_staging();
    const uint64_t total = 1ull << n_;
    for (uint64_t begin = 0; begin < total; begin += staging_count_)
    {
        const uint64_t cnt = std::min<uint64_t>(staging_count_, total - begin);
        const size_t bytes = sizeof(double2) * cnt;
        if (to_host)
        {
            const double2 *src = stage_chunk_out(begin, cnt);
            QCSB_CUDA(cudaMemcpyAsync(staging_host_, src, bytes, cudaMemcpyDeviceToHost, stream_));
            QCSB_CUDA(cudaStreamSynchronize(stream_));
            fused_->check_device_error();
            std::memcpy(host + 2 * begin, staging_host_, bytes);
        }
        else
        {
            std::memcpy(staging_host_, host + 2 * begin, bytes);
            const bool direct = !c64() && identity_mapping();
            double2 *dst = direct ? static_cast<double2 *>(state_) + begin : staging_dev_;
            QCSB_CUDA(cudaMemcpyAsync(dst, staging_host_, bytes, cudaMemcpyHostToDevice, stream_));
            if (!direct)
            {
                if (identity_mapping())
                    stats.kernel_launches += launch_narrow<float>(staging_dev_, cnt, static_cast<float2 *>(state_) + begin, stream_);
                else
                    stats.kernel_launches += QCSB_ON_STATE(launch_scatter_logical, n_, perm_l2p_.data(), begin, cnt, staging_dev_, stream_);
            }
            QCSB_CUDA(cudaStreamSynchronize(stream_));
        }
    }
}

// Device pointer to logical amplitudes [begin, begin + cnt) as complex128:
// the register itself when it is complex128 in logical order, else the
// staging buffer filled by a gather or widening kernel.
const double2 *Simulator::stage_chunk_out(uint64_t begin, uint64_t cnt)
{
    const bool ident = identity_mapping();
    if (!c64() && ident)
        return static_cast<const double2 *>(state_) + begin;
    if (ident)
        stats.kernel_launches += launch_widen<float>(static_cast<const float2 *>(state_) + begin, cnt, staging_dev_, stream_);
    else
        stats.kernel_launches += QCSB_ON_STATE(launch_gather_logical, n_, perm_l2p_.data(), begin, cnt, staging_dev_, stream_);
    return staging_dev_;
}

void Simulator::save_statevector(const char *path)
{
    // reference save_statevector, src/qcs.cu:2494-2543: raw complex128 in
    // logical index order. Written sequentially, one chunk at a time.
    require_allocated("save_statevector");
    if (path == nullptr)
        throw std::runtime_error("save_statevector: output path must not be NULL");
    flush();
    FILE *fp = std::fopen(path, "wb");
    if (fp == nullptr)
        throw std::runtime_error("open failed");
    ensure_staging();
    const uint64_t total = 1ull << n_;
    for (uint64_t begin = 0; begin < total; begin += staging_count_)
    {
        const uint64_t cnt = std::min<uint64_t>(staging_count_, total - begin);
        const double2 *src = stage_chunk_out(begin, cnt);
        QCSB_CUDA(cudaMemcpyAsync(staging_host_, src, sizeof(double2) * cnt, cudaMemcpyDeviceToHost, stream_));
        QCSB_CUDA(cudaStreamSynchronize(stream_));
        if (std::fwrite(staging_host_, sizeof(double2), cnt, fp) != cnt)
        {
            std::fclose(fp);
            throw std::runtime_error("fwrite failed");
        }
    }
    std::fflush(fp);
    std::fclose(fp);
}

void Simulator::get_statevector(double *out, uint64_t count)
{
    require_allocated("get_statevector");
    if (out == nullptr)
        throw std::runtime_error("get_statevector: output pointer must not be NULL");
    if (count < (1ull << n_))
        throw std::runtime_error(strformat("get_statevector: buffer holds %llu amplitudes, the register has %llu",
                                           (unsigned long long)count, (unsigned long long)(1ull << n_)));
    flush();
    logical_transfer(out, count, true);
}

void Simulator::set_statevector(const double *in, uint64_t count)
{
    require_allocated("set_statevector");
    if (in == nullptr)
        throw std::runtime_error("set_statevector: input pointer must not be NULL");
    if (count != (1ull << n_))
        throw std::runtime_error(strformat("set_statevector: got %llu amplitudes, the register has %llu",
                                           (unsigned long long)count, (unsigned long long)(1ull << n_)));
    discard_pending();
    clear_measurement_state();
    restore_reference_layout();
    logical_transfer(const_cast<double *>(in), count, false);
    norm_target_ = -1.0;
}

void Simulator::expectation_z(double *out, double *norm)
{
    require_allocated("expectation_z");
    if (out == nullptr)
        throw std::runtime_error("expectation_z: output pointer must not be NULL");
    flush();
    stats.kernel_launches += QCSB_ON_STATE(launch_zsums, n_, zsum_partials_, zsum_result_, stream_);
    double *h = static_cast<double *>(host_pinned_);
    QCSB_CUDA(cudaMemcpyAsync(h, zsum_result_, sizeof(double) * (n_ + 1), cudaMemcpyDeviceToHost, stream_));
    QCSB_CUDA(cudaStreamSynchronize(stream_));
    fused_->check_device_error();
    const double total = h[0];
    for (int q = 0; q < n_; ++q)
    {
        const double p1 = h[1 + perm_l2p_[q]];
        out[q] = total > 0.0 ? (total - 2.0 * p1) / total : 0.0;
    }
    if (norm)
        *norm = total;
}

void Simulator::sample(uint32_t num_shots, uint64_t *out)
{
    require_allocated("sample");
    if (n_ > 64)
        throw std::runtime_error("sample: more than 64 qubits do not fit a 64-bit outcome");
    if (num_shots > 0 && out == nullptr)
        throw std::runtime_error("sample: output pointer must not be NULL");
    flush();
    int split = 0;
    const size_t tree_bytes = sampler_tree_bytes(n_, &split);
    const size_t nu = (size_t)num_shots * n_;
    const size_t need_host = std::max(sizeof(double) * nu, sizeof(uint64_t) * (size_t)num_shots);
    if (need_host > host_pinned_bytes_)
    {
        QCSB_CUDA(cudaStreamSynchronize(stream_));
        QCSB_CUDA(cudaFreeHost(host_pinned_));
        host_pinned_ = nullptr;
        host_pinned_bytes_ = need_host;
        QCSB_CUDA(cudaMallocHost(&host_pinned_, host_pinned_bytes_));
    }
    double *u = static_cast<double *>(host_pinned_);
    // same draws, in the same order, as num_shots rounds of measuring
    // qubits 0..n-1 (src/qcs.cu:2615-2617)
    std::uniform_real_distribution<double> dist(0.0, 1.0);
    for (size_t k = 0; k < nu; ++k)
        u[k] = dist(engine_);
    // one device buffer: tree, then uniforms, then outcomes (256-byte aligned)
    auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t u_off = up(tree_bytes), bits_off = u_off + up(sizeof(double) * std::max<size_t>(nu, 1));
    const size_t need_dev = bits_off + up(sizeof(uint64_t) * std::max<uint32_t>(num_shots, 1));
    if (need_dev > sampler_bytes_)
    {
        QCSB_CUDA(cudaStreamSynchronize(stream_));
        cudaFree(sampler_dev_);
        sampler_dev_ = nullptr;
        sampler_bytes_ = 0;
        QCSB_CUDA(cudaMalloc(&sampler_dev_, need_dev));
        sampler_bytes_ = need_dev;
    }
    char *base = static_cast<char *>(sampler_dev_);
    double *tree = reinterpret_cast<double *>(base);
    double *u_dev = reinterpret_cast<double *>(base + u_off);
    uint64_t *bits_dev = reinterpret_cast<uint64_t *>(base + bits_off);
    QCSB_CUDA(cudaMemcpyAsync(u_dev, u, sizeof(double) * nu, cudaMemcpyHostToDevice, stream_));
    stats.kernel_launches += QCSB_ON_STATE(launch_sampler, n_, perm_l2p_.data(), num_shots, u_dev, bits_dev, tree, split, stream_);
    QCSB_CUDA(cudaStreamSynchronize(stream_));   // the pinned buffer is reused below
    QCSB_CUDA(cudaMemcpyAsync(host_pinned_, bits_dev, sizeof(uint64_t) * num_shots, cudaMemcpyDeviceToHost, stream_));
    QCSB_CUDA(cudaStreamSynchronize(stream_));
    fused_->check_device_error();
    std::memcpy(out, host_pinned_, sizeof(uint64_t) * num_shots);
}

KernelTimer::~KernelTimer()
{
    clear();
    for (cudaEvent_t e : pool_)
        cudaEventDestroy(e);
}

cudaEvent_t KernelTimer::take()
{
    if (!pool_.empty())
    {
        cudaEvent_t e = pool_.back();
        pool_.pop_back();
        return e;
    }
    cudaEvent_t e;
    QCSB_CUDA(cudaEventCreate(&e));
    return e;
}

void KernelTimer::begin(cudaStream_t stream, int cls, double bytes, const PassFeatures *features)
{
    Rec r{cls, bytes, take(), take(), PassFeatures{{0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}}};
    if (features)
        r.feat = *features;
    QCSB_CUDA(cudaEventRecord(r.a, stream));
    recs_.push_back(r);
}

void KernelTimer::take_pass_log(std::vector<PassFeatures> &features, std::vector<float> &ms)
{
    qcs_b200_kernel_times unused;
    collect(unused);
    features.swap(log_feat_);
    ms.swap(log_ms_);
    log_feat_.clear();
    log_ms_.clear();
}

void KernelTimer::end(cudaStream_t stream) { QCSB_CUDA(cudaEventRecord(recs_.back().b, stream)); }

void KernelTimer::collect(qcs_b200_kernel_times &out)
{
    out = qcs_b200_kernel_times{};
    for (const Rec &r : recs_)
    {
        QCSB_CUDA(cudaEventSynchronize(r.b));
        float ms = 0.0f;
        QCSB_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        if (r.cls == kFused)
        {
            ++out.fused_launches;
            out.fused_ms += ms;
            out.fused_bytes += r.bytes;
            log_feat_.push_back(r.feat);
            log_ms_.push_back(ms);
        }
        else
        {
            ++out.plain_launches;
            out.plain_ms += ms;
            out.plain_bytes += r.bytes;
        }
    }
    clear();
}

void KernelTimer::clear()
{
    for (const Rec &r : recs_)
    {
        pool_.push_back(r.a);
        pool_.push_back(r.b);
    }
    recs_.clear();
}

void Simulator::get_amplitudes(const uint64_t *indices, uint64_t count, double *out)
{
    require_allocated("get_amplitudes");
    if (count > 0 && (indices == nullptr || out == nullptr))
        throw std::runtime_error("get_amplitudes: index and output pointers must not be NULL");
    const uint64_t total = 1ull << n_;
    for (uint64_t k = 0; k < count; ++k)
        if (indices[k] >= total)
            throw std::runtime_error(strformat("get_amplitudes: index %llu is outside the register of %llu amplitudes",
                                               (unsigned long long)indices[k], (unsigned long long)total));
    flush();
    ensure_staging();
    // physical indices go through the pinned staging buffer (16 bytes per
    // amplitude leaves room for the 8-byte index in its upper half)
    const uint64_t chunk = staging_count_ / 2;
    uint64_t *idx_host = reinterpret_cast<uint64_t *>(staging_host_ + chunk);
    uint64_t *idx_dev = reinterpret_cast<uint64_t *>(staging_dev_ + chunk);
    for (uint64_t begin = 0; begin < count; begin += chunk)
    {
        const uint64_t cnt = std::min<uint64_t>(chunk, count - begin);
        for (uint64_t k = 0; k < cnt; ++k)
        {
            const uint64_t l = indices[begin + k];
            uint64_t p = 0;
            for (int q = 0; q < n_; ++q)
                p |= ((l >> q) & 1ull) << perm_l2p_[q];
            idx_host[k] = p;
        }
        QCSB_CUDA(cudaMemcpyAsync(idx_dev, idx_host, sizeof(uint64_t) * cnt, cudaMemcpyHostToDevice, stream_));
        stats.kernel_launches += QCSB_ON_STATE(launch_gather_indices, idx_dev, cnt, staging_dev_, stream_);
        QCSB_CUDA(cudaMemcpyAsync(staging_host_, staging_dev_, sizeof(double2) * cnt, cudaMemcpyDeviceToHost, stream_));
        QCSB_CUDA(cudaStreamSynchronize(stream_));
        std::memcpy(out + 2 * begin, staging_host_, sizeof(double2) * cnt);
    }
}

void Simulator::compare(Simulator &a, Simulator &b, double *overlap_re, double *overlap_im, double *max_abs_diff,
                        double *norm_a, double *norm_b)
{
    a.require_allocated("compare");
    b.require_allocated("compare");
    if (a.n_ != b.n_)
        throw std::runtime_error(strformat("compare: registers of %d and %d qubits", a.n_, b.n_));
    if (a.device_ != b.device_)
        throw std::runtime_error("compare: the simulators are on different devices");
    a.flush();
    b.flush();
    QCSB_CUDA(cudaStreamSynchronize(b.stream_));
    a.ensure_staging();
    b.ensure_staging();
    double *partials = nullptr, *host = nullptr;
    const size_t pbytes = sizeof(double) * 5 * kReduceBlocks;
    QCSB_CUDA(cudaMalloc(&partials, pbytes));
    if (cudaMallocHost(&host, pbytes) != cudaSuccess)
    {
        cudaFree(partials);
        throw std::runtime_error("compare: cudaMallocHost failed");
    }
    double re = 0.0, im = 0.0, mx = 0.0, na = 0.0, nb = 0.0;
    const uint64_t total = 1ull << a.n_;
    cudaError_t err = cudaSuccess;
    for (uint64_t begin = 0; begin < total && err == cudaSuccess; begin += a.staging_count_)
    {
        const uint64_t cnt = std::min<uint64_t>(a.staging_count_, total - begin);
        const double2 *y = b.stage_chunk_out(begin, cnt);
        err = cudaStreamSynchronize(b.stream_);
        if (err != cudaSuccess)
            break;
        const double2 *x = a.stage_chunk_out(begin, cnt);
        a.stats.kernel_launches += launch_compare(x, y, cnt, partials, a.stream_);
        err = cudaMemcpyAsync(host, partials, pbytes, cudaMemcpyDeviceToHost, a.stream_);
        if (err == cudaSuccess)
            err = cudaStreamSynchronize(a.stream_);
        for (int i = 0; i < kReduceBlocks && err == cudaSuccess; ++i)
        {
            re += host[5 * i];
            im += host[5 * i + 1];
            mx = std::max(mx, host[5 * i + 2]);
            na += host[5 * i + 3];
            nb += host[5 * i + 4];
        }
    }
    cudaFree(partials);
    cudaFreeHost(host);
    QCSB_CUDA(err);
    if (overlap_re)
        *overlap_re = re;
    if (overlap_im)
        *overlap_im = im;
    if (max_abs_diff)
        *max_abs_diff = mx;
    if (norm_a)
        *norm_a = na;
    if (norm_b)
        *norm_b = nb;
}

int Simulator::event_create()
{
    if (disposed_)
        throw std::runtime_error("event_create: the simulator has been disposed");
    cudaEvent_t e;
    QCSB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDefault));
    events_.push_back(e);
    return (int)events_.size() - 1;
}

void Simulator::event_record(int event_num)
{
    if (disposed_)
        throw std::runtime_error("event_record: the simulator has been disposed");
    if (event_num < 0 || event_num >= (int)events_.size())
        throw std::runtime_error(strformat("event %d does not exist", event_num));
    flush();
    QCSB_CUDA(cudaEventRecordWithFlags(events_[event_num], stream_, cudaEventDefault));
}

double Simulator::event_elapsed(int start, int stop)
{
    // reference event_get_elapsed_time, src/qcs.cu:2862-2897: seconds
    if (disposed_)
        throw std::runtime_error("event_get_elapsed_time: the simulator has been disposed");
    for (int e : {start, stop})
        if (e < 0 || e >= (int)events_.size())
            throw std::runtime_error(strformat("event %d does not exist", e));
    QCSB_CUDA(cudaEventSynchronize(events_[start]));
    QCSB_CUDA(cudaEventSynchronize(events_[stop]));
    float ms = 0.0f;
    QCSB_CUDA(cudaEventElapsedTime(&ms, events_[start], events_[stop]));
    return ms * 1e-3;
}

} // namespace qcsb
