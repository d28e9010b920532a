// Batched execution of many independent circuits.
//
// Layout: all registers live in one arena, grouped by gate structure (the
// same gates on the same qubits, parameters aside); a group's registers are
// stored back to back, 2^n amplitudes each. Every group has one plan of
// fused passes, built from "shape" ops (each gate evaluated at generic
// parameters, so that the plan does not depend on parameter values: an RY
// that happens to be the identity still gets its slot). Each register's gate
// entries sit in its own block of the entry buffer, in the order the plan's
// FOps read them, so one launch of the batched pass kernel runs a pass over
// every register of the group.
//
// A run: copy the entries to the device, run every group's passes (the first
// pass builds |0..0> in shared memory instead of reading the register), reduce
// <Z> of every register, copy the expectations back. It is captured once as a
// CUDA graph and replayed; new parameters only change the entry buffer.
//
// Tuning: on the first run each group's plan is built for each candidate
// number of local qubits, timed with CUDA events, and the fastest is kept.

#include "batch.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <thread>

namespace qcsb
{
namespace
{

// generic parameters: no gate of the API is the identity, diagonal or a
// permutation at these values unless it is one for every value
const double kProbe[4] = {0.7309, 1.1763, 0.4217, 2.0389};

uint64_t mix(uint64_t h, uint64_t v)
{
    h ^= v;
    h *= 1099511628211ull;
    return h;
}

uint64_t dbits(double x)
{
    uint64_t u;
    std::memcpy(&u, &x, sizeof(u));
    return u;
}

// The GateOp of an actual parameter set laid over the shape's active set.
GateOp op_like(const GateOp &shape, const GateMatrix &g)
{
    GateOp op = shape;
    const int d = 1 << g.nt;
    if (shape.diag)
    {
        for (int a = 0; a < shape.na; ++a)
            op.mat[a] = g.m[shape.act[a] * d + shape.act[a]];
    }
    else
    {
        for (int a = 0; a < shape.na; ++a)
            for (int b = 0; b < shape.na; ++b)
                op.mat[a * shape.na + b] = g.m[shape.act[a] * d + shape.act[b]];
    }
    return op;
}

constexpr size_t kBatchTensorMatsBytes = size_t(2) << 30;   // stage matrices of one batched tensor pass

bool tune_enabled()
{
    const char *e = std::getenv("QCS_BATCH_TUNE");
    return !(e && e[0] == '0');
}

} // namespace

Batch::Batch(int amplitude_bits)
{
    if (amplitude_bits != 128 && amplitude_bits != 64)
        throw std::runtime_error(strformat("precision %d is not 128 (complex128) or 64 (complex64)", amplitude_bits));
    amp_bytes_ = amplitude_bits / 8;
    QCSB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    QCSB_CUDA(cudaEventCreate(&ev0_));
    QCSB_CUDA(cudaEventCreate(&ev1_));
}

Batch::~Batch()
{
    if (stream_)
        cudaStreamSynchronize(stream_);
    release_device();
    if (ev0_)
        cudaEventDestroy(ev0_);
    if (ev1_)
        cudaEventDestroy(ev1_);
    if (stream_)
        cudaStreamDestroy(stream_);
}

void Batch::release_device()
{
    for (cudaGraphExec_t e : execs_)
        cudaGraphExecDestroy(e);
    execs_.clear();
    cudaFree(arena_);
    cudaFree(mats_dev_);
    cudaFree(zitems_dev_);
    cudaFree(zregs_dev_);
    cudaFree(zpartials_dev_);
    cudaFree(zout_dev_);
    cudaFree(tmats_dev_);
    tmats_dev_ = nullptr;
    tmats_bytes_ = 0;
    if (mats_host_)
        cudaFreeHost(mats_host_);
    if (zout_host_)
        cudaFreeHost(zout_host_);
    arena_ = nullptr;
    mats_dev_ = mats_host_ = nullptr;
    zitems_dev_ = nullptr;
    zregs_dev_ = nullptr;
    zpartials_dev_ = zout_dev_ = zout_host_ = nullptr;
}

void Batch::invalidate()
{
    if (stream_)
        QCSB_CUDA(cudaStreamSynchronize(stream_));
    release_device();
    groups_.clear();
    built_ = false;
    ran_ = false;
}

uint32_t Batch::add_circuit(int n, const qcs_b200_gate *gates, uint32_t count)
{
    if (n < fused_min_qubits() || n > 30)
        throw std::runtime_error(strformat("batch registers hold %d to 30 qubits, got %d", fused_min_qubits(), n));
    if (count > 0 && gates == nullptr)
        throw std::runtime_error("add_circuit: gates must not be NULL");
    Circuit c;
    c.n = n;
    c.gates.reserve(count);
    uint64_t params = 0;
    for (uint32_t i = 0; i < count; ++i)
    {
        const qcs_b200_gate &in = gates[i];
        Gate g;
        std::memset(&g, 0, sizeof(g));
        if (std::memchr(in.name, '\0', sizeof(in.name)) == nullptr)
            throw std::runtime_error(strformat("gate %u: name is not NUL-terminated", i));
        std::memcpy(g.name, in.name, sizeof(g.name));
        g.id = gate_id(g.name);
        g.np = gate_nparams(g.id);
        const int arity = gate_arity(g.name);
        if (arity > 2)
            throw std::runtime_error(strformat("gate %u (%s): batches take gates on at most two targets", i, g.name));
        if (in.num_targets != arity)
            throw std::runtime_error(strformat("gate %u (%s) takes %d target qubits, got %d", i, g.name, arity,
                                               (int)in.num_targets));
        if (in.num_negctrls < 0 || in.num_ctrls < 0 || arity + in.num_negctrls + in.num_ctrls > 12)
            throw std::runtime_error(strformat("gate %u (%s): bad control counts", i, g.name));
        uint64_t seen = 0;
        const int total = arity + in.num_negctrls + in.num_ctrls;
        for (int j = 0; j < total; ++j)
        {
            const int q = in.qubits[j];
            if (q < 0 || q >= n)
                throw std::runtime_error(strformat("gate %u (%s): qubit %d is out of range [0, %d)", i, g.name, q, n));
            if ((seen >> q) & 1)
                throw std::runtime_error(strformat("gate %u (%s): qubit %d appears more than once", i, g.name, q));
            seen |= 1ull << q;
            if (j < arity)
                g.tq[j] = q;
            else
            {
                g.cmask |= 1ull << q;
                if (j >= arity + in.num_negctrls)
                    g.cval |= 1ull << q;
            }
        }
        for (int j = 0; j < g.np; ++j)
            g.params[j] = in.params[j];
        params += g.np;
        c.gates.push_back(g);
    }
    invalidate();
    circuits_.push_back(std::move(c));
    num_params_ += params;
    return static_cast<uint32_t>(circuits_.size() - 1);
}

void Batch::set_parameters(const double *params, uint64_t count)
{
    if (count != num_params_)
        throw std::runtime_error(strformat("set_parameters: the batch has %llu parameters, got %llu",
                                           (unsigned long long)num_params_, (unsigned long long)count));
    if (count > 0 && params == nullptr)
        throw std::runtime_error("set_parameters: params must not be NULL");
    uint64_t i = 0;
    for (Circuit &c : circuits_)
        for (Gate &g : c.gates)
            for (int j = 0; j < g.np; ++j)
                g.params[j] = params[i++];
    // the entries are filled by the next run, group by group, while the GPU
    // runs the groups before
    dirty_ = built_;
}

void Batch::plan_group(Group &g, int k, bool tensor)
{
    g.k = k;
    g.passes.clear();
    const int low = std::min(kLowBits, k);
    const std::vector<Segment> segs = plan_greedy(g.shape, g.n, k, low, kFusedMaxOps);
    for (const Segment &s : segs)
    {
        if (!s.fused)
            throw std::runtime_error("batch: a gate of this circuit cannot run in a fused pass");
        if (tensor && s.pass.k == kTensorLocal)
        {
            // the pass replanned with 8 x 8 stages, as a tensor pass where
            // every piece allows it
            PlannedPass p3 = s.pass;
            p3.stage_width = 3;
            std::vector<FPassParams> params3;
            std::vector<std::vector<FOpSource>> srcs3;
            std::vector<std::vector<StageCond>> conds3;
            bool ok = build_pieces(g.shape, p3, g.n, params3, &srcs3, nullptr, nullptr, &conds3);
            std::vector<Pass> tpasses(ok ? params3.size() : 0);
            for (size_t i = 0; ok && i < params3.size(); ++i)
            {
                Pass &p = tpasses[i];
                p.prm = params3[i];
                p.src = std::move(srcs3[i]);
                p.tensor = make_tensor_params(p.prm, conds3[i], amp_bytes_, p.tp, p.tb, 3);
                // every register's matrices of a pass live on the device at
                // once: beyond kBatchTensorMatsBytes the pass stays on the
                // register path
                ok = p.tensor && static_cast<double>(p.tb.nmats) * kTensor3Fragments * 32 * 16 * g.members.size() <=
                                     static_cast<double>(kBatchTensorMatsBytes);
            }
            if (ok)
            {
                for (Pass &p : tpasses)
                    g.passes.push_back(std::move(p));
                continue;
            }
        }
        std::vector<FPassParams> params;
        std::vector<std::vector<FOpSource>> srcs;
        if (!build_pieces(g.shape, s.pass, g.n, params, &srcs))
            throw std::runtime_error("batch: a gate of this circuit does not fit a pass");
        for (size_t i = 0; i < params.size(); ++i)
        {
            Pass p;
            p.prm = params[i];
            p.src = std::move(srcs[i]);
            g.passes.push_back(std::move(p));
        }
    }
    // entry offsets within a register's block of the entry buffer
    uint32_t off = 0;
    double2 scratch[16];
    for (Pass &p : g.passes)
    {
        for (int f = 0; f < p.prm.nops; ++f)
        {
            FOp &op = p.prm.ops[f];
            if (op.kind == F_SIGNT)
                continue;   // moff holds the term's slot mask, no entries
            if (off > 0xffffu)
                throw std::runtime_error("batch: too many gate entries in one circuit");
            op.moff = static_cast<uint16_t>(off);
            off += layer_kind(op.kind) ? layer_entries(g.shape, p.src[f], op.kind, scratch)
                                      : fop_entries(g.shape[p.src[f].op], op, p.src[f].swapped, scratch);
        }
    }
    g.stride = off;
}

void Batch::layout_entries()
{
    uint64_t off = 0;
    for (Group &g : groups_)
    {
        g.mats_off = off;
        off += (uint64_t)g.stride * g.members.size();
    }
    if (off != mats_count_ || mats_dev_ == nullptr)
    {
        if (stream_)
            QCSB_CUDA(cudaStreamSynchronize(stream_));
        cudaFree(mats_dev_);
        if (mats_host_)
            cudaFreeHost(mats_host_);
        mats_dev_ = mats_host_ = nullptr;
        mats_count_ = off;
        const size_t bytes = sizeof(double2) * std::max<uint64_t>(off, 1);
        QCSB_CUDA(cudaMalloc(&mats_dev_, bytes));
        QCSB_CUDA(cudaMallocHost(&mats_host_, bytes));
    }
    for (Group &g : groups_)
        for (Pass &p : g.passes)
        {
            p.prm.mats = mats_dev_ + g.mats_off;
            p.prm.mat_stride = g.stride;
        }
}

void Batch::fill_group_range(const Group &g, size_t first, size_t last)
{
    std::vector<GateOp> ops(g.shape.size());
    for (size_t s = first; s < last; ++s)
    {
        const Circuit &c = circuits_[g.members[s]];
        for (size_t i = 0; i < c.gates.size(); ++i)
        {
            const Gate &gt = c.gates[i];
            ops[i] = op_like(g.shape[i], gate_matrix(gt.id, gt.params, gt.np));
        }
        double2 *block = mats_host_ + g.mats_off + (uint64_t)s * g.stride;
        for (const Pass &p : g.passes)
            for (int f = 0; f < p.prm.nops; ++f)
            {
                const FOp &op = p.prm.ops[f];
                if (op.kind == F_SIGNT)
                    continue;
                if (layer_kind(op.kind))
                    layer_entries(ops, p.src[f], op.kind, block + op.moff);
                else
                    fop_entries(ops[p.src[f].op], op, p.src[f].swapped, block + op.moff);
            }
        if (amp_bytes_ == (int)sizeof(float2))
            entries_to_float(block, g.stride);
    }
}

void Batch::fill_entries(int only_group)
{
    // work units: (group, slot range); spread over the host's cores
    struct Unit
    {
        int group;
        size_t first, last;
    };
    std::vector<Unit> units;
    for (int gi = 0; gi < (int)groups_.size(); ++gi)
    {
        if (only_group >= 0 && gi != only_group)
            continue;
        const size_t m = groups_[gi].members.size();
        const size_t step = 64;
        for (size_t a = 0; a < m; a += step)
            units.push_back({gi, a, std::min(m, a + step)});
    }
    unsigned hw = std::thread::hardware_concurrency();
    const unsigned workers = std::max(1u, std::min<unsigned>(hw ? hw : 1, std::min<size_t>(units.size(), 64)));
    if (workers <= 1)
    {
        for (const Unit &u : units)
            fill_group_range(groups_[u.group], u.first, u.last);
        return;
    }
    std::vector<std::thread> pool;
    std::vector<std::exception_ptr> errors(workers);
    for (unsigned w = 0; w < workers; ++w)
        pool.emplace_back([&, w] {
            try
            {
                for (size_t i = w; i < units.size(); i += workers)
                    fill_group_range(groups_[units[i].group], units[i].first, units[i].last);
            }
            catch (...)
            {
                errors[w] = std::current_exception();
            }
        });
    for (auto &t : pool)
        t.join();
    for (auto &e : errors)
        if (e)
            std::rethrow_exception(e);
}

// The stage-matrix buffer: the largest tensor pass's matrices over all its
// group's registers (8 x 8 stages: kTensor3Fragments x 32 lanes x 16 bytes
// per matrix). Grown before any graph is captured.
void Batch::ensure_tensor_mats()
{
    size_t need = 0;
    for (const Group &g : groups_)
        for (const Pass &p : g.passes)
            if (p.tensor)
                need = std::max(need, static_cast<size_t>(p.tb.nmats) * kTensor3Fragments * 32 * 16 * g.members.size());
    if (need <= tmats_bytes_)
        return;
    if (stream_)
        QCSB_CUDA(cudaStreamSynchronize(stream_));
    cudaFree(tmats_dev_);
    tmats_dev_ = nullptr;
    tmats_bytes_ = 0;
    QCSB_CUDA(cudaMalloc(&tmats_dev_, need));
    tmats_bytes_ = need;
}

void Batch::set_tensor_mode(int mode)
{
    if (mode < 0 || mode > 2)
        throw std::runtime_error(strformat("batch tensor mode %d is not 0 (never), 1 (tuned) or 2 (always)", mode));
    tensor_mode_ = mode;
    invalidate();
}

void Batch::enqueue_passes(const Group &g, cudaStream_t s, int *launches)
{
    void *base = static_cast<char *>(arena_) + g.amp_off * amp_bytes_;
    if (g.passes.empty())
    {
        QCSB_CUDA(cudaMemsetAsync(base, 0, ((size_t)amp_bytes_ << g.n) * g.members.size(), s));
        *launches += amp_bytes_ == 8 ? launch_batch_set_ones<float>(base, 1ull << g.n, (uint32_t)g.members.size(), s)
                                     : launch_batch_set_ones<double>(base, 1ull << g.n, (uint32_t)g.members.size(), s);
        return;
    }
    for (size_t pi = 0; pi < g.passes.size(); ++pi)
    {
        Pass &pass = const_cast<Pass &>(g.passes[pi]);
        FPassParams &prm = pass.prm;
        prm.chunks = (uint64_t)g.members.size() << (g.n - g.k);
        prm.from_zero = pi == 0 ? 1 : 0;
        if (pass.tensor)
        {
            TBuildParams &tb = pass.tb;
            TPassParams &tp = pass.tp;
            tb.out = static_cast<double2 *>(tmats_dev_);
            tb.regs = static_cast<uint32_t>(g.members.size());
            tb.batch_float = amp_bytes_ == 8 ? 1 : 0;
            *launches += launch_stage_matrices<double>(prm, tb, s);
            tp.state = base;
            tp.mats = static_cast<const double2 *>(tmats_dev_);
            tp.reg_mats = tb.nmats;
            tp.batch_cbits = g.n - g.k;
            tp.chunks = prm.chunks;
            tp.from_zero = prm.from_zero;
            tp.err = nullptr;
            *launches += amp_bytes_ == 8 ? launch_tensor_pass<float>(tp, s) : launch_tensor_pass<double>(tp, s);
            continue;
        }
        *launches += amp_bytes_ == 8 ? launch_fused_batch<float>(base, g.k, prm, s)
                                     : launch_fused_batch<double>(base, g.k, prm, s);
    }
}

void Batch::enqueue_group(int gi, cudaStream_t s, int *launches)
{
    const Group &g = groups_[gi];
    const size_t count = (size_t)g.stride * g.members.size();
    if (count > 0)
        QCSB_CUDA(cudaMemcpyAsync(mats_dev_ + g.mats_off, mats_host_ + g.mats_off, sizeof(double2) * count,
                                  cudaMemcpyHostToDevice, s));
    enqueue_passes(g, s, launches);
}

void Batch::enqueue_results(cudaStream_t s, int *launches)
{
    *launches += amp_bytes_ == 8
                     ? launch_batch_zsums<float>(arena_, zitems_dev_, num_zitems_, zregs_dev_,
                                                 (uint32_t)circuits_.size(), zpartials_dev_, zout_dev_, s)
                     : launch_batch_zsums<double>(arena_, zitems_dev_, num_zitems_, zregs_dev_,
                                                  (uint32_t)circuits_.size(), zpartials_dev_, zout_dev_, s);
    QCSB_CUDA(cudaMemcpyAsync(zout_host_, zout_dev_, sizeof(double) * zout_count_, cudaMemcpyDeviceToHost, s));
}

void Batch::tune()
{
    for (int gi = 0; gi < (int)groups_.size(); ++gi)
    {
        Group &g = groups_[gi];
        // candidates: register passes at k = 9..11, and 8 x 8 tensor passes
        // (k = 11) unless the mode excludes them
        std::vector<std::pair<int, bool>> cands;
        for (int k = kStageBits + 5; k <= kDefaultLocal; ++k)
        {
            const int kk = clamp_local_bits(k, g.n);
            if (std::find(cands.begin(), cands.end(), std::make_pair(kk, false)) == cands.end())
                cands.push_back({kk, false});
        }
        const bool tensor_ok = g.n >= kTensorLocal && tensor_mode_ != 0;
        if (tensor_mode_ == 2 && tensor_ok)
        {
            plan_group(g, kTensorLocal, true);
            continue;
        }
        const int default_k = clamp_local_bits(kDefaultLocal, g.n);   // the largest register-path k
        if (tensor_ok)
            cands.push_back({kTensorLocal, true});
        if (cands.size() < 2 || !tune_enabled())
        {
            plan_group(g, default_k);
            continue;
        }
        std::pair<int, bool> best = cands.front();
        float best_ms = 0.0f;
        for (const auto &cand : cands)
        {
            plan_group(g, cand.first, cand.second);
            layout_entries();
            ensure_tensor_mats();
            fill_entries(gi);
            QCSB_CUDA(cudaMemcpyAsync(mats_dev_ + g.mats_off, mats_host_ + g.mats_off,
                                      sizeof(double2) * g.stride * g.members.size(), cudaMemcpyHostToDevice, stream_));
            int launches = 0;
            enqueue_passes(g, stream_, &launches);   // warm-up
            QCSB_CUDA(cudaEventRecord(ev0_, stream_));
            enqueue_passes(g, stream_, &launches);
            QCSB_CUDA(cudaEventRecord(ev1_, stream_));
            QCSB_CUDA(cudaEventSynchronize(ev1_));
            float ms = 0.0f;
            QCSB_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
            if (cand == cands.front() || ms < best_ms)
            {
                best_ms = ms;
                best = cand;
            }
        }
        plan_group(g, best.first, best.second);
    }
}

void Batch::build()
{
    if (circuits_.empty())
        throw std::runtime_error("run: the batch has no circuits");
    // A build that threw part way (a gate that fits no pass, too little
    // memory) leaves its buffers and graphs behind; a rebuild starts from
    // nothing so that retries do not leak device or pinned memory.
    if (stream_)
        QCSB_CUDA(cudaStreamSynchronize(stream_));
    release_device();
    mats_count_ = 0;
    groups_.clear();
    // group by structure
    for (uint32_t ci = 0; ci < circuits_.size(); ++ci)
    {
        Circuit &c = circuits_[ci];
        std::vector<GateOp> shape;
        shape.reserve(c.gates.size());
        uint64_t sig = mix(1469598103934665603ull, (uint64_t)c.n);
        for (const Gate &gt : c.gates)
        {
            const GateMatrix gm = gate_matrix(gt.id, kProbe, gt.np);
            const GateOp op = make_gate_op(gm, gt.tq, gt.cmask, gt.cval);
            sig = mix(sig, (uint64_t)op.nt | ((uint64_t)op.na << 8) | ((uint64_t)op.diag << 16));
            for (int i = 0; i < op.nt; ++i)
                sig = mix(sig, (uint64_t)op.tq[i]);
            sig = mix(mix(sig, op.cmask), op.cval);
            const int ne = op.diag ? op.na : op.na * op.na;
            for (int e = 0; e < ne; ++e)
                sig = mix(mix(sig, dbits(op.mat[e].re)), dbits(op.mat[e].im));
            shape.push_back(op);
        }
        sig = mix(sig, c.gates.size());
        int gi = -1;
        for (int i = 0; i < (int)groups_.size(); ++i)
            if (groups_[i].signature == sig && groups_[i].n == c.n && groups_[i].shape.size() == shape.size())
                gi = i;
        if (gi < 0)
        {
            Group g;
            g.n = c.n;
            g.signature = sig;
            g.shape = std::move(shape);
            groups_.push_back(std::move(g));
            gi = (int)groups_.size() - 1;
        }
        c.group = gi;
        c.slot = (uint32_t)groups_[gi].members.size();
        groups_[gi].members.push_back(ci);
    }
    // arena and <Z> work lists
    total_amps_ = 0;
    for (Group &g : groups_)
    {
        g.amp_off = total_amps_;
        total_amps_ += (uint64_t)g.members.size() << g.n;
    }
    std::vector<BatchZItem> items;
    std::vector<BatchZReg> regs(circuits_.size());
    zout_count_ = 0;
    for (uint32_t ci = 0; ci < circuits_.size(); ++ci)
    {
        Circuit &c = circuits_[ci];
        c.z_off = zout_count_;
        zout_count_ += c.n;
    }
    for (const Group &g : groups_)
        for (uint32_t s = 0; s < g.members.size(); ++s)
        {
            const Circuit &c = circuits_[g.members[s]];
            const int sb = std::min(c.n, kBatchZSliceBits);
            BatchZReg r;
            r.first = (uint32_t)items.size();
            r.count = 1u << (c.n - sb);
            r.n = c.n;
            r.out_off = (uint32_t)c.z_off;
            for (uint32_t sl = 0; sl < r.count; ++sl)
                items.push_back({g.amp_off + ((uint64_t)s << g.n), c.n, sl});
            regs[g.members[s]] = r;
        }
    num_zitems_ = (uint32_t)items.size();
    size_t free_b = 0, total_b = 0;
    QCSB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t arena_bytes = (size_t)total_amps_ * amp_bytes_;
    if (arena_bytes + (256ull << 20) > free_b)
        throw std::runtime_error(strformat("batch: the registers need %.2f GB, %.2f GB are free", arena_bytes / 1e9,
                                           free_b / 1e9));
    QCSB_CUDA(cudaMalloc(&arena_, arena_bytes));
    QCSB_CUDA(cudaMalloc(&zitems_dev_, sizeof(BatchZItem) * items.size()));
    QCSB_CUDA(cudaMalloc(&zregs_dev_, sizeof(BatchZReg) * regs.size()));
    QCSB_CUDA(cudaMalloc(&zpartials_dev_, sizeof(double) * kBatchZPartials * items.size()));
    QCSB_CUDA(cudaMalloc(&zout_dev_, sizeof(double) * zout_count_));
    QCSB_CUDA(cudaMallocHost(&zout_host_, sizeof(double) * zout_count_));
    QCSB_CUDA(cudaMemcpy(zitems_dev_, items.data(), sizeof(BatchZItem) * items.size(), cudaMemcpyHostToDevice));
    QCSB_CUDA(cudaMemcpy(zregs_dev_, regs.data(), sizeof(BatchZReg) * regs.size(), cudaMemcpyHostToDevice));

    // plans: tuned per group, then the final entry layout
    for (Group &g : groups_)
        plan_group(g, clamp_local_bits(kDefaultLocal, g.n));
    layout_entries();
    tune();
    layout_entries();
    ensure_tensor_mats();
    fill_entries();

    // capture the run: a graph per group, then the results (after dropping
    // those of a build that stopped part way)
    for (cudaGraphExec_t e : execs_)
        cudaGraphExecDestroy(e);
    execs_.clear();
    int launches = 0;
    for (int gi = 0; gi <= (int)groups_.size(); ++gi)
        execs_.push_back(capture(gi, &launches));
    launches_per_run_ = (uint32_t)launches;
    built_ = true;
    dirty_ = false;
}

// Graph of group gi (gi == number of groups: the results).
cudaGraphExec_t Batch::capture(int gi, int *launches)
{
    cudaGraph_t graph = nullptr;
    QCSB_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed));
    try
    {
        if (gi < (int)groups_.size())
            enqueue_group(gi, stream_, launches);
        else
            enqueue_results(stream_, launches);
    }
    catch (...)
    {
        cudaStreamEndCapture(stream_, &graph);
        if (graph)
            cudaGraphDestroy(graph);
        throw;
    }
    QCSB_CUDA(cudaStreamEndCapture(stream_, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t err = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    QCSB_CUDA(err);
    return exec;
}

void Batch::run()
{
    if (!built_)
        build();
    // new parameters: each group's entries are filled on the host while the
    // GPU runs the groups launched before it (the copies of a group read only
    // its own part of the pinned entry buffer)
    const bool fill = dirty_;
    for (size_t gi = 0; gi < groups_.size(); ++gi)
    {
        if (fill)
            fill_entries((int)gi);
        if (gi == 0)
            QCSB_CUDA(cudaEventRecord(ev0_, stream_));
        QCSB_CUDA(cudaGraphLaunch(execs_[gi], stream_));
    }
    if (groups_.empty())
        QCSB_CUDA(cudaEventRecord(ev0_, stream_));
    QCSB_CUDA(cudaGraphLaunch(execs_.back(), stream_));
    dirty_ = false;
    QCSB_CUDA(cudaEventRecord(ev1_, stream_));
    QCSB_CUDA(cudaStreamSynchronize(stream_));
    float ms = 0.0f;
    QCSB_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    last_ms_ = ms;
    ran_ = true;
}

void Batch::expectation_z(double *out, uint64_t count) const
{
    if (!ran_)
        throw std::runtime_error("expectation_z: run the batch first");
    if (count < zout_count_)
        throw std::runtime_error(strformat("expectation_z: the batch has %llu expectations, the buffer holds %llu",
                                           (unsigned long long)zout_count_, (unsigned long long)count));
    if (out == nullptr)
        throw std::runtime_error("expectation_z: output pointer must not be NULL");
    std::memcpy(out, zout_host_, sizeof(double) * zout_count_);
}

void Batch::get_statevector(uint32_t index, double *out, uint64_t count)
{
    if (!ran_)
        throw std::runtime_error("get_statevector: run the batch first");
    if (index >= circuits_.size())
        throw std::runtime_error(strformat("get_statevector: no circuit %u", index));
    const Circuit &c = circuits_[index];
    const uint64_t amps = 1ull << c.n;
    if (out == nullptr || count < amps)
        throw std::runtime_error("get_statevector: the buffer must hold 2^n amplitudes");
    const Group &g = groups_[c.group];
    const char *src = static_cast<const char *>(arena_) + (g.amp_off + ((uint64_t)c.slot << c.n)) * amp_bytes_;
    if (amp_bytes_ == 16)
    {
        QCSB_CUDA(cudaMemcpy(out, src, 16 * amps, cudaMemcpyDeviceToHost));
        return;
    }
    std::vector<float> tmp(2 * amps);
    QCSB_CUDA(cudaMemcpy(tmp.data(), src, 8 * amps, cudaMemcpyDeviceToHost));
    for (uint64_t i = 0; i < 2 * amps; ++i)
        out[i] = tmp[i];
}

void Batch::info(qcs_b200_batch_info *out) const
{
    std::memset(out, 0, sizeof(*out));
    out->circuits = (uint32_t)circuits_.size();
    out->parameters = num_params_;
    uint64_t amps = 0;
    for (const Circuit &c : circuits_)
        amps += 1ull << c.n;
    out->amplitudes = amps;
    if (built_)
    {
        out->groups = (uint32_t)groups_.size();
        double bytes = 0.0;
        for (const Group &g : groups_)
        {
            out->passes += (uint32_t)g.passes.size();
            for (const Pass &p : g.passes)
                out->tensor_passes += p.tensor ? 1u : 0u;
            const double reg = std::ldexp((double)amp_bytes_, g.n) * g.members.size();
            if (!g.passes.empty())
                bytes += reg * (2.0 * g.passes.size() - 1.0);
        }
        out->pass_bytes = bytes;
        out->launches_per_run = launches_per_run_;
    }
    out->last_run_ms = last_ms_;
}

} // namespace qcsb
