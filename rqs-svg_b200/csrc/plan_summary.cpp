// Host-only view of how the fused planner would run a gate list: passes,
// stages and pass ops by kind, without a GPU (qcs_b200_plan_summary).
#include "fused_pass.h"
#include "qcs_b200.h"

#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace qcsb
{

static_assert(F_DENSE1 == 0 && F_SWAP1 == 1 && F_DENSE2 == 2 && F_SWAP2 == 3 && F_PHASE == 4 && F_DIAG == 5 &&
                  F_TERM == 6 && F_DENSE1R == 7 && F_MULI == 9 && F_DENSE1X4 == 10 && F_DENSE1RX4 == 11 &&
                  F_PRUN == 12 && F_SIGNS == 13 && F_SIGNT == 14 && F_DENSE1X2 == 15,
              "op kinds as documented in qcs_b200.h");
static_assert(sizeof(qcs_b200_plan_summary) == 4 * 4 + 4 * QCS_B200_PLAN_KINDS + 8 + 4 * 4,
              "qcs_b200_plan_summary layout");

void plan_summary(int n, const qcs_b200_gate *gates, uint64_t count, qcs_b200_plan_summary &out)
{
    if (n < 1 || n > kMaxQubits)
        throw std::runtime_error("plan_summary: num_qubits must be in [1, " + std::to_string(kMaxQubits) + "]");
    if (count > 0 && gates == nullptr)
        throw std::runtime_error("plan_summary: gates must not be NULL");
    std::memset(&out, 0, sizeof(out));
    // logical -> physical map: uncontrolled SWAPs only relabel qubits, as
    // the simulator's fused modes do
    std::vector<int> l2p(n);
    for (int q = 0; q < n; ++q)
        l2p[q] = q;
    std::vector<GateOp> queue;
    queue.reserve(count);
    for (uint64_t i = 0; i < count; ++i)
    {
        const qcs_b200_gate &in = gates[i];
        if (std::memchr(in.name, '\0', sizeof(in.name)) == nullptr)
            throw std::runtime_error("plan_summary: gate " + std::to_string(i) + ": name is not NUL-terminated");
        const int id = gate_id(in.name);
        const int arity = gate_arity(id);
        if (in.num_targets != arity || in.num_negctrls < 0 || in.num_ctrls < 0 ||
            arity + in.num_negctrls + in.num_ctrls > 12)
            throw std::runtime_error("plan_summary: gate " + std::to_string(i) + " (" + in.name +
                                     "): bad target or control counts");
        int tq[4] = {0, 0, 0, 0};
        uint64_t cm = 0, cv = 0, seen = 0;
        const int total = arity + in.num_negctrls + in.num_ctrls;
        for (int j = 0; j < total; ++j)
        {
            const int lq = in.qubits[j];
            if (lq < 0 || lq >= n || ((seen >> lq) & 1))
                throw std::runtime_error("plan_summary: gate " + std::to_string(i) + " (" + in.name +
                                         "): qubit out of range or repeated");
            seen |= 1ull << lq;
            const int q = l2p[lq];
            if (j < arity)
                tq[j] = q;
            else
            {
                cm |= 1ull << q;
                if (j >= arity + in.num_negctrls)
                    cv |= 1ull << q;
            }
        }
        if (arity == 2 && cm == 0 && std::strcmp(in.name, "swap") == 0)
        {
            std::swap(l2p[in.qubits[0]], l2p[in.qubits[1]]);
            continue;
        }
        const GateMatrix g = gate_matrix(id, in.params, gate_nparams(id));
        queue.push_back(make_gate_op(g, tq, cm, cv));
    }
    if (n < fused_min_qubits())
    {
        out.plain_gates = static_cast<uint32_t>(queue.size());
        return;
    }
    queue = defer_x(queue);
    const int k = clamp_local_bits(kDefaultLocal, n);
    const std::vector<Segment> segs = plan_greedy(queue, n, k, std::min(kLowBits, k), kFusedMaxOps);
    std::vector<double2> tables;
    for (const Segment &s : segs)
    {
        if (!s.fused)
        {
            ++out.plain_gates;
            continue;
        }
        std::vector<FPassParams> params;
        std::vector<PlannedPass> pieces;
        std::vector<std::vector<StageCond>> conds;
        if (!build_pieces(queue, s.pass, n, params, nullptr, &pieces, &tables, &conds))
        {
            out.plain_gates += static_cast<uint32_t>(s.pass.ops.size());
            continue;
        }
        for (size_t pi = 0; pi < params.size(); ++pi)
        {
            TPassParams tp;
            TBuildParams tb;
            if (make_tensor_params(params[pi], conds[pi], 16, tp, tb))
                ++out.tensor_eligible;
        }
        // the executor's choice for a complex128 register (automatic mode)
        PassChoice choice;
        choose_execution(queue, s.pass, n, 16, 1, params, pieces, conds, &tables, choice, 0);
        for (size_t pi = 0; pi < params.size(); ++pi)
        {
            const FPassParams &p = params[pi];
            const int t = choice.tensor[pi];
            if (t >= 0)
            {
                ++out.tensor_passes;
                out.tensor_matrices += choice.tbuild[t].nmats;
                if (choice.tparams[t].width == 3)
                    ++out.tensor8_passes;
            }
            ++out.passes;
            out.stages += static_cast<uint32_t>(p.nstages);
            out.ops += static_cast<uint32_t>(p.nops);
            for (int o = 0; o < p.nops; ++o)
                if (p.ops[o].kind < QCS_B200_PLAN_KINDS)
                    ++out.kinds[p.ops[o].kind];
        }
    }
    out.table_entries = tables.size();
}

} // namespace qcsb
