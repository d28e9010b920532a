// C ABI of libqcs.so: the reference's extern "C" entry points and C++ *_cxx
// functions (include/qcs.h), plus the B200 extensions (include/qcs_b200.h).
//
// Error convention (reference src/qcs.cu:2935-3000): every extern "C"
// function runs its body inside a try block, returns 1 on success and 0 when
// anything throws, handing the exception text to the process-wide callback.

#include "qcs.h"
#include "qcs_b200.h"
#include "batch.h"
#include "cost_model.h"
#include "simulator.h"

#include <algorithm>
#include <cstring>
#include <exception>
#include <new>

struct qcs_simulator
{
    qcsb::Simulator *core = nullptr;
};

namespace
{

qcs_exception_callback g_callback = nullptr;

void report(const char *msg)
{
    if (g_callback != nullptr)
        g_callback(msg, std::strlen(msg));
}

template <typename F>
int guarded(F &&f)
{
    try
    {
        f();
        return 1;
    }
    catch (const std::exception &e)
    {
        report(e.what());
    }
    catch (...)
    {
        report("Unknown C++ exception");
    }
    return 0;
}

template <typename R, typename V>
void write_result(R *out, V v)
{
    if (out == nullptr)
        throw std::runtime_error("result pointer must not be NULL");
    *out = static_cast<R>(v);
}

qcsb::Simulator &core(qcs_simulator *sim)
{
    if (sim == nullptr)
        throw std::runtime_error("simulator handle must not be NULL");
    if (sim->core == nullptr)
        throw std::runtime_error("the simulator has been disposed");
    return *sim->core;
}

const qcsb::Simulator &core(const qcs_simulator *sim)
{
    return core(const_cast<qcs_simulator *>(sim));
}

// reference qcs_vector_from_array, src/qcs.cu:2914-2925
std::vector<int> to_vector(const bit_num_t *values, bit_num_t count)
{
    if (count < 0)
        throw std::runtime_error("array element count must be non-negative");
    if (count > 0 && values == nullptr)
        throw std::runtime_error("array pointer must not be NULL when element count is positive");
    return std::vector<int>(values, values + count);
}

// Qubit list of a gate call copied to ints; a list longer than any register
// holds a repeated or out-of-range qubit, which the simulator reports.
struct QubitList
{
    int q[qcsb::kMaxQubits + 1];
    int n;
    QubitList(const bit_num_t *values, bit_num_t count)
    {
        if (count < 0)
            throw std::runtime_error("array element count must be non-negative");
        if (count > 0 && values == nullptr)
            throw std::runtime_error("array pointer must not be NULL when element count is positive");
        n = std::min<int>(count, qcsb::kMaxQubits + 1);
        for (int i = 0; i < n; ++i)
            q[i] = values[i];
    }
};

void gate(qcs_simulator *sim, const char *name, std::initializer_list<double> params,
          const bit_num_t *t, bit_num_t nt, const bit_num_t *neg, bit_num_t nneg, const bit_num_t *ctl, bit_num_t nctl)
{
    const QubitList targets(t, nt), negs(neg, nneg), ctls(ctl, nctl);
    double p[4];
    int np = 0;
    for (double v : params)
        p[np++] = v;
    core(sim).apply_gate(name, p, np, targets.q, targets.n, negs.q, negs.n, ctls.q, ctls.n);
}

} // namespace

void qcsb::report_error(const char *message) { report(message); }

// ------------------------------------------------------------ C++ API

qcs_simulator *qcs_simulator_create_cxx()
{
    qcs_simulator *sim = new qcs_simulator();
    try
    {
        sim->core = new qcsb::Simulator();
    }
    catch (...)
    {
        delete sim;
        throw;
    }
    return sim;
}

void qcs_simulator_dispose_cxx(qcs_simulator *sim)
{
    if (sim == nullptr)
        throw std::runtime_error("simulator handle must not be NULL");
    if (sim->core == nullptr)
        throw std::runtime_error("the simulator has already been disposed");
    qcsb::Simulator *c = sim->core;
    sim->core = nullptr;
    try
    {
        c->dispose();
    }
    catch (...)
    {
        delete c;
        throw;
    }
    delete c;
}

void qcs_simulator_destroy_cxx(qcs_simulator *sim)
{
    if (sim == nullptr)
        return;
    if (sim->core != nullptr)
    {
        qcsb::Simulator *c = sim->core;
        sim->core = nullptr;
        try
        {
            c->dispose();
        }
        catch (...)
        {
            delete c;
            delete sim;
            throw;
        }
        delete c;
    }
    delete sim;
}

void qcs_simulator_allocate_memory_cxx(qcs_simulator *sim) { core(sim).allocate_memory(); }
int qcs_simulator_get_num_procs_cxx(qcs_simulator *sim) { (void)core(sim); return 1; }
int qcs_simulator_get_proc_num_cxx(qcs_simulator *sim) { (void)core(sim); return 0; }
int qcs_simulator_get_num_qubits_cxx(const qcs_simulator *sim) { return core(sim).num_qubits_cfg; }
int qcs_simulator_get_num_clbits_cxx(const qcs_simulator *sim) { return core(sim).num_clbits; }

void qcs_simulator_set_num_qubits_cxx(qcs_simulator *sim, bit_num_t num_qubits)
{
    auto &c = core(sim);
    if (c.allocated())
        throw std::runtime_error("set_num_qubits: memory is already allocated");
    c.num_qubits_cfg = num_qubits;
}

void qcs_simulator_set_mapping_cxx(qcs_simulator *sim, const bit_num_t *perm_p2l, bit_num_t perm_p2l_count)
{
    auto perm = to_vector(perm_p2l, perm_p2l_count);
    core(sim).set_mapping(perm);
}

void qcs_simulator_set_num_clbits_cxx(qcs_simulator *sim, bit_num_t num_clbits)
{
    if (num_clbits < 0)
        throw std::runtime_error("num_clbits must be non-negative");
    auto &c = core(sim);
    c.num_clbits = num_clbits;
    c.clbits.resize(num_clbits, 0);
}

void qcs_simulator_get_clbits_cxx(const qcs_simulator *sim, bit_t *clbits)
{
    const auto &c = core(sim);
    if (clbits == nullptr && c.num_clbits > 0)
        throw std::runtime_error("clbits pointer must not be NULL");
    for (int i = 0; i < c.num_clbits; ++i)
        clbits[i] = c.clbits[i] ? 1 : 0;
}

void qcs_simulator_get_clbits_string_cxx(const qcs_simulator *sim, char *clbits_string)
{
    // most significant (highest-numbered) clbit first, src/qcs.cu:3371-3377
    const auto &c = core(sim);
    if (clbits_string == nullptr)
        throw std::runtime_error("clbits_string pointer must not be NULL");
    int out = 0;
    for (int i = (int)c.clbits.size() - 1; i >= 0; --i)
        clbits_string[out++] = c.clbits[i] ? '1' : '0';
    clbits_string[out] = '\0';
}

void qcs_simulator_reset_cxx(qcs_simulator *sim, bit_num_t qubit_num) { core(sim).reset_qubit(qubit_num); }
void qcs_simulator_set_zero_state_cxx(qcs_simulator *sim) { core(sim).set_zero_state(); }
void qcs_simulator_set_sequential_state_cxx(qcs_simulator *sim) { core(sim).set_sequential_state(); }
void qcs_simulator_set_flat_state_cxx(qcs_simulator *sim) { core(sim).set_flat_state(); }
void qcs_simulator_set_entangled_state_cxx(qcs_simulator *sim) { core(sim).set_entangled_state(); }
void qcs_simulator_set_random_state_cxx(qcs_simulator *sim) { core(sim).set_random_state(); }

void qcs_simulator_reset_clbits_cxx(qcs_simulator *sim)
{
    auto &c = core(sim);
    std::fill(c.clbits.begin(), c.clbits.end(), 0);
}

void qcs_simulator_reset_measurement_state_cxx(qcs_simulator *sim) { core(sim).clear_measurement_state(); }
void qcs_simulator_reinitialize_mapping_cxx(qcs_simulator *sim) { core(sim).reinitialize_mapping(); }

#define QCSB_TARGETS const bit_num_t *t, bit_num_t nt, const bit_num_t *neg, bit_num_t nneg, const bit_num_t *ctl, bit_num_t nctl
#define QCSB_TARGET_ARGS t, nt, neg, nneg, ctl, nctl

void qcs_simulator_gate_global_phase_cxx(qcs_simulator *sim, double theta, const bit_num_t *neg, bit_num_t nneg,
                                         const bit_num_t *ctl, bit_num_t nctl)
{
    gate(sim, "global_phase", {theta}, nullptr, 0, neg, nneg, ctl, nctl);
}

#define QCSB_GATE0(NAME)                                                   \
    void qcs_simulator_gate_##NAME##_cxx(qcs_simulator *sim, QCSB_TARGETS) \
    {                                                                      \
        gate(sim, #NAME, {}, QCSB_TARGET_ARGS);                            \
    }
#define QCSB_GATE1(NAME, A)                                                          \
    void qcs_simulator_gate_##NAME##_cxx(qcs_simulator *sim, double A, QCSB_TARGETS) \
    {                                                                                \
        gate(sim, #NAME, {A}, QCSB_TARGET_ARGS);                                     \
    }
#define QCSB_GATE2(NAME, A, B)                                                                 \
    void qcs_simulator_gate_##NAME##_cxx(qcs_simulator *sim, double A, double B, QCSB_TARGETS) \
    {                                                                                          \
        gate(sim, #NAME, {A, B}, QCSB_TARGET_ARGS);                                            \
    }
#define QCSB_GATE3(NAME, A, B, C)                                                                        \
    void qcs_simulator_gate_##NAME##_cxx(qcs_simulator *sim, double A, double B, double C, QCSB_TARGETS) \
    {                                                                                                    \
        gate(sim, #NAME, {A, B, C}, QCSB_TARGET_ARGS);                                                   \
    }

QCSB_GATE0(h)
QCSB_GATE0(x)
QCSB_GATE0(y)
QCSB_GATE0(z)
QCSB_GATE0(s)
QCSB_GATE0(sdg)
QCSB_GATE0(t)
QCSB_GATE0(tdg)
QCSB_GATE0(sx)
QCSB_GATE1(rx, theta)
QCSB_GATE1(ry, theta)
QCSB_GATE1(rz, theta)
void qcs_simulator_gate_u4_cxx(qcs_simulator *sim, double theta, double phi, double lambda, double gamma, QCSB_TARGETS)
{
    gate(sim, "u4", {theta, phi, lambda, gamma}, QCSB_TARGET_ARGS);
}
QCSB_GATE3(u3, theta, phi, lambda)
QCSB_GATE2(u2, phi, lambda)
QCSB_GATE1(u1, lambda)
QCSB_GATE3(u, theta, phi, lambda)
QCSB_GATE1(p, theta)
QCSB_GATE0(swap)
QCSB_GATE0(iswap)
QCSB_GATE0(id)
QCSB_GATE0(sxdg)
QCSB_GATE2(r, theta, phi)
QCSB_GATE1(rxx, theta)
QCSB_GATE1(ryy, theta)
QCSB_GATE1(rzz, theta)
QCSB_GATE1(rzx, theta)
QCSB_GATE0(dcx)
QCSB_GATE0(ecr)
QCSB_GATE2(xx_plus_yy, theta, beta)
QCSB_GATE2(xx_minus_yy, theta, beta)
QCSB_GATE0(rccx)
QCSB_GATE0(rcccx)

int qcs_simulator_measure_cxx(qcs_simulator *sim, bit_num_t qubit_num) { return core(sim).measure(qubit_num); }

int qcs_simulator_measure_to_clbit_cxx(qcs_simulator *sim, bit_num_t qubit_num, bit_num_t clbit_num)
{
    auto &c = core(sim);
    if (clbit_num < 0 || clbit_num >= c.num_clbits)
        throw std::runtime_error(qcsb::strformat("clbit %d is out of range [0, %d)", clbit_num, c.num_clbits));
    const int r = c.measure(qubit_num);
    c.clbits[clbit_num] = static_cast<uint8_t>(r);
    return r;
}

int qcs_simulator_read_cxx(qcs_simulator *sim, bit_num_t clbit_num)
{
    auto &c = core(sim);
    if (clbit_num < 0 || clbit_num >= c.num_clbits)
        throw std::runtime_error(qcsb::strformat("clbit %d is out of range [0, %d)", clbit_num, c.num_clbits));
    return c.clbits[clbit_num];
}

void qcs_simulator_save_statevector_cxx(qcs_simulator *sim, const char *outfn) { core(sim).save_statevector(outfn); }
int qcs_simulator_event_create_cxx(qcs_simulator *sim) { return core(sim).event_create(); }
void qcs_simulator_event_record_cxx(qcs_simulator *sim, int event_num) { core(sim).event_record(event_num); }
double qcs_simulator_event_get_elapsed_time_cxx(qcs_simulator *sim, event_num_t start_event_num, event_num_t stop_event_num)
{
    return core(sim).event_elapsed(start_event_num, stop_event_num);
}

// ------------------------------------------------------------ C API

extern "C" int qcs_set_exception_callback(qcs_exception_callback callback)
{
    g_callback = callback;
    return 1;
}

extern "C" int qcs_simulator_create(qcs_simulator **result)
{
    return guarded([&] {
        if (result == nullptr)
            throw std::runtime_error("result pointer must not be NULL");
        *result = qcs_simulator_create_cxx();
    });
}

extern "C" int qcs_simulator_destroy(qcs_simulator *sim) { return guarded([&] { qcs_simulator_destroy_cxx(sim); }); }
extern "C" int qcs_simulator_allocate_memory(qcs_simulator *sim) { return guarded([&] { qcs_simulator_allocate_memory_cxx(sim); }); }
extern "C" int qcs_simulator_dispose(qcs_simulator *sim) { return guarded([&] { qcs_simulator_dispose_cxx(sim); }); }
extern "C" int qcs_simulator_get_num_procs(qcs_simulator *sim, bit_t *result)
{
    return guarded([&] { write_result(result, qcs_simulator_get_num_procs_cxx(sim)); });
}
extern "C" int qcs_simulator_get_proc_num(qcs_simulator *sim, bit_t *result)
{
    return guarded([&] { write_result(result, qcs_simulator_get_proc_num_cxx(sim)); });
}
extern "C" int qcs_simulator_get_num_qubits(const qcs_simulator *sim, bit_t *result)
{
    return guarded([&] { write_result(result, qcs_simulator_get_num_qubits_cxx(sim)); });
}
extern "C" int qcs_simulator_get_num_clbits(const qcs_simulator *sim, bit_t *result)
{
    return guarded([&] { write_result(result, qcs_simulator_get_num_clbits_cxx(sim)); });
}
extern "C" int qcs_simulator_set_num_qubits(qcs_simulator *sim, bit_num_t num_qubits)
{
    return guarded([&] { qcs_simulator_set_num_qubits_cxx(sim, num_qubits); });
}
extern "C" int qcs_simulator_set_mapping(qcs_simulator *sim, const bit_num_t *perm_p2l, bit_num_t perm_p2l_count)
{
    return guarded([&] { qcs_simulator_set_mapping_cxx(sim, perm_p2l, perm_p2l_count); });
}
extern "C" int qcs_simulator_set_num_clbits(qcs_simulator *sim, bit_num_t num_clbits)
{
    return guarded([&] { qcs_simulator_set_num_clbits_cxx(sim, num_clbits); });
}
extern "C" int qcs_simulator_get_clbits(const qcs_simulator *sim, bit_t *clbits)
{
    return guarded([&] { qcs_simulator_get_clbits_cxx(sim, clbits); });
}
extern "C" int qcs_simulator_get_clbits_string(const qcs_simulator *sim, char *clbits_string)
{
    return guarded([&] { qcs_simulator_get_clbits_string_cxx(sim, clbits_string); });
}
extern "C" int qcs_simulator_reset(qcs_simulator *sim, bit_num_t qubit_num) { return guarded([&] { qcs_simulator_reset_cxx(sim, qubit_num); }); }
extern "C" int qcs_simulator_set_zero_state(qcs_simulator *sim) { return guarded([&] { qcs_simulator_set_zero_state_cxx(sim); }); }
extern "C" int qcs_simulator_set_sequential_state(qcs_simulator *sim) { return guarded([&] { qcs_simulator_set_sequential_state_cxx(sim); }); }
extern "C" int qcs_simulator_set_flat_state(qcs_simulator *sim) { return guarded([&] { qcs_simulator_set_flat_state_cxx(sim); }); }
extern "C" int qcs_simulator_set_entangled_state(qcs_simulator *sim) { return guarded([&] { qcs_simulator_set_entangled_state_cxx(sim); }); }
extern "C" int qcs_simulator_set_random_state(qcs_simulator *sim) { return guarded([&] { qcs_simulator_set_random_state_cxx(sim); }); }
extern "C" int qcs_simulator_reset_clbits(qcs_simulator *sim) { return guarded([&] { qcs_simulator_reset_clbits_cxx(sim); }); }
extern "C" int qcs_simulator_reset_measurement_state(qcs_simulator *sim) { return guarded([&] { qcs_simulator_reset_measurement_state_cxx(sim); }); }
extern "C" int qcs_simulator_reinitialize_mapping(qcs_simulator *sim) { return guarded([&] { qcs_simulator_reinitialize_mapping_cxx(sim); }); }

extern "C" int qcs_simulator_gate_global_phase(qcs_simulator *sim, double theta, const bit_num_t *neg, bit_num_t nneg,
                                               const bit_num_t *ctl, bit_num_t nctl)
{
    return guarded([&] { qcs_simulator_gate_global_phase_cxx(sim, theta, neg, nneg, ctl, nctl); });
}

#define QCSB_CGATE0(NAME)                                                                                    \
    extern "C" int qcs_simulator_gate_##NAME(qcs_simulator *sim, QCSB_TARGETS)                               \
    {                                                                                                        \
        return guarded([&] { qcs_simulator_gate_##NAME##_cxx(sim, QCSB_TARGET_ARGS); });                     \
    }
#define QCSB_CGATE1(NAME)                                                                                    \
    extern "C" int qcs_simulator_gate_##NAME(qcs_simulator *sim, double a, QCSB_TARGETS)                     \
    {                                                                                                        \
        return guarded([&] { qcs_simulator_gate_##NAME##_cxx(sim, a, QCSB_TARGET_ARGS); });                  \
    }
#define QCSB_CGATE2(NAME)                                                                                    \
    extern "C" int qcs_simulator_gate_##NAME(qcs_simulator *sim, double a, double b, QCSB_TARGETS)           \
    {                                                                                                        \
        return guarded([&] { qcs_simulator_gate_##NAME##_cxx(sim, a, b, QCSB_TARGET_ARGS); });               \
    }
#define QCSB_CGATE3(NAME)                                                                                    \
    extern "C" int qcs_simulator_gate_##NAME(qcs_simulator *sim, double a, double b, double c, QCSB_TARGETS) \
    {                                                                                                        \
        return guarded([&] { qcs_simulator_gate_##NAME##_cxx(sim, a, b, c, QCSB_TARGET_ARGS); });            \
    }

QCSB_CGATE0(h)
QCSB_CGATE0(x)
QCSB_CGATE0(y)
QCSB_CGATE0(z)
QCSB_CGATE0(s)
QCSB_CGATE0(sdg)
QCSB_CGATE0(t)
QCSB_CGATE0(tdg)
QCSB_CGATE0(sx)
QCSB_CGATE1(rx)
QCSB_CGATE1(ry)
QCSB_CGATE1(rz)
extern "C" int qcs_simulator_gate_u4(qcs_simulator *sim, double a, double b, double c, double d, QCSB_TARGETS)
{
    return guarded([&] { qcs_simulator_gate_u4_cxx(sim, a, b, c, d, QCSB_TARGET_ARGS); });
}
QCSB_CGATE3(u3)
QCSB_CGATE2(u2)
QCSB_CGATE1(u1)
QCSB_CGATE3(u)
QCSB_CGATE1(p)
QCSB_CGATE0(swap)
QCSB_CGATE0(iswap)
QCSB_CGATE0(id)
QCSB_CGATE0(sxdg)
QCSB_CGATE2(r)
QCSB_CGATE1(rxx)
QCSB_CGATE1(ryy)
QCSB_CGATE1(rzz)
QCSB_CGATE1(rzx)
QCSB_CGATE0(dcx)
QCSB_CGATE0(ecr)
QCSB_CGATE2(xx_plus_yy)
QCSB_CGATE2(xx_minus_yy)
QCSB_CGATE0(rccx)
QCSB_CGATE0(rcccx)

extern "C" int qcs_simulator_measure(qcs_simulator *sim, bit_num_t qubit_num, bit_t *result)
{
    return guarded([&] {
        if (result == nullptr)
            throw std::runtime_error("result pointer must not be NULL");
        write_result(result, qcs_simulator_measure_cxx(sim, qubit_num));
    });
}
extern "C" int qcs_simulator_measure_to_clbit(qcs_simulator *sim, bit_num_t qubit_num, bit_num_t clbit_num, bit_t *result)
{
    return guarded([&] {
        if (result == nullptr)
            throw std::runtime_error("result pointer must not be NULL");
        write_result(result, qcs_simulator_measure_to_clbit_cxx(sim, qubit_num, clbit_num));
    });
}
extern "C" int qcs_simulator_read(qcs_simulator *sim, bit_num_t clbit_num, bit_t *result)
{
    return guarded([&] { write_result(result, qcs_simulator_read_cxx(sim, clbit_num)); });
}
extern "C" int qcs_simulator_save_statevector(qcs_simulator *sim, const char *outfn)
{
    return guarded([&] { qcs_simulator_save_statevector_cxx(sim, outfn); });
}
extern "C" int qcs_simulator_event_create(qcs_simulator *sim, bit_t *result)
{
    return guarded([&] {
        if (result == nullptr)
            throw std::runtime_error("result pointer must not be NULL");
        write_result(result, qcs_simulator_event_create_cxx(sim));
    });
}
extern "C" int qcs_simulator_event_record(qcs_simulator *sim, int event_num)
{
    return guarded([&] { qcs_simulator_event_record_cxx(sim, event_num); });
}
extern "C" int qcs_simulator_event_get_elapsed_time(qcs_simulator *sim, event_num_t start_event_num, event_num_t stop_event_num, double *result)
{
    return guarded([&] {
        if (result == nullptr)
            throw std::runtime_error("result pointer must not be NULL");
        write_result(result, qcs_simulator_event_get_elapsed_time_cxx(sim, start_event_num, stop_event_num));
    });
}

// ------------------------------------------------------------ extensions

extern "C" int qcs_simulator_set_fusion(qcs_simulator *sim, int mode) { return guarded([&] { core(sim).set_fusion(mode); }); }
extern "C" int qcs_simulator_get_fusion(const qcs_simulator *sim, int *mode)
{
    return guarded([&] { write_result(mode, core(sim).fusion()); });
}
extern "C" int qcs_simulator_set_seed(qcs_simulator *sim, uint32_t seed) { return guarded([&] { core(sim).set_seed(seed); }); }
extern "C" int qcs_simulator_synchronize(qcs_simulator *sim) { return guarded([&] { core(sim).synchronize(); }); }
extern "C" int qcs_simulator_get_statevector(qcs_simulator *sim, double *amplitudes, uint64_t count)
{
    return guarded([&] { core(sim).get_statevector(amplitudes, count); });
}
extern "C" int qcs_simulator_set_statevector(qcs_simulator *sim, const double *amplitudes, uint64_t count)
{
    return guarded([&] { core(sim).set_statevector(amplitudes, count); });
}
extern "C" int qcs_simulator_expectation_z(qcs_simulator *sim, double *expectations, double *norm)
{
    return guarded([&] { core(sim).expectation_z(expectations, norm); });
}
extern "C" int qcs_simulator_sample(qcs_simulator *sim, uint32_t num_shots, uint64_t *bitstrings)
{
    return guarded([&] { core(sim).sample(num_shots, bitstrings); });
}
extern "C" int qcs_simulator_get_stats(const qcs_simulator *sim, qcs_b200_stats *stats)
{
    return guarded([&] {
        if (stats == nullptr)
            throw std::runtime_error("stats pointer must not be NULL");
        *stats = core(sim).stats;
    });
}
extern "C" int qcs_simulator_reset_stats(qcs_simulator *sim)
{
    return guarded([&] { core(sim).stats = qcs_b200_stats{}; });
}
extern "C" int qcs_simulator_set_kernel_timing(qcs_simulator *sim, int enable)
{
    return guarded([&] {
        auto &c = core(sim);
        c.flush();
        c.timer.enabled = enable != 0;
    });
}
extern "C" int qcs_simulator_get_kernel_times(qcs_simulator *sim, qcs_b200_kernel_times *times)
{
    return guarded([&] {
        if (times == nullptr)
            throw std::runtime_error("times pointer must not be NULL");
        auto &c = core(sim);
        c.flush();
        c.timer.collect(*times);
    });
}

// ------------------------------------------------------------ planner and cost model

struct qcs_b200_cost_model
{
    qcsb::CostModel *m = nullptr;
};

namespace
{
qcsb::CostModel &model_of(qcs_b200_cost_model *model)
{
    if (model == nullptr || model->m == nullptr)
        throw std::runtime_error("cost model handle must not be NULL");
    return *model->m;
}
} // namespace

extern "C" int qcs_simulator_set_planner_options(qcs_simulator *sim, int max_gates_per_pass, int local_qubits)
{
    return guarded([&] { core(sim).set_planner_options(max_gates_per_pass, local_qubits); });
}

extern "C" int qcs_simulator_set_tensor_passes(qcs_simulator *sim, int mode)
{
    return guarded([&] { core(sim).set_tensor_mode(mode); });
}
extern "C" int qcs_simulator_get_tensor_passes(const qcs_simulator *sim, int *mode)
{
    return guarded([&] { write_result(mode, core(sim).tensor_mode()); });
}
extern "C" int qcs_simulator_set_tensor_engine(qcs_simulator *sim, int engine)
{
    return guarded([&] { core(sim).set_tensor_engine(engine); });
}
extern "C" int qcs_simulator_get_tensor_engine(const qcs_simulator *sim, int *engine)
{
    return guarded([&] { write_result(engine, core(sim).tensor_engine()); });
}

extern "C" int qcs_simulator_get_pass_records(qcs_simulator *sim, float *features, float *milliseconds,
                                              uint32_t capacity, uint32_t *count)
{
    return guarded([&] {
        if (count == nullptr || (capacity > 0 && (features == nullptr || milliseconds == nullptr)))
            throw std::runtime_error("get_pass_records: output pointers must not be NULL");
        auto &c = core(sim);
        c.flush();
        std::vector<qcsb::PassFeatures> f;
        std::vector<float> ms;
        c.timer.take_pass_log(f, ms);
        const uint32_t n = static_cast<uint32_t>(std::min<size_t>(capacity, f.size()));
        for (uint32_t i = 0; i < n; ++i)
        {
            for (int j = 0; j < QCS_PASS_FEATURES; ++j)
                features[QCS_PASS_FEATURES * i + j] = f[i].f[j];
            milliseconds[i] = ms[i];
        }
        *count = n;
    });
}

extern "C" int qcs_b200_cost_model_create(qcs_b200_cost_model **model, uint32_t seed)
{
    return guarded([&] {
        if (model == nullptr)
            throw std::runtime_error("result pointer must not be NULL");
        auto *h = new qcs_b200_cost_model();
        try
        {
            h->m = new qcsb::CostModel(seed);
        }
        catch (...)
        {
            delete h;
            throw;
        }
        *model = h;
    });
}

extern "C" int qcs_b200_cost_model_destroy(qcs_b200_cost_model *model)
{
    return guarded([&] {
        if (model == nullptr)
            return;
        delete model->m;
        delete model;
    });
}

extern "C" int qcs_b200_cost_model_train(qcs_b200_cost_model *model, const float *features, const float *targets,
                                         uint32_t count, uint32_t epochs, uint32_t batch, float learning_rate,
                                         float *final_loss)
{
    return guarded([&] {
        if (features == nullptr || targets == nullptr)
            throw std::runtime_error("cost model train: data pointers must not be NULL");
        const float loss = model_of(model).train(features, targets, (int)count, (int)epochs, (int)batch,
                                                 learning_rate, 12345u);
        if (final_loss)
            *final_loss = loss;
    });
}

extern "C" int qcs_b200_cost_model_predict(qcs_b200_cost_model *model, const float *features, uint32_t count,
                                           float *predictions)
{
    return guarded([&] {
        if (features == nullptr || predictions == nullptr)
            throw std::runtime_error("cost model predict: pointers must not be NULL");
        model_of(model).predict(features, (int)count, predictions);
    });
}

extern "C" int qcs_b200_cost_model_gradients(qcs_b200_cost_model *model, const float *inputs, const float *targets,
                                             uint32_t count, float *gradients, float *loss)
{
    return guarded([&] {
        if (inputs == nullptr || targets == nullptr || gradients == nullptr || count == 0)
            throw std::runtime_error("cost model gradients: pointers must not be NULL and count positive");
        const float l = model_of(model).gradients(inputs, targets, (int)count, gradients);
        if (loss)
            *loss = l;
    });
}

extern "C" int qcs_b200_cost_model_get_params(qcs_b200_cost_model *model, float *params, float *scaling)
{
    return guarded([&] {
        auto &m = model_of(model);
        if (params)
            m.get_params(params);
        if (scaling)
            m.get_scaling(scaling);
    });
}

extern "C" int qcs_b200_cost_model_set_params(qcs_b200_cost_model *model, const float *params, const float *scaling)
{
    return guarded([&] {
        auto &m = model_of(model);
        if (params)
            m.set_params(params);
        if (scaling)
            m.set_scaling(scaling);
    });
}

extern "C" int qcs_simulator_set_cost_model(qcs_simulator *sim, qcs_b200_cost_model *model)
{
    return guarded([&] { core(sim).set_cost_model(model ? model->m : nullptr); });
}

extern "C" int qcs_simulator_get_planner_judge(qcs_simulator *sim, int *learned_plan, double *greedy_ms,
                                               double *learned_ms)
{
    return guarded([&] {
        auto &c = core(sim);
        c.flush();
        auto *f = c.fused_executor();
        if (f == nullptr)
            throw std::runtime_error("get_planner_judge: allocate_memory must be called first");
        if (learned_plan)
            *learned_plan = f->last_plan_learned;
        if (greedy_ms)
            *greedy_ms = f->last_greedy_ms;
        if (learned_ms)
            *learned_ms = f->last_learned_ms;
    });
}

extern "C" int qcs_simulator_set_precision(qcs_simulator *sim, int amplitude_bits)
{
    return guarded([&] { core(sim).set_precision(amplitude_bits); });
}

extern "C" int qcs_simulator_get_precision(const qcs_simulator *sim, int *amplitude_bits)
{
    return guarded([&] { write_result(amplitude_bits, core(sim).precision()); });
}

extern "C" int qcs_simulator_get_amplitudes(qcs_simulator *sim, const uint64_t *indices, uint64_t count, double *amplitudes)
{
    return guarded([&] { core(sim).get_amplitudes(indices, count, amplitudes); });
}

extern "C" int qcs_simulator_get_device_state(qcs_simulator *sim, void **state, int *amplitude_bits)
{
    return guarded([&] {
        if (state == nullptr || amplitude_bits == nullptr)
            throw std::runtime_error("result pointer must not be NULL");
        void *p = core(sim).device_state_in_logical_order();
        *state = p;
        *amplitude_bits = core(sim).precision();
    });
}

extern "C" int qcs_simulator_compare(qcs_simulator *a, qcs_simulator *b, double *overlap_re, double *overlap_im,
                                     double *max_abs_diff, double *norm_a, double *norm_b)
{
    return guarded([&] {
        qcsb::Simulator::compare(core(a), core(b), overlap_re, overlap_im, max_abs_diff, norm_a, norm_b);
    });
}

// ------------------------------------------------------------------ batches

struct qcs_b200_batch
{
    qcsb::Batch *b = nullptr;
};

namespace
{
qcsb::Batch &batch_of(qcs_b200_batch *batch)
{
    if (batch == nullptr || batch->b == nullptr)
        throw std::runtime_error("batch handle is NULL");
    return *batch->b;
}
} // namespace

extern "C" int qcs_b200_batch_create(qcs_b200_batch **batch, int amplitude_bits)
{
    return guarded([&] {
        if (batch == nullptr)
            throw std::runtime_error("result pointer must not be NULL");
        auto *h = new qcs_b200_batch();
        try
        {
            h->b = new qcsb::Batch(amplitude_bits);
        }
        catch (...)
        {
            delete h;
            throw;
        }
        *batch = h;
    });
}

extern "C" int qcs_b200_batch_destroy(qcs_b200_batch *batch)
{
    return guarded([&] {
        if (batch == nullptr)
            throw std::runtime_error("batch handle is NULL");
        delete batch->b;
        delete batch;
    });
}

extern "C" int qcs_b200_batch_add_circuit(qcs_b200_batch *batch, int num_qubits, const qcs_b200_gate *gates,
                                          uint32_t num_gates, uint32_t *index)
{
    return guarded([&] {
        const uint32_t i = batch_of(batch).add_circuit(num_qubits, gates, num_gates);
        if (index)
            *index = i;
    });
}

namespace qcsb
{
void plan_summary(int n, const qcs_b200_gate *gates, uint64_t count, qcs_b200_plan_summary &out);
}

extern "C" int qcs_b200_plan_summary_get(int num_qubits, const qcs_b200_gate *gates, uint64_t num_gates,
                                         qcs_b200_plan_summary *summary)
{
    return guarded([&] {
        if (summary == nullptr)
            throw std::runtime_error("plan_summary: summary must not be NULL");
        qcsb::plan_summary(num_qubits, gates, num_gates, *summary);
    });
}

extern "C" int qcs_b200_batch_set_parameters(qcs_b200_batch *batch, const double *params, uint64_t count)
{
    return guarded([&] { batch_of(batch).set_parameters(params, count); });
}

extern "C" int qcs_b200_batch_run(qcs_b200_batch *batch)
{
    return guarded([&] { batch_of(batch).run(); });
}

extern "C" int qcs_b200_batch_expectation_z(qcs_b200_batch *batch, double *expectations, uint64_t count)
{
    return guarded([&] { batch_of(batch).expectation_z(expectations, count); });
}

extern "C" int qcs_b200_batch_get_statevector(qcs_b200_batch *batch, uint32_t index, double *amplitudes,
                                              uint64_t count)
{
    return guarded([&] { batch_of(batch).get_statevector(index, amplitudes, count); });
}

extern "C" int qcs_b200_batch_set_tensor_passes(qcs_b200_batch *batch, int mode)
{
    return guarded([&] { batch_of(batch).set_tensor_mode(mode); });
}

extern "C" int qcs_b200_batch_get_info(qcs_b200_batch *batch, qcs_b200_batch_info *info)
{
    return guarded([&] {
        if (info == nullptr)
            throw std::runtime_error("result pointer must not be NULL");
        batch_of(batch).info(info);
    });
}
