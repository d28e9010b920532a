// bin/qcs: runs a circuit shared object against libqcs.so.
//
// Command line and output match the reference driver (src/qcs_main.cpp,
// options from src/qcs_args.ggo:8-11):
//   qcs [-s N | --num-samples N] [--mapping p2l.csv] [-r | --reversed-mapping]
//       [--output-statevector FILE] circuit.so
// The circuit exports circuit_init(qcs_simulator*) and
// circuit_run(qcs_simulator*); circuit_run is executed once per sample and
// each sample prints
//   {"sample_num": i, "clbits": "<highest clbit first>", "elapsed_time": s}
// Between samples the mapping, state, clbits and measurement bookkeeping are
// reset (src/qcs_main.cpp:186-192). Errors print a message to stderr and exit
// with status 1.

#include <qcs.h>

#include <dlfcn.h>
#include <getopt.h>

#include <cstdio>
#include <cstdlib>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace
{

void usage(FILE *out)
{
    std::fprintf(out,
                 "Usage: qcs [OPTIONS] USER_CIRCUIT_SO\n"
                 "B200 state-vector quantum circuit simulator\n\n"
                 "  -s, --num-samples=INT          Number of measurement samples (default 1)\n"
                 "      --mapping=STRING           Comma-separated physical-to-logical qubit mapping\n"
                 "  -r, --reversed-mapping         Reverse the qubit mapping (swap perm_p2l/perm_l2p)\n"
                 "      --output-statevector=FILE  Write final statevector to the specified file\n"
                 "  -h, --help                     Print help and exit\n"
                 "  -V, --version                  Print version and exit\n");
}

std::vector<bit_num_t> parse_mapping_csv(const std::string &text)
{
    if (text.empty())
        throw std::runtime_error("mapping string must not be empty");
    std::vector<bit_num_t> mapping;
    std::stringstream ss(text);
    std::string token;
    while (std::getline(ss, token, ','))
    {
        if (token.empty())
            throw std::runtime_error("mapping contains an empty entry");
        mapping.push_back(static_cast<bit_num_t>(std::stoi(token)));
    }
    return mapping;
}

std::vector<bit_num_t> invert_mapping(const std::vector<bit_num_t> &p2l, int n)
{
    if ((int)p2l.size() != n)
        throw std::runtime_error("mapping size " + std::to_string(p2l.size()) + " does not match num_qubits " + std::to_string(n));
    std::vector<bit_num_t> l2p(n, -1);
    for (int p = 0; p < n; ++p)
    {
        const int l = p2l[p];
        if (l < 0 || l >= n)
            throw std::runtime_error("mapping value " + std::to_string(l) + " is out of range [0, " + std::to_string(n) + ")");
        if (l2p[l] != -1)
            throw std::runtime_error("mapping value " + std::to_string(l) + " appears multiple times");
        l2p[l] = static_cast<bit_num_t>(p);
    }
    return l2p;
}

std::string g_last_error;
void on_error(const char *msg, size_t len) { g_last_error.assign(msg, len); }

void check(int ok, const char *what)
{
    if (!ok)
        throw std::runtime_error(std::string(what) + " failed" + (g_last_error.empty() ? "" : ": " + g_last_error));
}

int run(int argc, char **argv)
{
    int num_samples = 1;
    bool mapping_given = false, reversed = false;
    std::string mapping_text, output_path;
    static const option longopts[] = {
        {"num-samples", required_argument, nullptr, 's'},
        {"mapping", required_argument, nullptr, 'm'},
        {"reversed-mapping", no_argument, nullptr, 'r'},
        {"output-statevector", required_argument, nullptr, 'o'},
        {"help", no_argument, nullptr, 'h'},
        {"version", no_argument, nullptr, 'V'},
        {nullptr, 0, nullptr, 0},
    };
    int c;
    while ((c = getopt_long(argc, argv, "s:rhV", longopts, nullptr)) != -1)
    {
        switch (c)
        {
        case 's':
        {
            char *end = nullptr;
            const long v = std::strtol(optarg, &end, 10);
            if (end == optarg || *end != '\0')
                throw std::runtime_error("--num-samples requires an integer");
            num_samples = static_cast<int>(v);
            break;
        }
        case 'm':
            mapping_given = true;
            mapping_text = optarg;
            break;
        case 'r':
            reversed = true;
            break;
        case 'o':
            output_path = optarg;
            break;
        case 'h':
            usage(stdout);
            return 0;
        case 'V':
            std::printf("qcs 1.0 (B200)\n");
            return 0;
        default:
            usage(stderr);
            return 1;
        }
    }
    if (argc - optind != 1)
        throw std::runtime_error("user circuit shared object path is required");
    if (num_samples <= 0)
        throw std::runtime_error("num_samples must be greater than 0");

    qcs_set_exception_callback(on_error);
    qcs_simulator *sim = nullptr;
    check(qcs_simulator_create(&sim), "qcs_simulator_create");
    struct Guard
    {
        qcs_simulator *s;
        ~Guard() { qcs_simulator_destroy(s); }
    } guard{sim};

    char *abspath = realpath(argv[optind], nullptr);
    if (abspath == nullptr)
        throw std::runtime_error("realpath returned NULL");
    void *dl = dlopen(abspath, RTLD_LAZY);
    std::free(abspath);
    if (dl == nullptr)
        throw std::runtime_error(std::string("dlopen failed: ") + dlerror());
    using fn_t = void (*)(qcs_simulator *);
    auto circuit_init = reinterpret_cast<fn_t>(dlsym(dl, "circuit_init"));
    auto circuit_run = reinterpret_cast<fn_t>(dlsym(dl, "circuit_run"));
    if (circuit_init == nullptr || circuit_run == nullptr)
        throw std::runtime_error("circuit shared object must export circuit_init and circuit_run");

    circuit_init(sim);

    bit_t nq = 0;
    check(qcs_simulator_get_num_qubits(sim, &nq), "qcs_simulator_get_num_qubits");
    std::vector<bit_num_t> mapping;
    if (mapping_given)
        mapping = parse_mapping_csv(mapping_text);
    else
        for (int q = 0; q < nq; ++q)
            mapping.push_back(static_cast<bit_num_t>(q));
    if (reversed)
        mapping = invert_mapping(mapping, nq);
    check(qcs_simulator_set_mapping(sim, mapping.data(), static_cast<bit_num_t>(mapping.size())), "qcs_simulator_set_mapping");
    check(qcs_simulator_allocate_memory(sim), "qcs_simulator_allocate_memory");

    bit_t e1 = 0, e2 = 0;
    check(qcs_simulator_event_create(sim, &e1) && qcs_simulator_event_create(sim, &e2), "qcs_simulator_event_create");
    for (int sample = 0; sample < num_samples; ++sample)
    {
        check(qcs_simulator_event_record(sim, e1), "qcs_simulator_event_record");
        circuit_run(sim);
        check(qcs_simulator_event_record(sim, e2), "qcs_simulator_event_record");
        double elapsed = 0.0;
        check(qcs_simulator_event_get_elapsed_time(sim, e1, e2, &elapsed), "qcs_simulator_event_get_elapsed_time");
        bit_t ncl = 0;
        check(qcs_simulator_get_num_clbits(sim, &ncl), "qcs_simulator_get_num_clbits");
        std::vector<char> clbits(ncl + 1);
        check(qcs_simulator_get_clbits_string(sim, clbits.data()), "qcs_simulator_get_clbits_string");
        std::fprintf(stdout, "{\"sample_num\": %d, \"clbits\": \"%s\", \"elapsed_time\": %.18g}\n", sample, clbits.data(), elapsed);
        std::fflush(stdout);
        if (sample != num_samples - 1)
        {
            qcs_simulator_reinitialize_mapping(sim);
            qcs_simulator_set_zero_state(sim);
            qcs_simulator_reset_clbits(sim);
            qcs_simulator_reset_measurement_state(sim);
        }
    }
    if (!output_path.empty())
        check(qcs_simulator_save_statevector(sim, output_path.c_str()), "qcs_simulator_save_statevector");
    return 0;
}

} // namespace

int main(int argc, char **argv)
{
    try
    {
        return run(argc, argv);
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "qcs: %s\n", e.what());
        return 1;
    }
}
