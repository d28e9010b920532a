// LD_PRELOAD shim that pins std::random_device for shot-parity runs: the
// reference seeds its measurement engine with std::random_device()()
// (src/qcs.cu:1845-1852), which calls this member. The value comes from the
// environment variable QCS_REF_SEED (default 12345). Test infrastructure.
#include <cstdlib>
#include <random>

unsigned int std::random_device::_M_getval()
{
    const char *e = std::getenv("QCS_REF_SEED");
    return e ? static_cast<unsigned int>(std::strtoul(e, nullptr, 10)) : 12345u;
}
