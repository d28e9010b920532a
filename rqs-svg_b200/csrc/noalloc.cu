// Allocation-free entry point for the per-qubit squared-norm sums.
//
// Some callers cannot let a library allocate device memory: code that runs
// inside a framework whose caching allocator owns the GPU's memory (a
// cudaMalloc behind its back can fail or fragment its pool), real-time loops
// where an allocation's latency or possible failure is not acceptable, and
// code paths that must not synchronise the device, which cudaMalloc and
// cudaFree may do. qcs_b200_zsums_noalloc serves them: the caller passes the
// state and the output in its own device memory, and the reduction's scratch
// lives in the fixed-size array below, which every GPU that loads the
// library holds until the process exits.
//
// The array keeps the last call's contents between calls; every call writes
// each partial sum it reads before reading it, so nothing needs clearing.
// Calls share the array, so calls that overlap on the GPU (on different
// streams, or from different host threads, on the same device) race and
// must be serialised by the caller.

#include "qcs_internal.h"
#include "qcs_b200.h"

#include <cstring>
#include <mutex>

namespace qcsb
{
namespace
{

// Largest register the entry point accepts, and the scratch that needs:
// at most 512 partial blocks x (kNoAllocMaxQubits + 1) doubles = 168 KiB.
constexpr int kNoAllocMaxQubits = kMaxQubits;
constexpr int kNoAllocPartials = 512 * (kNoAllocMaxQubits + 1);

static __device__ __align__(256) double g_zsum_scratch[kNoAllocPartials];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, fetched once
// per device with that device current. In host code the array's name is a
// host-side stand-in, not a device address, so only this pointer is passed
// to kernels.
double *scratch_for_current_device()
{
    int dev = 0;
    QCSB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        throw std::runtime_error(strformat("qcs_b200_zsums_noalloc: device %d is beyond the supported %d", dev, kMaxDevices));
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_ptr[dev] == nullptr)
    {
        void *p = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&p, g_zsum_scratch);
        if (err != cudaSuccess || p == nullptr)
            throw std::runtime_error(strformat("qcs_b200_zsums_noalloc: cudaGetSymbolAddress failed: %s",
                                               cudaGetErrorString(err)));
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    return g_scratch_ptr[dev];
}

} // namespace
} // namespace qcsb

extern "C" int qcs_b200_zsums_noalloc(const double *state_device, int num_qubits, double *sums_device, void *stream)
{
    try
    {
        if (num_qubits < 1 || num_qubits > qcsb::kNoAllocMaxQubits)
            throw std::runtime_error(qcsb::strformat(
                "qcs_b200_zsums_noalloc: num_qubits %d is outside [1, %d], the largest register its fixed scratch serves",
                num_qubits, qcsb::kNoAllocMaxQubits));
        if (state_device == nullptr || sums_device == nullptr)
            throw std::runtime_error("qcs_b200_zsums_noalloc: state and sums pointers must not be NULL");
        if ((reinterpret_cast<uintptr_t>(state_device) & 15u) != 0)
            throw std::runtime_error("qcs_b200_zsums_noalloc: the state must be 16-byte aligned");
        double *scratch = qcsb::scratch_for_current_device();
        qcsb::launch_zsums(reinterpret_cast<const double2 *>(state_device), num_qubits, scratch, sums_device,
                           static_cast<cudaStream_t>(stream));
        return 1;
    }
    catch (const std::exception &e)
    {
        qcsb::report_error(e.what());
    }
    catch (...)
    {
        qcsb::report_error("Unknown C++ exception");
    }
    return 0;
}
