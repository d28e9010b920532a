#pragma once
#include "stub_common.hpp"
#include <cuda_runtime.h>

// The check runs the call unchanged. For parity tests at full register size
// it also notes every buffer the reference allocates through cudaMallocAsync
// (its state vector among them, src/qcs.cu:1956) and forgets it at
// cudaFreeAsync, so that a test in the same process can read the reference's
// amplitudes in place instead of through a multi-gigabyte file.
namespace atlc
{
namespace stub
{
struct device_buffer
{
    void *ptr;
    size_t bytes;
};
constexpr int kMaxBuffers = 64;
inline device_buffer buffers[kMaxBuffers];

template <typename... Args>
inline void note_call(const char *, cudaError_t, const Args &...)
{
}
template <typename T>
inline void note_call(const char *name, cudaError_t code, T **const &ptr, const size_t &bytes, const cudaStream_t &)
{
    if (code != cudaSuccess || std::string(name) != "cudaMallocAsync")
        return;
    for (device_buffer &b : buffers)
        if (b.ptr == nullptr)
        {
            b = {static_cast<void *>(*ptr), bytes};
            return;
        }
}
template <typename T>
inline void note_call(const char *name, cudaError_t code, T *const &ptr, const cudaStream_t &)
{
    if (code != cudaSuccess || std::string(name) != "cudaFreeAsync")
        return;
    for (device_buffer &b : buffers)
        if (b.ptr == static_cast<void *>(ptr))
            b = {nullptr, 0};
}
// code: the call's result (the call itself stays in the macro, so that
// overloads and templates resolve as they do without the note)
template <typename... Args>
inline cudaError_t noted(const char *name, cudaError_t code, const Args &...args)
{
    note_call(name, code, args...);
    return code;
}
} // namespace stub
} // namespace atlc

// The largest live buffer the reference allocated (its state vector once
// allocate_memory has run): 1 and its address and size, or 0 when none.
extern "C" __attribute__((visibility("default"), used)) inline int qcs_ref_stub_largest_buffer(void **ptr,
                                                                                              size_t *bytes)
{
    const atlc::stub::device_buffer *best = nullptr;
    for (const atlc::stub::device_buffer &b : atlc::stub::buffers)
        if (b.ptr != nullptr && (best == nullptr || b.bytes > best->bytes))
            best = &b;
    if (best == nullptr)
        return 0;
    *ptr = best->ptr;
    *bytes = best->bytes;
    return 1;
}

#define ATLC_CHECK_CUDA(func, ...)                                                                              \
    ::atlc::check_code<cudaError_t>(::atlc::stub::noted(#func, func(__VA_ARGS__), __VA_ARGS__), cudaSuccess, #func, \
                                    __FILE__, __LINE__)
