#pragma once
#include "stub_common.hpp"
#include <cuda_runtime.h>
namespace atlc
{
template <typename... KArgs, typename... Args>
cudaError_t cudaLaunchKernel(void (*kernel)(KArgs...), unsigned long long grid, unsigned long long block,
                             size_t shmem, cudaStream_t stream, Args &&...args)
{
    kernel<<<dim3((unsigned)grid), dim3((unsigned)block), shmem, stream>>>(std::forward<Args>(args)...);
    return cudaGetLastError();
}
} // namespace atlc
