#pragma once
#include "stub_common.hpp"
#include <cuda_runtime.h>
#define ATLC_CHECK_CUDA(func, ...) ::atlc::check_code<cudaError_t>(func(__VA_ARGS__), cudaSuccess, #func, __FILE__, __LINE__)
