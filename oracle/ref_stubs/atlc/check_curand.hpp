#pragma once
#include "stub_common.hpp"
#include <curand.h>
#define ATLC_CHECK_CURAND(func, ...) ::atlc::check_code<curandStatus_t>(func(__VA_ARGS__), CURAND_STATUS_SUCCESS, #func, __FILE__, __LINE__)
