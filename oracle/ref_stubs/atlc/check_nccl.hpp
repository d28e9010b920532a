#pragma once
#include "stub_common.hpp"
#include <nccl.h>
#define ATLC_CHECK_NCCL(func, ...) ::atlc::check_code<ncclResult_t>(func(__VA_ARGS__), ncclSuccess, #func, __FILE__, __LINE__)
