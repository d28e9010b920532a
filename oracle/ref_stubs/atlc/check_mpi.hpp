#pragma once
#include "stub_common.hpp"
#define ATLC_CHECK_MPI(func, ...) ::atlc::check_code<int>(func(__VA_ARGS__), 0, #func, __FILE__, __LINE__)
