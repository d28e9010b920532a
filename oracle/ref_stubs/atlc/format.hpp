#pragma once
#include "stub_common.hpp"
