// Host-side helpers shared by the C ABI translation units.
#pragma once

#include <string>

#include "../../include/ibgpu.h"
#include "layout.h"

namespace ibgpu {
int validate_case(const ibgpu_case *cs);
void fill_case_const(const ibgpu_case *cs, CaseConst &k);
void set_last_error(const std::string &msg);
}  // namespace ibgpu
