// Plan construction per transform kind / data type, and synchronous
// execution for plfft_plan_execute.
#pragma once
#include <string>

#include "../../include/plfft.h"
#include "plan.hpp"

namespace plfft_b200 {

// Fill p.root and the execution bookkeeping from p.cfg (already validated).
plfft_status_t build_plan(PlanData& p, std::string* why);

// plfft_plan_execute: host or device pointers, returns when done.
plfft_status_t execute_sync(const PlanData& p, const void* in, void* out);

}  // namespace plfft_b200
