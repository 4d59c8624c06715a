// qk_handles.h -- definitions of the opaque handles of the C ABI that more
// than one translation unit of the library needs.
#pragma once

#include "mc_plan.h"

struct qk_mc_plan {
    qkb::Plan plan;
};
