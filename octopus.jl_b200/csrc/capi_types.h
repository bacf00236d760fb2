// Definitions of the opaque C-ABI handles (include/octopus_b200.h).
#pragma once

#include "internal.h"

struct oct_ctx {
    oct::Ctx c;
};
struct oct_tree {
    oct::Tree t;
    oct_ctx* owner = nullptr;
};
