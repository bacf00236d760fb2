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

// Argument rules shared by oct_edges_count and oct_edges_count_noalloc: both
// trees built with the same ndims and dtype; exclude_self only for a tree
// searched against itself; a batched tree only against itself with self
// pairs excluded.  Returns an oct_status and sets the context's message.
int oct_check_count_pair(oct_ctx* ctx, const oct_tree* query, const oct_tree* target, int exclude_self);
