// skm_table.cuh -- phase-table fast path (stationary kernel on commensurate grids).
// Not planned for this evaluator: every call takes the generic kernels.
#pragma once

#include "skm_kernels.cuh"

namespace skm {

struct TablePlan {
    bool enabled = false;
};

inline int table_plan(TablePlan &t, const EvalParams &, int, cudaStream_t)
{
    t.enabled = false;
    return 0;
}

inline int table_value(TablePlan &, const EvalParams &, float4 *, double *, int, cudaStream_t) { return 3; }
inline int table_derivative(TablePlan &, const EvalParams &, const DerivParams &, int, cudaStream_t) { return 3; }
inline void table_free(TablePlan &) {}

}  // namespace skm
