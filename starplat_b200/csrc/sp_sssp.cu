#include "sp_internal.cuh"
namespace sp {
struct SsspPlan {};
void free_sssp_plan(SsspPlan* p) { delete p; }
}  // namespace sp
