#include "sp_internal.cuh"
namespace sp {
struct BcPlan {};
void free_bc_plan(BcPlan* p) { delete p; }
}  // namespace sp
