#include "sp_internal.cuh"
namespace sp {
struct LvPlan {};
void free_lv_plan(LvPlan* p) { delete p; }
}  // namespace sp
