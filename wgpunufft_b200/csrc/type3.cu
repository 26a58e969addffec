// Type-3 plans.
#include "type3.h"

namespace b200nufft {

Type3Plan::Type3Plan(const b200nufft_type3_config&) {
  throw NufftFailure{B200NUFFT_PRECISION_UNSUPPORTED, "type-3 plans are not built yet"};
}

void Type3Plan::set_points(int64_t, const void*, int64_t, const void*, cudaStream_t) {}
void Type3Plan::execute(int64_t, const void*, void*, cudaStream_t) {}
void Type3Plan::info(b200nufft_type3_info*) const {}

}  // namespace b200nufft
