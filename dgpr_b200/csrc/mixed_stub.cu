// Placeholder until the mixed-precision kernels land: the precision is
// rejected at dgb_create.
#include "../../include/dgb200.h"
#include "mixed.hpp"

namespace dgb {

struct MixedState {};

int mixed_create(MixedState**, const Ops1D&, const std::vector<double>&, const double*, const int*, long,
                 const DevParams&)
{
  return DGB_ERR_UNSUPPORTED;
}
void mixed_destroy(MixedState* m) { delete m; }
int mixed_residual(MixedState*, const double*, double*, double*, cudaStream_t) { return DGB_ERR_UNSUPPORTED; }
int mixed_step(MixedState*, int, double, double*, double*, double*, double*, double*, int*, int*, cudaStream_t,
               cudaEvent_t*)
{
  return DGB_ERR_UNSUPPORTED;
}
int mixed_initial_traces(MixedState*, const double*, cudaStream_t) { return DGB_ERR_UNSUPPORTED; }
long long mixed_launches_per_step(const MixedState*, int) { return 0; }

}  // namespace dgb
