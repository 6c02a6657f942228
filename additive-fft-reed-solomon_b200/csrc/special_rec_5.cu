// Recover kernel for n = 32.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_5(const RecoverArgs& a, cudaStream_t s) { return launch_rec<5>(a, s); }
}  // namespace spec
}  // namespace afrs
