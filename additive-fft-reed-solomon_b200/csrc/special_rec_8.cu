// Recover kernel for n = 256.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_8(const RecoverArgs& a, cudaStream_t s) { return launch_rec<8>(a, s); }
}  // namespace spec
}  // namespace afrs
