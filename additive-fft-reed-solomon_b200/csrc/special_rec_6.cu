// Recover kernels for n = 64.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_6(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<6>(a, sc, s);
}
}  // namespace spec
}  // namespace afrs
