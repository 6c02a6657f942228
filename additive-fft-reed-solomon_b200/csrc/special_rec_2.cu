// Recover kernels for n = 4.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_2(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<2>(a, sc, s);
}
}  // namespace spec
}  // namespace afrs
