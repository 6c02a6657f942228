// Recover kernels for n = 2.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_1(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<1>(a, sc, s);
}
}  // namespace spec
}  // namespace afrs
