// Recover kernels for n = 16.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_4(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<4>(a, sc, s);
}
}  // namespace spec
}  // namespace afrs
