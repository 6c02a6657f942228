// Recover kernels for n = 128.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_7(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<7>(a, sc, s);
}
}  // namespace spec
}  // namespace afrs
