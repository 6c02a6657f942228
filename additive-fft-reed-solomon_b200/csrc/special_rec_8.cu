// Recover kernels for n = 256.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_8(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<8>(a, sc, s);
}
}  // namespace spec
}  // namespace afrs
