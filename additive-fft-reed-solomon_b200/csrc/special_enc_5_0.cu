// Encode kernels for n = 32, t = 1.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_5_0(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_enc<5, 0>(a, sc, s);
}
}  // namespace spec
}  // namespace afrs
