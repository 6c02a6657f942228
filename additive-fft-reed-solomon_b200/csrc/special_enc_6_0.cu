// Encode kernels for n = 64, t = 1.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_6_0(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_enc<6, 0>(a, sc, s);
}
}  // namespace spec
}  // namespace afrs
