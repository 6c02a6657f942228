// Encode kernels for n = 64, t = 32.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_6_5(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_enc<6, 5>(a, sc, s);
}
}  // namespace spec
}  // namespace afrs
