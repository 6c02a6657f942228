// Encode kernels for n = 8, t = 4.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_3_2(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_enc<3, 2>(a, sc, s);
}
}  // namespace spec
}  // namespace afrs
