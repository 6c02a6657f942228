// Encode kernels for n = 128, t = 8.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_7_3(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_enc<7, 3>(a, sc, s);
}
}  // namespace spec
}  // namespace afrs
