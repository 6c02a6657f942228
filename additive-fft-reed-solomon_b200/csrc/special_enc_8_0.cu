// Encode kernel for n = 256, t = 1.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_8_0(const EncodeArgs& a, cudaStream_t s) { return launch_enc<8, 0>(a, s); }
}  // namespace spec
}  // namespace afrs
