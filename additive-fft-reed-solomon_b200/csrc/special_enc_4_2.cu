// Encode kernel for n = 16, t = 4.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_4_2(const EncodeArgs& a, cudaStream_t s) { return launch_enc<4, 2>(a, s); }
}  // namespace spec
}  // namespace afrs
