// Encode kernel for n = 32, t = 4.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_5_2(const EncodeArgs& a, cudaStream_t s) { return launch_enc<5, 2>(a, s); }
}  // namespace spec
}  // namespace afrs
