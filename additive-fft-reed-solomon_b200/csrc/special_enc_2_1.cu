// Encode kernel for n = 4, t = 2.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_2_1(const EncodeArgs& a, cudaStream_t s) { return launch_enc<2, 1>(a, s); }
}  // namespace spec
}  // namespace afrs
