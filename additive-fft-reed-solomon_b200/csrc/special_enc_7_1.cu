// Encode kernel for n = 128, t = 2.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_7_1(const EncodeArgs& a, cudaStream_t s) { return launch_enc<7, 1>(a, s); }
}  // namespace spec
}  // namespace afrs
