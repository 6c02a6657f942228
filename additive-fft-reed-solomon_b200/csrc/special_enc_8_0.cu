// Encode kernels for n = 256, t = 1.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_8_0(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_enc<8, 0>(a, sc, s);
}
cudaError_t launch_enc_jobs_8_0(const EncJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_enc_jobs<8, 0>(d, count, max_ncw, s);
}
}  // namespace spec
}  // namespace afrs
