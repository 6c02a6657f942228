// Encode kernels for n = 16, t = 1.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_4_0(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_enc<4, 0>(a, sc, s);
}
cudaError_t launch_enc_jobs_4_0(const EncJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_enc_jobs<4, 0>(d, count, max_ncw, s);
}
}  // namespace spec
}  // namespace afrs
