// Encode kernels for n = 2, t = 1.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_1_0(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_enc<1, 0>(a, sc, s);
}
cudaError_t launch_enc_jobs_1_0(const EncJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_enc_jobs<1, 0>(d, count, max_ncw, s);
}
}  // namespace spec
}  // namespace afrs
