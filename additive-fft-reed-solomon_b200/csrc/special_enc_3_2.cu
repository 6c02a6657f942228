// Encode kernels for n = 8, t = 4.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_3_2(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_enc<3, 2>(a, sc, s);
}
cudaError_t launch_enc_jobs_3_2(const EncJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_enc_jobs<3, 2>(d, count, max_ncw, s);
}
}  // namespace spec
}  // namespace afrs
