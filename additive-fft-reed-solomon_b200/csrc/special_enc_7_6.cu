// Encode kernels for n = 128, t = 64.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_7_6(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_enc<7, 6>(a, sc, s);
}
cudaError_t launch_enc_jobs_7_6(const EncJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_enc_jobs<7, 6>(d, count, max_ncw, s);
}
}  // namespace spec
}  // namespace afrs
