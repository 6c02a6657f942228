// Encode kernels for n = 32, t = 16.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_5_4(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_enc<5, 4>(a, sc, s);
}
cudaError_t launch_enc_jobs_5_4(const EncJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_enc_jobs<5, 4>(d, count, max_ncw, s);
}
}  // namespace spec
}  // namespace afrs
