// Encode kernels for n = 256, t = 32.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_8_5(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_enc<8, 5>(a, sc, s);
}
cudaError_t launch_enc_jobs_8_5(const EncJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_enc_jobs<8, 5>(d, count, max_ncw, s);
}
}  // namespace spec
}  // namespace afrs
