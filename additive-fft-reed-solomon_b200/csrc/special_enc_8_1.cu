// Encode kernels for n = 256, t = 2.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_enc_8_1(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_enc<8, 1>(a, sc, s);
}
cudaError_t launch_enc_jobs_8_1(const EncJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_enc_jobs<8, 1>(d, count, max_ncw, s);
}
}  // namespace spec
}  // namespace afrs
