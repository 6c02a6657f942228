// Recover kernels for n = 256.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_8(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<8>(a, sc, s);
}
cudaError_t launch_rec_jobs_8(RecJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_rec_jobs<8>(d, count, max_ncw, s);
}
cudaError_t launch_rec_few_jobs_8(const FewJob* d, int count, size_t max_ncw, int logt, cudaStream_t s) {
  return launch_rec_few_jobs<8>(d, count, max_ncw, logt, s);
}
cudaError_t preload_rec_8() { return preload_rec<8>(); }
}  // namespace spec
}  // namespace afrs
