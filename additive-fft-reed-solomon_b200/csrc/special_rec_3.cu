// Recover kernels for n = 8.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_3(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<3>(a, sc, s);
}
cudaError_t launch_rec_jobs_3(RecJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_rec_jobs<3>(d, count, max_ncw, s);
}
cudaError_t launch_rec_few_jobs_3(const FewJob* d, int count, size_t max_ncw, int logt, cudaStream_t s) {
  return launch_rec_few_jobs<3>(d, count, max_ncw, logt, s);
}
cudaError_t preload_rec_3() { return preload_rec<3>(); }
}  // namespace spec
}  // namespace afrs
