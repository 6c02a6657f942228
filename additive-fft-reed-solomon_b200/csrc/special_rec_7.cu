// Recover kernels for n = 128.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_7(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<7>(a, sc, s);
}
cudaError_t launch_rec_jobs_7(RecJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_rec_jobs<7>(d, count, max_ncw, s);
}
cudaError_t launch_rec_few_jobs_7(const FewJob* d, int count, size_t max_ncw, int logt, cudaStream_t s) {
  return launch_rec_few_jobs<7>(d, count, max_ncw, logt, s);
}
cudaError_t preload_rec_7() { return preload_rec<7>(); }
}  // namespace spec
}  // namespace afrs
