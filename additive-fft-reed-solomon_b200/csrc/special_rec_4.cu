// Recover kernels for n = 16.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_4(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<4>(a, sc, s);
}
cudaError_t launch_rec_jobs_4(RecJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_rec_jobs<4>(d, count, max_ncw, s);
}
cudaError_t launch_rec_few_jobs_4(const FewJob* d, int count, size_t max_ncw, int logt, cudaStream_t s) {
  return launch_rec_few_jobs<4>(d, count, max_ncw, logt, s);
}
cudaError_t preload_rec_4() { return preload_rec<4>(); }
}  // namespace spec
}  // namespace afrs
