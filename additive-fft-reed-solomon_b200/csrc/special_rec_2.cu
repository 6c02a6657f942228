// Recover kernels for n = 4.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_2(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<2>(a, sc, s);
}
cudaError_t launch_rec_jobs_2(RecJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_rec_jobs<2>(d, count, max_ncw, s);
}
cudaError_t launch_rec_few_jobs_2(const FewJob* d, int count, size_t max_ncw, int logt, cudaStream_t s) {
  return launch_rec_few_jobs<2>(d, count, max_ncw, logt, s);
}
cudaError_t preload_rec_2() { return preload_rec<2>(); }
}  // namespace spec
}  // namespace afrs
