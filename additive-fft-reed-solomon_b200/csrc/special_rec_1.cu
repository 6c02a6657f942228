// Recover kernels for n = 2.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_1(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<1>(a, sc, s);
}
cudaError_t launch_rec_jobs_1(RecJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_rec_jobs<1>(d, count, max_ncw, s);
}
cudaError_t launch_rec_few_jobs_1(const FewJob* d, int count, size_t max_ncw, int logt, cudaStream_t s) {
  return launch_rec_few_jobs<1>(d, count, max_ncw, logt, s);
}
cudaError_t preload_rec_1() { return preload_rec<1>(); }
}  // namespace spec
}  // namespace afrs
