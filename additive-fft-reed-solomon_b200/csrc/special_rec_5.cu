// Recover kernels for n = 32.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_5(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<5>(a, sc, s);
}
cudaError_t launch_rec_jobs_5(RecJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_rec_jobs<5>(d, count, max_ncw, s);
}
cudaError_t launch_rec_few_jobs_5(const FewJob* d, int count, size_t max_ncw, int logt, cudaStream_t s) {
  return launch_rec_few_jobs<5>(d, count, max_ncw, logt, s);
}
cudaError_t preload_rec_5() { return preload_rec<5>(); }
}  // namespace spec
}  // namespace afrs
