// Recover kernels for n = 64.
#include "special.cuh"

namespace afrs {
namespace spec {
cudaError_t launch_rec_6(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  return launch_rec<6>(a, sc, s);
}
cudaError_t launch_rec_jobs_6(RecJob* d, int count, size_t max_ncw, cudaStream_t s) {
  return launch_rec_jobs<6>(d, count, max_ncw, s);
}
cudaError_t launch_rec_few_jobs_6(const FewJob* d, int count, size_t max_ncw, int logt, cudaStream_t s) {
  return launch_rec_few_jobs<6>(d, count, max_ncw, logt, s);
}
cudaError_t preload_rec_6() { return preload_rec<6>(); }
}  // namespace spec
}  // namespace afrs
