// Compile-time-twiddle kernels for the throughput shapes (filled in below as
// they are built).  Shapes without a specialisation use generic_kernels.cu.
#include "afrs_internal.h"

namespace afrs {

cudaError_t launch_encode_special(const EncodeArgs&, cudaStream_t) { return cudaErrorNotSupported; }
cudaError_t launch_recover_special(const RecoverArgs&, cudaStream_t) { return cudaErrorNotSupported; }

}  // namespace afrs
