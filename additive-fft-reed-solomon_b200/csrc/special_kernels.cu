// Dispatch of the specialised (compile-time-twiddle) kernels by shape.
#include "special.cuh"

namespace afrs {

cudaError_t launch_encode_special(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  const int ln = __builtin_ctz((unsigned)a.n), lt = __builtin_ctz((unsigned)a.t);
  switch (ln) {
    case 1:
      switch (lt) {
        case 0: return spec::launch_enc_1_0(a, sc, s);
        default: return cudaErrorNotSupported;
      }
    case 2:
      switch (lt) {
        case 0: return spec::launch_enc_2_0(a, sc, s);
        case 1: return spec::launch_enc_2_1(a, sc, s);
        default: return cudaErrorNotSupported;
      }
    case 3:
      switch (lt) {
        case 0: return spec::launch_enc_3_0(a, sc, s);
        case 1: return spec::launch_enc_3_1(a, sc, s);
        case 2: return spec::launch_enc_3_2(a, sc, s);
        default: return cudaErrorNotSupported;
      }
    case 4:
      switch (lt) {
        case 0: return spec::launch_enc_4_0(a, sc, s);
        case 1: return spec::launch_enc_4_1(a, sc, s);
        case 2: return spec::launch_enc_4_2(a, sc, s);
        case 3: return spec::launch_enc_4_3(a, sc, s);
        default: return cudaErrorNotSupported;
      }
    case 5:
      switch (lt) {
        case 0: return spec::launch_enc_5_0(a, sc, s);
        case 1: return spec::launch_enc_5_1(a, sc, s);
        case 2: return spec::launch_enc_5_2(a, sc, s);
        case 3: return spec::launch_enc_5_3(a, sc, s);
        case 4: return spec::launch_enc_5_4(a, sc, s);
        default: return cudaErrorNotSupported;
      }
    case 6:
      switch (lt) {
        case 0: return spec::launch_enc_6_0(a, sc, s);
        case 1: return spec::launch_enc_6_1(a, sc, s);
        case 2: return spec::launch_enc_6_2(a, sc, s);
        case 3: return spec::launch_enc_6_3(a, sc, s);
        case 4: return spec::launch_enc_6_4(a, sc, s);
        case 5: return spec::launch_enc_6_5(a, sc, s);
        default: return cudaErrorNotSupported;
      }
    case 7:
      switch (lt) {
        case 0: return spec::launch_enc_7_0(a, sc, s);
        case 1: return spec::launch_enc_7_1(a, sc, s);
        case 2: return spec::launch_enc_7_2(a, sc, s);
        case 3: return spec::launch_enc_7_3(a, sc, s);
        case 4: return spec::launch_enc_7_4(a, sc, s);
        case 5: return spec::launch_enc_7_5(a, sc, s);
        case 6: return spec::launch_enc_7_6(a, sc, s);
        default: return cudaErrorNotSupported;
      }
    case 8:
      switch (lt) {
        case 0: return spec::launch_enc_8_0(a, sc, s);
        case 1: return spec::launch_enc_8_1(a, sc, s);
        case 2: return spec::launch_enc_8_2(a, sc, s);
        case 3: return spec::launch_enc_8_3(a, sc, s);
        case 4: return spec::launch_enc_8_4(a, sc, s);
        case 5: return spec::launch_enc_8_5(a, sc, s);
        case 6: return spec::launch_enc_8_6(a, sc, s);
        case 7: return spec::launch_enc_8_7(a, sc, s);
        default: return cudaErrorNotSupported;
      }
    default: return cudaErrorNotSupported;
  }
}

cudaError_t launch_recover_special(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  switch (__builtin_ctz((unsigned)a.n)) {
    case 1: return spec::launch_rec_1(a, sc, s);
    case 2: return spec::launch_rec_2(a, sc, s);
    case 3: return spec::launch_rec_3(a, sc, s);
    case 4: return spec::launch_rec_4(a, sc, s);
    case 5: return spec::launch_rec_5(a, sc, s);
    case 6: return spec::launch_rec_6(a, sc, s);
    case 7: return spec::launch_rec_7(a, sc, s);
    case 8: return spec::launch_rec_8(a, sc, s);
    default: return cudaErrorNotSupported;
  }
}

size_t scratch_bytes_encode(int n, int t, size_t L) { return spec::scratch_full_bytes_enc(n, t, L); }
size_t scratch_bytes_recover(int n, size_t L) { return spec::scratch_full_bytes_rec(n, L); }

}  // namespace afrs
