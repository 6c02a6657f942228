// Dispatch of the specialised (compile-time-twiddle) kernels by shape.
#include <cstring>

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

cudaError_t preload_recover_special() {
  cudaError_t (*const fns[])() = {spec::preload_rec_1, spec::preload_rec_2, spec::preload_rec_3, spec::preload_rec_4,
                                   spec::preload_rec_5, spec::preload_rec_6, spec::preload_rec_7, spec::preload_rec_8};
  for (auto f : fns) {
    cudaError_t e = f();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

size_t scratch_bytes_encode(int n, int t, size_t L) { return spec::scratch_full_bytes_enc(n, t, L); }
size_t scratch_bytes_recover(int n, size_t L) { return spec::scratch_full_bytes_rec(n, L); }


// ---- grouped launches (afrs_batch_dev) --------------------------------------

bool jobs_supported(int op, int n, int t) {
  return n >= (op == 2 ? 32 : 2) && n <= 256 && t >= 1 && t < n;
}

size_t job_desc_bytes(int op) {
  return op == 0 ? sizeof(spec::EncJob) : (op == 1 ? sizeof(spec::RecJob) : sizeof(spec::FewJob));
}

size_t job_scratch_bytes(int op, int n, int t, size_t L) {
  return op == 0 ? spec::scratch_full_bytes_enc(n, t, L) : (op == 1 ? spec::scratch_full_bytes_rec(n, L) : 0);
}

size_t job_colwords(size_t L) { return spec::total_colwords(L); }

void fill_enc_job(void* desc, const EncodeArgs& a, uint32_t* scratch) {
  spec::EncJob j{};
  j.a = a;
  j.s1 = scratch;
  j.ncw = spec::total_colwords(a.L);
  std::memcpy(desc, &j, sizeof j);
}

void fill_rec_job(void* desc, const RecoverArgs& a, uint32_t* scratch) {
  spec::RecJob j{};
  j.a = a;
  j.ncw = spec::total_colwords(a.L);
  j.s1 = scratch;
  j.s2 = scratch + (size_t)a.n * j.ncw * 8;
  // j.loc is filled on the device (k_rec_jobs_locator) before the kernels run.
  for (int q = 0; q < a.e; q++) j.gmask |= 1u << (a.pos[q] >> 4);
  std::memcpy(desc, &j, sizeof j);
}

cudaError_t launch_encode_jobs(int n, int t, const void* d_jobs, int count, size_t max_ncw, cudaStream_t s) {
  const auto* d = static_cast<const spec::EncJob*>(d_jobs);
  const int ln = __builtin_ctz((unsigned)n), lt = __builtin_ctz((unsigned)t);
  switch (ln) {
    case 1:
      switch (lt) {
        case 0: return spec::launch_enc_jobs_1_0(d, count, max_ncw, s);
        default: return cudaErrorNotSupported;
      }
    case 2:
      switch (lt) {
        case 0: return spec::launch_enc_jobs_2_0(d, count, max_ncw, s);
        case 1: return spec::launch_enc_jobs_2_1(d, count, max_ncw, s);
        default: return cudaErrorNotSupported;
      }
    case 3:
      switch (lt) {
        case 0: return spec::launch_enc_jobs_3_0(d, count, max_ncw, s);
        case 1: return spec::launch_enc_jobs_3_1(d, count, max_ncw, s);
        case 2: return spec::launch_enc_jobs_3_2(d, count, max_ncw, s);
        default: return cudaErrorNotSupported;
      }
    case 4:
      switch (lt) {
        case 0: return spec::launch_enc_jobs_4_0(d, count, max_ncw, s);
        case 1: return spec::launch_enc_jobs_4_1(d, count, max_ncw, s);
        case 2: return spec::launch_enc_jobs_4_2(d, count, max_ncw, s);
        case 3: return spec::launch_enc_jobs_4_3(d, count, max_ncw, s);
        default: return cudaErrorNotSupported;
      }
    case 5:
      switch (lt) {
        case 0: return spec::launch_enc_jobs_5_0(d, count, max_ncw, s);
        case 1: return spec::launch_enc_jobs_5_1(d, count, max_ncw, s);
        case 2: return spec::launch_enc_jobs_5_2(d, count, max_ncw, s);
        case 3: return spec::launch_enc_jobs_5_3(d, count, max_ncw, s);
        case 4: return spec::launch_enc_jobs_5_4(d, count, max_ncw, s);
        default: return cudaErrorNotSupported;
      }
    case 6:
      switch (lt) {
        case 0: return spec::launch_enc_jobs_6_0(d, count, max_ncw, s);
        case 1: return spec::launch_enc_jobs_6_1(d, count, max_ncw, s);
        case 2: return spec::launch_enc_jobs_6_2(d, count, max_ncw, s);
        case 3: return spec::launch_enc_jobs_6_3(d, count, max_ncw, s);
        case 4: return spec::launch_enc_jobs_6_4(d, count, max_ncw, s);
        case 5: return spec::launch_enc_jobs_6_5(d, count, max_ncw, s);
        default: return cudaErrorNotSupported;
      }
    case 7:
      switch (lt) {
        case 0: return spec::launch_enc_jobs_7_0(d, count, max_ncw, s);
        case 1: return spec::launch_enc_jobs_7_1(d, count, max_ncw, s);
        case 2: return spec::launch_enc_jobs_7_2(d, count, max_ncw, s);
        case 3: return spec::launch_enc_jobs_7_3(d, count, max_ncw, s);
        case 4: return spec::launch_enc_jobs_7_4(d, count, max_ncw, s);
        case 5: return spec::launch_enc_jobs_7_5(d, count, max_ncw, s);
        case 6: return spec::launch_enc_jobs_7_6(d, count, max_ncw, s);
        default: return cudaErrorNotSupported;
      }
    case 8:
      switch (lt) {
        case 0: return spec::launch_enc_jobs_8_0(d, count, max_ncw, s);
        case 1: return spec::launch_enc_jobs_8_1(d, count, max_ncw, s);
        case 2: return spec::launch_enc_jobs_8_2(d, count, max_ncw, s);
        case 3: return spec::launch_enc_jobs_8_3(d, count, max_ncw, s);
        case 4: return spec::launch_enc_jobs_8_4(d, count, max_ncw, s);
        case 5: return spec::launch_enc_jobs_8_5(d, count, max_ncw, s);
        case 6: return spec::launch_enc_jobs_8_6(d, count, max_ncw, s);
        case 7: return spec::launch_enc_jobs_8_7(d, count, max_ncw, s);
        default: return cudaErrorNotSupported;
      }
    default: return cudaErrorNotSupported;
  }
}

cudaError_t launch_recover_jobs(int n, void* d_jobs, int count, size_t max_ncw, cudaStream_t s) {
  auto* d = static_cast<spec::RecJob*>(d_jobs);
  switch (__builtin_ctz((unsigned)n)) {
    case 1: return spec::launch_rec_jobs_1(d, count, max_ncw, s);
    case 2: return spec::launch_rec_jobs_2(d, count, max_ncw, s);
    case 3: return spec::launch_rec_jobs_3(d, count, max_ncw, s);
    case 4: return spec::launch_rec_jobs_4(d, count, max_ncw, s);
    case 5: return spec::launch_rec_jobs_5(d, count, max_ncw, s);
    case 6: return spec::launch_rec_jobs_6(d, count, max_ncw, s);
    case 7: return spec::launch_rec_jobs_7(d, count, max_ncw, s);
    case 8: return spec::launch_rec_jobs_8(d, count, max_ncw, s);
    default: return cudaErrorNotSupported;
  }
}

bool fill_few_job(void* desc, const RecoverArgs& a) {
  spec::FewJob j{};
  j.a = a;
  if (!spec::host_few_table(a, &j.ft)) return false;
  std::memcpy(desc, &j, sizeof j);
  return true;
}

cudaError_t launch_recover_few_jobs(int n, int logt, const void* d_jobs, int count, size_t max_ncw, cudaStream_t s) {
  auto* d = static_cast<const spec::FewJob*>(d_jobs);
  switch (__builtin_ctz((unsigned)n)) {
    case 5: return spec::launch_rec_few_jobs_5(d, count, max_ncw, logt, s);
    case 6: return spec::launch_rec_few_jobs_6(d, count, max_ncw, logt, s);
    case 7: return spec::launch_rec_few_jobs_7(d, count, max_ncw, logt, s);
    case 8: return spec::launch_rec_few_jobs_8(d, count, max_ncw, logt, s);
    default: return cudaErrorNotSupported;
  }
}
}  // namespace afrs
