// Mixed-precision M2L on tcgen05 tensor cores (placeholder until the kernel lands).
#include "solver.cuh"

namespace bbfmm {
int tc_supported() { return 0; }
int tc_prepare_operators(int, const double *, int, void **out, cudaStream_t) {
  *out = nullptr;
  return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "tensor-core M2L not built");
}
void tc_free_operators(void *) {}
size_t tc_split_bytes(int r, int64_t ncell) { return (size_t)ncell * r * 4; }
int tc_split_multipoles(int, int64_t, const double *, int, void *, cudaStream_t) {
  return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "tensor-core M2L not built");
}
int launch_m2l_tc(int, const void *, const void *, float *, int, const int4 *, int, cudaStream_t) {
  return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "tensor-core M2L not built");
}
}  // namespace bbfmm
