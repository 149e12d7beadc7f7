// gemm_tc.cu - split-BF16 tcgen05 GEMMs (see gemm_tc.hpp).
#include "engine.hpp"
#include "gemm_tc.hpp"

namespace dnnf90 {

bool gemm_tc_available() { return false; }
void gemm_tc_release_weights(DevNet *) {}
int gemm_tc_prepare(DevNet *, cudaStream_t) { return RC_OK; }
int gemm_tc_fwd(const DevNet *, int, int, int, int, int, const void *, void *,
                cudaStream_t) {
  return RC_UNSUPPORTED;
}
int gemm_tc_dt(const DevNet *, int, int, int, int, const void *, void *,
               cudaStream_t) {
  return RC_UNSUPPORTED;
}
int gemm_tc_dw(const DevNet *, int, int, int, int, const void *, const void *,
               double *, cudaStream_t) {
  return RC_UNSUPPORTED;
}

int gemm_tc_syrk(const double *, int, int, double *, cudaStream_t) {
  return RC_UNSUPPORTED;
}

}  // namespace dnnf90
