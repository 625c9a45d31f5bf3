// Fused ZDT path for power-of-two Nf (placeholder: not yet enabled).
#include "zdt_ws.cuh"

namespace fdr {

bool zdt_fused_eligible(int64_t, int64_t, int64_t) { return false; }
int zdt_fused_setup(fdr_zdt*) { return FDR_OK; }
int zdt_fused_input(fdr_zdt*, const float*, cudaStream_t) { return FDR_ERR_INVALID_ARGUMENT; }
int zdt_fused_A_to_F(fdr_zdt*, cudaStream_t) { return FDR_ERR_INVALID_ARGUMENT; }
int zdt_fused_run(fdr_zdt*, float, float*, int, const double*, cudaStream_t) {
  return FDR_ERR_INVALID_ARGUMENT;
}
void zdt_fused_release(fdr_zdt*) {}

}  // namespace fdr
