// fss_align_combo.cu -- instantiations of the fused alignment kernel for vol_and_surf_esp
// (shape-steered pose, ShaEP ESP comparison in the tracked score).  Code variants: base and
// the one-CTA/SM register budget (the shape channel works on small heavy-atom clouds).
#include "fss_align_kernel.cuh"

namespace fss {

int launch_align_combo(int lpp, int var, const AlignParams& prm, int threads, int cps,
                       size_t smem, cudaStream_t st) {
  if (var == 2) return dispatch_lanes<FSS_MODE_ESP_COMBO, 2>(lpp, prm, threads, cps, smem, st);
  return dispatch_lanes<FSS_MODE_ESP_COMBO, 0>(lpp, prm, threads, cps, smem, st);
}

}  // namespace fss
