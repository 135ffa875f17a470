// fss_align_esp.cu -- instantiations of the fused alignment kernel for the ESP mode (FP32-lane variants and tensor-core sums).
#include "fss_align_kernel.cuh"

namespace fss {

int launch_align_esp(int lpp, int acc, int var, const AlignParams& prm, int threads, int cps, size_t smem,
         cudaStream_t st) {
  if (acc == 1) return launch_align<32, FSS_MODE_ESP, 1, 0>(prm, threads, cps, smem, st);
  if (acc == 2) return launch_align<32, FSS_MODE_ESP, 2, 0>(prm, threads, cps, smem, st);
  switch (var) {
    case 0: return dispatch_lanes<FSS_MODE_ESP, 0>(lpp, prm, threads, cps, smem, st);
    case 1: return dispatch_lanes<FSS_MODE_ESP, 1>(lpp, prm, threads, cps, smem, st);
    case 2: return dispatch_lanes<FSS_MODE_ESP, 2>(lpp, prm, threads, cps, smem, st);
    case 3: return dispatch_lanes<FSS_MODE_ESP, 3>(lpp, prm, threads, cps, smem, st);
    case 4: return dispatch_lanes<FSS_MODE_ESP, 4>(lpp, prm, threads, cps, smem, st);
    default: return set_error(FSS_ERR_INVALID, "fss_align: kernel_variant must be 0..5");
  }
}

}  // namespace fss
