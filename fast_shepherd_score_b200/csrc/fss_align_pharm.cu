// fss_align_pharm.cu -- instantiations of the fused alignment kernel for the modes with a
// pharmacophore channel (pharm, shape + directional pharm, shape + colour).  Their poses are
// small and tail-heavy, so only the base code variant is built.
#include "fss_align_kernel.cuh"

namespace fss {

int launch_align_pharm(int mode, int lpp, int ext, const AlignParams& prm, int threads,
                       int cps, size_t smem, cudaStream_t st) {
  switch (mode) {
    case FSS_MODE_PHARM:
      // ext: 0 cosine weights, 1 extended points + anchors, 2 extended points only
      if (ext == 1) return dispatch_lanes<FSS_MODE_PHARM, 0, 1>(lpp, prm, threads, cps, smem, st);
      if (ext == 2) return dispatch_lanes<FSS_MODE_PHARM, 0, 2>(lpp, prm, threads, cps, smem, st);
      return dispatch_lanes<FSS_MODE_PHARM, 0, 0>(lpp, prm, threads, cps, smem, st);
    case FSS_MODE_SHAPE_PHARM:
      return dispatch_lanes<FSS_MODE_SHAPE_PHARM, 0>(lpp, prm, threads, cps, smem, st);
    default: return dispatch_lanes<FSS_MODE_SHAPE_COLOR, 0>(lpp, prm, threads, cps, smem, st);
  }
}

}  // namespace fss
