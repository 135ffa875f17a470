// fss_probe.cu -- issue-rate probes that measure this GPU's roof for the pairwise kernels:
// ex2 (MUFU) throughput and FP32 FMA throughput.  The bench divides the kernels' achieved
// pair-term rate by the probe-derived ceiling, so the roofline is measured on the same
// device and clocks rather than taken from a datasheet.
#include "fss_internal.cuh"

namespace fss {
namespace {

constexpr int kChains = 8;

// MUFU: 8 independent ex2 chains per thread; each ex2 feeds the next through a cheap scale
// so the compiler cannot fold the loop.
__global__ void probe_ex2_kernel(int iters, float* out) {
  float v[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) v[c] = -1e-3f * (float)(threadIdx.x + c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = ex2(v[c]) - 1.0f;
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += v[c];
  if (s == 12345.f) out[blockIdx.x] = s;  // never true; keeps the work alive
}

// FP32: 8 independent FMA chains per thread.
__global__ void probe_ffma_kernel(int iters, float* out) {
  float v[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) v[c] = 1e-3f * (float)(threadIdx.x + c);
  const float a = 0.999f, b = 1e-4f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = fmaf(v[c], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += v[c];
  if (s == 12345.f) out[blockIdx.x] = s;
}

}  // namespace

int probe_launch(int which, int iters, int blocks_per_sm, float* out, long long* ops,
                 cudaStream_t st) {
  if (iters <= 0 || blocks_per_sm <= 0 || !out || !ops)
    return set_error(FSS_ERR_INVALID, "fss_probe_peak: bad arguments");
  const int threads = 256;
  const int grid = blocks_per_sm * num_sms();
  if (which == 0) {
    probe_ex2_kernel<<<grid, threads, 0, st>>>(iters, out);
  } else if (which == 1) {
    probe_ffma_kernel<<<grid, threads, 0, st>>>(iters, out);
  } else {
    return set_error(FSS_ERR_INVALID, "fss_probe_peak: which must be 0 (ex2) or 1 (ffma)");
  }
  *ops = (long long)grid * threads * (long long)iters * kChains;
  return check_launch("fss_probe_peak");
}

}  // namespace fss
