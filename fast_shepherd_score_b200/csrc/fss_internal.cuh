// fss_internal.cuh -- host/device plumbing shared by the libfss_cuda translation units.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/fss_cuda.h"
#include "fss_device.cuh"

namespace fss {

// Hard limit of points (or pharmacophore features) per molecule that the fused kernels
// stage in shared memory.  4096 float4 points = 64 KB per cloud.
constexpr int kMaxPoints = 4096;

// Thread-local error message + status helpers (fss_capi.cu).
int set_error(int code, const std::string& msg);
int check_launch(const char* what);

// A packed cloud in global memory: float32 (x, y, z, w) points, or float16 (x, y, z, w)
// points (8 bytes each, a library kept in float16 on the device) that are widened here, in
// the staging loads.  Only staging code reads through it; the pairwise loops read the
// staged float32 copies in shared memory.  The format flag is uniform across a launch.
struct Pts {
  const void* base;
  int f16;
  __host__ __device__ Pts() : base(nullptr), f16(0) {}
  __host__ __device__ Pts(const float4* p) : base(p), f16(0) {}  // NOLINT: implicit on purpose
  __host__ __device__ Pts(const void* p, int half) : base(p), f16(half) {}
  __device__ __forceinline__ float4 operator[](int i) const {
    if (!f16) return reinterpret_cast<const float4*>(base)[i];
    const uint2 raw = reinterpret_cast<const uint2*>(base)[i];
    const float2 xy = __half22float2(*reinterpret_cast<const __half2*>(&raw.x));
    const float2 zw = __half22float2(*reinterpret_cast<const __half2*>(&raw.y));
    return make_float4(xy.x, xy.y, zw.x, zw.y);
  }
  // A pharmacophore anchor: float32 storage carries the type in w's bits, float16 storage
  // carries it as a (small, exact) float16 value.
  __device__ __forceinline__ float4 anchor(int i) const {
    float4 a = (*this)[i];
    if (f16) a.w = __int_as_float(__float2int_rn(a.w));
    return a;
  }
  __host__ __device__ Pts operator+(int o) const {
    if (!base) return *this;
    return f16 ? Pts(reinterpret_cast<const uint2*>(base) + o, 1)
               : Pts(reinterpret_cast<const float4*>(base) + o, 0);
  }
  __host__ __device__ explicit operator bool() const { return base != nullptr; }
};

// Block-wide sum of a float3 (blockDim.x a multiple of 32, <= 1024); every thread gets it.
__device__ __forceinline__ float3 block_sum3(float3 v, float* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    v.z += __shfl_xor_sync(0xffffffffu, v.z, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (l == 0) { red[3 * w] = v.x; red[3 * w + 1] = v.y; red[3 * w + 2] = v.z; }
  __syncthreads();
  float3 s = make_float3(0.f, 0.f, 0.f);
  for (int i = 0; i < nw; ++i) { s.x += red[3 * i]; s.y += red[3 * i + 1]; s.z += red[3 * i + 2]; }
  return s;
}

// Centroid of n packed points; every thread of the block gets it.  The sum has a fixed order
// (lane-strided partial sums of warp 0, then a butterfly), so the centroid -- and the rounding
// of everything staged relative to it -- does not depend on the CTA size of the launch.
__device__ __forceinline__ float3 block_centroid(const Pts g, int n, float* red) {
  float3 s = make_float3(0.f, 0.f, 0.f);
  if (threadIdx.x < 32) {
    for (int i = threadIdx.x; i < n; i += 32) {
      const float4 p = g[i];
      s.x += p.x; s.y += p.y; s.z += p.z;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
      s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
      s.z += __shfl_xor_sync(0xffffffffu, s.z, o);
    }
  }
  __syncthreads();  // earlier readers of red are done
  if (threadIdx.x == 0) { red[0] = s.x; red[1] = s.y; red[2] = s.z; }
  __syncthreads();
  const float inv = 1.f / (float)(n > 0 ? n : 1);
  return make_float3(red[0] * inv, red[1] * inv, red[2] * inv);
}

// Stage a reference cloud (centred on c) in the expanded, duplicated form
//   sPd[2i] = (2k a.x, 2k a.x, 2k a.y, 2k a.y), sPd[2i+1] = (2k a.z, 2k a.z, P.w, P.w)
// with P.w = -k|a|^2 - e c^2, and for ESP sQd[i] = (2 e c_i, 2 e c_i).
template <bool ESP>
__device__ __forceinline__ void stage_ref(const Pts g, int n, float3 c, float k,
                                          float e, float4* sPd, float2* sQd) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float4 p = g[i];
    const float ax = p.x - c.x, ay = p.y - c.y, az = p.z - c.z;
    float w = -k * (ax * ax + ay * ay + az * az);
    if (ESP) {
      w = fmaf(-e * p.w, p.w, w);
      sQd[i] = make_float2(2.f * e * p.w, 2.f * e * p.w);
    }
    const float px = 2.f * k * ax, py = 2.f * k * ay, pz = 2.f * k * az;
    sPd[2 * i] = make_float4(px, px, py, py);
    sPd[2 * i + 1] = make_float4(pz, pz, w, w);
  }
}

__device__ __forceinline__ void stage_copy(const Pts g, int n, float4* s) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) s[i] = g[i];
}

// Pharmacophore type carried in a float's bits; anything outside the 9-entry tables is
// treated as Dummy (8), which the kernels skip.
__device__ __forceinline__ float clamp_type(float w) {
  const int t = __float_as_int(w);
  return __int_as_float((t < 0 || t > 8) ? 8 : t);
}

// Reference pharmacophores: anchors centred on c (type bits kept), unit vectors.  With `toff`
// the features are stored grouped by type -- a stable counting sort, so the features of one
// type keep their order -- and toff[t] is the first feature of type t (toff[9] = n): the typed
// overlap then visits only a fit feature's same-type reference features, in the order of the
// ungrouped loop, so its sums are unchanged.
__device__ __forceinline__ void stage_ref_pharm(const Pts ga, const Pts gv, int n, float3 c,
                                                float4* sA, float4* sV, int* toff = nullptr) {
  auto type_of = [&](int j) { return __float_as_int(clamp_type(ga.anchor(j).w)); };
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float4 a = ga.anchor(i);
    const float tw = clamp_type(a.w);
    int pos = i;
    if (toff) {
      const int t = __float_as_int(tw);
      pos = 0;
      for (int j = 0; j < n; ++j) {
        const int u = type_of(j);
        pos += (u < t || (u == t && j < i)) ? 1 : 0;
      }
    }
    sA[pos] = make_float4(a.x - c.x, a.y - c.y, a.z - c.z, tw);
    if (gv) {
      const float4 v = gv[i];
      sV[pos] = unit4(v.x, v.y, v.z);
    } else {
      sV[pos] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  if (toff) {
    for (int t = threadIdx.x; t < 10; t += blockDim.x) {
      int below = 0;
      for (int j = 0; j < n; ++j) below += type_of(j) < t ? 1 : 0;
      toff[t] = below;
    }
  }
}

// Fit pharmacophores in their body frame: anchors as given, unit vectors.
__device__ __forceinline__ void stage_fit_pharm(const Pts ga, const Pts gv, int n,
                                                float4* sA, float4* sV) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float4 a = ga.anchor(i);
    sA[i] = make_float4(a.x, a.y, a.z, clamp_type(a.w));
    if (gv) {
      const float4 v = gv[i];
      sV[i] = unit4(v.x, v.y, v.z);
    } else {
      sV[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
}

// Lookup tables of accel/kernels/... build_lookup_tables (analytical_gradients/_torch.py:177-220):
// alpha per type, K = (pi / (2 alpha))^1.5, category 0 isotropic, 1 directional,
// 2 aromatic (|cos|), 3 dummy (skipped).  directional = false maps every real type to 0.
PharmTables make_pharm_tables(bool directional);

int num_sms();

// Launchers behind the C ABI (each validates its arguments and returns an fss_status).
int align_launch(const fss_align_desc* d, cudaStream_t st);
int pick_best_launch(const float* rs, const float* rq, const float* rt, int P, int S, float* os,
                     float* oq, float* ot, cudaStream_t st);
int self_overlap_launch(const float* pts, const int32_t* off, int n_mol, int max_n, float alpha,
                        int esp, float inv_lam, int f16, float* out, cudaStream_t st);
int pharm_self_launch(const float* anc, const float* vec, const int32_t* off, int n_mol, int max_n,
                      int directional, int extended, int f16, float* out, cudaStream_t st);

}  // namespace fss
