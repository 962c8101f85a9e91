// IEEE-arithmetic stages (compiled without fast math): plane projection of
// baseline uvw, Stokes-I collapse, and the reduced-precision visibility
// storage of the precision form.
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "fip_common.cuh"
#include "fip_kernels.h"

namespace {

constexpr int kThreads = 256;
constexpr int kPlaneBlocks = 296;  // 2 x 148 SMs
constexpr double kLight = 299792458.0;

// Sample s = row + chan * rows (SVDPreprocessMain.cpp:36-38), in wavelengths
// (SVDPreprocessKernels.cu:41-61), FP64.
__device__ __forceinline__ void sample_lambda(const float* uvw, const float* freqs, size_t rows,
                                              size_t s, double x[3]) {
  const size_t r = s % rows, c = s / rows;
  const double sc = (double)freqs[c] / kLight;
  x[0] = (double)uvw[3 * r + 0] * sc;
  x[1] = (double)uvw[3 * r + 1] * sc;
  x[2] = (double)uvw[3 * r + 2] * sc;
}

// Block partial sums in FP64 (deterministic two-stage reduction).
// MODE 0: sum x (3 values); MODE 1: centred second moments (6 values).
template <int MODE>
__global__ void k_plane_moments(const float* uvw, const float* freqs, size_t rows, size_t chans,
                                const double* mean, double* partial) {
  constexpr int K = MODE == 0 ? 3 : 6;
  __shared__ double sh[K][kThreads];
  double acc[K];
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
  const size_t ns = rows * chans;
  double m[3] = {0, 0, 0};
  if (MODE == 1) {
    m[0] = mean[0]; m[1] = mean[1]; m[2] = mean[2];
  }
  for (size_t s = blockIdx.x * (size_t)kThreads + threadIdx.x; s < ns;
       s += (size_t)gridDim.x * kThreads) {
    double x[3];
    sample_lambda(uvw, freqs, rows, s, x);
    if (MODE == 0) {
      acc[0] += x[0]; acc[1] += x[1]; acc[2] += x[2];
    } else {
      const double a = x[0] - m[0], b = x[1] - m[1], c = x[2] - m[2];
      acc[0] += a * a; acc[1] += a * b; acc[2] += a * c;
      acc[3 % K] += b * b; acc[4 % K] += b * c; acc[5 % K] += c * c;
    }
  }
  for (int k = 0; k < K; ++k) sh[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int d = kThreads / 2; d > 0; d >>= 1) {
    if ((int)threadIdx.x < d)
      for (int k = 0; k < K; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + d];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < K; ++k) partial[blockIdx.x * K + k] = sh[k][0];
}

template <int K>
__global__ void k_plane_reduce(const double* partial, int nblocks, double scale, double* out) {
  if (threadIdx.x < K) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partial[b * K + threadIdx.x];
    out[threadIdx.x] = s * scale;
  }
}

// Cyclic Jacobi eigen-decomposition of the 3x3 covariance, then the basis
// of the reference: principal axes in descending order, each signed so its
// largest-magnitude component is positive (SVDPreprocessKernels.cu:115-206),
// third row their cross product.
__global__ void k_plane_basis(const double* cov6, double* basis_out, float* V) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double A[9] = {cov6[0], cov6[1], cov6[2], cov6[1], cov6[3], cov6[4], cov6[2], cov6[4], cov6[5]};
  double Q[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int sweep = 0; sweep < 64; ++sweep) {
    const double off = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
    if (off < 1e-300) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        const double apq = A[p * 3 + q];
        if (fabs(apq) < 1e-300) continue;
        const double app = A[p * 3 + p], aqq = A[q * 3 + q];
        const double tau = (aqq - app) / (2.0 * apq);
        const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
        for (int k = 0; k < 3; ++k) {
          const double akp = A[k * 3 + p], akq = A[k * 3 + q];
          A[k * 3 + p] = c * akp - s * akq;
          A[k * 3 + q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {
          const double apk = A[p * 3 + k], aqk = A[q * 3 + k];
          A[p * 3 + k] = c * apk - s * aqk;
          A[q * 3 + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          const double qkp = Q[k * 3 + p], qkq = Q[k * 3 + q];
          Q[k * 3 + p] = c * qkp - s * qkq;
          Q[k * 3 + q] = s * qkp + c * qkq;
        }
      }
  }
  const double d[3] = {A[0], A[4], A[8]};
  int big = 0;
  for (int k = 1; k < 3; ++k)
    if (d[k] > d[big]) big = k;
  int mid = -1;
  for (int k = 0; k < 3; ++k)
    if (k != big && (mid < 0 || d[k] > d[mid])) mid = k;
  double b[6];
  for (int a = 0; a < 3; ++a) {
    b[a] = Q[a * 3 + big];
    b[3 + a] = Q[a * 3 + mid];
  }
  for (int comp = 0; comp < 2; ++comp) {
    int ma = 0;
    double mv = fabs(b[comp * 3]);
    for (int a = 1; a < 3; ++a)
      if (fabs(b[comp * 3 + a]) > mv) {
        mv = fabs(b[comp * 3 + a]);
        ma = a;
      }
    if (b[comp * 3 + ma] < 0)
      for (int a = 0; a < 3; ++a) b[comp * 3 + a] = -b[comp * 3 + a];
  }
  for (int k = 0; k < 6; ++k) basis_out[k] = b[k];
  const double c0 = b[1] * b[5] - b[2] * b[4];
  const double c1 = b[2] * b[3] - b[0] * b[5];
  const double c2 = b[0] * b[4] - b[1] * b[3];
  for (int k = 0; k < 6; ++k) V[k] = (float)b[k];
  V[6] = (float)c0;
  V[7] = (float)c1;
  V[8] = (float)c2;
}

// B[s] = x_s . basis^T, uncentred (SVDPreprocessKernels.cu:142-165).
__global__ void k_plane_projectB(const float* uvw, const float* freqs, size_t rows, size_t chans,
                                 const double* basis, float* B) {
  const size_t ns = rows * chans;
  for (size_t s = blockIdx.x * (size_t)kThreads + threadIdx.x; s < ns;
       s += (size_t)gridDim.x * kThreads) {
    double x[3];
    sample_lambda(uvw, freqs, rows, s, x);
    B[2 * s + 0] = (float)(x[0] * basis[0] + x[1] * basis[1] + x[2] * basis[2]);
    B[2 * s + 1] = (float)(x[0] * basis[3] + x[1] * basis[4] + x[2] * basis[5]);
  }
}

// SVDPreprocessKernels.cu:208-237.
__global__ void k_collapse(const float* v0r, const float* v0i, const float* v3r, const float* v3i,
                           const unsigned char* f0, const unsigned char* f3, const float* w0,
                           const float* w3, float* out_re, float* out_im, size_t ns) {
  const FipRawVis r{v0r, v0i, v3r, v3i, f0, f3, w0, w3};
  for (size_t s = blockIdx.x * (size_t)kThreads + threadIdx.x; s < ns;
       s += (size_t)gridDim.x * kThreads)
    fip_collapse_sample(r, s, out_re[s], out_im[s]);
}

// Sample k of the visibilities: FP32 arrays, or raw polarisations collapsed
// to Stokes I on load.
struct F32Vis {
  const float* vr;
  const float* vi;
  __device__ __forceinline__ void operator()(size_t k, float& re, float& im) const {
    re = vr[k];
    im = vi[k];
  }
};
struct RawVis {
  FipRawVis r;
  __device__ __forceinline__ void operator()(size_t k, float& re, float& im) const {
    fip_collapse_sample(r, k, re, im);
  }
};

// One block of FIP_QBLOCK samples per CTA (kThreads threads, four samples
// each): the block's max-abs, its power-of-two scale 2^(e - 14) for a max-abs
// in [2^e, 2^(e+1)) (so the max lands in [2^14, 2^15), inside FP16's range,
// and the division by the scale is exact), then the values divided by it.
template <int VT, class L>
__global__ void __launch_bounds__(kThreads) k_quantize(const L load, size_t nb, void* qr,
                                                       void* qi, float* scales) {
  static_assert(FIP_QBLOCK == 4 * kThreads, "four samples per thread");
  __shared__ float s_max[kThreads / 32];
  const size_t base = (size_t)blockIdx.x * FIP_QBLOCK;
  float re[4], im[4];
  float m = 0.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const size_t i = base + (size_t)k * kThreads + threadIdx.x;
    re[k] = 0.f;
    im[k] = 0.f;
    if (i < nb) load(i, re[k], im[k]);
    m = fmaxf(m, fmaxf(fabsf(re[k]), fabsf(im[k])));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
  __syncthreads();
  m = s_max[0];
#pragma unroll
  for (int w = 1; w < kThreads / 32; ++w) m = fmaxf(m, s_max[w]);
  // The max's biased exponent E gives scale 2^(E - 141) (bits E - 14) and
  // inverse 2^(141 - E) (bits 268 - E).  E is held >= 15 so both are normal:
  // a block whose max is below 2^-112 (zero included) takes scale 2^-126.
  const int eb = max((int)((__float_as_uint(m) >> 23) & 0xffu), 15);
  const float scale = __uint_as_float((unsigned)(eb - 14) << 23);
  const float inv = __uint_as_float((unsigned)(268 - eb) << 23);
  if (threadIdx.x == 0) scales[blockIdx.x] = scale;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const size_t i = base + (size_t)k * kThreads + threadIdx.x;
    if (i >= nb) continue;
    if (VT == FIP_VIS_F16) {
      reinterpret_cast<__half*>(qr)[i] = __float2half_rn(re[k] * inv);
      reinterpret_cast<__half*>(qi)[i] = __float2half_rn(im[k] * inv);
    } else {
      reinterpret_cast<__nv_bfloat16*>(qr)[i] = __float2bfloat16_rn(re[k] * inv);
      reinterpret_cast<__nv_bfloat16*>(qi)[i] = __float2bfloat16_rn(im[k] * inv);
    }
  }
}

}  // namespace

cudaError_t fip_launch_plane_project(const float* uvw, const float* freqs, size_t rows,
                                     size_t chans, double* work, float* B, float* V,
                                     cudaStream_t s) {
  const size_t ns = rows * chans;
  const int blocks = (int)std::min<size_t>(kPlaneBlocks, (ns + kThreads - 1) / kThreads);
  double* w = work;
  cudaError_t e = cudaSuccess;
  bool own = false;
  if (!w) {
    e = cudaMallocAsync((void**)&w, (size_t)(blocks * 6 + 16) * sizeof(double), s);
    if (e != cudaSuccess) return e;
    own = true;
  }
  double* partial = w;
  double* mean = w + blocks * 6;
  double* cov = mean + 3;
  double* basis = cov + 6;
  k_plane_moments<0><<<blocks, kThreads, 0, s>>>(uvw, freqs, rows, chans, nullptr, partial);
  k_plane_reduce<3><<<1, 32, 0, s>>>(partial, blocks, 1.0 / (double)ns, mean);
  k_plane_moments<1><<<blocks, kThreads, 0, s>>>(uvw, freqs, rows, chans, mean, partial);
  k_plane_reduce<6><<<1, 32, 0, s>>>(partial, blocks, 1.0, cov);
  k_plane_basis<<<1, 32, 0, s>>>(cov, basis, V);
  k_plane_projectB<<<blocks, kThreads, 0, s>>>(uvw, freqs, rows, chans, basis, B);
  e = cudaGetLastError();
  if (own) {
    cudaError_t e2 = cudaFreeAsync(w, s);
    if (e == cudaSuccess) e = e2;
  }
  return e;
}

cudaError_t fip_launch_collapse(const float* v0r, const float* v0i, const float* v3r,
                                const float* v3i, const unsigned char* f0,
                                const unsigned char* f3, const float* w0, const float* w3,
                                float* out_re, float* out_im, size_t ns, cudaStream_t s) {
  const int blocks = (int)std::min<size_t>(4 * 148, (ns + kThreads - 1) / kThreads + 1);
  k_collapse<<<blocks, kThreads, 0, s>>>(v0r, v0i, v3r, v3i, f0, f3, w0, w3, out_re, out_im, ns);
  return cudaGetLastError();
}

template <class L>
static cudaError_t launch_quantize(const L& load, size_t nb, int vis_type, void* out_re,
                                  void* out_im, float* scales, cudaStream_t s) {
  const size_t blocks = fip_qblocks(nb);
  if (blocks == 0) return cudaSuccess;
  if (blocks > 0x7fffffffu) return cudaErrorInvalidValue;
  if (vis_type == FIP_VIS_F16)
    k_quantize<FIP_VIS_F16><<<(unsigned)blocks, kThreads, 0, s>>>(load, nb, out_re, out_im, scales);
  else
    k_quantize<FIP_VIS_BF16><<<(unsigned)blocks, kThreads, 0, s>>>(load, nb, out_re, out_im,
                                                                   scales);
  return cudaGetLastError();
}

cudaError_t fip_launch_quantize(const float* vr, const float* vi, size_t nb, int vis_type,
                                void* out_re, void* out_im, float* scales, cudaStream_t s) {
  return launch_quantize(F32Vis{vr, vi}, nb, vis_type, out_re, out_im, scales, s);
}

cudaError_t fip_launch_quantize_raw(const FipRawVis& raw, size_t nb, int vis_type, void* out_re,
                                    void* out_im, float* scales, cudaStream_t s) {
  return launch_quantize(RawVis{raw}, nb, vis_type, out_re, out_im, scales, s);
}
