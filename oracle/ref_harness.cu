// Test harness around the reference's own CUDA implementation.
//
// TEST INFRASTRUCTURE ONLY (the checker, never the product).  The reference's
// FIPkernels.cu is compiled unmodified from where it lies (the path comes in
// as FIP_REFERENCE_CU from oracle/Makefile) and this file adds C entry points:
//   ref_fipipe            the reference's FIpipe itself (host buffers in/out);
//   ref_image_snapshot    the reference kernels of one snapshot, launched in
//                         FIpipe's order and shapes (FIPkernels.cu:665-711),
//                         returning the images FIpipe keeps internal;
//   ref_trigger           the reference trigger kernels (FIPkernels.cu:831-840);
//   ref_pixel_targets     coordschange + p2p output (FIPkernels.cu:687-688).
// Every call allocates and frees its own device memory.
#include FIP_REFERENCE_CU

#include <cstdio>

#define RH_CHECK(x)                                                              \
  do {                                                                           \
    cudaError_t e_ = (x);                                                        \
    if (e_ != cudaSuccess) {                                                     \
      fprintf(stderr, "ref_harness: %s -> %s\n", #x, cudaGetErrorString(e_));   \
      return 1;                                                                  \
    }                                                                            \
  } while (0)

extern "C" int ref_fipipe(float* vr, float* vi, float* B, float* V, float* result, size_t nb,
                          size_t n, size_t nsnap, float cell, size_t t) {
  return FIpipe(vr, vi, B, V, result, nb, n, nsnap, cell, t);
}

extern "C" int ref_pixel_targets(const float* V, size_t n, float cell, float* out_oi) {
  float *d_oi = nullptr, *d_V = nullptr;
  RH_CHECK(cudaMalloc(&d_oi, n * n * 2 * sizeof(float)));
  RH_CHECK(cudaMalloc(&d_V, 9 * sizeof(float)));
  RH_CHECK(cudaMemcpy(d_V, V, 9 * sizeof(float), cudaMemcpyHostToDevice));
  RH_CHECK(cudaMemset(d_oi, 0, n * n * 2 * sizeof(float)));
  dim3 th(32, 32), bl((unsigned)((n + 31) / 32), (unsigned)((n + 31) / 32));
  coordschange<<<bl, th>>>(d_oi, d_V, n);
  p2p<<<bl, th>>>(d_oi, d_V, cell, n);
  RH_CHECK(cudaGetLastError());
  RH_CHECK(cudaMemcpy(out_oi, d_oi, n * n * 2 * sizeof(float), cudaMemcpyDeviceToHost));
  cudaFree(d_oi);
  cudaFree(d_V);
  return 0;
}

// One snapshot through the reference kernels.  Outputs (host, may be null):
// dirty [N*N], dirty_pre [N*N], max_out [1].
extern "C" int ref_image_snapshot(const float* vr, const float* vi, const float* B, const float* V,
                                  size_t nb, size_t n, float cell, float* dirty_out,
                                  float* dirty_pre_out, float* max_out) {
  const size_t g = static_cast<size_t>(computeCeil(1.5 * static_cast<float>(n)));
  const float r1r2_scale = cell * g;
  const float norm = 2.4937047051153827;
  const size_t region_num = 32;
  const size_t region_size =
      static_cast<size_t>(computeCeil(static_cast<float>(n) / static_cast<float>(region_num)));
  float *d_vr, *d_vi, *d_B, *d_V, *d_pre, *d_ck, *d_gr, *d_gi, *d_oi, *d_dirty, *d_mtmp, *d_max;
  cufftComplex* d_grid;
  RH_CHECK(cudaMalloc(&d_vr, nb * sizeof(float)));
  RH_CHECK(cudaMalloc(&d_vi, nb * sizeof(float)));
  RH_CHECK(cudaMalloc(&d_B, nb * 2 * sizeof(float)));
  RH_CHECK(cudaMalloc(&d_V, 9 * sizeof(float)));
  RH_CHECK(cudaMalloc(&d_pre, n * n * sizeof(float)));
  RH_CHECK(cudaMalloc(&d_ck, (n / 2 + 1) * sizeof(float)));
  RH_CHECK(cudaMalloc(&d_gr, g * g * sizeof(float)));
  RH_CHECK(cudaMalloc(&d_gi, g * g * sizeof(float)));
  RH_CHECK(cudaMalloc(&d_grid, g * g * sizeof(cufftComplex)));
  RH_CHECK(cudaMalloc(&d_oi, n * n * 2 * sizeof(float)));
  RH_CHECK(cudaMalloc(&d_dirty, n * n * sizeof(float)));
  RH_CHECK(cudaMalloc(&d_mtmp, region_num * region_num * sizeof(float)));
  RH_CHECK(cudaMalloc(&d_max, 3 * sizeof(float)));
  RH_CHECK(cudaMemcpy(d_vr, vr, nb * sizeof(float), cudaMemcpyHostToDevice));
  RH_CHECK(cudaMemcpy(d_vi, vi, nb * sizeof(float), cudaMemcpyHostToDevice));
  RH_CHECK(cudaMemcpy(d_B, B, nb * 2 * sizeof(float), cudaMemcpyHostToDevice));
  RH_CHECK(cudaMemcpy(d_V, V, 9 * sizeof(float), cudaMemcpyHostToDevice));
  RH_CHECK(cudaMemset(d_pre, 0, n * n * sizeof(float)));
  RH_CHECK(cudaMemset(d_ck, 0, (n / 2 + 1) * sizeof(float)));
  RH_CHECK(cudaMemset(d_gr, 0, g * g * sizeof(float)));
  RH_CHECK(cudaMemset(d_gi, 0, g * g * sizeof(float)));
  RH_CHECK(cudaMemset(d_oi, 0, n * n * 2 * sizeof(float)));
  RH_CHECK(cudaMemset(d_dirty, 0, n * n * sizeof(float)));
  RH_CHECK(cudaMemset(d_max, 0, 3 * sizeof(float)));

  cufftHandle plan;
  if (cufftPlan2d(&plan, (int)g, (int)g, CUFFT_C2C) != CUFFT_SUCCESS) return 2;

  size_t nt = 1024;
  size_t nblk = computeCeil(static_cast<float>(n / 2 + 1) / nt);
  convolveKernel<<<nblk, nt>>>(d_ck, n, g, norm);
  nblk = computeCeil(static_cast<float>(nb) / nt);
  computeVisWeighted<<<nblk, nt>>>(d_vr, d_vi, nb, d_V);
  gridding<<<nblk, nt>>>(d_B, d_gr, d_gi, d_vr, d_vi, r1r2_scale, g, nb);
  nblk = computeCeil(static_cast<float>(g * g) / nt);
  combineToComplex<<<nblk, nt>>>(d_gr, d_gi, d_grid, g);
  if (cufftExecC2C(plan, d_grid, d_grid, CUFFT_INVERSE) != CUFFT_SUCCESS) return 2;
  dim3 th(32, 32);
  dim3 bl(computeCeil(static_cast<float>(n) / 32), computeCeil(static_cast<float>(n) / 32));
  accumulation<<<bl, th>>>(d_pre, d_grid, n, g);
  scaling<<<bl, th>>>(d_pre, d_ck, n, norm);
  coordschange<<<bl, th>>>(d_oi, d_V, n);
  p2p<<<bl, th>>>(d_oi, d_V, cell, n);
  finalinterp<<<bl, th>>>(d_oi, d_pre, d_dirty, n, nb);
  max_large<<<region_num * region_num, 1024, 1024 * sizeof(float)>>>(d_dirty, d_mtmp, region_num,
                                                                      region_size, n);
  max_small<<<1, 1024, 1024 * sizeof(float)>>>(d_mtmp, d_max, n, 0);
  RH_CHECK(cudaGetLastError());
  RH_CHECK(cudaDeviceSynchronize());
  if (dirty_out) RH_CHECK(cudaMemcpy(dirty_out, d_dirty, n * n * 4, cudaMemcpyDeviceToHost));
  if (dirty_pre_out) RH_CHECK(cudaMemcpy(dirty_pre_out, d_pre, n * n * 4, cudaMemcpyDeviceToHost));
  if (max_out) RH_CHECK(cudaMemcpy(max_out, d_max, 4, cudaMemcpyDeviceToHost));
  cufftDestroy(plan);
  cudaFree(d_vr); cudaFree(d_vi); cudaFree(d_B); cudaFree(d_V); cudaFree(d_pre); cudaFree(d_ck);
  cudaFree(d_gr); cudaFree(d_gi); cudaFree(d_grid); cudaFree(d_oi); cudaFree(d_dirty);
  cudaFree(d_mtmp); cudaFree(d_max);
  return 0;
}

// Trigger kernels on three host images; maxall3 are the per-image maxima.
extern "C" int ref_trigger(const float* I1, const float* I2, const float* I3, const float* maxall3,
                           size_t n, size_t t, float* result) {
  const size_t u = n / t, sz = n * n;
  float *d1, *d2, *d3, *a, *b, *diff, *res, *mx;
  RH_CHECK(cudaMalloc(&d1, sz * 4)); RH_CHECK(cudaMalloc(&d2, sz * 4));
  RH_CHECK(cudaMalloc(&d3, sz * 4)); RH_CHECK(cudaMalloc(&a, sz * 4));
  RH_CHECK(cudaMalloc(&b, sz * 4)); RH_CHECK(cudaMalloc(&diff, sz * 4));
  RH_CHECK(cudaMalloc(&res, u * u * 4)); RH_CHECK(cudaMalloc(&mx, 3 * 4));
  RH_CHECK(cudaMemcpy(d1, I1, sz * 4, cudaMemcpyHostToDevice));
  RH_CHECK(cudaMemcpy(d2, I2, sz * 4, cudaMemcpyHostToDevice));
  RH_CHECK(cudaMemcpy(d3, I3, sz * 4, cudaMemcpyHostToDevice));
  RH_CHECK(cudaMemcpy(mx, maxall3, 3 * 4, cudaMemcpyHostToDevice));
  size_t nt = 1024, nblk = computeCeil(static_cast<float>(sz) / nt);
  subtraction<<<nblk, nt>>>(d1, d2, a, sz);
  subtraction<<<nblk, nt>>>(d2, d3, b, sz);
  setNonPositiveToC<<<nblk, nt>>>(d2, sz, 1e-6f);
  subtraction<<<nblk, nt>>>(a, b, diff, sz);
  tlisi<<<u * u, nt, 3 * nt * sizeof(float)>>>(diff, d2, res, t, n, u, mx);
  RH_CHECK(cudaGetLastError());
  RH_CHECK(cudaMemcpy(result, res, u * u * 4, cudaMemcpyDeviceToHost));
  cudaFree(d1); cudaFree(d2); cudaFree(d3); cudaFree(a); cudaFree(b); cudaFree(diff);
  cudaFree(res); cudaFree(mx);
  return 0;
}
