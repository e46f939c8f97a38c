// srk_b200.hpp — C++ drop-in layer over the C ABI (srk_b200.h).
//
// Same function names, argument order and argument meaning as the
// reference's operator headers, so a caller of
//   srkTrainingForward          (training/srk_training_forward.cuh:175-241)
//   srkForwardOaS               (srk_forward.cuh:468-501)
//   adjointSRK                  (adjoint/srk_adjoint.cuh:402-425)
//   shrinkageTangentOaS         (tan_tanadj/srk_tangent.cuh:111-151)
//   shrinkageTangentAdjointOaS  (tan_tanadj/srk_tangent_adjoint.cuh:105-159)
//   srkPrecomputeKernelFreq     (srk_forward.cuh:154-203)
// switches by changing the include and the workspace type.  Differences:
//   * the workspace is an srk::Workspace (wraps an srk_plan); its
//     allocate() takes the same sizes as the reference's allocate();
//   * the OaS operators take the spectra size as a template argument
//     exactly like the reference's template parameter M;
//   * every call returns srk_status instead of void and never aborts; like
//     the reference it synchronises the stream before returning (use the C
//     entry points for the asynchronous form).
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <vector>

#include "srk_b200.h"

namespace srk {

// Owns one srk_plan.  allocate(N, B) mirrors SrkTrainWorkspace::allocate;
// allocate_oas(N, W, M) mirrors SrkConvWorkspace / SrkAdjWorkspace /
// SrkTanWorkspace / SrkTanAdjWorkspace::allocate with the reference's M.
struct Workspace {
  srk_plan plan = nullptr;
  int N = 0, W = 0, erosion = -1, B_max = 0, M = 0;
  float dx = 0.f;

  srk_status ensure(int N_, int W_, int e_, float dx_, int B_, int M_) {
    if (plan && N_ == N && W_ == W && e_ == erosion && dx_ == dx && B_ <= B_max && M_ == M) return SRK_OK;
    release();
    const srk_status s = srk_plan_create(&plan, N_, W_, e_, dx_, B_, M_, SRK_F32, 0, 0);
    if (s == SRK_OK) { N = N_; W = W_; erosion = e_; dx = dx_; B_max = B_; M = M_; }
    return s;
  }
  void release() {
    if (plan) srk_plan_destroy(plan);
    plan = nullptr;
  }
  ~Workspace() { release(); }
};

inline srk_status srkTrainingForward(const float* d_E_batch, const float* d_I_batch, const cufftComplex* d_Gx_freq,
                                     const cufftComplex* d_Gy_freq, int N, int W, int erosion, float dx, int B,
                                     cudaStream_t stream, float* d_R_batch, Workspace& ws) {
  srk_status s = ws.ensure(N, W, erosion, dx, B, N);
  if (s != SRK_OK) return s;
  return srk_training_forward_sync(d_E_batch, d_I_batch, d_Gx_freq, d_Gy_freq, N, W, erosion, dx, B,
                                   reinterpret_cast<srk_stream_t>(stream), d_R_batch, ws.plan);
}

template <unsigned Arch, unsigned M, unsigned... Rest>
inline srk_status srkForwardOaS(const float* d_E_pad, const float* d_I_pad, const cufftComplex* d_Gx_freq,
                                const cufftComplex* d_Gy_freq, int N_large, int W, int erosion, float dx,
                                cudaStream_t stream, float* d_R, Workspace& ws, float* d_ux = nullptr,
                                float* d_uy = nullptr) {
  srk_status s = ws.ensure(N_large, W, erosion, dx, 1, (int)M);
  if (s != SRK_OK) return s;
  s = srk_forward_oas(d_E_pad, d_I_pad, d_Gx_freq, d_Gy_freq, N_large, W, erosion, dx,
                      reinterpret_cast<srk_stream_t>(stream), d_R, ws.plan, d_ux, d_uy);
  return s != SRK_OK ? s : (cudaStreamSynchronize(stream) == cudaSuccess ? SRK_OK : SRK_ERR_CUDA);
}

template <unsigned Arch, unsigned M, unsigned... Rest>
inline srk_status adjointSRK(const float* d_v, const float* d_ux, const float* d_uy, const float* d_I_pad,
                             const cufftComplex* d_Gx_freq, const cufftComplex* d_Gy_freq, int N_large, int W,
                             int erosion, float dx, cudaStream_t stream, float* d_dLdI, float* d_dLdE,
                             Workspace& ws) {
  srk_status s = ws.ensure(N_large, W, erosion, dx, 1, (int)M);
  if (s != SRK_OK) return s;
  s = srk_adjoint(d_v, d_ux, d_uy, d_I_pad, d_Gx_freq, d_Gy_freq, N_large, W, erosion, dx,
                  reinterpret_cast<srk_stream_t>(stream), d_dLdI, d_dLdE, ws.plan);
  return s != SRK_OK ? s : (cudaStreamSynchronize(stream) == cudaSuccess ? SRK_OK : SRK_ERR_CUDA);
}

template <unsigned Arch, unsigned M, unsigned... Rest>
inline srk_status shrinkageTangentOaS(const float* d_f_pad, const float* d_g_pad, const float* d_df_pad,
                                      const float* d_dg_pad, const cufftComplex* d_Gx_freq,
                                      const cufftComplex* d_Gy_freq, int N_large, int W, int erosion, float dx,
                                      cudaStream_t stream, float* d_dh, Workspace& ws) {
  srk_status s = ws.ensure(N_large, W, erosion, dx, 1, (int)M);
  if (s != SRK_OK) return s;
  s = srk_tangent(d_f_pad, d_g_pad, d_df_pad, d_dg_pad, d_Gx_freq, d_Gy_freq, N_large, W, erosion, dx,
                  reinterpret_cast<srk_stream_t>(stream), d_dh, ws.plan);
  return s != SRK_OK ? s : (cudaStreamSynchronize(stream) == cudaSuccess ? SRK_OK : SRK_ERR_CUDA);
}

template <unsigned Arch, unsigned M, unsigned... Rest>
inline srk_status shrinkageTangentAdjointOaS(const float* d_f_pad, const float* d_g_pad, const float* d_df_pad,
                                             const float* d_dg_pad, const float* d_lam_h, const float* d_dlam_h,
                                             const cufftComplex* d_Gx_freq, const cufftComplex* d_Gy_freq,
                                             int N_large, int W, int erosion, float dx, cudaStream_t stream,
                                             float* d_dLam_f, float* d_dLam_g, Workspace& ws) {
  srk_status s = ws.ensure(N_large, W, erosion, dx, 1, (int)M);
  if (s != SRK_OK) return s;
  s = srk_tangent_adjoint(d_f_pad, d_g_pad, d_df_pad, d_dg_pad, d_lam_h, d_dlam_h, d_Gx_freq, d_Gy_freq, N_large,
                          W, erosion, dx, reinterpret_cast<srk_stream_t>(stream), d_dLam_f, d_dLam_g, ws.plan);
  return s != SRK_OK ? s : (cudaStreamSynchronize(stream) == cudaSuccess ? SRK_OK : SRK_ERR_CUDA);
}

// Host kernel (kw x kh, column-major) -> device spectrum at size M, reference
// layout, computed in FP64 on the device (no host fftshift round trip).
inline srk_status srkPrecomputeKernelFreq(const std::vector<float>& h_G, int kw, int kh, int M,
                                          cufftComplex* d_G_freq, cudaStream_t stream) {
  if (kw != kh) return SRK_ERR_UNSUPPORTED;
  float* d_K = nullptr;
  if (cudaMallocAsync(&d_K, sizeof(float) * kw * kh, stream) != cudaSuccess) return SRK_ERR_ALLOC;
  cudaMemcpyAsync(d_K, h_G.data(), sizeof(float) * kw * kh, cudaMemcpyHostToDevice, stream);
  const srk_status s = srk_precompute_kernel_freq(d_K, kw, M, d_G_freq, reinterpret_cast<srk_stream_t>(stream));
  cudaFreeAsync(d_K, stream);
  cudaStreamSynchronize(stream);
  return s;
}

}  // namespace srk
