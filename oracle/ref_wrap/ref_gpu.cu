// ref_gpu.cu — TEST INFRASTRUCTURE ONLY.  C entry points around the
// reference's own GPU code, compiled from its sources where they lie
// (oracle/build.py), so GPU tests and the benchmark's reference leg can run
// the reference unmodified on the same device:
//   srkTrainingForward + SrkTrainWorkspace   training/srk_training_forward.cuh:117-241
//   MeasureCD_Batched                        third_party/src/metricUtil/cd_measure_util.cu:310-437
//   srkCudnnForward + SrkCudnnWorkspace      training/srk_cudnn_forward.cuh:92-269
#include "srk_training_forward.cuh"
#include "srk_cudnn_forward.cuh"
#include <metricUtil/cd_measure_util.cuh>
#include <cstring>

extern "C" void* ref_train_ws_create(int N, int B, cudaStream_t s) {
  auto* w = new SrkTrainWorkspace();
  w->allocate(N, B, s);
  cudaStreamSynchronize(s);
  return w;
}
extern "C" void ref_train_ws_destroy(void* w, cudaStream_t s) {
  auto* ws = static_cast<SrkTrainWorkspace*>(w);
  ws->release(s);
  cudaStreamSynchronize(s);
  delete ws;
}
extern "C" int ref_train_forward(const float* E, const float* I, const void* Gx, const void* Gy, int N, int W,
                                 int erosion, float dx, int B, cudaStream_t s, float* R, void* w) {
  srkTrainingForward(E, I, static_cast<const cufftComplex*>(Gx), static_cast<const cufftComplex*>(Gy), N, W, erosion,
                     dx, B, s, R, *static_cast<SrkTrainWorkspace*>(w));
  return (int)cudaGetLastError();
}
// CD of B signals [B][n] (device), L-fold upsampling, sinc half width A.
extern "C" int ref_measure_cd(const float* d_sig, int B, int n, int L, int A, cudaStream_t s, float* left,
                              float* right, float* cd) {
  const st::util::BatchCDResult r = st::util::MeasureCD_Batched(d_sig, B, n, L, A, s);
  for (int b = 0; b < B; ++b) {
    left[b] = r.cd[b].left_edge_px;
    right[b] = r.cd[b].right_edge_px;
    cd[b] = r.cd[b].cd_px;
  }
  return (int)cudaGetLastError();
}

// The reference's cuDNN forward (spatial kernels, column-major KW x KW).
extern "C" void* ref_cudnn_ws_create(int N, int W, int KW, int B, cudaStream_t s) {
  auto* w = new SrkCudnnWorkspace();
  w->allocate(B, N, KW, KW, W, s);
  cudaStreamSynchronize(s);
  return w;
}
extern "C" void ref_cudnn_ws_destroy(void* w, cudaStream_t s) {
  auto* ws = static_cast<SrkCudnnWorkspace*>(w);
  ws->release(s);
  cudaStreamSynchronize(s);
  delete ws;
}
extern "C" int ref_cudnn_forward(const float* E, const float* I, const float* Kx, const float* Ky, int N, int W,
                                 int erosion, float dx, int B, cudaStream_t s, float* R, void* w) {
  srkCudnnForward(E, I, Kx, Ky, N, W, erosion, dx, B, s, R, *static_cast<SrkCudnnWorkspace*>(w));
  return (int)cudaGetLastError();
}

