// engine.cuh — overlap-and-save (OaS) FFT convolution engine for the
// resist-shrinkage operator and its derivatives.
//
// Terminology
//   image      N x N, column-major buf[col*N + row] ("x" = column, "y" = row)
//   tile       M x M window of the (virtual) input image at origin
//              (tx*S, ty*S); its valid outputs are local x,y in [e, e+S)
//   work tile  (WT) one complex M x M field pair processed together:
//              either two real tiles packed as re/im (forward-type ops), the
//              base and tangent field of one tile (JVP-type ops), or two
//              packed tiles with two fields each (adjoint-type ops).
//
// One WT goes through three passes whose intermediates live in a scratch
// buffer (column-contiguous, 8-byte complex):
//   P1  per column x: load the field(s) (the op's loader computes them on
//       the fly: image values, or v*df/dx products for the adjoint), FFT
//       along y                                    -> S1[wt][k][x][ky]
//   P2  per block of 8 rows ky: FFT along x, spectral map with the kernel
//       spectra (Gx, Gy; conjugated for a true adjoint), inverse FFT along
//       kx, keep valid columns                    -> S2[wt][l][x'][ky]
//   P3  per valid column: inverse FFT along ky, then the op's epilogue
//       (central differences of f, combine, store) — conv(g,Gx), conv(g,Gy)
//       never leave registers.
//
// The reference performs the same linear "valid" convolution with cufftDX
// tiles (srk_forward.cuh:354-423) or whole-image cuFFT
// (training/srk_training_forward.cuh:175-241); with KW <= 2e+1 there is no
// circular wrap-around in either, so all of them equal
//     u[o] = dx^2 * sum_d E[o+e-d] * G[c+d]
// (adjoint/main_adjoint.cu:70-90) up to rounding.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cstdint>
#include "fft_warp.cuh"

namespace srk {

enum Op : int {
  OP_FWD = 0,       // R = ux*df/dx + uy*df/dy (pairs of tiles); optional ux/uy
  OP_VJP_F = 1,     // wx = ux*v, wy = uy*v (pairs of tiles) for dL/df
  OP_JVP = 2,       // dh from g + i*dg (one tile per WT)
  OP_TANADJ_F = 3,  // wx = dlam*ux_g + lam*ux_dg, wy likewise (one tile per WT)
  OP_ADJ = 4,       // dL/dg (full N x N) from hx + i*hy fields (pairs of tiles)
};

template <int OP> struct OpTraits;
template <> struct OpTraits<OP_FWD>      { static constexpr int K = 1, L = 2; static constexpr bool PAIRS = true; };
template <> struct OpTraits<OP_VJP_F>    { static constexpr int K = 1, L = 2; static constexpr bool PAIRS = true; };
template <> struct OpTraits<OP_JVP>      { static constexpr int K = 1, L = 2; static constexpr bool PAIRS = false; };
template <> struct OpTraits<OP_TANADJ_F> { static constexpr int K = 1, L = 2; static constexpr bool PAIRS = false; };
template <> struct OpTraits<OP_ADJ>      { static constexpr int K = 2, L = 1; static constexpr bool PAIRS = true; };

// Tile geometry of one launch.
struct Geom {
  int M;      // FFT tile size
  int e;      // erosion (kernel half width bound)
  int S;      // valid outputs per tile per axis (<= M - 2e)
  int T;      // tiles per axis
  int Nin;    // virtual input size (N for forward-type, N + 2e for adjoint)
  int Wout;   // output size (W for forward-type, N for adjoint)
  int TT;     // T*T
  int U;      // tiles in the whole batch (B*T*T)
};

// Operand pointers.  All images are column-major; batch strides are
// N*N for N-sized images and W*W for W-sized ones.
struct OpArgs {
  const void* E;    // convolved field g            [B][N][N]
  const void* I;    // differentiated field f       [B][N][N]
  const void* dE;   // tangent of g                 [B][N][N]
  const void* dI;   // tangent of f                 [B][N][N]
  const void* v;    // cotangent (lambda_h)         [B][W][W]
  const void* dv;   // tangent of the cotangent     [B][W][W]
  void* out0;       // R | dh | wx | dL/dg
  void* out1;       // wy
  void* out_ux;     // optional ux (OP_FWD)
  void* out_uy;     // optional uy (OP_FWD)
  int N, W, e;
};

// ---- storage types --------------------------------------------------------
template <typename T> __device__ __forceinline__ float ldf(const T* p, long long i);
template <> __device__ __forceinline__ float ldf<float>(const float* p, long long i) { return __ldg(p + i); }
template <> __device__ __forceinline__ float ldf<__half>(const __half* p, long long i) { return __half2float(p[i]); }
template <> __device__ __forceinline__ float ldf<__nv_bfloat16>(const __nv_bfloat16* p, long long i) {
  return __bfloat162float(p[i]);
}
template <typename T> __device__ __forceinline__ void stf(T* p, long long i, float v);
template <> __device__ __forceinline__ void stf<float>(float* p, long long i, float v) { p[i] = v; }
template <> __device__ __forceinline__ void stf<__half>(__half* p, long long i, float v) { p[i] = __float2half_rn(v); }
template <> __device__ __forceinline__ void stf<__nv_bfloat16>(__nv_bfloat16* p, long long i, float v) {
  p[i] = __float2bfloat16_rn(v);
}

// Central difference along columns (x) / rows (y) with zero outside [0,N),
// as srk_grad_x / srk_grad_y (srk_forward.cuh:429-445).
template <typename T>
__device__ __forceinline__ float grad_x(const T* f, int N, int gx, int gy) {
  const float r = (gx + 1 < N) ? ldf(f, (long long)(gx + 1) * N + gy) : 0.f;
  const float l = (gx > 0) ? ldf(f, (long long)(gx - 1) * N + gy) : 0.f;
  return (r - l) * 0.5f;
}
template <typename T>
__device__ __forceinline__ float grad_y(const T* f, int N, int gx, int gy) {
  const float d = (gy + 1 < N) ? ldf(f, (long long)gx * N + gy + 1) : 0.f;
  const float u = (gy > 0) ? ldf(f, (long long)gx * N + gy - 1) : 0.f;
  return (d - u) * 0.5f;
}

struct TileRef {
  int b, x0, y0;  // image index and tile origin in virtual input coordinates
  bool live;
};
__device__ __forceinline__ TileRef tile_of(const Geom& g, int u) {
  TileRef t;
  t.live = u < g.U;
  const int uu = t.live ? u : 0;
  t.b = uu / g.TT;
  const int r = uu - t.b * g.TT;
  const int tx = r / g.T, ty = r - (r / g.T) * g.T;
  t.x0 = tx * g.S;
  t.y0 = ty * g.S;
  return t;
}

// ---- loaders: value of field k of work tile w at local (x, y) ------------
// Forward-type: image value of g at virtual coords (== image coords).
template <typename T>
__device__ __forceinline__ float img_at(const T* p, const OpArgs& a, int b, int gx, int gy) {
  if (gx < 0 || gy < 0 || gx >= a.N || gy >= a.N) return 0.f;
  return ldf(p, (long long)b * a.N * a.N + (long long)gx * a.N + gy);
}

// Adjoint-type: h_x = v*df/dx (or dv*df/dx + v*d(df)/dx for the
// tangent-adjoint) on the valid window, zero elsewhere; virtual coords are
// shifted by +e so that the full N x N output is the valid part of the
// convolution of the zero-extended (N+2e)^2 field
// (srk_adj_load_tile, adjoint/srk_adjoint.cuh:169-200).
template <typename T>
__device__ __forceinline__ float h_at(const OpArgs& a, int b, int k, int px, int py) {
  const int qx = px - a.e, qy = py - a.e;            // image coords
  const int ox = qx - a.e, oy = qy - a.e;            // valid-window coords
  if (ox < 0 || oy < 0 || ox >= a.W || oy >= a.W) return 0.f;
  const long long vo = (long long)b * a.W * a.W + (long long)ox * a.W + oy;
  const T* f = static_cast<const T*>(a.I) + (long long)b * a.N * a.N;
  const float v = ldf(static_cast<const T*>(a.v), vo);
  const float g = (k == 0) ? grad_x(f, a.N, qx, qy) : grad_y(f, a.N, qx, qy);
  if (a.dI == nullptr) return v * g;
  const T* df = static_cast<const T*>(a.dI) + (long long)b * a.N * a.N;
  const float dv = ldf(static_cast<const T*>(a.dv), vo);
  const float dg = (k == 0) ? grad_x(df, a.N, qx, qy) : grad_y(df, a.N, qx, qy);
  return dv * g + v * dg;
}

template <int M, int OP, typename T>
__device__ __forceinline__ void load_column(const OpArgs& a, const Geom& g, int w, int k, int x, int lane,
                                            float2 (&z)[M / 32]) {
  constexpr int EPT = M / 32;
  if constexpr (OpTraits<OP>::PAIRS) {
    const TileRef t0 = tile_of(g, 2 * w), t1 = tile_of(g, 2 * w + 1);
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      const int y = lane + 32 * i;
      float re = 0.f, im = 0.f;
      if constexpr (OP == OP_ADJ) {
        re = h_at<T>(a, t0.b, k, t0.x0 + x, t0.y0 + y);
        if (t1.live) im = h_at<T>(a, t1.b, k, t1.x0 + x, t1.y0 + y);
      } else {
        const T* E = static_cast<const T*>(a.E);
        re = img_at(E, a, t0.b, t0.x0 + x, t0.y0 + y);
        if (t1.live) im = img_at(E, a, t1.b, t1.x0 + x, t1.y0 + y);
      }
      z[i] = make_float2(re, im);
    }
  } else {
    const TileRef t = tile_of(g, w);
    const T* E = static_cast<const T*>(a.E);
    const T* dE = static_cast<const T*>(a.dE);
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      const int y = lane + 32 * i;
      z[i] = make_float2(img_at(E, a, t.b, t.x0 + x, t.y0 + y), img_at(dE, a, t.b, t.x0 + x, t.y0 + y));
    }
  }
}

// ---- epilogues: P3 hands over column x (local, valid) of work tile w ------
// zx = IFFT(Z*Gx), zy = IFFT(Z*Gy) (OP != ADJ), or z = IFFT(sum) (ADJ).
template <int M, int OP, typename T>
__device__ __forceinline__ void epilogue_column(const OpArgs& a, const Geom& g, int w, int x, int lane,
                                                const float2 (&z0)[M / 32], const float2 (&z1)[M / 32]) {
  constexpr int EPT = M / 32;
  const int N = a.N, W = a.W, e = a.e;
  auto emit_fwd = [&](const TileRef& t, bool imag) {
    if (!t.live) return;
    const int ox = t.x0 + x - g.e;
    if (ox >= g.Wout) return;
    const T* f = static_cast<const T*>(a.I) + (long long)t.b * N * N;
    const long long ob = (long long)t.b * W * W + (long long)ox * W;
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      const int y = lane + 32 * i;
      const int oy = t.y0 + y - g.e;
      if (y < g.e || y >= g.e + g.S || oy >= g.Wout) continue;
      const float ux = imag ? z0[i].y : z0[i].x;
      const float uy = imag ? z1[i].y : z1[i].x;
      const int gx = ox + e, gy = oy + e;
      if constexpr (OP == OP_FWD) {
        if (a.out0) {
          const float r = ux * grad_x(f, N, gx, gy) + uy * grad_y(f, N, gx, gy);
          stf(static_cast<T*>(a.out0), ob + oy, r);
        }
        if (a.out_ux) stf(static_cast<T*>(a.out_ux), ob + oy, ux);
        if (a.out_uy) stf(static_cast<T*>(a.out_uy), ob + oy, uy);
      } else {  // OP_VJP_F: w = u * v
        const float v = ldf(static_cast<const T*>(a.v), ob + oy);
        stf(static_cast<float*>(a.out0), ob + oy, ux * v);
        stf(static_cast<float*>(a.out1), ob + oy, uy * v);
      }
    }
  };
  if constexpr (OP == OP_FWD || OP == OP_VJP_F) {
    emit_fwd(tile_of(g, 2 * w), false);
    emit_fwd(tile_of(g, 2 * w + 1), true);
  } else if constexpr (OP == OP_JVP || OP == OP_TANADJ_F) {
    const TileRef t = tile_of(g, w);
    const int ox = t.x0 + x - g.e;
    if (ox >= g.Wout) return;
    const long long ob = (long long)t.b * W * W + (long long)ox * W;
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      const int y = lane + 32 * i;
      const int oy = t.y0 + y - g.e;
      if (y < g.e || y >= g.e + g.S || oy >= g.Wout) continue;
      // re: conv of g, im: conv of dg
      if constexpr (OP == OP_JVP) {
        const T* f = static_cast<const T*>(a.I) + (long long)t.b * N * N;
        const T* df = static_cast<const T*>(a.dI) + (long long)t.b * N * N;
        const int gx = ox + e, gy = oy + e;
        // srk_tangent_combine (tan_tanadj/srk_tangent.cuh:28-52)
        const float dh = z0[i].y * grad_x(f, N, gx, gy) + z1[i].y * grad_y(f, N, gx, gy) +
                         z0[i].x * grad_x(df, N, gx, gy) + z1[i].x * grad_y(df, N, gx, gy);
        stf(static_cast<T*>(a.out0), ob + oy, dh);
      } else {
        const float lam = ldf(static_cast<const T*>(a.v), ob + oy);
        const float dlam = ldf(static_cast<const T*>(a.dv), ob + oy);
        stf(static_cast<float*>(a.out0), ob + oy, dlam * z0[i].x + lam * z0[i].y);
        stf(static_cast<float*>(a.out1), ob + oy, dlam * z1[i].x + lam * z1[i].y);
      }
    }
  } else {  // OP_ADJ: output is the full N x N image
    auto emit_adj = [&](const TileRef& t, bool imag) {
      if (!t.live) return;
      const int ox = t.x0 + x - g.e;
      if (ox >= g.Wout) return;
      const long long ob = (long long)t.b * N * N + (long long)ox * N;
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int y = lane + 32 * i;
        const int oy = t.y0 + y - g.e;
        if (y < g.e || y >= g.e + g.S || oy >= g.Wout) continue;
        stf(static_cast<T*>(a.out0), ob + oy, imag ? z0[i].y : z0[i].x);
      }
    };
    emit_adj(tile_of(g, 2 * w), false);
    emit_adj(tile_of(g, 2 * w + 1), true);
  }
}

// ---- phases ------------------------------------------------------------------
constexpr int kWarps = 8;
constexpr int kThreads = 32 * kWarps;

__device__ __forceinline__ void load_twiddles(float2* tw, const float2* __restrict__ twg, int M) {
  for (int i = threadIdx.x; i < M; i += blockDim.x) tw[i] = twg[i];
}

// Scratch of one work tile: S1 [K][M][M] then S2 [L][S][M] (float2).
template <int M, int OP>
__host__ __device__ constexpr size_t s1_elems() { return (size_t)OpTraits<OP>::K * M * M; }
template <int M, int OP>
__host__ __device__ inline size_t wt_elems(int S) { return s1_elems<M, OP>() + (size_t)OpTraits<OP>::L * S * M; }

template <int M>
constexpr size_t p1_smem_bytes() { return sizeof(float2) * (M + kWarps * fft_row_words(M)); }
template <int M>
constexpr size_t p3_smem_bytes() { return p1_smem_bytes<M>(); }
inline size_t p2_smem_bytes(int M, int K, int L, int S) {
  return sizeof(float2) * ((size_t)M + (size_t)K * kWarps * fft_row_words(M) + (size_t)L * S * 9);
}

// P1: warp `warp` transforms column x = xb*8 + warp of every field along y.
template <int M, int OP, typename T>
__device__ __forceinline__ void phase1(const OpArgs& a, const Geom& g, int w, int xb, float2* __restrict__ S1,
                                       float2* __restrict__ row, const float2* __restrict__ tw, int warp, int lane) {
  constexpr int EPT = M / 32;
  constexpr int K = OpTraits<OP>::K;
  const int x = xb * kWarps + warp;
#pragma unroll 1
  for (int k = 0; k < K; ++k) {
    float2 z[EPT];
    load_column<M, OP, T>(a, g, w, k, x, lane, z);
    fft<M, false>(z, row, tw, lane);
    float2* dst = S1 + ((size_t)k * M + x) * M + lane;
#pragma unroll
    for (int i = 0; i < EPT; ++i) __stcg(dst + 32 * i, z[i]);
  }
}

// P2: rows ky0 .. ky0+7: FFT along x, spectral map, inverse, keep the valid
// columns, write S2 column-contiguous through a padded transpose buffer.
// Needs __syncthreads-uniform control flow (all threads of the CTA).
template <int M, int OP>
__device__ __forceinline__ void phase2(const float2* __restrict__ S1, float2* __restrict__ S2,
                                       const float2* __restrict__ Gx, const float2* __restrict__ Gy, int conjG,
                                       const Geom& g, int ky0, float2* __restrict__ buf,
                                       const float2* __restrict__ tw, int warp, int lane) {
  constexpr int EPT = M / 32;
  constexpr int K = OpTraits<OP>::K;
  constexpr int L = OpTraits<OP>::L;
  constexpr int RW = fft_row_words(M);
  float2* in = buf;                      // [K][8][RW]
  float2* out = buf + K * kWarps * RW;   // [L][S][9]
  const int S = g.S, e = g.e;
  for (int idx = threadIdx.x; idx < K * M * 4; idx += kThreads) {
    const int k = idx / (M * 4);
    const int rem = idx - k * (M * 4);
    const int x = rem >> 2, rp = rem & 3;
    const float4 q = __ldcg(reinterpret_cast<const float4*>(S1 + ((size_t)k * M + x) * M + ky0 + 2 * rp));
    in[(k * kWarps + 2 * rp) * RW + fft_pad(x)] = make_float2(q.x, q.y);
    in[(k * kWarps + 2 * rp + 1) * RW + fft_pad(x)] = make_float2(q.z, q.w);
  }
  __syncthreads();
  const int ky = ky0 + warp;
  float2* row0 = in + warp * RW;
  const float2* rd0 = row0 + lane + (lane >> 4);
  float2 z0[EPT];
#pragma unroll
  for (int i = 0; i < EPT; ++i) z0[i] = rd0[34 * i];
  fft<M, false>(z0, row0, tw, lane);
  const float2* gxr = Gx + (size_t)ky * M + lane;
  const float2* gyr = Gy + (size_t)ky * M + lane;
  auto spec = [&](float2 z, float2 G) { return conjG ? cmulc(z, G) : cmul(z, G); };
  auto park = [&](const float2 (&o)[EPT], int l) {
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      const int xv = lane + 32 * i - e;
      if (xv >= 0 && xv < S) out[(l * S + xv) * 9 + warp] = o[i];
    }
  };
  if constexpr (K == 1) {
    float2 o[EPT];
#pragma unroll
    for (int i = 0; i < EPT; ++i) o[i] = spec(z0[i], __ldg(gxr + 32 * i));
    fft<M, true>(o, row0, tw, lane);
    park(o, 0);
#pragma unroll
    for (int i = 0; i < EPT; ++i) o[i] = spec(z0[i], __ldg(gyr + 32 * i));
    fft<M, true>(o, row0, tw, lane);
    park(o, 1);
  } else {
    float2* row1 = in + (kWarps + warp) * RW;
    const float2* rd1 = row1 + lane + (lane >> 4);
    float2 z1[EPT];
#pragma unroll
    for (int i = 0; i < EPT; ++i) z1[i] = rd1[34 * i];
    fft<M, false>(z1, row1, tw, lane);
#pragma unroll
    for (int i = 0; i < EPT; ++i) z0[i] = cadd(spec(z0[i], __ldg(gxr + 32 * i)), spec(z1[i], __ldg(gyr + 32 * i)));
    fft<M, true>(z0, row0, tw, lane);
    park(z0, 0);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < L * S * 4; idx += kThreads) {
    const int l = idx / (S * 4);
    const int rem = idx - l * (S * 4);
    const int xv = rem >> 2, rp = rem & 3;
    const float2 lo = out[(l * S + xv) * 9 + 2 * rp];
    const float2 hi = out[(l * S + xv) * 9 + 2 * rp + 1];
    __stcg(reinterpret_cast<float4*>(S2 + ((size_t)l * S + xv) * M + ky0 + 2 * rp),
           make_float4(lo.x, lo.y, hi.x, hi.y));
  }
}

// P3: warp `warp` finishes valid column xv = xb*8 + warp (if < S).
template <int M, int OP, typename T>
__device__ __forceinline__ void phase3(const float2* __restrict__ S2, const OpArgs& a, const Geom& g, int w, int xb,
                                       float2* __restrict__ row, const float2* __restrict__ tw, int warp, int lane) {
  constexpr int EPT = M / 32;
  constexpr int L = OpTraits<OP>::L;
  const int xv = xb * kWarps + warp;
  if (xv >= g.S) return;
  float2 z0[EPT], z1[EPT];
  {
    const float2* src = S2 + (size_t)xv * M + lane;
#pragma unroll
    for (int i = 0; i < EPT; ++i) z0[i] = __ldcg(src + 32 * i);
    fft<M, true>(z0, row, tw, lane);
  }
  if constexpr (L == 2) {
    const float2* src = S2 + ((size_t)g.S + xv) * M + lane;
#pragma unroll
    for (int i = 0; i < EPT; ++i) z1[i] = __ldcg(src + 32 * i);
    fft<M, true>(z1, row, tw, lane);
  } else {
#pragma unroll
    for (int i = 0; i < EPT; ++i) z1[i] = make_float2(0.f, 0.f);
  }
  epilogue_column<M, OP, T>(a, g, w, xv + g.e, lane, z0, z1);
}

// ---- three-launch schedule (one kernel per phase over a chunk of WTs) ------
template <int M, int OP, typename T>
__global__ void __launch_bounds__(kThreads, 2)
k_p1(OpArgs a, Geom g, const float2* __restrict__ twg, int w0, float2* __restrict__ scratch, int S) {
  extern __shared__ float2 sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  load_twiddles(sm, twg, M);
  __syncthreads();
  const int wl = blockIdx.y;
  phase1<M, OP, T>(a, g, w0 + wl, blockIdx.x, scratch + wl * wt_elems<M, OP>(S), sm + M + warp * fft_row_words(M),
                   sm, warp, lane);
}

template <int M, int OP>
__global__ void __launch_bounds__(kThreads, 2)
k_p2(float2* __restrict__ scratch, const float2* __restrict__ Gx, const float2* __restrict__ Gy, int conjG, Geom g,
     const float2* __restrict__ twg) {
  extern __shared__ float2 sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  load_twiddles(sm, twg, M);
  float2* base = scratch + blockIdx.y * wt_elems<M, OP>(g.S);
  phase2<M, OP>(base, base + s1_elems<M, OP>(), Gx, Gy, conjG, g, blockIdx.x * kWarps, sm + M, sm, warp, lane);
}

template <int M, int OP, typename T>
__global__ void __launch_bounds__(kThreads, 2)
k_p3(float2* __restrict__ scratch, OpArgs a, Geom g, const float2* __restrict__ twg, int w0) {
  extern __shared__ float2 sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  load_twiddles(sm, twg, M);
  __syncthreads();
  const int wl = blockIdx.y;
  phase3<M, OP, T>(scratch + wl * wt_elems<M, OP>(g.S) + s1_elems<M, OP>(), a, g, w0 + wl, blockIdx.x,
                   sm + M + warp * fft_row_words(M), sm, warp, lane);
}

// ---- persistent schedule ---------------------------------------------------------
// One launch processes every WT.  Work is a ticket queue of rounds; round r
// holds the P1 units of WT r, the P2 units of WT r-kLag and the P3 units of
// WT r-2*kLag.  A WT's scratch lives in slot w mod nslot of a small ring that
// stays in L2.  Per-slot counters (monotonic over the slot's reuses) order
// the phases:
//   P1(w) needs c2[slot] >= gen*n2       (previous user's P2 done reading S1)
//   P2(w) needs c1[slot] >= (gen+1)*n1   (its S1 complete)
//           and c3[slot] >= gen*n3       (previous user's P3 done reading S2)
//   P3(w) needs c2[slot] >= (gen+1)*n2   (its S2 complete)
// Every dependency points to a smaller ticket, and a ticket is only ever held
// by a running CTA, so the smallest unfinished ticket can always proceed.
// Waits are bounded anyway: a wait that exceeds `spin_limit` polls sets
// ctl->abort (with the place in ctl->where) and every CTA returns.
constexpr int kLag = 2;
constexpr int kMaxSlots = 16;

struct Ctl {
  unsigned int ticket;
  unsigned int abort;
  unsigned int where;
  unsigned int pad;
  unsigned int c1[kMaxSlots], c2[kMaxSlots], c3[kMaxSlots];
};

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Thread-0 wait: returns false if the kernel must stop.
__device__ __forceinline__ bool wait_geq(const unsigned int* p, unsigned int target, unsigned long long limit,
                                         Ctl* ctl, unsigned int where) {
  unsigned long long it = 0;
  while (ld_acquire(p) < target) {
    if (ld_acquire(&ctl->abort)) return false;
    if (++it > limit) {
      atomicExch(&ctl->where, where);
      atomicExch(&ctl->abort, 1u);
      return false;
    }
    __nanosleep(64);
  }
  return true;
}

template <int M, int OP, typename T>
__global__ void __launch_bounds__(kThreads, 2)
k_persist(OpArgs a, Geom g, const float2* __restrict__ Gx, const float2* __restrict__ Gy, int conjG,
          const float2* __restrict__ twg, float2* __restrict__ scratch, int nslot, int nwt, Ctl* ctl,
          unsigned long long spin_limit) {
  extern __shared__ float2 sm[];
  __shared__ int s_t[2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n1 = M / kWarps, n2 = M / kWarps, n3 = (g.S + kWarps - 1) / kWarps;
  const int round = n1 + n2 + n3;
  const long long total = (long long)(nwt + 2 * kLag) * round;
  const size_t slot_elems = wt_elems<M, OP>(g.S);
  float2* tw = sm;
  float2* buf = sm + M;
  load_twiddles(tw, twg, M);
  if (threadIdx.x == 0) s_t[0] = (int)atomicAdd(&ctl->ticket, 1u);
  __syncthreads();
  int cur = s_t[0];
  while (cur < total) {
    // prefetch the next ticket while this unit runs
    unsigned int nxt = 0;
    if (threadIdx.x == 0) nxt = atomicAdd(&ctl->ticket, 1u);
    const int r = cur / round, u = cur - (cur / round) * round;
    int phase, w, unit;
    if (u < n1) { phase = 1; w = r; unit = u; }
    else if (u < n1 + n2) { phase = 2; w = r - kLag; unit = u - n1; }
    else { phase = 3; w = r - 2 * kLag; unit = u - n1 - n2; }
    const bool live = (w >= 0 && w < nwt);
    const int slot = live ? w % nslot : 0;
    const unsigned int gen = live ? (unsigned int)(w / nslot) : 0u;
    if (threadIdx.x == 0) {
      bool ok = ld_acquire(&ctl->abort) == 0u;
      if (ok && live) {
        if (phase == 1) ok = wait_geq(&ctl->c2[slot], gen * n2, spin_limit, ctl, 1);
        else if (phase == 2) ok = wait_geq(&ctl->c1[slot], (gen + 1) * n1, spin_limit, ctl, 2) &&
                                  wait_geq(&ctl->c3[slot], gen * n3, spin_limit, ctl, 3);
        else ok = wait_geq(&ctl->c2[slot], (gen + 1) * n2, spin_limit, ctl, 4);
      }
      s_t[1] = ok ? 1 : 0;
    }
    __syncthreads();
    if (!s_t[1]) return;
    if (live) {
      float2* base = scratch + (size_t)slot * slot_elems;
      if (phase == 1) {
        phase1<M, OP, T>(a, g, w, unit, base, buf + warp * fft_row_words(M), tw, warp, lane);
      } else if (phase == 2) {
        phase2<M, OP>(base, base + s1_elems<M, OP>(), Gx, Gy, conjG, g, unit * kWarps, buf, tw, warp, lane);
      } else {
        phase3<M, OP, T>(base + s1_elems<M, OP>(), a, g, w, unit, buf + warp * fft_row_words(M), tw, warp, lane);
      }
    }
    __syncthreads();  // every thread's scratch stores of this unit are issued
    if (threadIdx.x == 0) {
      if (live) {
        __threadfence();
        atomicAdd(phase == 1 ? &ctl->c1[slot] : phase == 2 ? &ctl->c2[slot] : &ctl->c3[slot], 1u);
      }
      s_t[0] = (int)nxt;
    }
    __syncthreads();
    cur = s_t[0];
  }
}

// Bounded-wait self test: thread 0 of one CTA waits for a counter that
// nothing increments; the wait must give up and raise the abort flag.
__global__ void k_wait_selftest(Ctl* ctl, unsigned long long spin_limit) {
  if (threadIdx.x == 0) wait_geq(&ctl->c1[0], 1u, spin_limit, ctl, 99);
}

// dL/df = D_x^T(wx) + D_y^T(wy) on N x N, with wx, wy given on the W x W
// window (zero outside); adjoint of the central difference
// (adjointWrtI_kernel, adjoint/srk_adjoint.cuh:25-59).  With ux, uy, v
// given instead (the reference contract) w = u*v is formed on the fly.
template <typename T, bool FROM_U>
__global__ void k_adj_wrt_f(const float* __restrict__ wx, const float* __restrict__ wy, const T* __restrict__ v,
                            const T* __restrict__ ux, const T* __restrict__ uy, int N, int W, int e, int B,
                            T* __restrict__ out) {
  const int gy = blockIdx.x * blockDim.x + threadIdx.x;
  const int gx = blockIdx.y * blockDim.y + threadIdx.y;
  const int b = blockIdx.z;
  if (gx >= N || gy >= N) return;
  const long long wb = (long long)b * W * W;
  auto WX = [&](int r, int c) -> float {
    if (r < 0 || r >= W || c < 0 || c >= W) return 0.f;
    const long long i = wb + (long long)c * W + r;
    if constexpr (FROM_U) return ldf(ux, i) * ldf(v, i);
    else return wx[i];
  };
  auto WY = [&](int r, int c) -> float {
    if (r < 0 || r >= W || c < 0 || c >= W) return 0.f;
    const long long i = wb + (long long)c * W + r;
    if constexpr (FROM_U) return ldf(uy, i) * ldf(v, i);
    else return wy[i];
  };
  const int ox = gx - e, oy = gy - e;
  const float val = (WX(oy, ox - 1) - WX(oy, ox + 1)) * 0.5f + (WY(oy - 1, ox) - WY(oy + 1, ox)) * 0.5f;
  stf(out, (long long)b * N * N + (long long)gx * N + gy, val);
}

}  // namespace srk
