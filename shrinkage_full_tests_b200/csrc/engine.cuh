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
#include <type_traits>
#include "fft_warp.cuh"

// CTAs per SM the kernels are compiled for (register cap 65536/(256*n)).
#ifndef SRK_MIN_BLOCKS
#define SRK_MIN_BLOCKS 4
#endif
#ifndef SRK_P1_MIN_BLOCKS
#define SRK_P1_MIN_BLOCKS SRK_MIN_BLOCKS
#endif
#ifndef SRK_P2_MIN_BLOCKS
#define SRK_P2_MIN_BLOCKS SRK_MIN_BLOCKS
#endif
#ifndef SRK_P3_MIN_BLOCKS
#define SRK_P3_MIN_BLOCKS SRK_MIN_BLOCKS
#endif

namespace srk {

constexpr int kWarps = 8;
constexpr int kThreads = 32 * kWarps;
constexpr int kThreadsStage = kThreads;

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

// One image of a ragged batch: its size and where it starts in the
// concatenated N-sized and W-sized batch arrays (elements).  A column slab
// of one image is a one-image table whose offsets are negative (the
// caller's pointers address the slab's first column) and whose stencil
// blocks cover only the pixel columns [cx0, cx1).
struct RagImage {
  long long on, ow;
  int N, W;
  int blk0;      // first block of this image in the ragged stencil launch
  int cx0, cx1;  // pixel columns of the N x N output the stencil writes
  int pad;
};

// Tile geometry of one launch.  A uniform batch tiles every image alike
// (tile u -> image u / TT); a ragged batch of images of different N lists
// its tiles in `rtile` (image, x0, y0) and its images in `rimg`.
struct Geom {
  int M;      // FFT tile size
  int e;      // erosion (kernel half width bound)
  int S;      // valid outputs per tile per axis (<= M - 2e)
  int T;      // tiles per axis (uniform batch)
  int Nin;    // virtual input size (N for forward-type, N + 2e for adjoint)
  int Wout;   // output size (W for forward-type, N for adjoint)
  int TT;     // T*T
  int U;      // tiles in the whole batch
  int N, W;   // image and valid-output size (uniform batch)
  int wout_n; // outputs are N x N (adjoint-type) rather than W x W
  const int4* __restrict__ rtile;      // ragged: tile -> (image, x0, y0, 0); else nullptr
  const RagImage* __restrict__ rimg;   // ragged: per-image sizes and offsets
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

// a*b + c*d with one fixed rounding sequence, so every kernel that inlines
// an epilogue produces bit-identical results.
__device__ __forceinline__ float dot2(float a, float b, float c, float d) { return __fmaf_rn(a, b, __fmul_rn(c, d)); }

struct TileRef {
  int b, x0, y0;     // image index and tile origin in virtual input coordinates
  bool live;
  int N, W, Wout;    // this image's size, valid-output size and output size
  long long on, ow;  // offset of this image in N-sized / W-sized batch arrays
};
__device__ __forceinline__ TileRef tile_of(const Geom& g, int u) {
  TileRef t;
  t.live = u < g.U;
  const int uu = t.live ? u : 0;
  if (g.rtile) {
    const int4 q = g.rtile[uu];
    const RagImage im = g.rimg[q.x];
    t.b = q.x;
    t.x0 = q.y;
    t.y0 = q.z;
    t.N = im.N;
    t.W = im.W;
    t.on = im.on;
    t.ow = im.ow;
  } else {
    if (g.TT == 1) {  // one tile per image (tile size >= image): no divisions
      t.b = uu;
      t.x0 = 0;
      t.y0 = 0;
    } else {
      t.b = uu / g.TT;
      const int r = uu - t.b * g.TT;
      const int tx = r / g.T, ty = r - (r / g.T) * g.T;
      t.x0 = tx * g.S;
      t.y0 = ty * g.S;
    }
    t.N = g.N;
    t.W = g.W;
    t.on = (long long)t.b * g.N * g.N;
    t.ow = (long long)t.b * g.W * g.W;
  }
  t.Wout = g.wout_n ? t.N : t.W;
  return t;
}

// ---- loaders: value of field k of work tile w at local (x, y) ------------
// Adjoint-type: h_x = v*df/dx (or dv*df/dx + v*d(df)/dx for the
// tangent-adjoint) on the valid window, zero elsewhere; virtual coords are
// shifted by +e so that the full N x N output is the valid part of the
// convolution of the zero-extended (N+2e)^2 field
// (srk_adj_load_tile, adjoint/srk_adjoint.cuh:169-200).
template <typename T>
__device__ __forceinline__ float h_at(const OpArgs& a, const TileRef& t, int k, int px, int py) {
  const int qx = px - a.e, qy = py - a.e;            // image coords
  const int ox = qx - a.e, oy = qy - a.e;            // valid-window coords
  if (ox < 0 || oy < 0 || ox >= t.W || oy >= t.W) return 0.f;
  const long long vo = t.ow + (long long)ox * t.W + oy;
  const T* f = static_cast<const T*>(a.I) + t.on;
  const float v = ldf(static_cast<const T*>(a.v), vo);
  const float g = (k == 0) ? grad_x(f, t.N, qx, qy) : grad_y(f, t.N, qx, qy);
  if (a.dI == nullptr) return v * g;
  const T* df = static_cast<const T*>(a.dI) + t.on;
  const float dv = ldf(static_cast<const T*>(a.dv), vo);
  const float dg = (k == 0) ? grad_x(df, t.N, qx, qy) : grad_y(df, t.N, qx, qy);
  return dot2(dv, g, v, dg);
}

// Column x of one real tile of image `img` (forward-type ops): values at
// rows y = lane + 32 i, zero outside the image.  Pointers are hoisted so the
// loads are (base + immediate); bounds are tested per element only for a
// tile that crosses the bottom edge.
template <int M, typename T>
__device__ __forceinline__ void load_tile_column(const T* __restrict__ img, const TileRef& t, int x, int lane,
                                                 float (&v)[M / tpf_of<M>()]) {
  constexpr int TPF = tpf_of<M>();
  constexpr int EPT = M / TPF;
  const int N = t.N;
  const int gx = t.x0 + x;
  if (!t.live || gx >= N) {
#pragma unroll
    for (int i = 0; i < EPT; ++i) v[i] = 0.f;
    return;
  }
  const T* col = img + t.on + (long long)gx * N + t.y0 + lane;
  const int rows = N - t.y0 - lane;  // rows available below this lane's first element
  if (N - t.y0 >= M) {
#pragma unroll
    for (int i = 0; i < EPT; ++i) v[i] = ldf(col, TPF * i);
  } else {
#pragma unroll
    for (int i = 0; i < EPT; ++i) v[i] = (TPF * i < rows) ? ldf(col, TPF * i) : 0.f;
  }
}

template <int M, int OP, typename T>
__device__ __forceinline__ void load_column(const OpArgs& a, const Geom& g, int w, int k, int x, int lane,
                                            float2 (&z)[M / tpf_of<M>()]) {
  constexpr int TPF = tpf_of<M>();
  constexpr int EPT = M / TPF;
  if constexpr (OP == OP_ADJ) {
    const TileRef t0 = tile_of(g, 2 * w), t1 = tile_of(g, 2 * w + 1);
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      const int y = lane + TPF * i;
      const float re = h_at<T>(a, t0, k, t0.x0 + x, t0.y0 + y);
      const float im = t1.live ? h_at<T>(a, t1, k, t1.x0 + x, t1.y0 + y) : 0.f;
      z[i] = make_float2(re, im);
    }
  } else if constexpr (OpTraits<OP>::PAIRS) {
    float re[EPT], im[EPT];
    const T* E = static_cast<const T*>(a.E);
    load_tile_column<M, T>(E, tile_of(g, 2 * w), x, lane, re);
    load_tile_column<M, T>(E, tile_of(g, 2 * w + 1), x, lane, im);
#pragma unroll
    for (int i = 0; i < EPT; ++i) z[i] = make_float2(re[i], im[i]);
  } else {
    float re[EPT], im[EPT];
    const TileRef t = tile_of(g, w);
    load_tile_column<M, T>(static_cast<const T*>(a.E), t, x, lane, re);
    load_tile_column<M, T>(static_cast<const T*>(a.dE), t, x, lane, im);
#pragma unroll
    for (int i = 0; i < EPT; ++i) z[i] = make_float2(re[i], im[i]);
  }
}

// Both adjoint-type fields of one P1 column at once (erosion >= 1, so every
// gradient neighbour of the valid window lies inside the image): zx = h_x of
// the two tiles of WT w (re / im) at virtual column x, rows lane + TPF i,
// and h_y of the same element straight into this thread's stash slot
// st[kThreads i].  Per element one load of v (and dv) and the four
// neighbours of f (and df), shared by h_x and h_y; the arithmetic is h_at's.
// TAN: the tangent-adjoint's fields (dv, df given), a compile-time choice so
// that the plain adjoint carries none of their registers.
template <int M, typename T, bool TAN>
__device__ __forceinline__ void load_adj_column(const OpArgs& a, const Geom& g, int w, int x, int lane,
                                                float2 (&zx)[M / tpf_of<M>()], float2* __restrict__ st) {
  constexpr int TPF = tpf_of<M>();
  constexpr int EPT = M / TPF;
  const T* vc[2];
  const T* fc[2];
  const T* dvc[2];
  const T* dfc[2];
  int N[2], W[2], oy0[2];
  bool on[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const TileRef tr = tile_of(g, 2 * w + h);
    const int qx = tr.x0 + x - a.e, ox = qx - a.e;  // image / valid-window column
    on[h] = tr.live && ox >= 0 && ox < tr.W;
    const int qy0 = tr.y0 + lane - a.e;
    oy0[h] = qy0 - a.e;
    N[h] = tr.N;
    W[h] = tr.W;
    const long long vo = tr.ow + (long long)ox * tr.W + oy0[h];
    const long long fo = tr.on + (long long)qx * tr.N + qy0;
    vc[h] = static_cast<const T*>(a.v) + vo;
    fc[h] = static_cast<const T*>(a.I) + fo;
    dvc[h] = TAN ? static_cast<const T*>(a.dv) + vo : vc[h];
    dfc[h] = TAN ? static_cast<const T*>(a.dI) + fo : fc[h];
  }
#pragma unroll
  for (int i = 0; i < EPT; ++i) {
    const int o = TPF * i;
    float hx[2], hy[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const bool in = on[h] && (unsigned)(oy0[h] + o) < (unsigned)W[h];
      const int n = N[h];
      const float v = in ? ldf(vc[h], o) : 0.f;
      const float gx = ((in ? ldf(fc[h] + n, o) : 0.f) - (in ? ldf(fc[h] - n, o) : 0.f)) * 0.5f;
      const float gy = ((in ? ldf(fc[h] + 1, o) : 0.f) - (in ? ldf(fc[h] - 1, o) : 0.f)) * 0.5f;
      hx[h] = v * gx;
      hy[h] = v * gy;
      if constexpr (TAN) {
        const float dv = in ? ldf(dvc[h], o) : 0.f;
        const float dgx = ((in ? ldf(dfc[h] + n, o) : 0.f) - (in ? ldf(dfc[h] - n, o) : 0.f)) * 0.5f;
        const float dgy = ((in ? ldf(dfc[h] + 1, o) : 0.f) - (in ? ldf(dfc[h] - 1, o) : 0.f)) * 0.5f;
        hx[h] = dot2(dv, gx, v, dgx);
        hy[h] = dot2(dv, gy, v, dgy);
      }
      if (!in) hx[h] = hy[h] = 0.f;
    }
    zx[i] = make_float2(hx[0], hx[1]);
    st[kThreads * i] = make_float2(hy[0], hy[1]);
  }
}

// Central differences of f at image column gx for this lane's rows
// gy = gy0 + 32 i: fx = (f[gx+1] - f[gx-1])/2, fy = (f[gy+1] - f[gy-1])/2.
// With erosion >= 1 every valid output has its 4 neighbours inside the
// image, so the zero-padding rule of srk_grad_x/_y never applies and the
// loads need no test; erosion 0 takes the tested path.
template <typename T>
struct GradCol {
  const T* __restrict__ c;   // f + gx*N + gy0
  int N;
  bool tested;
  int gx, gy0;
  int st;  // row step between a thread's elements (threads per transform)
  __device__ __forceinline__ void at(int i, float& fx, float& fy) const {
    if (!tested) {
      fx = (ldf(c + N, st * i) - ldf(c - N, st * i)) * 0.5f;
      fy = (ldf(c + 1, st * i) - ldf(c - 1, st * i)) * 0.5f;
    } else {
      const int gy = gy0 + st * i;
      const float r = (gx + 1 < N) ? ldf(c + N, st * i) : 0.f;
      const float l = (gx > 0) ? ldf(c - N, st * i) : 0.f;
      const float d = (gy + 1 < N) ? ldf(c + 1, st * i) : 0.f;
      const float u = (gy > 0) ? ldf(c - 1, st * i) : 0.f;
      fx = (r - l) * 0.5f;
      fy = (d - u) * 0.5f;
    }
  }
};
template <typename T>
__device__ __forceinline__ GradCol<T> grad_col(const T* f_img, int N, int e, int gx, int gy0, int st) {
  GradCol<T> gc;
  gc.st = st;
  gc.c = f_img + (long long)gx * N + gy0;
  gc.N = N;
  gc.tested = e < 1;
  gc.gx = gx;
  gc.gy0 = gy0;
  return gc;
}

// Rows of this lane that carry valid outputs, as a bit mask over i.
template <int M>
__device__ __forceinline__ unsigned valid_rows(const Geom& g, const TileRef& t, int lane) {
  // rows y = lane + TPF*i are valid for e <= y < yhi: a contiguous run of i
  constexpr int TPF = tpf_of<M>();
  constexpr int EPT = M / TPF;
  const int yhi = min(g.e + g.S, t.Wout - t.y0 + g.e);
  const int ilo = max(0, (g.e - lane + TPF - 1) / TPF);        // first i with y >= e (g.e - lane > -TPF)
  const int ihi = yhi - lane > 0 ? (yhi - lane + TPF - 1) / TPF : 0;  // first i with y >= yhi
  const int hi = min(ihi, EPT);
  return hi > ilo ? (((1u << hi) - 1u) & ~((1u << ilo) - 1u)) : 0u;
}

template <int M, int OP, typename T>
__device__ __forceinline__ void epilogue_column(const OpArgs& a, const Geom& g, int w, int x, int lane,
                                                float2 (&z0)[M / tpf_of<M>()], float2 (&z1)[M / tpf_of<M>()]) {
  constexpr int TPF = tpf_of<M>();
  constexpr int EPT = M / TPF;
  const int e = a.e;
  if constexpr (OP == OP_FWD || OP == OP_VJP_F) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const TileRef t = tile_of(g, 2 * w + h);
      const int ox = t.x0 + x - g.e;
      if (!t.live || ox >= t.Wout) continue;
      const unsigned vm = valid_rows<M>(g, t, lane);
      // output row oy = y0 + y - e  ->  offset of row (y0 - e + lane)
      const long long ob = t.ow + (long long)ox * t.W + t.y0 - g.e + lane;
      if constexpr (OP == OP_FWD) {
        T* __restrict__ R = static_cast<T*>(a.out0);
        T* __restrict__ UX = static_cast<T*>(a.out_ux);
        T* __restrict__ UY = static_cast<T*>(a.out_uy);
        if (UX) {
#pragma unroll
          for (int i = 0; i < EPT; ++i)
            if (vm >> i & 1u) stf(UX, ob + TPF * i, h ? z0[i].y : z0[i].x);
        }
        if (UY) {
#pragma unroll
          for (int i = 0; i < EPT; ++i)
            if (vm >> i & 1u) stf(UY, ob + TPF * i, h ? z1[i].y : z1[i].x);
        }
        if (R) {
          const GradCol<T> gc = grad_col(static_cast<const T*>(a.I) + t.on, t.N, e, ox + e, t.y0 + lane, TPF);
          // gradients for all rows first (every load in flight before the
          // first store); the result overwrites this image's half of z0
#pragma unroll
          for (int i = 0; i < EPT; ++i) {
            float fx = 0.f, fy = 0.f;
            if (vm >> i & 1u) gc.at(i, fx, fy);
            float& o = h ? z0[i].y : z0[i].x;
            o = dot2(o, fx, h ? z1[i].y : z1[i].x, fy);
          }
#pragma unroll
          for (int i = 0; i < EPT; ++i)
            if (vm >> i & 1u) stf(R, ob + TPF * i, h ? z0[i].y : z0[i].x);
        }
      } else {  // OP_VJP_F: w = u * v
        const T* __restrict__ V = static_cast<const T*>(a.v);
        float* __restrict__ WX = static_cast<float*>(a.out0);
        float* __restrict__ WY = static_cast<float*>(a.out1);
        float v[EPT];
#pragma unroll
        for (int i = 0; i < EPT; ++i) v[i] = (vm >> i & 1u) ? ldf(V, ob + TPF * i) : 0.f;
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
          if (!(vm >> i & 1u)) continue;
          WX[ob + TPF * i] = (h ? z0[i].y : z0[i].x) * v[i];
          WY[ob + TPF * i] = (h ? z1[i].y : z1[i].x) * v[i];
        }
      }
    }
  } else if constexpr (OP == OP_JVP || OP == OP_TANADJ_F) {
    const TileRef t = tile_of(g, w);
    const int ox = t.x0 + x - g.e;
    if (ox >= t.Wout) return;
    const unsigned vm = valid_rows<M>(g, t, lane);
    const long long ob = t.ow + (long long)ox * t.W + t.y0 - g.e + lane;
    if constexpr (OP == OP_JVP) {
      // srk_tangent_combine (tan_tanadj/srk_tangent.cuh:28-52); re: conv of g, im: conv of dg
      const GradCol<T> gf = grad_col(static_cast<const T*>(a.I) + t.on, t.N, e, ox + e, t.y0 + lane, TPF);
      const GradCol<T> gd = grad_col(static_cast<const T*>(a.dI) + t.on, t.N, e, ox + e, t.y0 + lane, TPF);
      T* __restrict__ DH = static_cast<T*>(a.out0);
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        float fx = 0.f, fy = 0.f, dfx = 0.f, dfy = 0.f;
        if (vm >> i & 1u) {
          gf.at(i, fx, fy);
          gd.at(i, dfx, dfy);
        }
        z0[i].x = __fmaf_rn(z1[i].x, dfy, __fmaf_rn(z0[i].x, dfx, dot2(z0[i].y, fx, z1[i].y, fy)));
      }
#pragma unroll
      for (int i = 0; i < EPT; ++i)
        if (vm >> i & 1u) stf(DH, ob + TPF * i, z0[i].x);
    } else {
      const T* __restrict__ LAM = static_cast<const T*>(a.v);
      const T* __restrict__ DLAM = static_cast<const T*>(a.dv);
      float* __restrict__ WX = static_cast<float*>(a.out0);
      float* __restrict__ WY = static_cast<float*>(a.out1);
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        if (!(vm >> i & 1u)) continue;
        const float lam = ldf(LAM, ob + TPF * i), dlam = ldf(DLAM, ob + TPF * i);
        WX[ob + TPF * i] = dot2(dlam, z0[i].x, lam, z0[i].y);
        WY[ob + TPF * i] = dot2(dlam, z1[i].x, lam, z1[i].y);
      }
    }
  } else {  // OP_ADJ: output is the full N x N image
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const TileRef t = tile_of(g, 2 * w + h);
      const int ox = t.x0 + x - g.e;
      if (!t.live || ox >= t.Wout) continue;
      const unsigned vm = valid_rows<M>(g, t, lane);
      const long long ob = t.on + (long long)ox * t.N + t.y0 - g.e + lane;
      T* __restrict__ O = static_cast<T*>(a.out0);
#pragma unroll
      for (int i = 0; i < EPT; ++i)
        if (vm >> i & 1u) stf(O, ob + TPF * i, h ? z0[i].y : z0[i].x);
    }
  }
}

// ---- unit geometry ----------------------------------------------------------------
// A CTA of kWarps warps processes one unit of LPU lines (columns in P1/P3,
// rows in P2); each line is one transform over TPF threads (line = thread /
// TPF, t = thread % TPF, named barrier 1 + line when TPF > 32).
template <int M>
__host__ __device__ constexpr int lpu_of() { return kThreads / tpf_of<M>(); }

// ---- staged gradients -------------------------------------------------------------
// The LPU output columns of a P3 unit need the image columns gx-1 ..
// gx+LPU and rows gy-1 .. gy+S.  They are staged into shared memory, one
// warp per window column: window column c <-> image column x0 + e - 1 + c;
// window row r <-> image row gy0 + r, gy0 = y0 + e - 1, stored at column
// offset off + r.  Out-of-image elements are zero (the central-difference
// rule).  With 16-byte copies the column starts at the aligned row
// gy0 - off (off = gy0 mod 4); otherwise off = 0.  The pitch is a multiple
// of 4 floats (16-byte aligned columns).
__host__ __device__ inline int gwin_pitch(int S) { return (S + 8) & ~3; }
// The same for a window of raw storage values (16-byte chunks of EPC
// elements): a multiple of EPC that holds off + S + 2 for any off < EPC.
template <typename T>
__host__ __device__ inline int gwin_pitch_t(int S) {
  constexpr int EPC = 16 / (int)sizeof(T);
  return (S + 2 + 2 * (EPC - 1)) / EPC * EPC;
}
// Shared-memory window value as float.
template <typename T> __device__ __forceinline__ float swin(const T* p);
template <> __device__ __forceinline__ float swin<float>(const float* p) { return *p; }
template <> __device__ __forceinline__ float swin<__half>(const __half* p) { return __half2float(*p); }
template <> __device__ __forceinline__ float swin<__nv_bfloat16>(const __nv_bfloat16* p) { return __bfloat162float(*p); }
// (LPU + 2) * gwin_pitch(S) floats <= (LPU + 2) * (M + 4) <= 2 * LPU * (M + M/16 + 2)
// for S <= M - 2: one image's window always fits the LPU staging rows of the
// second field.
struct GradWin {
  int gx0, gy0;  // image coordinates of window column 0, row 0
  int ncol, S;   // columns, and S + 2 rows
  int HP, off;   // column pitch (floats), offset of row 0 in a column
};

// Synchronous staging (any storage type; values converted to float).
template <typename T>
__device__ __forceinline__ void stage_grad_window(const T* __restrict__ img, int N, const GradWin& gw,
                                                  float* __restrict__ dst) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int H = gw.S + 2;
  for (int c = warp; c < gw.ncol; c += kWarps) {
    const int gx = gw.gx0 + c;
    const bool colin = gx >= 0 && gx < N;
    const T* col = img + (long long)(colin ? gx : 0) * N;
    float* d = dst + c * gw.HP;
    for (int r = lane; r < H; r += 32) {
      const int gy = gw.gy0 + r;
      d[r] = (colin && gy >= 0 && gy < N) ? ldf(col, gy) : 0.f;
    }
  }
}

// Asynchronous staging with cp.async (FP32 images): the caller commits the
// group and waits for it later, so the loads overlap other work.
__device__ __forceinline__ void cp_async4_zfill(float* dst, const float* src, bool valid) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async16_zfill(float* dst, const float* src, bool valid) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Raw storage values of the window.  vec16: 16-byte chunks of EPC values
// (needs N % EPC == 0 and a 16-byte aligned image, so every chunk lies
// wholly inside or wholly outside the image); else 4-byte copies (FP32 only).
template <typename T>
__device__ __forceinline__ void stage_grad_window_async(const T* __restrict__ img, int N, const GradWin& gw,
                                                        bool vec16, T* __restrict__ dst) {
  constexpr int EPC = 16 / (int)sizeof(T);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int c = warp; c < gw.ncol; c += kWarps) {
    const int gx = gw.gx0 + c;
    const bool colin = gx >= 0 && gx < N;
    const T* col = img + (long long)(colin ? gx : 0) * N;
    T* d = dst + c * gw.HP;
    if (vec16) {
      // chunk q of the column: rows gya + EPC*q ..; gya = gy0 - off >= 0, so
      // a chunk is outside the image only past its last row (or off its columns)
      const int gya = gw.gy0 - gw.off;
      const int nch = (gw.off + gw.S + 2 + EPC - 1) / EPC;
      const int glim = colin ? N : -1;
      const char* src = reinterpret_cast<const char*>(col + gya) + 16 * lane;
      unsigned dsm = static_cast<unsigned>(__cvta_generic_to_shared(d)) + 16u * lane;
      int gy = gya + EPC * lane;
      for (int q = lane; q < nch; q += 32, src += 512, dsm += 512u, gy += 32 * EPC) {
        const bool in = gy < glim;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dsm), "l"(in ? src : (const char*)img),
                     "r"(in ? 16 : 0)
                     : "memory");
      }
    } else if constexpr (std::is_same<T, float>::value) {
      for (int r = lane; r < gw.S + 2; r += 32) {
        const int gy = gw.gy0 + r;
        const bool in = colin && gy >= 0 && gy < N;
        cp_async4_zfill(d + r, in ? col + gy : img, in);
      }
    }
  }
}
// Floats of one staged window at tile size M (S <= M - 2 when erosion >= 1);
// a window of 2-byte values needs at most (LPU + 2) * (M + 8) of them.
template <int M>
__host__ __device__ constexpr int p3_window_floats() { return (lpu_of<M>() + 2) * (M + 4); }
// P3 of the three-launch schedule prefetches the first window asynchronously
// into a buffer of its own (forward / tangent epilogues).
template <int OP, typename T>
__host__ __device__ constexpr bool p3_async_window() {
  return OP == OP_FWD || OP == OP_JVP;
}

// Forward / tangent epilogue, round h, with the central differences read
// from the staged window (window column line+1 is this line's image
// column).  FWD: round h finishes image h of the pair.  JVP: round 0
// (window = f) leaves the f terms in z0.y, round 1 (window = df) adds the df
// terms.  z0 stays stashed in the line's padded row (z0s = row + t +
// (t >> 4), element i at z0s[(TPF + TPF/16) i]) to keep registers free.
template <int M, int OP, typename T, typename WT>
__device__ __forceinline__ void epilogue_staged(const OpArgs& a, const Geom& g, const TileRef& tr, int x, int line,
                                                int t, int h, float2* __restrict__ z0s,
                                                const float2 (&z1)[M / tpf_of<M>()], const WT* __restrict__ win,
                                                const GradWin& gw) {
  constexpr int TPF = tpf_of<M>();
  constexpr int EPT = M / TPF;
  constexpr int RSP = TPF + TPF / 16;
  const int W = tr.W;
  const int rb = gw.off + t - g.e + 1;     // window row of element 0: y - e + 1, y = t
  const WT* cm = win + line * gw.HP + rb;  // image column gx - 1
  const WT* cc = cm + gw.HP;               // gx
  const WT* cp = cc + gw.HP;               // gx + 1
  const int ox = tr.x0 + x - g.e;
  if (!tr.live || ox >= tr.Wout) return;
  const unsigned vm = valid_rows<M>(g, tr, t);
  const long long ob = tr.ow + (long long)ox * W + tr.y0 - g.e + t;
  if constexpr (OP == OP_FWD) {
    T* __restrict__ R = static_cast<T*>(a.out0);
    T* __restrict__ UX = static_cast<T*>(a.out_ux);
    T* __restrict__ UY = static_cast<T*>(a.out_uy);
    if (!UX && !UY) {
      // R only (R is never NULL here): the common case; of the stashed z0
      // only this round's half is read
      T* __restrict__ Rp = R + ob;
      const float* z0h = reinterpret_cast<const float*>(z0s) + h;
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        if (!(vm >> i & 1u)) continue;
        const float ux = z0h[2 * RSP * i];
        const float uy = h ? z1[i].y : z1[i].x;
        // the central differences' factor 1/2 applied once: halving is
        // exact, so dot2(ux, dx/2, uy, dy/2) == dot2(ux, dx, uy, dy)/2
        const float dx = swin(cp + TPF * i) - swin(cm + TPF * i);
        const float dy = swin(cc + TPF * i + 1) - swin(cc + TPF * i - 1);
        stf(Rp, TPF * i, dot2(ux, dx, uy, dy) * 0.5f);
      }
      return;
    }
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      if (!(vm >> i & 1u)) continue;
      const float2 z0i = z0s[RSP * i];
      const float ux = h ? z0i.y : z0i.x;
      const float uy = h ? z1[i].y : z1[i].x;
      if (UX) stf(UX, ob + TPF * i, ux);
      if (UY) stf(UY, ob + TPF * i, uy);
      if (R) {
        const float dx = swin(cp + TPF * i) - swin(cm + TPF * i);
        const float dy = swin(cc + TPF * i + 1) - swin(cc + TPF * i - 1);
        stf(R, ob + TPF * i, dot2(ux, dx, uy, dy) * 0.5f);
      }
    }
  } else {
    // srk_tangent_combine (tan_tanadj/srk_tangent.cuh:28-52):
    // dh = Im(zx) fx + Im(zy) fy + Re(zx) dfx + Re(zy) dfy
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      if (!(vm >> i & 1u)) continue;
      const float dx_ = (swin(cp + TPF * i) - swin(cm + TPF * i)) * 0.5f;
      const float dy_ = (swin(cc + TPF * i + 1) - swin(cc + TPF * i - 1)) * 0.5f;
      float2 z0i = z0s[RSP * i];
      if (h == 0) {
        z0i.y = dot2(z0i.y, dx_, z1[i].y, dy_);
        z0s[RSP * i] = z0i;
      } else {
        stf(static_cast<T*>(a.out0), ob + TPF * i, __fmaf_rn(z1[i].x, dy_, __fmaf_rn(z0i.x, dx_, z0i.y)));
      }
    }
  }
}

// ---- phases ------------------------------------------------------------------
__device__ __forceinline__ void load_twiddles(float2* tw, const float2* __restrict__ twg, int M) {
  for (int i = threadIdx.x; i < tw_entries(M); i += blockDim.x) tw[i] = twg[i];
}

// Staging rows: fft_row_words(M) or a little more, so that the rows of a
// transposing copy fall into different banks.
template <int M>
__host__ __device__ constexpr int row_stride() {
  // stage_rows writes 2 (LPU = 4) or 4 (LPU = 8) rows per half-warp: their
  // strides must land on disjoint banks (RS = 4 or 2 mod 8 complex values)
  int w = fft_row_words(M) + 1;
  while (w % 8 != (lpu_of<M>() == 4 ? 4 : 2)) ++w;
  return w;
}
// Valid columns x' of S2 rounded up to a multiple of 8 (>= LPU).
__host__ __device__ inline int s2_pitch(int S) { return (S + 7) & ~7; }
// S2 layout.  Blocked (M = 512, LPU = 4): S2[l][x'/LPU][ky][x' % LPU], so
// the LPU columns a P3 unit needs are one contiguous run of M*LPU values
// (instead of 32-byte pieces of every row), and the LPU x LPU block a P2
// unit produces per column block is contiguous too; P2 assembles the blocks
// in a shared tile of pitch s2_block_pitch per block (LPU^2 values + padding
// that keeps its writes free of bank conflicts).  Row layout (LPU = 8):
// S2[l][ky][x'], pitch s2_pitch(S) — with 64-byte pieces per row the extra
// tile pass in P2 costs more than it saves in P3.
template <int M>
__host__ __device__ constexpr bool s2_blocked() { return lpu_of<M>() == 4; }
// S1 likewise (M = 512): S1[k][ky/LPU][x][ky % LPU], assembled by P1 in its
// staging rows (free after the transforms), staged by P2 from one
// contiguous run of M*LPU values.  At LPU = 8 the rows are read in 64-byte
// pieces already and the blocked form measured no faster.
template <int M>
__host__ __device__ constexpr bool s1_blocked() { return lpu_of<M>() == 4; }
template <int M>
__host__ __device__ constexpr int s2_block_pitch() { return lpu_of<M>() == 4 ? 20 : 72; }
template <int M>
__host__ __device__ inline size_t p2_tile_bytes(int S) {
  return s2_blocked<M>() ? sizeof(float2) * (size_t)(s2_pitch(S) / lpu_of<M>()) * s2_block_pitch<M>() : 0;
}
// Twiddle slots at the start of every kernel's shared memory.
template <int M>
__host__ __device__ constexpr int tw_slots() { return (tw_entries(M) + 7) & ~7; }

// Scratch of one work tile: S1 [K][x < M][ky < M] then S2 (L fields of M x pitch(S), see above) (float2).
template <int M, int OP>
__host__ __device__ constexpr size_t s1_elems() { return (size_t)OpTraits<OP>::K * M * M; }
template <int M, int OP>
__host__ __device__ inline size_t wt_elems(int S) {
  return s1_elems<M, OP>() + (size_t)OpTraits<OP>::L * M * s2_pitch(S);
}

// Shared memory of every phase: the twiddle table and 2 x LPU staging rows
// (P2 adds its block tile, P3 its first gradient window).
template <int M>
constexpr size_t phase_smem_bytes() { return sizeof(float2) * (tw_slots<M>() + 2 * lpu_of<M>() * row_stride<M>()); }
// P1 of the adjoint-type op adds the stash of the second field.
template <int M, int OP>
constexpr size_t p1_smem_bytes() {
  return phase_smem_bytes<M>() + (OP == OP_ADJ ? sizeof(float2) * kThreads * (M / tpf_of<M>()) : 0);
}

// Copies between a thread's registers (strided order) and a padded row.
template <int M>
__device__ __forceinline__ void row_to_regs(const float2* __restrict__ row, float2 (&z)[M / tpf_of<M>()], int t) {
  constexpr int TPF = tpf_of<M>();
  const float2* rd = row + t + (t >> 4);
#pragma unroll
  for (int i = 0; i < M / TPF; ++i) z[i] = rd[(TPF + TPF / 16) * i];
}
template <int M>
__device__ __forceinline__ void regs_to_row(float2* __restrict__ row, const float2 (&z)[M / tpf_of<M>()], int t) {
  constexpr int TPF = tpf_of<M>();
  float2* wr = row + t + (t >> 4);
#pragma unroll
  for (int i = 0; i < M / TPF; ++i) wr[(TPF + TPF / 16) * i] = z[i];
}

// P1: line `line` transforms column x = xb*LPU + line of every field along y.
// P1 output of one field: the line's transform z (ky = t + TPF*i) of
// column xb*LPU + line -> S1.
template <int M>
__device__ __forceinline__ void p1_store(const float2 (&z)[M / tpf_of<M>()], float2* __restrict__ S1k, int xb,
                                         float2* __restrict__ rows, int line, int t) {
  constexpr int TPF = tpf_of<M>();
  constexpr int EPT = M / TPF;
  constexpr int LPU = lpu_of<M>();
  if constexpr (s1_blocked<M>()) {
    // the unit's LPU columns -> shared tile of (ky/LPU) blocks -> whole
    // LPU x LPU blocks of S1 (the staging rows are free after the transforms)
    constexpr int PB = s2_block_pitch<M>();
    constexpr int F4B = LPU * LPU / 2;
    __syncthreads();
    // ky = t + TPF*i: block t/LPU + i*TPF/LPU, position t % LPU in it
    float2* rl = rows + (t / LPU) * PB + line * LPU + (t % LPU);
#pragma unroll
    for (int i = 0; i < EPT; ++i) rl[(TPF / LPU) * PB * i] = z[i];
    __syncthreads();
    float2* dst = S1k + (size_t)xb * LPU * LPU;
    for (int j = threadIdx.x; j < (M / LPU) * F4B; j += kThreads) {
      const int q = j / F4B, v = j - (j / F4B) * F4B;
      __stcg(reinterpret_cast<float4*>(dst + (size_t)q * M * LPU + 2 * v),
             *reinterpret_cast<const float4*>(rows + q * PB + 2 * v));
    }
    __syncthreads();  // the rows are the next transform's exchange rows
  } else {
    float2* dst = S1k + (size_t)(xb * LPU + line) * M + t;
#pragma unroll
    for (int i = 0; i < EPT; ++i) __stcg(dst + TPF * i, z[i]);
  }
}

// L2 prefetch of the image columns that P1 units xb2 .. xb2+NU-1 of WT w2
// load (single-field ops: the two tiles of a pair, or E and dE of one
// tile).  One 128-byte line per thread; only addresses inside the images.
template <int M, int OP, typename T, int NU>
__device__ __forceinline__ void p1_prefetch(const OpArgs& a, const Geom& g, int w2, int xb2) {
  constexpr int C = lpu_of<M>() * NU;                     // columns per field
  constexpr int RPL = 128 / (int)sizeof(T);              // rows per line
  constexpr int LC = (M + RPL - 1) / RPL;                 // lines per column
  static_assert(C * LC <= kThreads / 2, "one line per thread and field");
  const int h = threadIdx.x / (kThreads / 2), r = threadIdx.x % (kThreads / 2);
  if (r >= C * LC) return;
  const TileRef tr = OpTraits<OP>::PAIRS ? tile_of(g, 2 * w2 + h) : tile_of(g, w2);
  const int gx = tr.x0 + xb2 * lpu_of<M>() + r / LC;
  const int gy = tr.y0 + (r % LC) * RPL;
  if (!tr.live || gx >= tr.N || gy >= tr.N) return;
  const T* img = static_cast<const T*>(OpTraits<OP>::PAIRS || h == 0 ? a.E : a.dE);
  asm volatile("prefetch.global.L2 [%0];" ::"l"(img + tr.on + (long long)gx * tr.N + gy));
}

// The same for the adjoint-type P1 unit xb of WT w2: the v (and dv) columns
// and the f (and df) columns around them that load_adj_column reads, for
// both tiles of the pair; one 128-byte line per thread and iteration.
template <int M, typename T>
__device__ __forceinline__ void p1_prefetch_adj(const OpArgs& a, const Geom& g, int w2, int xb2) {
  constexpr int LPU = lpu_of<M>();
  constexpr int RPL = 128 / (int)sizeof(T);
  constexpr int LV = (M + RPL - 1) / RPL + 1;      // lines of a v column (start not line-aligned)
  constexpr int LF = (M + 2 + RPL - 1) / RPL + 1;  // lines of an f column
  constexpr int PER = LPU * LV + (LPU + 2) * LF;   // per tile and array pair
  const int npair = a.dI != nullptr ? 2 : 1;
  const int e = a.e;
  for (int idx = threadIdx.x; idx < 2 * PER * npair; idx += kThreads) {
    const int d = idx / (2 * PER), h = (idx / PER) & 1, r = idx % PER;
    const TileRef tr = tile_of(g, 2 * w2 + h);
    if (!tr.live) continue;
    const int x = tr.x0 + xb2 * LPU;
    if (r < LPU * LV) {
      const int col = x + r / LV - 2 * e, row0 = tr.y0 - 2 * e;
      const int row = max(row0, 0) + (r % LV) * RPL;
      if (col < 0 || col >= tr.W || row >= tr.W || row >= row0 + M) continue;
      const T* v = static_cast<const T*>(d ? a.dv : a.v);
      asm volatile("prefetch.global.L2 [%0];" ::"l"(v + tr.ow + (long long)col * tr.W + row));
    } else {
      const int rf = r - LPU * LV;
      const int col = x + rf / LF - e - 1, row0 = tr.y0 - e - 1;
      const int row = max(row0, 0) + (rf % LF) * RPL;
      if (col < 0 || col >= tr.N || row >= tr.N || row >= row0 + M + 2) continue;
      const T* f = static_cast<const T*>(d ? a.dI : a.I);
      asm volatile("prefetch.global.L2 [%0];" ::"l"(f + tr.on + (long long)col * tr.N + row));
    }
  }
}

// P1: line `line` transforms column x = xb*LPU + line of every field along
// y.  NU consecutive units (xb, xb+1, ...) per call, single-field ops only:
// the next unit's columns are loaded before the current transform, so their
// latency overlaps it, and the columns of the CTA `ahead` launch positions
// later (about one per SM: it starts when this one is nearly done) are
// prefetched into L2.
template <int M, int OP, typename T, int NU = 1, bool TAN = false>
__device__ __forceinline__ void phase1(const OpArgs& a, const Geom& g, int w, int xb, float2* __restrict__ S1,
                                       float2* __restrict__ rows, const float2* __restrict__ tw, int line, int t,
                                       int ahead = 0, float2* __restrict__ stash = nullptr) {
  constexpr int TPF = tpf_of<M>();
  constexpr int EPT = M / TPF;
  constexpr int K = OpTraits<OP>::K;
  constexpr int LPU = lpu_of<M>();
  constexpr int RS = row_stride<M>();
  static_assert(NU == 1 || (NU == 2 && K == 1), "two units per call for single-field ops only");
  float2* row = rows + line * RS;
  if constexpr (NU == 2) {
    if (ahead > 0) {
      const int lin = (int)(blockIdx.y * gridDim.x + blockIdx.x) + ahead;
      p1_prefetch<M, OP, T, NU>(a, g, w - (int)blockIdx.y + lin / (int)gridDim.x, (lin % (int)gridDim.x) * NU);
    }
    float2 za[EPT], zb[EPT];
    load_column<M, OP, T>(a, g, w, 0, xb * LPU + line, t, za);
    load_column<M, OP, T>(a, g, w, 0, (xb + 1) * LPU + line, t, zb);
    fft<M, false>(za, row, tw, t, 1 + line);
    p1_store<M>(za, S1, xb, rows, line, t);
    fft<M, false>(zb, row, tw, t, 1 + line);
    p1_store<M>(zb, S1, xb + 1, rows, line, t);
  } else {
    if constexpr (OP == OP_ADJ) {
      // both fields from one pass over the inputs; h_y waits in the
      // stash (kThreads x EPT values after the rows, each thread its own)
      if (stash && a.e >= 1) {
        if (ahead > 0) {
          const int lin = (int)(blockIdx.y * gridDim.x + blockIdx.x) + ahead;
          p1_prefetch_adj<M, T>(a, g, w - (int)blockIdx.y + lin / (int)gridDim.x, lin % (int)gridDim.x);
        }
        float2 zx[EPT];
        float2* st = stash + threadIdx.x;
        load_adj_column<M, T, TAN>(a, g, w, xb * LPU + line, t, zx, st);
        fft<M, false>(zx, row, tw, t, 1 + line);
        p1_store<M>(zx, S1, xb, rows, line, t);
#pragma unroll
        for (int i = 0; i < EPT; ++i) zx[i] = st[kThreads * i];
        fft<M, false>(zx, row, tw, t, 1 + line);
        p1_store<M>(zx, S1 + (size_t)M * M, xb, rows, line, t);
        return;
      }
    }
#pragma unroll 1
    for (int k = 0; k < K; ++k) {
      float2 z[EPT];
      load_column<M, OP, T>(a, g, w, k, xb * LPU + line, t, z);
      fft<M, false>(z, row, tw, t, 1 + line);
      p1_store<M>(z, S1 + (size_t)k * M * M, xb, rows, line, t);
    }
  }
}

// Transposing copy of an M x LPU block (M lines of LPU consecutive complex
// values, line pitch `pitch`) into LPU staging rows of M values each.  All
// threads of the CTA take part; every load is in flight before the
// scattered shared stores.
template <int M>
__device__ __forceinline__ void stage_rows(const float2* __restrict__ src, int pitch, float2* __restrict__ rows) {
  constexpr int RS = row_stride<M>();
  constexpr int LPU = lpu_of<M>();
  constexpr int Q = LPU / 2;                 // float4 per line
  constexpr int NIT = M * Q / kThreads;      // float4 loads per thread
  static_assert(M * Q % kThreads == 0, "staging loop must divide evenly");
  // element j of this thread: line y0 + j*YS, value pair cp (YS is a multiple
  // of 16, so fft_pad(y0 + j*YS) = fft_pad(y0) + fft_pad(j*YS))
  constexpr int YS = kThreads / Q;
  static_assert(YS % 16 == 0, "line step must keep the padding separable");
  const int y0 = threadIdx.x / Q, cp = threadIdx.x % Q;
  const float4* sp = reinterpret_cast<const float4*>(src + (size_t)y0 * pitch + 2 * cp);
  const size_t sstep = (size_t)YS * pitch / 2;  // float4 per j (pitch is even)
  float4 q[NIT];
#pragma unroll
  for (int j = 0; j < NIT; ++j) q[j] = __ldcg(sp + j * sstep);
  float2* r0 = rows + (2 * cp) * RS + fft_pad(y0);
  float2* r1 = r0 + RS;
#pragma unroll
  for (int j = 0; j < NIT; ++j) {
    r0[fft_pad(j * YS)] = make_float2(q[j].x, q[j].y);
    r1[fft_pad(j * YS)] = make_float2(q[j].z, q[j].w);
  }
}

// stage_rows for a rotated S2 block (the tensor-core row pass's layout):
// block line y holds frequency row (y - rot) mod M, which lands in the rows
// at that index.  Rotating the lines by the column block spreads the row
// pass's 32-byte pieces of one ky over the L2 instead of stacking them at one
// offset of blocks 16 KB apart.
template <int M>
__device__ __forceinline__ void stage_rows_rot(const float2* __restrict__ src, int rot, float2* __restrict__ rows) {
  constexpr int RS = row_stride<M>();
  constexpr int LPU = lpu_of<M>();
  constexpr int Q = LPU / 2;
  constexpr int NIT = M * Q / kThreads;
  constexpr int YS = kThreads / Q;
  const int y0 = threadIdx.x / Q, cp = threadIdx.x % Q;
  const float4* sp = reinterpret_cast<const float4*>(src + (size_t)y0 * LPU + 2 * cp);
  constexpr size_t sstep = (size_t)YS * LPU / 2;
  float4 q[NIT];
#pragma unroll
  for (int j = 0; j < NIT; ++j) q[j] = __ldcg(sp + j * sstep);
  float2* r0 = rows + (2 * cp) * RS;
  float2* r1 = r0 + RS;
#pragma unroll
  for (int j = 0; j < NIT; ++j) {
    const int ky = (y0 + j * YS - rot) & (M - 1);
    r0[fft_pad(ky)] = make_float2(q[j].x, q[j].y);
    r1[fft_pad(ky)] = make_float2(q[j].z, q[j].w);
  }
}

// P2: rows ky0 .. ky0+LPU-1: FFT along x, spectral map, inverse, keep the
// valid columns, write S2 rows.  All threads of the CTA take part.
template <int M, int OP>
__device__ __forceinline__ void phase2(const float2* __restrict__ S1, float2* __restrict__ S2,
                                       const float2* __restrict__ Gx, const float2* __restrict__ Gy, int conjG,
                                       const Geom& g, int ky0, float2* __restrict__ rows,
                                       const float2* __restrict__ tw, int line, int t, float2* __restrict__ tile) {
  constexpr int TPF = tpf_of<M>();
  constexpr int EPT = M / TPF;
  constexpr int RSP = TPF + TPF / 16;
  constexpr int K = OpTraits<OP>::K;
  constexpr int RS = row_stride<M>();
  constexpr int LPU = lpu_of<M>();
  const int S = g.S, e = g.e, P = s2_pitch(S);
  const int bar = 1 + line;
  // S1[k][x][ky0 + c]: a transposing copy of LPU consecutive ky of every column x
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if constexpr (s1_blocked<M>())
      stage_rows<M>(S1 + (size_t)k * M * M + (size_t)ky0 * M, LPU, rows + k * LPU * RS);
    else
      stage_rows<M>(S1 + (size_t)k * M * M + ky0, M, rows + k * LPU * RS);
  }
  __syncthreads();
  const int ky = ky0 + line;
  float2* row0 = rows + line * RS;           // field 0 / exchange
  float2* row1 = rows + (LPU + line) * RS;   // field 1 or the stash
  const float2* gxr = Gx + (size_t)ky * M + t;
  const float2* gyr = Gy + (size_t)ky * M + t;
  auto spec = [&](float2 z, float2 G) { return conjG ? cmulc(z, G) : cmul(z, G); };
  // valid columns of field l -> the shared block tile -> whole LPU x LPU
  // blocks of S2 (16-byte stores, each block one contiguous run)
  constexpr int PB = s2_block_pitch<M>();
  constexpr int F4B = LPU * LPU / 2;  // float4 per block
  const int nblk = P / LPU;
  auto emit = [&](const float2 (&o)[EPT], int l) {
    if constexpr (!s2_blocked<M>()) {
      float2* dst = S2 + ((size_t)l * M + ky) * P - e + t;
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int xv = t + TPF * i - e;
        if (xv >= 0 && xv < S) __stcg(dst + TPF * i, o[i]);
      }
      return;
    }
    {
      // xv = xb0 + TPF*i lies in block floor(xb0 / LPU) + i*TPF/LPU at
      // position xb0 mod LPU (an arithmetic shift and a mask also for the
      // negative xb0 of the columns left of the valid range, never stored)
      const int xb0 = t - e;
      constexpr int LS = LPU == 4 ? 2 : 3;
      float2* tl = tile + (xb0 >> LS) * PB + line * LPU + (xb0 & (LPU - 1));
#pragma unroll
      for (int i = 0; i < EPT; ++i)
        if ((unsigned)(xb0 + TPF * i) < (unsigned)S) tl[(TPF / LPU) * PB * i] = o[i];
    }
    __syncthreads();
    // thread: value pair w of blocks q = q0, q0 + QS, ... (QS blocks per sweep)
    constexpr int QS = kThreads / F4B;
    const int q0 = threadIdx.x / F4B, w = threadIdx.x % F4B;
    float4* dst = reinterpret_cast<float4*>(S2 + ((size_t)l * nblk * M + ky0) * LPU + (size_t)q0 * M * LPU + 2 * w);
    const float4* src = reinterpret_cast<const float4*>(tile + q0 * PB + 2 * w);
    for (int q = q0; q < nblk; q += QS, dst += (size_t)QS * M * LPU / 2, src += QS * PB / 2) __stcg(dst, *src);
    __syncthreads();  // the tile is reused by the next field
  };
  float2 z[EPT];
  row_to_regs<M>(row0, z, t);
  fft<M, false>(z, row0, tw, t, bar);
  if constexpr (K == 1) {
    // both spectral products at once; Z*Gy waits in the line's second row
    // (each thread rereads only its own elements)
    float2* st = row1 + t + (t >> 4);
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
      const float2 zi = z[i];
      st[RSP * i] = spec(zi, __ldg(gyr + TPF * i));
      z[i] = spec(zi, __ldg(gxr + TPF * i));
    }
    fft<M, true>(z, row0, tw, t, bar);
    emit(z, 0);
#pragma unroll
    for (int i = 0; i < EPT; ++i) z[i] = st[RSP * i];
    fft<M, true>(z, row0, tw, t, bar);
    emit(z, 1);
  } else {
    group_sync<TPF>(bar);
    regs_to_row<M>(row0, z, t);  // stash Z0(ky, .) in its own row
    row_to_regs<M>(row1, z, t);
    fft<M, false>(z, row1, tw, t, bar);
    const float2* st = row0 + t + (t >> 4);
#pragma unroll
    for (int i = 0; i < EPT; ++i)
      z[i] = cadd(spec(st[RSP * i], __ldg(gxr + TPF * i)), spec(z[i], __ldg(gyr + TPF * i)));
    fft<M, true>(z, row1, tw, t, bar);
    emit(z, 0);
  }
}

// P3: columns x' = xb*LPU .. +LPU-1: stage them, inverse FFT along ky,
// epilogue.  All threads of the CTA take part (lines without a valid column
// still join the barriers).  For the forward and tangent epilogues with
// erosion >= 1 the image columns the central differences need are staged in
// shared memory after the transforms, in the rows they no longer use.
// S2 layouts P3 reads: the engine's (blocked for M = 512), the blocked one
// with rotated lines, or the plain one [field][ky][P] (the latter two written
// by the tensor-core row pass).
enum S2Layout : int { kS2Engine = 0, kS2Rotated = 1, kS2Plain = 2 };
template <int M, int OP, typename T, bool ASYNC = false, int S2L = kS2Engine>
__device__ __forceinline__ void phase3(const float2* __restrict__ S2, const OpArgs& a, const Geom& g, int w, int xb,
                                       float2* __restrict__ rows, const float2* __restrict__ tw, int line, int t,
                                       T* __restrict__ win0 = nullptr) {
  constexpr int TPF = tpf_of<M>();
  constexpr int EPT = M / TPF;
  constexpr int L = OpTraits<OP>::L;
  constexpr int RS = row_stride<M>();
  constexpr int LPU = lpu_of<M>();
  constexpr bool GRAD = (OP == OP_FWD || OP == OP_JVP);
  static_assert(!ASYNC || p3_async_window<OP, T>(), "asynchronous window only for the forward / tangent");
  constexpr int EPC = 16 / (int)sizeof(T);  // storage values per 16-byte copy
  const int P = s2_pitch(g.S);
  const int x0 = xb * LPU;
  const int bar = 1 + line;
  // window of round h: image (pair member h, or f / df) columns
  // x0+e-1 .. x0+e+LPU, rows y0+e-1 .. y0+e+S
  // raw: the asynchronous copy of storage values (else floats staged by the threads)
  auto window_of = [&](int h, const TileRef& tr, bool vec16, bool raw) {
    GradWin gw;
    gw.gx0 = tr.x0 + x0 + a.e - 1;
    gw.gy0 = tr.y0 + a.e - 1;
    gw.ncol = LPU + 2;
    gw.S = g.S;
    gw.HP = raw ? gwin_pitch_t<T>(g.S) : gwin_pitch(g.S);
    gw.off = vec16 ? (gw.gy0 % EPC) : 0;
    return gw;
  };
  auto tile_h = [&](int h) { return tile_of(g, OP == OP_FWD ? 2 * w + h : w); };
  auto image_h = [&](int h) { return static_cast<const T*>(OP == OP_FWD || h == 0 ? a.I : a.dI); };
  // 16-byte window copies: N % EPC == 0, a 16-byte aligned image start
  auto vec16_of = [&](int h, const TileRef& tr) {
    return ASYNC && tr.N % EPC == 0 &&
           ((reinterpret_cast<uintptr_t>(image_h(h)) + sizeof(T) * (uintptr_t)tr.on) & 15) == 0;
  };
  auto issue_window = [&](int h, T* dst) {
    if constexpr (ASYNC) {
      const TileRef tr = tile_h(h);
      const bool vec16 = vec16_of(h, tr);
      if (tr.live) stage_grad_window_async<T>(image_h(h) + tr.on, tr.N, window_of(h, tr, vec16, true), vec16, dst);
      cp_async_commit();
    }
  };
  // 2-byte storage needs the 16-byte form for both windows; else the
  // threads stage converted floats (below)
  bool async_win = false;
  if constexpr (ASYNC) {
    async_win = a.e >= 1;
    if constexpr (!std::is_same<T, float>::value)
      async_win = async_win && vec16_of(0, tile_h(0)) && vec16_of(1, tile_h(1));
    if (async_win) issue_window(0, win0);  // in flight during the staging and the transforms
  }
#pragma unroll
  for (int l = 0; l < L; ++l) {
    if constexpr (S2L == kS2Rotated) {
      static_assert(s2_blocked<M>(), "rotated blocks of the blocked layout");
      stage_rows_rot<M>(S2 + ((size_t)l * (P / LPU) + xb) * M * LPU, xb & (M - 1), rows + l * LPU * RS);
    } else if constexpr (s2_blocked<M>() && S2L == kS2Engine)
      stage_rows<M>(S2 + ((size_t)l * (P / LPU) + xb) * M * LPU, LPU, rows + l * LPU * RS);
    else
      stage_rows<M>(S2 + (size_t)l * M * P + x0, P, rows + l * LPU * RS);
  }
  __syncthreads();
  const int xv = x0 + line;
  const bool active = xv < g.S;
  float2* row0 = rows + line * RS;
  float2* row1 = rows + (LPU + line) * RS;
  float2 z0[EPT], z1[EPT];
  if (active) {
    row_to_regs<M>(row0, z0, t);
    fft<M, true>(z0, row0, tw, t, bar);
    if constexpr (L == 2) {
      group_sync<TPF>(bar);
      regs_to_row<M>(row0, z0, t);   // stash, reread after the second transform
      row_to_regs<M>(row1, z1, t);
      fft<M, true>(z1, row1, tw, t, bar);
    }
  }
  if constexpr (L == 1) {
#pragma unroll
    for (int i = 0; i < EPT; ++i) z1[i] = make_float2(0.f, 0.f);
  }
  if constexpr (ASYNC) {
    if (async_win) {
      // window 0 has been arriving in its own buffer; window 1 goes to the
      // second field's rows once every line is done with them
      T* win1 = reinterpret_cast<T*>(rows + LPU * RS);
      float2* z0s = row0 + t + (t >> 4);
      __syncthreads();
      issue_window(1, win1);
      cp_async_wait<1>();
      __syncthreads();
      const TileRef tr0 = tile_h(0);
      if (active)
        epilogue_staged<M, OP, T, T>(a, g, tr0, xv + g.e, line, t, 0, z0s, z1, win0,
                                     window_of(0, tr0, vec16_of(0, tr0), true));
      cp_async_wait<0>();
      __syncthreads();
      const TileRef tr1 = tile_h(1);
      if (active)
        epilogue_staged<M, OP, T, T>(a, g, tr1, xv + g.e, line, t, 1, z0s, z1, win1,
                                     window_of(1, tr1, vec16_of(1, tr1), true));
      return;
    }
  }
  if constexpr (GRAD) {
    if (a.e >= 1) {
      // two rounds, one image window each, in the second field's rows
      float* win = reinterpret_cast<float*>(rows + LPU * RS);
      float2* z0s = row0 + t + (t >> 4);
#pragma unroll 1
      for (int h = 0; h < 2; ++h) {
        __syncthreads();  // rows of field 1 no longer used (round 0) / window consumed (round 1)
        const TileRef tr = tile_h(h);
        const GradWin gw = window_of(h, tr, false, false);
        if (tr.live) stage_grad_window<T>(image_h(h) + tr.on, tr.N, gw, win);
        __syncthreads();
        if (active) epilogue_staged<M, OP, T, float>(a, g, tr, xv + g.e, line, t, h, z0s, z1, win, gw);
      }
      return;
    }
  }
  if (!active) return;
  if constexpr (L == 2) {
    group_sync<TPF>(bar);
    row_to_regs<M>(row0, z0, t);
  }
  epilogue_column<M, OP, T>(a, g, w, xv + g.e, t, z0, z1);
}

// ---- three-launch schedule (one kernel per phase over a chunk of WTs) ------
// Units per P1 CTA (see phase1): two for single-field ops (the second
// unit's loads overlap the first transform; -4% at N=512), else one.
#ifndef SRK_P1_UNITS
#define SRK_P1_UNITS 2
#endif
template <int M, int OP>
__host__ __device__ constexpr int p1_units() { return OpTraits<OP>::K == 1 ? SRK_P1_UNITS : 1; }
template <int M, int OP, typename T, bool TAN = false>
__global__ void __launch_bounds__(kThreads, SRK_P1_MIN_BLOCKS)
k_p1(OpArgs a, Geom g, const float2* __restrict__ twg, int w0, float2* __restrict__ scratch, int S, int ahead) {
  // TAN (adjoint-type op of the tangent-adjoint, dv and df given) is chosen
  // by the launch: a.dI != nullptr exactly when TAN
  extern __shared__ float2 sm[];
  constexpr int TPF = tpf_of<M>();
  const int line = threadIdx.x / TPF, t = threadIdx.x % TPF;
  load_twiddles(sm, twg, M);
  __syncthreads();
  const int wl = blockIdx.y;
  constexpr int NU = p1_units<M, OP>();
  float2* stash = OP == OP_ADJ ? sm + tw_slots<M>() + 2 * lpu_of<M>() * row_stride<M>() : nullptr;
  phase1<M, OP, T, NU, TAN>(a, g, w0 + wl, blockIdx.x * NU, scratch + wl * wt_elems<M, OP>(S), sm + tw_slots<M>(),
                            sm, line, t, ahead, stash);
}

template <int M, int OP>
__global__ void __launch_bounds__(kThreads, SRK_P2_MIN_BLOCKS)
k_p2(float2* __restrict__ scratch, const float2* __restrict__ Gx, const float2* __restrict__ Gy, int conjG, Geom g,
     const float2* __restrict__ twg) {
  extern __shared__ float2 sm[];
  constexpr int TPF = tpf_of<M>();
  const int line = threadIdx.x / TPF, t = threadIdx.x % TPF;
  load_twiddles(sm, twg, M);
  float2* base = scratch + blockIdx.y * wt_elems<M, OP>(g.S);
  float2* rows = sm + tw_slots<M>();
  phase2<M, OP>(base, base + s1_elems<M, OP>(), Gx, Gy, conjG, g, blockIdx.x * lpu_of<M>(), rows, sm, line, t,
                rows + 2 * lpu_of<M>() * row_stride<M>());
}

// S2L: the S2 layout (S2Layout).
template <int M, int OP, typename T, int S2L = kS2Engine>
__global__ void __launch_bounds__(kThreads, SRK_P3_MIN_BLOCKS)
k_p3(float2* __restrict__ scratch, OpArgs a, Geom g, const float2* __restrict__ twg, int w0, int ahead) {
  extern __shared__ float2 sm[];
  constexpr int TPF = tpf_of<M>();
  const int line = threadIdx.x / TPF, t = threadIdx.x % TPF;
  load_twiddles(sm, twg, M);
  const int wl = blockIdx.y;
  constexpr bool ASYNC = p3_async_window<OP, T>();
  T* win0 = ASYNC ? reinterpret_cast<T*>(sm + tw_slots<M>() + 2 * lpu_of<M>() * row_stride<M>()) : nullptr;
  {
    // L2 prefetch of the S2 columns of the CTA one SM-count of launch
    // positions later: one contiguous run per field in the blocked layout,
    // one 8-value row piece per ky in the plain one
    constexpr int L = OpTraits<OP>::L;
    const int lin = (int)(blockIdx.y * gridDim.x + blockIdx.x) + ahead;
    const int by2 = lin / (int)gridDim.x, bx2 = lin % (int)gridDim.x;
    if (ahead > 0 && by2 < (int)gridDim.y) {
      const float2* s2 = scratch + by2 * wt_elems<M, OP>(g.S) + s1_elems<M, OP>();
      if constexpr (s2_blocked<M>() && S2L != kS2Plain) {
        constexpr int LINES = M * lpu_of<M>() * (int)sizeof(float2) / 128;  // per field
        static_assert(L * LINES <= kThreads, "one line per thread");
        if (threadIdx.x < L * LINES) {
          const int l = threadIdx.x / LINES, r = threadIdx.x % LINES;
          const float2* blk = s2 + ((size_t)l * (s2_pitch(g.S) / lpu_of<M>()) + bx2) * M * lpu_of<M>();
          asm volatile("prefetch.global.L2 [%0];" ::"l"(blk + r * (128 / sizeof(float2))));
        }
      } else {
        const float2* col = s2 + bx2 * lpu_of<M>();
        for (int idx = threadIdx.x; idx < L * M; idx += kThreads)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(col + (size_t)idx * s2_pitch(g.S)));
      }
    }
  }
  phase3<M, OP, T, ASYNC, S2L>(scratch + wl * wt_elems<M, OP>(g.S) + s1_elems<M, OP>(), a, g, w0 + wl, blockIdx.x,
                          sm + tw_slots<M>(), sm, line, t, win0);
}

// ---- persistent schedule ---------------------------------------------------------
// One launch processes every WT.  Work is a ticket queue of rounds; round r
// holds the P1 units of WT r, the P2 units of WT r-lag and the P3 units of
// WT r-2*lag.  A WT's scratch lives in slot w mod nslot of a small ring that
// stays in L2.  Per-slot counters (monotonic over the slot's reuses) order
// the phases:
//   P1(w) needs c2[slot] >= gen*n2       (previous user's P2 done reading S1)
//   P2(w) needs c1[slot] >= (gen+1)*n1   (its S1 complete)
//           and c3[slot] >= gen*n3       (previous user's P3 done reading S2)
//   P3(w) needs c2[slot] >= (gen+1)*n2   (its S2 complete)
// Every dependency points to a smaller ticket, and a ticket is only ever held
// by a running CTA (a CTA holds at most its current ticket and one
// prefetched larger one), so the smallest unfinished ticket can always
// proceed.  The lag and the ring size only decide how often a unit finds its
// dependency not yet met.  Waits are bounded anyway: a wait that exceeds
// `spin_limit` polls sets ctl->abort (with the place in ctl->where) and every
// CTA returns.
constexpr int kMaxSlots = 32;

struct Ctl {
  unsigned int ticket;
  unsigned int abort;
  unsigned int where;
  unsigned int pad;
  unsigned long long spins;  // polls that found a dependency unmet (diagnostic)
  unsigned int c1[kMaxSlots], c2[kMaxSlots], c3[kMaxSlots];
};

struct PersistParams {
  int lag;        // rounds between the phases of one WT
  int nslot;      // scratch ring slots (> lag)
  int prefetch;   // fetch the next ticket while running the current one
  int pad;
  unsigned long long spin_limit;
};

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Thread-0 wait: returns false if the kernel must stop.
__device__ __forceinline__ bool wait_geq(const unsigned int* p, unsigned int target, unsigned long long limit,
                                         Ctl* ctl, unsigned int where, unsigned long long& spins) {
  unsigned long long it = 0;
  while (ld_acquire(p) < target) {
    if (ld_acquire(&ctl->abort)) return false;
    if (++it > limit) {
      atomicExch(&ctl->where, where);
      atomicExch(&ctl->abort, 1u);
      return false;
    }
    __nanosleep(32);
  }
  spins += it;
  return true;
}

template <int M, int OP, typename T>
__global__ void __launch_bounds__(kThreads, SRK_MIN_BLOCKS)
k_persist(OpArgs a, Geom g, const float2* __restrict__ Gx, const float2* __restrict__ Gy, int conjG,
          const float2* __restrict__ twg, float2* __restrict__ scratch, int nwt, Ctl* ctl, PersistParams pp) {
  extern __shared__ float2 sm[];
  __shared__ int s_t[2];
  constexpr int TPF = tpf_of<M>();
  constexpr int LPU = lpu_of<M>();
  const int line = threadIdx.x / TPF, t = threadIdx.x % TPF;
  const int n1 = M / LPU, n2 = M / LPU, n3 = (g.S + LPU - 1) / LPU;
  const int round = n1 + n2 + n3;
  const int lag = pp.lag, nslot = pp.nslot;
  const long long total = (long long)(nwt + 2 * lag) * round;
  const size_t slot_elems = wt_elems<M, OP>(g.S);
  unsigned long long spins = 0;
  float2* tw = sm;
  float2* buf = sm + tw_slots<M>();
  load_twiddles(tw, twg, M);
  if (threadIdx.x == 0) s_t[0] = (int)atomicAdd(&ctl->ticket, 1u);
  __syncthreads();
  int cur = s_t[0];
  while (cur < total) {
    unsigned int nxt = 0;
    if (threadIdx.x == 0 && pp.prefetch) nxt = atomicAdd(&ctl->ticket, 1u);
    const int r = cur / round, u = cur - (cur / round) * round;
    int phase, w, unit;
    if (u < n1) { phase = 1; w = r; unit = u; }
    else if (u < n1 + n2) { phase = 2; w = r - lag; unit = u - n1; }
    else { phase = 3; w = r - 2 * lag; unit = u - n1 - n2; }
    const bool live = (w >= 0 && w < nwt);
    const int slot = live ? w % nslot : 0;
    const unsigned int gen = live ? (unsigned int)(w / nslot) : 0u;
    if (threadIdx.x == 0) {
      bool ok = ld_acquire(&ctl->abort) == 0u;
      if (ok && live) {
        if (phase == 1) ok = wait_geq(&ctl->c2[slot], gen * n2, pp.spin_limit, ctl, 1, spins);
        else if (phase == 2) ok = wait_geq(&ctl->c1[slot], (gen + 1) * n1, pp.spin_limit, ctl, 2, spins) &&
                                  wait_geq(&ctl->c3[slot], gen * n3, pp.spin_limit, ctl, 3, spins);
        else ok = wait_geq(&ctl->c2[slot], (gen + 1) * n2, pp.spin_limit, ctl, 4, spins);
      }
      s_t[1] = ok ? 1 : 0;
    }
    __syncthreads();
    if (!s_t[1]) break;
    if (live) {
      float2* base = scratch + (size_t)slot * slot_elems;
      if (phase == 1) {
        phase1<M, OP, T>(a, g, w, unit, base, buf, tw, line, t);
      } else if (phase == 2) {
        phase2<M, OP>(base, base + s1_elems<M, OP>(), Gx, Gy, conjG, g, unit * LPU, buf, tw, line, t,
                      buf + 2 * LPU * row_stride<M>());
      } else {
        phase3<M, OP, T>(base + s1_elems<M, OP>(), a, g, w, unit, buf, tw, line, t);
      }
    }
    __syncthreads();  // every thread's scratch stores of this unit are issued
    if (threadIdx.x == 0) {
      if (live) {
        __threadfence();
        atomicAdd(phase == 1 ? &ctl->c1[slot] : phase == 2 ? &ctl->c2[slot] : &ctl->c3[slot], 1u);
      }
      s_t[0] = pp.prefetch ? (int)nxt : (int)atomicAdd(&ctl->ticket, 1u);
    }
    __syncthreads();
    cur = s_t[0];
  }
  if (threadIdx.x == 0 && spins) atomicAdd(&ctl->spins, spins);
}

// Bounded-wait self test: thread 0 of one CTA waits for a counter that
// nothing increments; the wait must give up and raise the abort flag.
static __global__ void k_wait_selftest(Ctl* ctl, unsigned long long spin_limit) {
  unsigned long long spins = 0;
  if (threadIdx.x == 0) wait_geq(&ctl->c1[0], 1u, spin_limit, ctl, 99, spins);
}

// dL/df = D_x^T(wx) + D_y^T(wy) on N x N, with wx, wy given on the W x W
// window (zero outside); adjoint of the central difference
// (adjointWrtI_kernel, adjoint/srk_adjoint.cuh:25-59).  With ux, uy, v
// given instead (the reference contract) w = u*v is formed on the fly.
// A thread computes kStencilCols consecutive columns of one row: the
// kStencilCols + 2 values of wx it needs are loaded once, and every load is
// issued before the first use.
constexpr int kStencilCols = 4;
template <typename T, bool FROM_U>
__device__ __forceinline__ void adj_wrt_f_cols(const float* __restrict__ wx, const float* __restrict__ wy,
                                               const T* __restrict__ v, const T* __restrict__ ux,
                                               const T* __restrict__ uy, long long wo, long long oo, int N, int W,
                                               int e, int gx0, int gx1, int gy, T* __restrict__ out) {
  constexpr int CX = kStencilCols;
  if (gy >= N) return;
  const int oy = gy - e;
  auto w_at = [&](const float* w, const T* u, int r, int c, bool in) -> float {
    const long long i = wo + (long long)c * W + r;
    if constexpr (FROM_U) return in ? __fmul_rn(ldf(u, i), ldf(v, i)) : 0.f;
    else return in ? w[i] : 0.f;
  };
  const bool rin = (unsigned)oy < (unsigned)W;
  const bool uin = (unsigned)(oy - 1) < (unsigned)W, din = (unsigned)(oy + 1) < (unsigned)W;
  float wxv[CX + 2];
#pragma unroll
  for (int j = 0; j < CX + 2; ++j) {
    const int c = gx0 - e - 1 + j;
    wxv[j] = w_at(wx, ux, oy, c, rin && (unsigned)c < (unsigned)W);
  }
  float wyu[CX], wyd[CX];
#pragma unroll
  for (int j = 0; j < CX; ++j) {
    const int c = gx0 - e + j;
    const bool cin = (unsigned)c < (unsigned)W;
    wyu[j] = w_at(wy, uy, oy - 1, c, uin && cin);
    wyd[j] = w_at(wy, uy, oy + 1, c, din && cin);
  }
#pragma unroll
  for (int j = 0; j < CX; ++j) {
    const int gx = gx0 + j;
    if (gx >= gx1) break;
    const float val = __fadd_rn(__fmul_rn(__fsub_rn(wxv[j], wxv[j + 2]), 0.5f),
                                __fmul_rn(__fsub_rn(wyu[j], wyd[j]), 0.5f));
    stf(out, oo + (long long)gx * N + gy, val);
  }
}

// Uniform batch: grid (N/32, N/(8*kStencilCols), B) of 32 x 8 blocks.
template <typename T, bool FROM_U>
__global__ void k_adj_wrt_f(const float* __restrict__ wx, const float* __restrict__ wy, const T* __restrict__ v,
                            const T* __restrict__ ux, const T* __restrict__ uy, int N, int W, int e, int B,
                            T* __restrict__ out) {
  const int gy = blockIdx.x * blockDim.x + threadIdx.x;
  const int gx0 = (blockIdx.y * blockDim.y + threadIdx.y) * kStencilCols;
  const int b = blockIdx.z;
  adj_wrt_f_cols<T, FROM_U>(wx, wy, v, ux, uy, (long long)b * W * W, (long long)b * N * N, N, W, e, gx0, N, gy,
                            out);
}

// The same for a ragged batch or a column slab: 32 x 8 blocks over the
// pixel columns [cx0, cx1) of each image, the blocks of image b starting at
// rimg[b].blk0.
template <typename T, bool FROM_U>
__global__ void k_adj_wrt_f_rag(const float* __restrict__ wx, const float* __restrict__ wy, const T* __restrict__ v,
                                const T* __restrict__ ux, const T* __restrict__ uy,
                                const RagImage* __restrict__ rimg, int B, int e, T* __restrict__ out) {
  int lo = 0, hi = B - 1;
  const int blk = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (rimg[mid].blk0 <= blk) lo = mid; else hi = mid - 1;
  }
  const RagImage im = rimg[lo];
  const int nby = (im.N + 31) / 32;
  const int k = blk - im.blk0;
  const int gy = (k % nby) * 32 + threadIdx.x;
  const int gx0 = im.cx0 + ((k / nby) * 8 + threadIdx.y) * kStencilCols;
  adj_wrt_f_cols<T, FROM_U>(wx, wy, v, ux, uy, im.ow, im.on, im.N, im.W, e, gx0, im.cx1, gy, out);
}

}  // namespace srk
