// hybrid.cu — the row pass (P2) of SRK_SCHEDULE_TENSOR_ROWS on the
// 5th-generation tensor cores, for FP16/BF16 storage plans at tile M = 512.
//
// After the column FFT along y (P1), the convolution along x is, for every
// frequency row ky, a 1-D convolution with a short complex kernel:
//   U_G[ky][x'] = sum_x g_{G,ky}[x' - x] Z[ky][x],  |x' - x| <= e,
//   g_{G,ky}[d] = sum_kx G[ky][kx] exp(+2 pi i d kx / M)
// where G is the plan's engine-layout spectrum (dx^2/M^2 folded in) — exactly
// the row FFT, spectral product and inverse row FFT of the FFT row pass
// (engine.cuh phase2) for the valid outputs, without the transforms.  The
// inverse column FFT and the epilogue (P3) are unchanged: U is written to S2
// in P3's blocked FP32 layout with the lines of column block b rotated by b
// (k_p3<.., ROT = true> undoes it while staging): one item has one ky, so
// its stores are 32-byte pieces, and unrotated those sat at one offset of
// blocks 16 KB apart (measured 159 -> 150 us per 128 work tiles).
//
// GEMM form per item (one ky, 128 outputs x' = e + 128 j .., 128 work tiles):
//   D[m][n] = sum_k T[m][k] Z_n[ky][128 j + k],  T[m][k] = g[m - k + e],
// complex: Ur = Tr Zr - Ti Zi, Ui = Tr Zi + Ti Zr, four real MMAs of
// 128 x 128 x 16 per K step and field (the minus sign by the instruction
// descriptor's negate-A bit).  N = 128 keeps the operand reads from shared
// memory (A 4 KB + B 4 KB per MMA) within what the tensor cores can fetch
// while they compute; N = 64 (A re-read for half the work) measured twice
// as many shared-memory wavefronts per output.
// * B (Z planes, FP16, written by k_p1h) by TMA with the 128-byte swizzle:
//   box {64 columns x, 128 work tiles, 1 plane}, the K-major SWIZZLE_128B
//   operand, streamed through a ring of NS atoms of 64 columns.
// * A (the band T) never materialised: rows reversed, one slot table of
//   KT/8 + 16 slots x 128 bytes per (ky, field, part), read through a
//   descriptor with leading = stride byte offset = 128 (direct.cu explains the
//   identity).  Tables scaled by a power of two (max |g| in [8, 16)).
// * Persistent, one CTA per SM; per item one pass per field over the same
//   atoms, into that field's TMEM set (2 x 128 columns), so the S2 stores of
//   one field overlap the MMAs of the other.
// * Precision: FP16 operands (Z and g rounded once), FP32 accumulation — for
//   the FP16/BF16 storage forms (rel 1e-2 / abs 1e-3).
#include <cuda.h>
#include <cudaTypedefs.h>

#include "hybrid_p1g.cuh"
#include "hybrid_scale.cuh"
#include "internal.h"
#include "tc.cuh"

namespace srk {
namespace hyb {
using namespace srk::tc;

constexpr int M = 512;
constexpr int MT = 128;        // outputs x' per tile = TMEM lanes
constexpr int NB = 128;        // work tiles per item = MMA N (128 x 128 x 16 MMAs)
constexpr int NS = 5;          // ring slots of plane atoms
#ifndef SRK_HYB_EPI_WARPS
#define SRK_HYB_EPI_WARPS 8
#endif
// a multiple of 4, each TMEM lane quarter split by columns; measured per 128
// work tiles: 4 warps 170 us, 8 warps 159 us, 16 warps 191 us
constexpr int kEpiWarps = SRK_HYB_EPI_WARPS;
static_assert(kEpiWarps >= 4 && kEpiWarps % 4 == 0 && NB / (kEpiWarps / 4) % 16 == 0, "whole lane quarters");
constexpr int kThreadsH = 32 * (kEpiWarps + 2);    // + the load warp and the MMA warp
constexpr int kLoadWarp = kEpiWarps, kMmaWarp = kEpiWarps + 1;
constexpr int kMaxE = 64;

// input columns per tile, a whole number of 64-column (128-byte) swizzle atoms
__host__ __device__ constexpr int kt_of(int e) { return ((MT + 2 * e) + 63) / 64 * 64; }
__host__ __device__ constexpr int qs_of(int e) { return kt_of(e) / 8 + MT / 8; }           // band slots

struct Args {
  const uint16_t* tabs;   // [M ky][2 field][2 part][QS][8][8] FP16 bits
  const int* tab_exp;     // tables hold g * 2^tab_exp
  const unsigned int* mx; // largest |Z| per work tile (float bits): its planes hold Z * 2^plane_exp(mx[wl])
  float2* scratch;        // chunk base: S2 of work tile wl at scratch + wl*per + s1
  size_t per, s1;         // float2 per work tile, offset of S2 in it
  unsigned int* err;
  unsigned long long spin_limit;
  int c, e, S, P;         // work tiles in the chunk, erosion, valid stride, S2 pitch
};

// One plane atom: 64 columns x of NB work tiles, both parts (re, im), each
// part a TMA box of NB rows x 128 bytes with the 128-byte swizzle.
constexpr uint32_t kPartBytes = (uint32_t)NB * 128;
constexpr uint32_t kAtomBytes = 2 * kPartBytes;
// The band tables of one ky: 2 fields x 2 parts x QS slots of 128 bytes.
__host__ __device__ inline size_t band_bytes(int e) { return 4 * (size_t)qs_of(e) * 128; }
// barriers | NS atoms | 2 band buffers
__host__ __device__ inline size_t smem_bytes(int e) { return 1024 + (size_t)NS * kAtomBytes + 2 * band_bytes(e); }

__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}

// Persistent: one CTA per SM walks the items (x'-tile j, ky, batch of NB work
// tiles) with a stride of the grid.  An item runs as two passes, one per
// field, over the same resident planes, each into its own TMEM accumulator
// set (2 x NB columns), so the epilogue of one field drains while the MMAs of
// the other run.  The planes stream through a ring of NS atoms (a slot is
// freed by the field-1 pass); the band tables of an item are double-buffered.
//   zfull[s] : atom slot s loaded (TMA bytes)        zempty[s]: slot s read by both passes (commit)
//   bfull[b] : band buffer b loaded (bulk copy)      bempty[b]: buffer b read (commit)
//   tfull[f] : accumulators of field f complete      tempty[f]: drained (every epilogue warp)
__global__ void __launch_bounds__(kThreadsH, 1) k_p2h(const __grid_constant__ CUtensorMap zmap, Args a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int e = a.e, KT = kt_of(e), KB = KT / 64, QS = qs_of(e);
  const uint32_t tab = (uint32_t)QS * 128;      // one (field, part) band
  uint64_t* zfull = reinterpret_cast<uint64_t*>(smem);  // [NS]
  uint64_t* zempty = zfull + NS;                        // [NS]
  uint64_t* bfull = zempty + NS;                        // [2]
  uint64_t* bempty = bfull + 2;                         // [2]
  uint64_t* tfull = bempty + 2;                         // [2]
  uint64_t* tempty = tfull + 2;                         // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  unsigned char* Zs = smem + 1024;                      // NS atoms (1024-byte aligned: swizzle atoms)
  unsigned char* Ts = Zs + (size_t)NS * kAtomBytes;     // 2 band buffers
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntx = (a.S + MT - 1) / MT, nbatch = (a.c + NB - 1) / NB;
  const int items = ntx * M * nbatch;
  const unsigned long long lim = a.spin_limit;

  if (threadIdx.x == 0) {
    *abort_flag = (smem_u32(Zs) & 1023u) != 0;
    if (*abort_flag) atomicCAS(a.err, 0u, 14u);
    for (int i = 0; i < NS; ++i) {
      mbar_init(zfull + i, 1);
      mbar_init(zempty + i, 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(bfull + i, 1);
      mbar_init(bempty + i, 1);
      mbar_init(tfull + i, 1);
      mbar_init(tempty + i, kEpiWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(4 * NB));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  auto decode = [&](int item, int& j, int& ky, int& batch) {
    j = item % ntx;
    const int r = item / ntx;
    ky = r % M;
    batch = r / M;
  };

  if (warp == kLoadWarp) {
    if (lane == 0) {
      long long r = 0;  // atoms issued
      int nb = 0;       // band buffers issued
      for (int k = 0, item = blockIdx.x; item < items && !*abort_flag; ++k, item += gridDim.x) {
        int j, ky, batch;
        decode(item, j, ky, batch);
        const int b = k & 1;
        if (k >= 2 && !mbar_wait(bempty + b, (unsigned)((k / 2 - 1) & 1), lim)) {
          atomicCAS(a.err, 0u, 13u);
          *abort_flag = 1;
          break;
        }
        mbar_expect_tx(bfull + b, 4 * tab);
        bulk_g2s(Ts + (size_t)b * 4 * tab, a.tabs + (size_t)ky * 4 * QS * 64, 4 * tab, bfull + b);
        ++nb;
        for (int at = 0; at < KB; ++at) {
          const int slot = (int)(r % NS);
          if (r >= NS && !mbar_wait(zempty + slot, (unsigned)((r / NS - 1) & 1), lim)) {
            atomicCAS(a.err, 0u, 13u);
            *abort_flag = 1;
            break;
          }
          unsigned char* Zd = Zs + (size_t)slot * kAtomBytes;
          mbar_expect_tx(zfull + slot, kAtomBytes);
          for (int part = 0; part < 2; ++part)
            tma_load_3d(Zd + part * kPartBytes, &zmap, MT * j + 64 * at, NB * batch, ky * 2 + part, zfull + slot);
          ++r;
        }
      }
      // every copy issued has landed before the CTA can leave (also on the error path)
      for (long long q = r > NS ? r - NS : 0; q < r; ++q) mbar_wait(zfull + (int)(q % NS), (unsigned)((q / NS) & 1), lim);
      for (int q = nb > 2 ? nb - 2 : 0; q < nb; ++q) mbar_wait(bfull + (q & 1), (unsigned)((q / 2) & 1), lim);
    }
    __syncwarp();
  } else if (warp == kMmaWarp) {
    if (lane == 0) {
      const uint32_t id = idesc_f16(0, MT, NB);
      const uint32_t idn = id | (1u << 13);  // negate A
      long long r = 0;                       // first atom of the item
      bool ok = true;
      for (int k = 0, item = blockIdx.x; item < items && ok; ++k, item += gridDim.x, r += KB) {
        const int b = k & 1;
        ok = mbar_wait(bfull + b, (unsigned)((k / 2) & 1), lim) && !*abort_flag;
        const uint32_t a0 = smem_u32(Ts + (size_t)b * 4 * tab);
        for (int f = 0; f < 2 && ok; ++f) {
          // accumulator set f, drained by the epilogue of the previous item's field f
          if (k >= 1 && !mbar_wait(tempty + f, (unsigned)((k - 1) & 1), lim)) ok = false;
          const uint32_t dr = tmem + (uint32_t)f * 2 * NB, di = dr + NB;
          for (int at = 0; at < KB && ok; ++at) {
            const long long q = r + at;
            const int slot = (int)(q % NS);
            if (f == 0 && !mbar_wait(zfull + slot, (unsigned)((q / NS) & 1), lim)) ok = false;
            if (!ok) break;
            tc_fence_after();
            const uint32_t b0 = smem_u32(Zs + (size_t)slot * kAtomBytes);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
              const int ks = 4 * at + kk;
              const uint64_t dbr = sdesc_sw128(b0 + (uint32_t)kk * 32);
              const uint64_t dbi = sdesc_sw128(b0 + kPartBytes + (uint32_t)kk * 32);
              const uint64_t dar = sdesc(a0 + (uint32_t)(f * 2 + 0) * tab + (uint32_t)ks * 256, 128, 128);
              const uint64_t dai = sdesc(a0 + (uint32_t)(f * 2 + 1) * tab + (uint32_t)ks * 256, 128, 128);
              mma_f16(dr, dar, dbr, id, ks > 0);   // + Tr Zr
              mma_f16(dr, dai, dbi, idn, true);    // - Ti Zi
              mma_f16(di, dar, dbi, id, ks > 0);   // + Tr Zi
              mma_f16(di, dai, dbr, id, true);     // + Ti Zr
            }
            if (f == 1) mma_commit(zempty + slot);  // both passes have read the atom
          }
          if (ok) mma_commit(tfull + f);
        }
        if (ok) mma_commit(bempty + b);
      }
      if (!ok) {
        atomicCAS(a.err, 0u, 11u);
        *abort_flag = 1;
      }
    }
    __syncwarp();
  } else {
    // epilogue warp: TMEM lane quarter (warp % 4) and its share of the NB columns
    constexpr int kCols = NB / (kEpiWarps / 4);
    static_assert(NB == 128, "four column factors per lane");
    const int quarter = warp & 3, colh = warp >> 2;
    const int mrow = quarter * 32 + lane;         // TMEM lane (rows reversed)
    const int tab_exp = __ldg(a.tab_exp);
    const uint32_t trow = tmem + ((uint32_t)(quarter * 32) << 16);
    const size_t fo = (size_t)a.P * M;            // S2 field stride
    bool ok = true;
    for (int k = 0, item = blockIdx.x; item < items && ok; ++k, item += gridDim.x) {
      int j, ky, batch;
      decode(item, j, ky, batch);
      const int wl0 = NB * batch;
      // largest |Z| words of the columns lane + 32 h, loaded before the wait so their latency hides behind it
      unsigned int zw[4];
#pragma unroll
      for (int h = 0; h < 4; ++h) zw[h] = __ldg(a.mx + min(wl0 + 32 * h + lane, a.c - 1));
      const int xv = MT * j + MT - 1 - mrow;      // valid-column index x' - e
      // rotated blocked layout: S2 block xv >> 2 holds ky at line (ky + xv >> 2) mod M;
      // plain layout: row ky, column xv
      const size_t xo = kHybS2Layout == 2
                            ? (size_t)ky * a.P + xv
                            : (size_t)(xv >> 2) * M * 4 + (size_t)((ky + (xv >> 2)) & (M - 1)) * 4 + (xv & 3);
      float sp[4];
      for (int f = 0; f < 2; ++f) {
        bool w = true;
        if (lane == 0) w = mbar_wait(tfull + f, (unsigned)(k & 1), lim) && !*abort_flag;
        if (__shfl_sync(0xffffffffu, w ? 1 : 0, 0) == 0) {
          if (lane == 0) {
            atomicCAS(a.err, 0u, 12u);
            *abort_flag = 1;
          }
          ok = false;
          break;
        }
        tc_fence_after();
        if (f == 0) {
#pragma unroll
          for (int h = 0; h < 4; ++h) sp[h] = ldexpf(1.f, -plane_exp(zw[h]) - tab_exp);  // 2^-(p + tab_exp)
        }
        const uint32_t tb = trow + (uint32_t)f * 2 * NB;
        float2* out = a.scratch + a.s1 + xo + (size_t)f * fo;
        for (int n0 = colh * kCols; n0 < (colh + 1) * kCols; n0 += 16) {
          float re[16], im[16];
          tmem_ld16(tb + (uint32_t)n0, re);
          tmem_ld16(tb + NB + (uint32_t)n0, im);
          tmem_wait_ld();
          // the 16 columns' factors (whole warp, before the per-lane exit)
          const float spn = n0 < 64 ? (n0 < 32 ? sp[0] : sp[1]) : (n0 < 96 ? sp[2] : sp[3]);
          float spq[16];
#pragma unroll
          for (int q = 0; q < 16; ++q) spq[q] = __shfl_sync(0xffffffffu, spn, (n0 + q) & 31);
          if (xv >= a.S) continue;
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int wl = wl0 + n0 + q;
            if (wl >= a.c) break;
            __stcg(out + (size_t)wl * a.per, make_float2(re[q] * spq[q], im[q] * spq[q]));
          }
        }
        // accumulators f are free for the next item
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(tempty + f);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(4 * NB));
  }
}

// g_{G,ky}[d] for d = -e .. e from the engine-layout spectra (FP32 values,
// FP64 sums): gbuf[(f * M + ky) * (2e+1) + d + e].
__global__ void k_hyb_g(const float2* __restrict__ Gx, const float2* __restrict__ Gy, int e,
                        const double2* __restrict__ tab, double2* __restrict__ gbuf) {
  const int KW = 2 * e + 1;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 2 * M * KW) return;
  const int f = idx / (M * KW), rem = idx - f * M * KW;
  const int ky = rem / KW, d = rem - (rem / KW) * KW - e;
  const float2* G = (f == 0 ? Gx : Gy) + (size_t)ky * M;
  double re = 0.0, im = 0.0;
  for (int kx = 0; kx < M; ++kx) {
    const float2 v = G[kx];
    int m = (d * kx) % M;
    if (m < 0) m += M;
    const double2 w = tab[m];  // (cos, sin)(2 pi m / M): exp(+i ...)
    re += (double)v.x * w.x - (double)v.y * w.y;
    im += (double)v.x * w.y + (double)v.y * w.x;
  }
  gbuf[idx] = make_double2(re, im);
}

// Power of two with 2^exp * max|g| in [8, 16).  One block.
__global__ void k_hyb_scale(const double2* __restrict__ gbuf, int n, int* __restrict__ exp_out) {
  __shared__ double red[256];
  double mx = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) mx = fmax(mx, fmax(fabs(gbuf[i].x), fabs(gbuf[i].y)));
  red[threadIdx.x] = mx;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int e2 = 0;
    if (red[0] > 0.0) {
      frexp(red[0], &e2);
      e2 = 4 - e2;
    }
    *exp_out = e2 < -60 ? -60 : (e2 > 60 ? 60 : e2);
  }
}

// tabs[ky][f][part][q][r][t] = part of g_{f,ky}[e - jj] * 2^exp, jj = 8q + r + t - 127
// (zero off the band).
__global__ void k_hyb_tabs(const double2* __restrict__ gbuf, const int* __restrict__ exp_in, int e,
                           uint16_t* __restrict__ tabs) {
  const int KW = 2 * e + 1, QS = qs_of(e);
  const long long total = (long long)M * 4 * QS * 64;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int w = (int)(idx % (QS * 64));
  const long long blk = idx / (QS * 64);  // ky * 4 + f * 2 + part
  const int part = (int)(blk & 1), f = (int)((blk >> 1) & 1), ky = (int)(blk >> 2);
  const int q = w / 64, r = (w / 8) % 8, t = w % 8;
  const int jj = 8 * q + r + t - (MT - 1);
  double v = 0.0;
  if (jj >= 0 && jj < KW) {
    const double2 gv = gbuf[((size_t)f * M + ky) * KW + (e - jj) + e];
    v = ldexp(part ? gv.y : gv.x, *exp_in);
  }
  tabs[idx] = __half_as_ushort(__double2half(v));
}

}  // namespace hyb

// ---- host side ------------------------------------------------------------------------------
bool tensor_rows_supported(const srk_plan_s* p, std::string* why) {
  char buf[160];
  if (p->dtype == SRK_F32) snprintf(buf, sizeof buf, "needs FP16 or BF16 storage (FP16 operands)");
  else if (p->M != hyb::M) snprintf(buf, sizeof buf, "needs tile M = 512 (plan has %d)", p->M);
  else if (p->e < 1 || p->e > hyb::kMaxE) snprintf(buf, sizeof buf, "needs 1 <= erosion <= %d", hyb::kMaxE);
  else return true;
  if (why) *why = buf;
  return false;
}

size_t tensor_rows_tab_bytes(const srk_plan_s* p) { return (size_t)hyb::M * 4 * hyb::qs_of(p->e) * 128; }
size_t tensor_rows_g_bytes(const srk_plan_s* p) { return sizeof(double2) * 2 * hyb::M * (2 * p->e + 1); }

// Band tables from the plan's engine-layout spectra (stream-ordered).
srk_status tensor_rows_build_tables(srk_plan_s* p, cudaStream_t s) {
  const int KW = 2 * p->e + 1;
  const int n = 2 * hyb::M * KW;
  int* exp_slot = reinterpret_cast<int*>(p->direct_err + 2);
  hyb::k_hyb_g<<<(n + 127) / 128, 128, 0, s>>>(p->G[0], p->G[1], p->e, p->imp_tab, p->hyb_g);
  hyb::k_hyb_scale<<<1, 256, 0, s>>>(p->hyb_g, n, exp_slot);
  const long long total = (long long)hyb::M * 4 * hyb::qs_of(p->e) * 64;
  hyb::k_hyb_tabs<<<(int)((total + 255) / 256), 256, 0, s>>>(p->hyb_g, exp_slot, p->e, p->hyb_tabs);
  return cuda_status(cudaGetLastError(), "tensor-row tables");
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn_h() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }
  return fn;
}
}  // namespace

// The column-DFT tables of k_p1g (C and S rows of both parities over y < M/2,
// 256 KB), in the plan's storage type.
size_t tensor_rows_p1g_tab_bytes() { return (size_t)2 * (p1g::M / 2) * (p1g::M / 2) * 2; }
srk_status tensor_rows_p1g_tables(srk_plan_s* p, cudaStream_t s) {
  const int n = 2 * (p1g::M / 2) * (p1g::M / 2);
  if (p->dtype == SRK_BF16)
    p1g::k_p1g_tables<__nv_bfloat16><<<(n + 255) / 256, 256, 0, s>>>(static_cast<__nv_bfloat16*>(p->p1g_tab));
  else
    p1g::k_p1g_tables<__half><<<(n + 255) / 256, 256, 0, s>>>(static_cast<__half*>(p->p1g_tab));
  return cuda_status(cudaGetLastError(), "column-DFT tables");
}

// Tensor maps of k_p1g: the tables (box 64 y x 128 rows) and the images
// ([nimg][N][N] column-major, box 64 y x 64 x x 1), both with the 128-byte
// swizzle.  The caller checks N % 8 == 0 and a 16-byte aligned image array.
srk_status tensor_rows_p1g_maps(const srk_plan_s* p, const void* img, int N, int nimg, CUtensorMap* tmap,
                                CUtensorMap* smap) {
  auto enc = encode_fn_h();
  if (!enc) return fail(SRK_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is unavailable");
  const CUtensorMapDataType dt = p->dtype == SRK_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
  {
    std::memset(tmap, 0, sizeof(*tmap));
    const cuuint64_t dims[2] = {(cuuint64_t)p1g::M / 2, (cuuint64_t)p1g::M};
    const cuuint64_t strides[1] = {(cuuint64_t)p1g::M / 2 * 2};
    const cuuint32_t box[2] = {64, (cuuint32_t)p1g::KR};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(tmap, dt, 2, p->p1g_tab, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(SRK_ERR_CUDA, "cuTensorMapEncodeTiled (DFT tables) failed (%d)", (int)r);
  }
  {
    std::memset(smap, 0, sizeof(CUtensorMap));
    const cuuint64_t dims[3] = {(cuuint64_t)N, (cuuint64_t)N, (cuuint64_t)nimg};
    const cuuint64_t strides[2] = {(cuuint64_t)N * 2, (cuuint64_t)N * N * 2};
    const cuuint32_t box[3] = {64, (cuuint32_t)p1g::XB, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(smap, dt, 3, const_cast<void*>(img), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(SRK_ERR_CUDA, "cuTensorMapEncodeTiled (images) failed (%d)", (int)r);
  }
  return SRK_OK;
}

// The planes [2M][c][M] as [ky][part][wl][x] for k_p1g's stores: box {64 x,
// 1 work tile, 2 parts, 256 ky traversed with stride 2} = 128 rows of one ky
// parity, 128-byte swizzle.
srk_status tensor_rows_p1g_store_map(const __half* planes, int c, CUtensorMap* out) {
  auto enc = encode_fn_h();
  if (!enc) return fail(SRK_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is unavailable");
  std::memset(out, 0, sizeof(*out));
  const cuuint64_t dims[4] = {(cuuint64_t)p1g::M, (cuuint64_t)c, 2, (cuuint64_t)p1g::M};
  const cuuint64_t strides[3] = {(cuuint64_t)p1g::M * 2, (cuuint64_t)c * p1g::M * 2, (cuuint64_t)2 * c * p1g::M * 2};
  const cuuint32_t box[4] = {(cuuint32_t)p1g::XB, 1, 2, 2 * p1g::KR};
  const cuuint32_t estr[4] = {1, 1, 1, 2};
  const CUresult r = enc(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 4, const_cast<__half*>(planes), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? SRK_OK : fail(SRK_ERR_CUDA, "cuTensorMapEncodeTiled (plane stores) failed (%d)", (int)r);
}

srk_status tensor_rows_plane_map(const __half* planes, int c, unsigned box_x, unsigned box_w, unsigned box_p,
                                 CUtensorMap* out, bool swizzle128) {
  auto enc = encode_fn_h();
  if (!enc) return fail(SRK_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is unavailable");
  std::memset(out, 0, sizeof(*out));
  const cuuint64_t dims[3] = {(cuuint64_t)hyb::M, (cuuint64_t)c, (cuuint64_t)(2 * hyb::M)};
  const cuuint64_t strides[2] = {(cuuint64_t)hyb::M * 2, (cuuint64_t)c * hyb::M * 2};
  const cuuint32_t box[3] = {box_x, box_w, box_p};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, const_cast<__half*>(planes), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE,
                         swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? SRK_OK : fail(SRK_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
}

// The row pass of one chunk of c work tiles: planes [2M][c][M] FP16 (k_p1h,
// work tile wl scaled by 2^plane_exp(mx[wl])) -> S2 of every work tile at
// scratch + wl*per + s1 (P3's layout).
srk_status tensor_rows_p2(srk_plan_s* p, const __half* planes, const unsigned int* mx, int c, float2* scratch,
                          size_t per, size_t s1, int S, int P, cudaStream_t s) {
  CUtensorMap map;
  SRK_TRY(tensor_rows_plane_map(planes, c, 64, hyb::NB, 1, &map, true));
  hyb::Args a;
  a.tabs = p->hyb_tabs;
  a.tab_exp = reinterpret_cast<const int*>(p->direct_err + 2);
  a.mx = mx;
  a.scratch = scratch;
  a.per = per;
  a.s1 = s1;
  a.err = p->direct_err;
  a.spin_limit = 1ull << 22;
  a.c = c;
  a.e = p->e;
  a.S = S;
  a.P = P;
  const size_t sm = hyb::smem_bytes(p->e);
  SRK_CUDA(cudaFuncSetAttribute(hyb::k_p2h, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const long long items = (long long)((S + hyb::MT - 1) / hyb::MT) * hyb::M * ((c + hyb::NB - 1) / hyb::NB);
  const int grid = (int)std::min<long long>(items, p->nsm > 0 ? p->nsm : 148);
  hyb::k_p2h<<<grid, hyb::kThreadsH, sm, s>>>(map, a);
  return cuda_status(cudaGetLastError(), "tensor-row pass launch");
}

}  // namespace srk
