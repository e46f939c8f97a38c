// direct.cu — the small-KW forward as a direct convolution on the
// 5th-generation tensor cores (tcgen05.mma, accumulators in TMEM, operands
// staged by TMA and bulk copies).
//
// u_x(x', y') = sum_{i,j} E(x'+i, y'+j) Kf_x(i, j),  Kf(i, j) = K(KW-1-i, KW-1-j)
// (the true convolution of the reference, u[o] = sum_d E[o+e-d] G[c+d],
// adjoint/main_adjoint.cu:70-90), and u_y likewise, then
// R = dx^2 (u_x dI/dx + u_y dI/dy) with the central differences of
// srk_forward.cuh:429-445 — the same result as srkTrainingForward
// (training/srk_training_forward.cuh:175-241) and srkCudnnForward
// (training/srk_cudnn_forward.cuh:194-269), computed without FFTs.
//
// GEMM form (one CTA per output tile of MT = 128 rows y' x NT = 128 columns x'):
//   D[m][n] = sum_i sum_k A_i[m][k] B_i[k][n],  B_i[k][n] = E(x0+n+i, y0+k),
//   A_i[m][k] = Kf(i, k-m) for 0 <= k-m < KW (a band: Toeplitz in (m, k)).
// * B_i for every i comes from ONE shared-memory tile of the image: the
//   K-major operand (rows n = image columns, 16-byte chunks of 8 image rows)
//   of kernel column i is the same tile with its start moved by i rows
//   (16 bytes): the image window is staged once per output tile.
// * A_i is never materialised: with the rows in reverse order (lane m' holds
//   output row y0 + 127 - m') the 16-byte chunk (m', C) of the band holds
//   Kf(i, 8(C + g') + r' + t - 127), t < 8, m' = 8 g' + r' — a function of
//   (C + g', r') only.  So a descriptor with leading and stride byte offsets
//   both equal to 128 bytes reads the whole band from QS = KT/8 + 16 slots of
//   8 x 16 bytes: 4.6 KB per kernel column instead of 40 KB.
// * FP16/BF16 storage: one MMA pass (kind::f16, A and B of the storage type,
//   FP32 accumulation).  FP32 storage: three passes over an exact split
//   x = hi + lo into FP16 halves (A_hi B_hi + A_hi B_lo + A_lo B_hi), ~22-bit
//   products with FP32 accumulation.
//
// Roles (192 threads): warps 0-3 run the epilogue (TMEM lanes 32w..32w+31),
// warp 4 streams the band tables through a ring of NST stages (bulk copies
// completing on mbarriers) after issuing the image window (TMA, FP16/BF16)
// and warp 5 owns the TMEM allocation and issues the MMAs from one thread.
// Every wait is bounded: on expiry the kernel records the site in a
// plan-owned error word, stops issuing, and still frees its TMEM.
//
// The FFT overlap-and-save path does the same work in O(log M) per output
// pixel; this path does (MT + KW - 1) * KW * 2 multiply-adds per pixel on the
// tensor pipe, so it only pays for small kernels (the tuner times both).
#include <cuda.h>
#include <cudaTypedefs.h>

#include "internal.h"
#include "tc.cuh"

using namespace srk;

namespace srk {
namespace direct {
using namespace srk::tc;

constexpr int MT = 128;     // output rows per tile = TMEM lanes
constexpr int NT = 128;     // output columns per tile (MMA N)
constexpr int NST = 4;      // band-table stages in flight
constexpr int kThreadsD = 192;
constexpr int kMaxKW = 63;

__host__ __device__ constexpr int kt_of(int KW) { return ((MT + KW - 1) + 15) / 16 * 16; }  // K extent (image rows)
__host__ __device__ constexpr int nr_of(int KW) { return ((NT + KW - 1) + 7) / 8 * 8; }     // image columns staged
__host__ __device__ constexpr int qs_of(int KW) { return kt_of(KW) / 8 + MT / 8; }           // band slots

template <typename T> struct OperandOf { using type = __half; static constexpr int fmt = 0; };
template <> struct OperandOf<__nv_bfloat16> { using type = __nv_bfloat16; static constexpr int fmt = 1; };
template <typename T> constexpr int npass_of() { return std::is_same<T, float>::value ? 3 : 1; }
template <typename T> constexpr int nsplit_of() { return std::is_same<T, float>::value ? 2 : 1; }

struct Args {
  const void* E;            // convolved image(s)  [B][N][N]
  const void* I;            // differentiated image(s)
  void* R;                  // [B][W][W]
  const uint16_t* tabs;     // band tables [KW][2][NSPLIT][QS][8][8] operand values
  unsigned int* err;        // error word (0 = ok, else 1 + wait site)
  const int* tab_exp;       // the band tables hold K * 2^tab_exp (K scaled into [8, 16))
  unsigned long long spin_limit;
  int N, W, e, KW;
  int tiles_x, tiles_y;     // per image
  float scale;              // 0.5 * dx^2 (central differences' 1/2 folded in)
};

// ---- the kernel -------------------------------------------------------------------------
// Dynamic shared memory: [0, 128) mbarriers and the TMEM address; B tile(s)
// from byte 1024; the NST band stages after them.
template <typename T>
__global__ void __launch_bounds__(kThreadsD, 1) k_direct(const __grid_constant__ CUtensorMap tmap, Args a) {
  using OT = typename OperandOf<T>::type;
  constexpr int NPASS = npass_of<T>();
  constexpr int NSPLIT = nsplit_of<T>();
  constexpr bool TMA = !std::is_same<T, float>::value;
  extern __shared__ __align__(1024) unsigned char smem[];
  const int KW = a.KW, KT = kt_of(KW), KC = KT / 8, NR = nr_of(KW), QS = qs_of(KW);
  const uint32_t lboB = (uint32_t)NR * 16;                 // bytes between 8-row chunks of B
  const uint32_t bbytes = (uint32_t)KC * lboB;             // one B copy
  const uint32_t tab_bytes = (uint32_t)QS * 128;           // one (kernel, split) band
  const uint32_t stage_bytes = 2u * NSPLIT * tab_bytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);      // [NST]
  uint64_t* empty = full + NST;                            // [NST]
  uint64_t* bfull = empty + NST;
  uint64_t* accfull = bfull + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accfull + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  unsigned char* Bs = smem + 1024;
  unsigned char* As = Bs + ((NSPLIT * bbytes + 1023) & ~1023u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  const int per_img = a.tiles_x * a.tiles_y;
  const int b = blockIdx.x / per_img;
  const int rt = blockIdx.x - b * per_img;
  const int x0 = (rt / a.tiles_y) * NT;
  const int y0 = (rt - (rt / a.tiles_y) * a.tiles_y) * MT;
  const long long on = (long long)b * a.N * a.N;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(bfull, 1);
    mbar_init(accfull, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * NT));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if constexpr (!TMA) {
    // FP32 storage: every thread stages hi / lo chunks of the image window
    // (row n = image column x0 + n, chunk c = image rows y0 + 8c ..), zero
    // outside the image; a warp writes 32 consecutive rows of one chunk.
    const float* E = static_cast<const float*>(a.E) + on;
    for (int idx = threadIdx.x; idx < KC * NR; idx += kThreadsD) {
      const int c = idx / NR, n = idx - (idx / NR) * NR;
      const int gx = x0 + n, gy = y0 + 8 * c;
      float v[8];
      if (gx < a.N && gy + 8 <= a.N) {
        const float4* p = reinterpret_cast<const float4*>(E + (long long)gx * a.N + gy);
        const float4 q0 = __ldg(p), q1 = __ldg(p + 1);
        v[0] = q0.x; v[1] = q0.y; v[2] = q0.z; v[3] = q0.w; v[4] = q1.x; v[5] = q1.y; v[6] = q1.z; v[7] = q1.w;
      } else {
#pragma unroll
        for (int t = 0; t < 8; ++t) v[t] = (gx < a.N && gy + t < a.N) ? __ldg(E + (long long)gx * a.N + gy + t) : 0.f;
      }
      __align__(16) __half hi[8], lo[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) split_half(v[t], hi[t], lo[t]);
      const uint32_t off = (uint32_t)c * lboB + (uint32_t)n * 16;
      *reinterpret_cast<uint4*>(Bs + off) = *reinterpret_cast<const uint4*>(hi);
      *reinterpret_cast<uint4*>(Bs + bbytes + off) = *reinterpret_cast<const uint4*>(lo);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const unsigned long long lim = a.spin_limit;

  if (warp == 4) {
    if (lane == 0) {
      if constexpr (TMA) {
        mbar_expect_tx(bfull, bbytes);
        for (int c = 0; c < KC; ++c) tma_load_3d(Bs + (size_t)c * lboB, &tmap, y0 + 8 * c, x0, b, bfull);
      }
      const unsigned char* src = reinterpret_cast<const unsigned char*>(a.tabs);
      int issued = 0;
      for (int i = 0; i < KW; ++i) {
        const int s = i % NST;
        if (i >= NST && !mbar_wait(empty + s, (unsigned)((i / NST - 1) & 1), lim)) {
          atomicCAS(a.err, 0u, 1u);
          *abort_flag = 1;
          break;
        }
        if (*abort_flag) break;
        mbar_expect_tx(full + s, stage_bytes);
        bulk_g2s(As + (size_t)s * stage_bytes, src + (size_t)i * stage_bytes, stage_bytes, full + s);
        ++issued;
      }
      if (*abort_flag) {
        // let the copies still in flight land before the CTA releases its shared memory
        for (int j = issued > NST ? issued - NST : 0; j < issued; ++j) mbar_wait(full + j % NST, (unsigned)((j / NST) & 1), lim);
        if constexpr (TMA) mbar_wait(bfull, 0, lim);
      }
    }
    __syncwarp();
  } else if (warp == 5) {
    if (lane == 0) {
      const uint32_t idesc = idesc_f16(OperandOf<T>::fmt, MT, NT);
      const uint32_t b_base = smem_u32(Bs), a_base = smem_u32(As);
      bool ok = true;
      if constexpr (TMA) ok = mbar_wait(bfull, 0, lim);
      if (!ok) {
        atomicCAS(a.err, 0u, 2u);
        *abort_flag = 1;
      }
      for (int i = 0; ok && i < KW; ++i) {
        const int s = i % NST;
        if (!mbar_wait(full + s, (unsigned)((i / NST) & 1), lim)) {
          atomicCAS(a.err, 0u, 3u);
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t st = a_base + (uint32_t)s * stage_bytes;
        for (int ks = 0; ks < KT / 16; ++ks) {
#pragma unroll
          for (int p = 0; p < NPASS; ++p) {
            const int pa = (p == 2), pb = (p == 1);  // (hi,hi), (hi,lo), (lo,hi)
            const uint64_t db = sdesc(b_base + (uint32_t)pb * bbytes + (uint32_t)i * 16 + (uint32_t)ks * 2 * lboB,
                                      lboB, 128);
#pragma unroll
            for (int kern = 0; kern < 2; ++kern) {
              const uint64_t da =
                  sdesc(st + (uint32_t)(kern * NSPLIT + pa) * tab_bytes + (uint32_t)ks * 256, 128, 128);
              mma_f16(tmem + (uint32_t)(kern * NT), da, db, idesc, (i | ks | p) != 0);
            }
          }
        }
        mma_commit(empty + s);  // the stage is free once these MMAs have read it
      }
      mma_commit(accfull);
    }
    __syncwarp();
  } else {
    // epilogue: lane quarter `warp` of the accumulators
    bool ok = true;
    if (lane == 0) ok = mbar_wait(accfull, 0, lim);
    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    if (!ok && lane == 0) atomicCAS(a.err, 0u, 4u);
    if (ok && !*abort_flag) {
      tc_fence_after();
      const int mrow = warp * 32 + lane;              // TMEM lane
      const int yo = y0 + MT - 1 - mrow;              // output row (rows stored in reverse)
      const T* I = static_cast<const T*>(a.I) + on;
      T* R = static_cast<T*>(a.R) + (long long)b * a.W * a.W;
      const int N = a.N, e = a.e;
      const float scale = ldexpf(a.scale, -__ldg(a.tab_exp));  // undo the tables' power-of-two scaling (exact)
      const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
      for (int c0 = 0; c0 < NT; c0 += 16) {
        float ux[16], uy[16];
        tmem_ld16(trow + (uint32_t)c0, ux);
        tmem_ld16(trow + (uint32_t)(NT + c0), uy);
        tmem_wait_ld();
        if (yo >= a.W) continue;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int xo = x0 + c0 + k;
          if (xo >= a.W) break;
          const long long ci = (long long)(xo + e) * N + yo + e;
          const float fx = ldf(I, ci + N) - ldf(I, ci - N);
          const float fy = ldf(I, ci + 1) - ldf(I, ci - 1);
          stf(R, (long long)xo * a.W + yo, dot2(ux[k], fx, uy[k], fy) * scale);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 5) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * NT));
  }
}

// Band tables from the FP64 spatial kernel Kd (column-major KW x KW):
// tab[i][kern][split][q][r][t] = Kf(i, 8q + r + t - 127) (zero off the band),
// Kf(i, j) = K(KW-1-i, KW-1-j); split 0 = the operand-type value, split 1 =
// the FP16 remainder (FP32 storage only).
// Power-of-two scale of both kernels' band tables: 2^exp * max|K| in [8, 16)
// (FP16 keeps every small tap a normal number; exact to undo).  One block.
__global__ void k_direct_scale(const double* __restrict__ kx, const double* __restrict__ ky, int n, int* __restrict__ exp_out) {
  __shared__ double red[256];
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fmax(fabs(kx[i]), fabs(ky[i])));
  red[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int e2 = 0;
    if (red[0] > 0.0) {
      frexp(red[0], &e2);   // max = f * 2^e2, f in [0.5, 1)
      e2 = 4 - e2;          // max * 2^(4 - e2) in [8, 16)
    }
    *exp_out = e2 < -60 ? -60 : (e2 > 60 ? 60 : e2);
  }
}

template <typename OT>
__global__ void k_direct_tables(const double* __restrict__ Kd, const int* __restrict__ exp_in, int KW, int kern,
                                int nsplit, uint16_t* __restrict__ tab) {
  const int QS = qs_of(KW);
  const int per = QS * 64;  // values per (kernel, split) band
  const long long total = (long long)KW * nsplit * per;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int i = (int)(idx / ((long long)nsplit * per));
  const int rem = (int)(idx - (long long)i * nsplit * per);
  const int split = rem / per, w = rem - (rem / per) * per;
  const int q = w / 64, r = (w / 8) % 8, t = w % 8;
  const int j = 8 * q + r + t - (MT - 1);
  double v = 0.0;
  if (j >= 0 && j < KW) v = ldexp(Kd[(long long)(KW - 1 - i) * KW + (KW - 1 - j)], *exp_in);
  uint16_t bits;
  if constexpr (std::is_same<OT, __half>::value) {
    const __half hi = __double2half(v);
    const __half out = split == 0 ? hi : __double2half(v - (double)__half2float(hi));
    bits = __half_as_ushort(out);
  } else {
    bits = __bfloat16_as_ushort(__double2bfloat16(v));
  }
  tab[(((long long)i * 2 + kern) * nsplit + split) * per + w] = bits;
}

}  // namespace direct
}  // namespace srk

// ---- host side ------------------------------------------------------------------------------
namespace srk {

bool direct_supported(const srk_plan_s* p, int N, std::string* why) {
  const int KW = 2 * p->e + 1;
  char buf[160];
  if (p->e < 1) snprintf(buf, sizeof buf, "needs erosion >= 1 (got %d)", p->e);
  else if (KW > direct::kMaxKW) snprintf(buf, sizeof buf, "kernel width %d > %d", KW, direct::kMaxKW);
  else if (N % 8) snprintf(buf, sizeof buf, "needs N %% 8 == 0 (got N=%d)", N);
  else return true;
  if (why) *why = buf;
  return false;
}

size_t direct_tab_bytes(const srk_plan_s* p) {
  const int KW = 2 * p->e + 1;
  const int nsplit = p->dtype == SRK_F32 ? 2 : 1;
  return (size_t)KW * 2 * nsplit * direct::qs_of(KW) * 128;
}

// Band tables of one kernel (kern 0 = Gx, 1 = Gy) from the plan's FP64
// spatial kernel in imp_Kd (stream-ordered, no allocation).
srk_status direct_build_tables(srk_plan_s* p, int kern, cudaStream_t s) {
  const int KW = 2 * p->e + 1;
  const int nsplit = p->dtype == SRK_F32 ? 2 : 1;
  const long long total = (long long)KW * nsplit * direct::qs_of(KW) * 64;
  const int blocks = (int)((total + 255) / 256);
  int* exp_slot = reinterpret_cast<int*>(p->direct_err + 1);
  if (kern == 0) direct::k_direct_scale<<<1, 256, 0, s>>>(p->kd[0], p->kd[1], KW * KW, exp_slot);
  if (p->dtype == SRK_BF16)
    direct::k_direct_tables<__nv_bfloat16><<<blocks, 256, 0, s>>>(p->kd[kern], exp_slot, KW, kern, nsplit,
                                                                   p->direct_tabs);
  else
    direct::k_direct_tables<__half><<<blocks, 256, 0, s>>>(p->kd[kern], exp_slot, KW, kern, nsplit, p->direct_tabs);
  return cuda_status(cudaGetLastError(), "direct band tables");
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
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

template <typename T>
size_t direct_smem(int KW) {
  const size_t bbytes = (size_t)(direct::kt_of(KW) / 8) * direct::nr_of(KW) * 16;
  const size_t stage = 2u * direct::nsplit_of<T>() * direct::qs_of(KW) * 128;
  const size_t need = 1024 + ((direct::nsplit_of<T>() * bbytes + 1023) & ~(size_t)1023) + direct::NST * stage;
  // at least 80 KB: at most two CTAs share an SM, so their two TMEM
  // allocations (256 columns each) always fit the SM's 512 columns
  return need > (80u << 10) ? need : (80u << 10);
}

template <typename T>
srk_status direct_launch(srk_plan_s* p, const void* E, const void* I, void* R, int B, cudaStream_t s) {
  const int KW = 2 * p->e + 1;
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  if constexpr (!std::is_same<T, float>::value) {
    auto enc = encode_fn();
    if (!enc) return fail(SRK_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is unavailable");
    if (reinterpret_cast<uintptr_t>(E) & 15) return fail(SRK_ERR_INVALID_ARG, "E must be 16-byte aligned");
    const cuuint64_t dims[3] = {(cuuint64_t)p->N, (cuuint64_t)p->N, (cuuint64_t)B};
    const cuuint64_t strides[2] = {(cuuint64_t)p->N * sizeof(T), (cuuint64_t)p->N * p->N * sizeof(T)};
    const cuuint32_t box[3] = {8, (cuuint32_t)direct::nr_of(KW), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(&map, std::is_same<T, __half>::value ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                                : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16,
                           3, const_cast<void*>(E), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(SRK_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  }
  direct::Args a;
  a.E = E; a.I = I; a.R = R;
  a.tabs = p->direct_tabs;
  a.err = p->direct_err;
  a.tab_exp = reinterpret_cast<const int*>(p->direct_err + 1);
  a.spin_limit = 1ull << 22;
  a.N = p->N; a.W = p->W; a.e = p->e; a.KW = KW;
  a.tiles_x = (p->W + direct::NT - 1) / direct::NT;
  a.tiles_y = (p->W + direct::MT - 1) / direct::MT;
  a.scale = 0.5f * p->dx * p->dx;
  const size_t sm = direct_smem<T>(KW);
  SRK_CUDA(cudaFuncSetAttribute(direct::k_direct<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const long long grid = (long long)B * a.tiles_x * a.tiles_y;
  if (grid > 0x7fffffffLL) return fail(SRK_ERR_UNSUPPORTED, "too many direct tiles");
  direct::k_direct<T><<<(unsigned)grid, direct::kThreadsD, sm, s>>>(map, a);
  p->last_launches = 1;
  return cuda_status(cudaGetLastError(), "direct launch");
}

}  // namespace

// The training forward (E, I: [B][N][N]) on the direct path.
srk_status direct_forward(srk_plan_s* p, const void* E, const void* I, void* R, int B, cudaStream_t s) {
  std::string why;
  if (!direct_supported(p, p->N, &why)) return fail(SRK_ERR_UNSUPPORTED, "direct schedule: %s", why.c_str());
  if (!p->direct_tabs || !p->direct_ready) return fail(SRK_ERR_INVALID_ARG, "direct schedule: no kernel bound");
  switch (p->dtype) {
    case SRK_F32: return direct_launch<float>(p, E, I, R, B, s);
    case SRK_F16: return direct_launch<__half>(p, E, I, R, B, s);
    case SRK_BF16: return direct_launch<__nv_bfloat16>(p, E, I, R, B, s);
  }
  return fail(SRK_ERR_UNSUPPORTED, "dtype %d", (int)p->dtype);
}

}  // namespace srk
