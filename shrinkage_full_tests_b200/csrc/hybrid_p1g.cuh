// hybrid_p1g.cuh — the column pass of SRK_SCHEDULE_TENSOR_ROWS as a DFT on
// the 5th-generation tensor cores, for uniform batches of FP16/BF16 images.
//
// The column transform of a work tile is Z[ky][x] = sum_y W^(ky y) z[y][x],
// W = exp(-2 pi i / M), z = a + i b (a, b: the work tile's two real source
// tiles, the two images of a pair).  Because a and b are
// real, A = DFT(a) and B = DFT(b) are Hermitian in ky and
//   Z[ky]     = (Re A - Im B) + i (Im A + Re B)
//   Z[M - ky] = (Re A + Im B) + i (Re B - Im A),
// so ky = 0 .. M/2 - 1 give every row but the Nyquist row M/2.  Per item
// (128 ky rows, 64 columns x of both sources) two real GEMMs with K = y:
//   Dr = C  [a | b],   C[ky][y]  = cos(2 pi ky y / M)
//   Di = S  [a | b],   S[ky][y]  = -sin(2 pi ky y / M)
// (N = 128: 64 columns of a, then the same 64 of b).  The row ky = 0 of S is
// zero; the table holds the Nyquist row (-1)^y there instead, so that lane
// also yields Re A[M/2], Re B[M/2] (Im of both is zero at ky = 0 and M/2).
// The tables and images are FP16 (or BF16 for BF16 storage) operands with
// FP32 accumulation: the planes are FP16 anyway.
//
// Data movement: the tables (128 ky x 64 y boxes) and the source tiles
// (64 x x 64 y boxes, the images' own column-major layout is the K-major
// operand) by TMA with the 128-byte swizzle through a ring of stages; the
// planes leave through shared memory by TMA stores of 256 plane rows x 64
// columns (128-byte rows), the Nyquist row by the threads.
// Used with tile origins on 8-row boundaries (TMA's innermost coordinate):
// one tile per image, or a tile stride that is a multiple of 8.  The tables'
// FP16 rounding adds an error relative to the larger image of the pair, of
// the order of the planes' own rounding.
#pragma once
#include <cuda.h>

#include "engine.cuh"
#include "tc.cuh"

namespace srk {
namespace p1g {
using namespace srk::tc;

constexpr int M = 512;
constexpr int KR = 128;                  // ky rows per item (TMEM lanes)
constexpr int XB = 64;                   // columns x per item and source
constexpr int NA = M / 64;               // K atoms of 64 rows y
// Staging buffers (1: one pair of blocks, each item waits for the previous
// item's stores to read it; 2: one pair per item parity, with a ring of 2
// stages to fit), epilogue warps (4 or 8: one or two per TMEM lane quarter).
// Measured (B = 5000 FP16 step): 1 / 4 8.50 ms, 1 / 8 8.50 ms, 2 / 8 8.81 ms
// (two stages starve the MMAs).
#ifndef SRK_P1G_STAGING
#define SRK_P1G_STAGING 1
#endif
#ifndef SRK_P1G_EPI
#define SRK_P1G_EPI 4
#endif
constexpr int kStagings = SRK_P1G_STAGING;
constexpr int NSG = kStagings == 2 ? 2 : 3;  // ring stages (one atom each)
constexpr int kEpi = SRK_P1G_EPI;
static_assert((kEpi == 4 || kEpi == 8) && XB == 64 && (kStagings == 1 || kStagings == 2), "configuration");
constexpr int kColsW = XB / (kEpi / 4);  // columns of each source per epilogue warp
constexpr int kThreadsG = 32 * (kEpi + 2);
constexpr int kLoadWarp = kEpi, kMmaWarp = kEpi + 1;
constexpr uint32_t kTabBox = KR * 128;   // 128 table rows x 64 y, 16 KB
constexpr uint32_t kSrcBox = XB * 128;   // 64 columns x 64 y, 8 KB
constexpr uint32_t kStage = 2 * kTabBox + 2 * kSrcBox;
constexpr uint32_t kStaging = 256 * 128;  // 256 plane rows x 64 FP16 columns
// barriers | NSG stages | staging (per buffer: rows ky, rows M - ky)
__host__ __device__ constexpr size_t smem_bytes() {
  return 1024 + (size_t)NSG * kStage + 2 * (size_t)kStagings * kStaging;
}

struct Args {
  __half* planes;            // the chunk's planes [2M][c][M] (the Nyquist row is stored directly)
  unsigned int* zmax;        // largest |Z| per work tile (float bits, zeroed before the launch)
  unsigned int* err;         // plan error word
  unsigned long long spin_limit;
  Geom g;                    // tile geometry (uniform batch)
  int w0, c;                 // first work tile and work tiles of the chunk
  int nimg;                  // images in the image map (a coordinate there reads zeros)
};

// C and S tables (rows part * 256 + ky, ky < 256; columns y < M), in the
// storage type's 16-bit format.
template <typename T>
__global__ void k_p1g_tables(T* __restrict__ tab) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 2 * (M / 2) * M) return;
  const int y = idx % M, row = idx / M, part = row / (M / 2), ky = row % (M / 2);
  const int m = (ky * y) % M;
  double s, c;
  sincospi(2.0 * m / M, &s, &c);
  double v = part == 0 ? c : -s;
  if (part == 1 && ky == 0) v = (y & 1) ? -1.0 : 1.0;  // the Nyquist row
  tab[idx] = T(static_cast<float>(v));
}

__device__ __forceinline__ void mbar_arrive_g(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
// Position of 16-byte chunk `ch` of row `row` in a 128-byte-swizzled block.
__device__ __forceinline__ uint32_t sw128(uint32_t row, uint32_t ch) { return row * 128 + ((ch ^ (row & 7)) << 4); }
// Two FP16 plane values in one word (x at the lower address).
__device__ __forceinline__ uint32_t pack_h2(float x, float y) {
  const __half2 h = __floats2half2_rn(x, y);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// Persistent, one CTA per SM; an item is (work tile wl, column block xb,
// ky block kt) with kt fastest (both ky blocks read the same source boxes).
//   full[s] / empty[s]: ring stage s loaded (TMA bytes) / read by the MMAs (commit)
//   tfull[t] / tempty[t]: accumulator set t complete (commit) / drained (epilogue warps)
template <typename T>
__global__ void __launch_bounds__(kThreadsG, 1)
k_p1g(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap smap,
      const __grid_constant__ CUtensorMap pmap, Args a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);  // [NSG]
  uint64_t* empty = full + NSG;                        // [NSG]
  uint64_t* tfull = empty + NSG;                       // [2]
  uint64_t* tempty = tfull + 2;                        // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  volatile int* go = abort_flag + 1;                   // the epilogue's per-item decision
  unsigned char* St = smem + 1024;                     // NSG stages: C | S | source a | source b
  unsigned char* Sg = St + (size_t)NSG * kStage;       // staging [item parity][rows ky | rows M - ky]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int items = a.c * (M / XB) * 2;
  const unsigned long long lim = a.spin_limit;

  if (threadIdx.x == 0) {
    *abort_flag = (smem_u32(St) & 1023u) != 0;
    if (*abort_flag) atomicCAS(a.err, 0u, 19u);
    for (int i = 0; i < NSG; ++i) {
      mbar_init(full + i, 1);
      mbar_init(empty + i, 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(tfull + i, 1);
      mbar_init(tempty + i, kEpi);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  auto decode = [&](int item, int& wl, int& xb, int& kt) {
    kt = item & 1;
    xb = (item >> 1) % (M / XB);
    wl = (item >> 1) / (M / XB);
  };

  if (warp == kLoadWarp) {
    if (lane == 0) {
      long long q = 0;  // atoms issued
      for (int item = blockIdx.x; item < items && !*abort_flag; item += gridDim.x) {
        int wl, xb, kt;
        decode(item, wl, xb, kt);
        const int w = a.w0 + wl;
        const TileRef t0 = tile_of(a.g, 2 * w), t1 = tile_of(a.g, 2 * w + 1);
        // a tile that does not exist reads zeros (image index past the map)
        const int i0 = t0.live ? t0.b : a.nimg, i1 = t1.live ? t1.b : a.nimg;
        for (int at = 0; at < NA; ++at, ++q) {
          const int st = (int)(q % NSG);
          if (q >= NSG && !mbar_wait(empty + st, (unsigned)((q / NSG - 1) & 1), lim)) {
            atomicCAS(a.err, 0u, 16u);
            *abort_flag = 1;
            break;
          }
          unsigned char* S = St + (size_t)st * kStage;
          mbar_expect_tx(full + st, kStage);
          tma_load_2d(S, &tmap, 64 * at, kt * KR, full + st);                        // C rows
          tma_load_2d(S + kTabBox, &tmap, 64 * at, M / 2 + kt * KR, full + st);      // S rows
          tma_load_3d(S + 2 * kTabBox, &smap, t0.y0 + 64 * at, t0.x0 + XB * xb, i0, full + st);
          tma_load_3d(S + 2 * kTabBox + kSrcBox, &smap, t1.y0 + 64 * at, t1.x0 + XB * xb, i1, full + st);
        }
      }
      for (long long r = q > NSG ? q - NSG : 0; r < q; ++r) mbar_wait(full + (int)(r % NSG), (unsigned)((r / NSG) & 1), lim);
    }
    __syncwarp();
  } else if (warp == kMmaWarp) {
    if (lane == 0) {
      constexpr int kFmt = std::is_same<T, __nv_bfloat16>::value ? 1 : 0;
      const uint32_t id = idesc_f16(kFmt, KR, 2 * XB);
      long long q = 0;
      bool ok = true;
      for (int k = 0, item = blockIdx.x; item < items && ok; ++k, item += gridDim.x) {
        const int t = k & 1;
        if (k >= 2 && !mbar_wait(tempty + t, (unsigned)((k / 2 - 1) & 1), lim)) ok = false;
        const uint32_t dr = tmem + (uint32_t)t * 256, di = dr + 128;
        for (int at = 0; at < NA && ok; ++at, ++q) {
          const int st = (int)(q % NSG);
          if (!mbar_wait(full + st, (unsigned)((q / NSG) & 1), lim) || *abort_flag) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t base = smem_u32(St + (size_t)st * kStage);
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const uint64_t dc = sdesc_sw128(base + (uint32_t)kk * 32);
            const uint64_t ds = sdesc_sw128(base + kTabBox + (uint32_t)kk * 32);
            const uint64_t db = sdesc_sw128(base + 2 * kTabBox + (uint32_t)kk * 32);
            mma_f16(dr, dc, db, id, (at | kk) != 0);
            mma_f16(di, ds, db, id, (at | kk) != 0);
          }
          mma_commit(empty + st);
        }
        if (ok) mma_commit(tfull + t);
      }
      if (!ok) {
        atomicCAS(a.err, 0u, 17u);
        *abort_flag = 1;
      }
    }
    __syncwarp();
  } else {
    // epilogue warp: TMEM lanes 32 (warp % 4) .. + 31 = rows r of the ky
    // block, columns kColsW (warp / 4) .. of each source
    const int quarter = warp & 3, colh = warp >> 2;
    const int r = quarter * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(quarter * 32) << 16);
    const uint32_t rk = 2 * r, rm = 2 * (KR - 1 - r);  // staging rows of ky and of M - ky (part 0; part 1 = +1)
    for (int k = 0, item = blockIdx.x; item < items; ++k, item += gridDim.x) {
      const int t = k & 1;
      int wl, xb, kt;
      decode(item, wl, xb, kt);
      // One thread decides for all epilogue warps, so that they leave together
      // (they meet at named barriers): the accumulators are complete and the
      // staging blocks free (the stores that last used them have read them).
      if (threadIdx.x == 0) {
        if (kStagings == 2)
          bulk_wait_read_but1();  // item k - 2 used this parity's buffer
        else
          bulk_wait_read();
        const bool w = mbar_wait(tfull + t, (unsigned)((k / 2) & 1), lim) && !*abort_flag;
        *go = w ? 1 : 0;
        if (!w) {
          atomicCAS(a.err, 0u, 18u);
          *abort_flag = 1;
        }
      }
      named_sync(1, 32 * kEpi);
      if (!*go) break;
      mbar_wait(tfull + t, (unsigned)((k / 2) & 1), lim);  // completed: returns at once
      tc_fence_after();
      const bool nyq = kt == 0 && r == 0;  // rows 0 and M/2 instead of 0 and its mirror
      const uint32_t tb = trow + (uint32_t)t * 256;
      unsigned char* Sk = Sg + (size_t)(kStagings == 2 ? (k & 1) : 0) * 2 * kStaging;
      unsigned char* Sm = Sk + kStaging;
      const uint32_t sk = smem_u32(Sk), sm = smem_u32(Sm);
      float m = 0.f;
#pragma unroll 1
      for (int n0 = colh * kColsW; n0 < colh * kColsW + kColsW; n0 += 16) {
        float ar[16], br[16], ai[16], bi[16];
        tmem_ld16(tb + (uint32_t)n0, ar);              // Re A (source a), columns n0 ..
        tmem_ld16(tb + XB + (uint32_t)n0, br);         // Re B (source b)
        tmem_ld16(tb + 128 + (uint32_t)n0, ai);        // Im A
        tmem_ld16(tb + 128 + XB + (uint32_t)n0, bi);   // Im B
        tmem_wait_ld();
        uint32_t kre[8], kim[8], mre[8], mim[8];
#pragma unroll
        for (int j = 0; j < 16; j += 2) {
          float kr[2], ki[2], mr[2], mi[2];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const float ra = ar[j + h], rb = br[j + h], ia = ai[j + h], ib = bi[j + h];
            kr[h] = nyq ? ra : ra - ib;
            ki[h] = nyq ? rb : ia + rb;
            mr[h] = nyq ? ia : ra + ib;  // the Nyquist row: Re A[M/2], Re B[M/2]
            mi[h] = nyq ? ib : rb - ia;
            m = fmaxf(m, fmaxf(fmaxf(fabsf(kr[h]), fabsf(ki[h])), fmaxf(fabsf(mr[h]), fabsf(mi[h]))));
          }
          kre[j / 2] = pack_h2(kr[0], kr[1]);
          kim[j / 2] = pack_h2(ki[0], ki[1]);
          mre[j / 2] = pack_h2(mr[0], mr[1]);
          mim[j / 2] = pack_h2(mi[0], mi[1]);
        }
        const uint32_t c0 = (uint32_t)n0 / 8;  // first 16-byte chunk of these 16 columns
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sk + sw128(rk, c0 + h)), "r"(kre[4 * h]),
                       "r"(kre[4 * h + 1]), "r"(kre[4 * h + 2]), "r"(kre[4 * h + 3]) : "memory");
          asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sk + sw128(rk + 1, c0 + h)), "r"(kim[4 * h]),
                       "r"(kim[4 * h + 1]), "r"(kim[4 * h + 2]), "r"(kim[4 * h + 3]) : "memory");
          asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sm + sw128(rm, c0 + h)), "r"(mre[4 * h]),
                       "r"(mre[4 * h + 1]), "r"(mre[4 * h + 2]), "r"(mre[4 * h + 3]) : "memory");
          asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sm + sw128(rm + 1, c0 + h)), "r"(mim[4 * h]),
                       "r"(mim[4 * h + 1]), "r"(mim[4 * h + 2]), "r"(mim[4 * h + 3]) : "memory");
        }
        if (nyq) {
          // planes M (re) and M + 1 (im) of work tile wl, columns XB xb + n0 ..
          uint4* pr = reinterpret_cast<uint4*>(a.planes + ((size_t)M * a.c + wl) * M + XB * xb + n0);
          uint4* pi = reinterpret_cast<uint4*>(a.planes + ((size_t)(M + 1) * a.c + wl) * M + XB * xb + n0);
          pr[0] = make_uint4(mre[0], mre[1], mre[2], mre[3]);
          pr[1] = make_uint4(mre[4], mre[5], mre[6], mre[7]);
          pi[0] = make_uint4(mim[0], mim[1], mim[2], mim[3]);
          pi[1] = make_uint4(mim[4], mim[5], mim[6], mim[7]);
        }
      }
      // accumulators t are free for item k + 2
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_g(tempty + t);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (lane == 0 && m > 0.f) atomicMax(a.zmax + wl, __float_as_uint(m));
      // staging complete: two stores of 256 plane rows x 64 columns (rows past the planes are dropped)
      fence_async_smem();
      named_sync(1, 32 * kEpi);
      if (threadIdx.x == 0) {
        tma_store_3d(&pmap, XB * xb, wl, 2 * kt * KR, Sk);
        tma_store_3d(&pmap, XB * xb, wl, 2 * (M - kt * KR - (KR - 1)), Sm);
        bulk_commit();
      }
    }
    if (threadIdx.x == 0) bulk_wait_all();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
  }
}

}  // namespace p1g
}  // namespace srk
