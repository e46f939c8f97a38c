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
// (128 ky rows of one parity, 64 columns x of both sources) two real GEMMs
// with K = y:
//   Dr = C [a | b],   C[ky][y] = cos(2 pi ky y / M)
//   Di = S [a | b],   S[ky][y] = -sin(2 pi ky y / M)
// (N = 128: 64 columns of a, then the same 64 of b).  Items take the even
// or the odd ky < M/2: C and S at y + M/2 are (-1)^ky times their values
// at y, so the tables cover y < M/2 only and each table atom multiplies the
// image atoms at y and at y + M/2 (the second with the instruction's
// negate-A bit for odd ky) — half the table bytes per unit of work.  The
// row ky = 0 of S is zero; the table holds the Nyquist row (-1)^y there
// instead (even at y + M/2 too), so that lane also yields Re A[M/2] and
// Re B[M/2] (Im of both is zero at ky = 0 and M/2).  The tables and images
// are FP16 (or BF16 for BF16 storage) operands with FP32 accumulation: the
// planes are FP16 anyway.
//
// Data movement: the tables (128 ky x 64 y boxes) and the source tiles
// (64 x x 64 y boxes, the images' own column-major layout is the K-major
// operand) by TMA with the 128-byte swizzle through a ring of stages; the
// planes leave through shared memory by 4-D TMA stores whose ky dimension
// steps by 2 (128 rows of one parity, both parts, 64 columns: 128-byte
// rows), the Nyquist row by the threads.
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
constexpr int NA = M / 2 / 64;           // table atoms of 64 rows y (each with the image atoms y and y + M/2)
constexpr int NSG = 3;                   // ring stages (one table atom each)
constexpr int kEpi = 4;                  // epilogue warps, one per TMEM lane quarter
constexpr int kThreadsG = 32 * (kEpi + 2);
constexpr int kLoadWarp = kEpi, kMmaWarp = kEpi + 1;
constexpr uint32_t kTabBox = KR * 128;   // 128 table rows x 64 y, 16 KB
constexpr uint32_t kSrcBox = XB * 128;   // 64 columns x 64 y, 8 KB
constexpr uint32_t kSrcAtom = 2 * kSrcBox;                 // both sources: the MMA's 128 B operand rows
constexpr uint32_t kStage = 2 * kTabBox + 2 * kSrcAtom;    // C | S | images at y | images at y + M/2
constexpr uint32_t kStaging = 256 * 128;  // 128 ky rows x 2 parts x 64 FP16 columns
// barriers | NSG stages | staging (rows ky, then rows M - ky, of one item)
__host__ __device__ constexpr size_t smem_bytes() { return 1024 + (size_t)NSG * kStage + kStaging; }

struct Args {
  __half* planes;            // the chunk's planes [2M][c][M] (the Nyquist row is stored directly)
  unsigned int* zmax;        // largest |Z| per work tile (float bits, zeroed before the launch)
  unsigned int* err;         // plan error word
  unsigned long long spin_limit;
  Geom g;                    // tile geometry (uniform batch)
  int w0, c;                 // first work tile and work tiles of the chunk
  int nimg;                  // images in the image map (a coordinate there reads zeros)
};

// C and S tables: rows part * 256 + p * 128 + r for ky = p + 2 r (parity p),
// columns y < M/2, in the storage type's 16-bit format.
template <typename T>
__global__ void k_p1g_tables(T* __restrict__ tab) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 2 * (M / 2) * (M / 2)) return;
  const int y = idx % (M / 2), row = idx / (M / 2), part = row / (M / 2);
  const int par = (row % (M / 2)) / KR, r = row % KR, ky = par + 2 * r;
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

// Persistent, one CTA per SM; an item is (work tile wl, column block xb, ky
// parity kt) with kt fastest (both parities read the same source boxes).
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
  unsigned char* St = smem + 1024;                     // NSG stages: C | S | images at y | images at y + M/2
  unsigned char* Sk = St + (size_t)NSG * kStage;       // staging: rows ky, then rows M - ky
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
          tma_load_2d(S, &tmap, 64 * at, kt * KR, full + st);                        // C rows of parity kt
          tma_load_2d(S + kTabBox, &tmap, 64 * at, M / 2 + kt * KR, full + st);      // S rows
          for (int h = 0; h < 2; ++h) {                                              // y and y + M/2
            unsigned char* D = S + 2 * kTabBox + h * kSrcAtom;
            const int y = 64 * at + h * (M / 2);
            tma_load_3d(D, &smap, t0.y0 + y, t0.x0 + XB * xb, i0, full + st);
            tma_load_3d(D + kSrcBox, &smap, t1.y0 + y, t1.x0 + XB * xb, i1, full + st);
          }
        }
      }
      for (long long r = q > NSG ? q - NSG : 0; r < q; ++r) mbar_wait(full + (int)(r % NSG), (unsigned)((r / NSG) & 1), lim);
    }
    __syncwarp();
  } else if (warp == kMmaWarp) {
    if (lane == 0) {
      constexpr int kFmt = std::is_same<T, __nv_bfloat16>::value ? 1 : 0;
      const uint32_t id = idesc_f16(kFmt, KR, 2 * XB);
      const uint32_t idn = id | (1u << 13);  // negate A: the odd rows' tables at y + M/2
      long long q = 0;
      bool ok = true;
      for (int k = 0, item = blockIdx.x; item < items && ok; ++k, item += gridDim.x) {
        const int t = k & 1;
        const uint32_t idh = (item & 1) ? idn : id;  // parity kt = item & 1
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
            const uint64_t dlo = sdesc_sw128(base + 2 * kTabBox + (uint32_t)kk * 32);
            const uint64_t dhi = sdesc_sw128(base + 2 * kTabBox + kSrcAtom + (uint32_t)kk * 32);
            mma_f16(dr, dc, dlo, id, (at | kk) != 0);
            mma_f16(dr, dc, dhi, idh, true);
            mma_f16(di, ds, dlo, id, (at | kk) != 0);
            mma_f16(di, ds, dhi, idh, true);
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
    // epilogue warp: TMEM lanes 32 warp .. + 31 = rows r of the item, ky = kt + 2 r
    const int r = warp * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t sk = smem_u32(Sk);
    for (int k = 0, item = blockIdx.x; item < items; ++k, item += gridDim.x) {
      const int t = k & 1;
      int wl, xb, kt;
      decode(item, wl, xb, kt);
      // One thread decides for all epilogue warps, so that they leave together
      // (they meet at named barriers): the accumulators are complete and the
      // staging block free (the previous item's stores have read it).
      if (threadIdx.x == 0) {
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
      float m = 0.f;
      // pass 0: rows ky (staging row 2 r + part) -> store from ky = kt;
      // pass 1: rows M - ky (staging row 2 (127 - r) + part) -> store from
      // ky = M/2 + 2 - kt (the row past M, r = 0 at kt = 0, is dropped) and
      // the Nyquist row by the threads
#pragma unroll 1
      for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
          if (threadIdx.x == 0) bulk_wait_read();  // the rows-ky store has read the staging block
          named_sync(1, 32 * kEpi);
        }
        const uint32_t row = pass == 0 ? 2 * r : 2 * (KR - 1 - r);
#pragma unroll 1
        for (int n0 = 0; n0 < XB; n0 += 16) {
          float ar[16], br[16], ai[16], bi[16];
          tmem_ld16(tb + (uint32_t)n0, ar);              // Re A (source a), columns n0 ..
          tmem_ld16(tb + XB + (uint32_t)n0, br);         // Re B (source b)
          tmem_ld16(tb + 128 + (uint32_t)n0, ai);        // Im A
          tmem_ld16(tb + 128 + XB + (uint32_t)n0, bi);   // Im B
          tmem_wait_ld();
          uint32_t vre[8], vim[8];
#pragma unroll
          for (int j = 0; j < 16; j += 2) {
            float zr[2], zi[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const float ra = ar[j + h], rb = br[j + h], ia = ai[j + h], ib = bi[j + h];
              if (pass == 0) {
                zr[h] = nyq ? ra : ra - ib;  // Z[ky]
                zi[h] = nyq ? rb : ia + rb;
                // bounds every |component| of Z[ky] and Z[M - ky] (the Nyquist row too)
                m = fmaxf(m, fmaxf(fabsf(ra) + fabsf(ib), fabsf(ia) + fabsf(rb)));
              } else {
                zr[h] = nyq ? ia : ra + ib;  // Z[M - ky]; the Nyquist row: Re A[M/2], Re B[M/2]
                zi[h] = nyq ? ib : rb - ia;
              }
            }
            vre[j / 2] = pack_h2(zr[0], zr[1]);
            vim[j / 2] = pack_h2(zi[0], zi[1]);
          }
          const uint32_t c0 = (uint32_t)n0 / 8;  // first 16-byte chunk of these 16 columns
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sk + sw128(row, c0 + h)), "r"(vre[4 * h]),
                         "r"(vre[4 * h + 1]), "r"(vre[4 * h + 2]), "r"(vre[4 * h + 3]) : "memory");
            asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sk + sw128(row + 1, c0 + h)),
                         "r"(vim[4 * h]), "r"(vim[4 * h + 1]), "r"(vim[4 * h + 2]), "r"(vim[4 * h + 3]) : "memory");
          }
          if (pass == 1 && nyq) {
            // planes M (re) and M + 1 (im) of work tile wl, columns XB xb + n0 ..
            uint4* pr = reinterpret_cast<uint4*>(a.planes + ((size_t)M * a.c + wl) * M + XB * xb + n0);
            uint4* pi = reinterpret_cast<uint4*>(a.planes + ((size_t)(M + 1) * a.c + wl) * M + XB * xb + n0);
            pr[0] = make_uint4(vre[0], vre[1], vre[2], vre[3]);
            pr[1] = make_uint4(vre[4], vre[5], vre[6], vre[7]);
            pi[0] = make_uint4(vim[0], vim[1], vim[2], vim[3]);
            pi[1] = make_uint4(vim[4], vim[5], vim[6], vim[7]);
          }
        }
        fence_async_smem();
        named_sync(1, 32 * kEpi);
        if (threadIdx.x == 0) {
          tma_store_4d(&pmap, XB * xb, wl, 0, pass == 0 ? kt : M / 2 + 2 - kt, Sk);
          bulk_commit();
        }
      }
      // accumulators t are free for item k + 2
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_g(tempty + t);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (lane == 0 && m > 0.f) atomicMax(a.zmax + wl, __float_as_uint(m));
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
