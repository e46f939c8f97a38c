// fft_warp.cuh — complex FFT of length M (128..512) by one warp or a warp pair, sm_100a.
//
// Layout contract (both directions): the TPF threads of a transform (a warp,
// or a pair of warps for M = 512) hold x[i] = X[t + TPF*i], i < M/TPF
// ("strided" order), so each warp loads/stores one contiguous column with
// fully coalesced requests, and the result comes back in the same order
// (natural frequency order, no bit reversal).
//
// Algorithm: Stockham auto-sort, one radix-R pass per stage (mixed radix,
// R in {2,4,8,16}).  Pass p with span Ns (product of the previous radices)
// runs M/R butterflies; butterfly j reads x[j + r*M/R], multiplies by
// W_{Ns*R}^{r*(j mod Ns)}, does an R-point DFT and writes
// y[(j/Ns)*Ns*R + (j mod Ns) + r*Ns].  Each lane owns EPT/R butterflies
// (j = t + 32*b), so the first pass reads straight from registers and the
// last pass writes straight back to registers in strided order; the
// passes in between exchange through a per-warp shared-memory row of
// M + M/16 float2 (one pad word per 16, which makes the scatter of the
// first pass bank-conflict free).
//
// Twiddles come from a table in shared memory, one block per pass
// (tw_entry), filled from double-precision cos/sin rounded once to float;
// the inverse transform uses their conjugates.  The transforms are
// unnormalised in both directions.
#pragma once
#include <cuda_runtime.h>

namespace srk {

// Complex arithmetic with every rounding spelled out (no compiler
// contraction of a product into a later sum): each kernel that inlines a
// transform computes bit-identical results, whatever the schedule.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y)); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(__fmaf_rn(a.x, b.x, -__fmul_rn(a.y, b.y)), __fmaf_rn(a.x, b.y, __fmul_rn(a.y, b.x)));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(__fmaf_rn(a.x, b.x, __fmul_rn(a.y, b.y)), __fmaf_rn(a.y, b.x, -__fmul_rn(a.x, b.y)));
}
template <bool INV>
__device__ __forceinline__ float2 twmul(float2 a, float2 w) {
  return INV ? cmulc(a, w) : cmul(a, w);
}

// Padded positions in a transform's shared row.  fft_pad is the layout of
// rows handed between phases (staging, stashes) and of the first exchange;
// the later exchanges of a transform use their own padding (exch_pad),
// chosen so that the 8-byte writes of that exchange and the reads after it
// keep every half-warp on distinct banks.
__host__ __device__ constexpr int fft_pad(int i) { return i + (i >> 4); }
template <int K>
__host__ __device__ constexpr int padk(int i) {
  return K == 0 ? i + (i >> 4) : K == 1 ? i + 8 * (i >> 6) : i + 4 * (i >> 4);
}
// Padding of the exchange that follows pass p of an M-point transform.
__host__ __device__ constexpr int exch_pad(int M, int p) { return p == 1 ? (M == 128 ? 2 : 1) : 0; }
// Row length (complex values) that holds every padding used on the row.
__host__ __device__ constexpr int fft_row_words(int M) {
  const int a = fft_pad(M - 1) + 1;
  const int b = (M == 128 ? padk<2>(M - 1) : padk<1>(M - 1)) + 1;
  return a > b ? a : b;
}

// Multiply by W_16^m = exp(-+ i*pi*m/8) for a compile-time m in [0,8).
template <int m, bool INV>
__device__ __forceinline__ float2 rot16(float2 v) {
  constexpr float R2 = 0.70710678118654752440f;   // cos(pi/4)
  constexpr float C1 = 0.92387953251128675613f;   // cos(pi/8)
  constexpr float S1 = 0.38268343236508977173f;   // sin(pi/8)
  if constexpr (m == 0) {
    return v;
  } else if constexpr (m == 4) {                  // -i (forward) / +i (inverse)
    return INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
  } else if constexpr (m == 2) {                  // (1 -+ i)/sqrt2
    const float p = __fadd_rn(v.x, v.y), q = __fsub_rn(v.x, v.y);
    return INV ? make_float2(__fmul_rn(q, R2), __fmul_rn(p, R2)) : make_float2(__fmul_rn(p, R2), __fmul_rn(-q, R2));
  } else if constexpr (m == 6) {                  // (-1 -+ i)/sqrt2
    const float p = __fadd_rn(v.x, v.y), q = __fsub_rn(v.x, v.y);
    return INV ? make_float2(__fmul_rn(-p, R2), __fmul_rn(q, R2)) : make_float2(__fmul_rn(-q, R2), __fmul_rn(-p, R2));
  } else {
    constexpr float c = (m == 1) ? C1 : (m == 3) ? S1 : (m == 5) ? -S1 : -C1;
    constexpr float s = (m == 1) ? S1 : (m == 3) ? C1 : (m == 5) ? C1 : S1;
    // forward: v*(c - i s); inverse: v*(c + i s)
    return INV ? make_float2(__fmaf_rn(v.x, c, -__fmul_rn(v.y, s)), __fmaf_rn(v.y, c, __fmul_rn(v.x, s)))
               : make_float2(__fmaf_rn(v.x, c, __fmul_rn(v.y, s)), __fmaf_rn(v.y, c, -__fmul_rn(v.x, s)));
  }
}

// In-register R-point DFT (natural order in and out), radix-2 decimation in
// time applied recursively.
template <int R, bool INV>
struct Dft {
  template <int K>
  __device__ __forceinline__ static void combine(float2* a, const float2* e, const float2* o) {
    if constexpr (K < R / 2) {
      const float2 t = rot16<(16 / R) * K, INV>(o[K]);
      a[K] = cadd(e[K], t);
      a[K + R / 2] = csub(e[K], t);
      combine<K + 1>(a, e, o);
    }
  }
  __device__ __forceinline__ static void run(float2* a) {
    float2 e[R / 2], o[R / 2];
#pragma unroll
    for (int i = 0; i < R / 2; ++i) { e[i] = a[2 * i]; o[i] = a[2 * i + 1]; }
    Dft<R / 2, INV>::run(e);
    Dft<R / 2, INV>::run(o);
    combine<0>(a, e, o);
  }
};
template <bool INV>
struct Dft<2, INV> {
  __device__ __forceinline__ static void run(float2* a) {
    const float2 t = a[0];
    a[0] = cadd(t, a[1]);
    a[1] = csub(t, a[1]);
  }
};

// ---- radix schedule and twiddle-table layout ---------------------------------
// Passes of the M-point transform: (radix R, span NS before the pass).
struct PassDesc { int R, NS; };
__host__ __device__ constexpr int fft_npasses(int M) { return M == 128 ? 4 : 3; }
__host__ __device__ constexpr PassDesc fft_pass_desc(int M, int p) {
  return M == 128   ? (p == 0 ? PassDesc{4, 1} : p == 1 ? PassDesc{4, 4} : p == 2 ? PassDesc{4, 16} : PassDesc{2, 64})
         : M == 256 ? (p == 0 ? PassDesc{8, 1} : p == 1 ? PassDesc{8, 8} : PassDesc{4, 64})
                    : (p == 0 ? PassDesc{8, 1} : p == 1 ? PassDesc{8, 8} : PassDesc{8, 64});
}
// The twiddle table holds, for every pass p >= 1, the NS entries
// W_{NS R}^k = exp(-2 pi i k / (NS R)), k < NS, one block per pass; a thread
// reads the one entry of its butterfly (consecutive threads read consecutive
// k or the same word: no bank conflicts) and forms the powers W^{r k},
// r < R, by complex products (tw_powers).
__host__ __device__ constexpr int tw_offset(int M, int p) {
  int off = 0;
  for (int q = 1; q < p; ++q) off += fft_pass_desc(M, q).NS;
  return off;
}
__host__ __device__ constexpr int tw_entries(int M) { return tw_offset(M, fft_npasses(M)); }
// Exponent of table entry idx as the fraction num/den of a full turn.
__host__ __device__ inline void tw_entry(int M, int idx, int& num, int& den) {
  for (int p = 1; p < fft_npasses(M); ++p) {
    const PassDesc d = fft_pass_desc(M, p);
    if (idx < d.NS) {
      num = idx;
      den = d.NS * d.R;
      return;
    }
    idx -= d.NS;
  }
  num = 0;
  den = 1;
}

// w[r] = w1^r for 1 <= r < R, by at most three dependent products (w[0] is
// not set): the rounding error stays within a few units of the last place.
template <int R>
__device__ __forceinline__ void tw_powers(float2 w1, float2 (&w)[R]) {
  w[1] = w1;
  if constexpr (R >= 4) {
    w[2] = cmul(w1, w1);
    w[3] = cmul(w[2], w1);
  }
  if constexpr (R == 8) {
    w[4] = cmul(w[2], w[2]);
    w[5] = cmul(w[4], w1);
    w[6] = cmul(w[4], w[2]);
    w[7] = cmul(w[4], w[3]);
  }
}

// Per-thread part P(t) and compile-time part C(b, r) of the write index
// (j/NS)*NS*R + (j mod NS) + r*NS of butterfly j = t + TPF*b, where TPF is
// the number of threads that share one transform (32 or 64).
template <int R, int NS, int TPF>
__host__ __device__ constexpr int pass_P(int t) {
  return NS >= TPF ? t : (t / NS) * NS * R + (t % NS);
}
template <int R, int NS, int TPF>
__host__ __device__ constexpr int pass_C(int b, int r) {
  return NS >= TPF ? ((TPF * b) / NS) * NS * R + (TPF * b) % NS + r * NS : TPF * b * R + r * NS;
}
// padk<K>(P + C) == padk<K>(P) + padk<K>(C) for every thread, butterfly and
// leg: then every shared-memory write is (per-thread base) + (immediate).
template <int M, int R, int NS, int TPF, int K>
__host__ __device__ constexpr bool pad_separable() {
  for (int t = 0; t < TPF; ++t)
    for (int b = 0; b < M / TPF / R; ++b)
      for (int r = 0; r < R; ++r) {
        const int P = pass_P<R, NS, TPF>(t), C = pass_C<R, NS, TPF>(b, r);
        if (padk<K>(P + C) != padk<K>(P) + padk<K>(C)) return false;
      }
  return true;
}
// The same for the reads X[t + TPF i].
template <int M, int TPF, int K>
__host__ __device__ constexpr bool read_separable() {
  for (int t = 0; t < TPF; ++t)
    for (int i = 0; i < M / TPF; ++i)
      if (padk<K>(t + TPF * i) != padk<K>(t) + padk<K>(TPF * i)) return false;
  return true;
}

// Barrier over the threads of one transform: the warp itself, or a named
// barrier (id >= 1) over the TPF threads of a multi-warp group.
template <int TPF>
__device__ __forceinline__ void group_sync(int bar) {
  if constexpr (TPF == 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "n"(TPF) : "memory");
  }
}

// One Stockham pass.  sm: this transform's padded exchange row; tw: W_M table.
// PIN / POUT: padding (padk) of the exchange read before / written after
// the pass.
template <int M, int TPF, int R, int NS, bool FIRST, bool LAST, bool INV, int TWOFF, int PIN, int POUT>
__device__ __forceinline__ void fft_pass(float2 (&x)[M / TPF], float2* __restrict__ sm,
                                         const float2* __restrict__ tw, int t, int bar) {
  constexpr int EPT = M / TPF;
  constexpr int NB = EPT / R;
  static_assert(EPT % R == 0, "radix must divide elements per thread");
  static_assert(LAST || pad_separable<M, R, NS, TPF, POUT>(), "padded write index must split into base + immediate");
  static_assert(FIRST || read_separable<M, TPF, PIN>(), "padded read index must split into base + immediate");
  if constexpr (!FIRST) {
    const float2* rd = sm + padk<PIN>(t);
#pragma unroll
    for (int i = 0; i < EPT; ++i) x[i] = rd[padk<PIN>(TPF * i)];
    group_sync<TPF>(bar);
  }
  float2* wr = nullptr;
  if constexpr (!LAST) wr = sm + padk<POUT>(pass_P<R, NS, TPF>(t));
  const float2* twp = tw + TWOFF;  // this pass's W_{NS R}^k block
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    float2 a[R];
#pragma unroll
    for (int r = 0; r < R; ++r) a[r] = x[b + r * NB];
    if constexpr (!FIRST) {
      // k = (t + TPF b) mod NS
      const int k = (NS <= TPF) ? (t & (NS - 1)) : (t + ((TPF * b) & (NS - 1)));
      float2 w[R];
      tw_powers<R>(twp[k], w);
#pragma unroll
      for (int r = 1; r < R; ++r) a[r] = twmul<INV>(a[r], w[r]);
    }
    Dft<R, INV>::run(a);
    if constexpr (LAST) {
#pragma unroll
      for (int r = 0; r < R; ++r) x[b + r * NB] = a[r];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) wr[padk<POUT>(pass_C<R, NS, TPF>(b, r))] = a[r];
    }
  }
  if constexpr (!LAST) group_sync<TPF>(bar);
}

// Threads per transform: a warp for M <= 256, a 64-thread pair of warps for
// M = 512 (8 values per thread keeps registers low enough for 5 CTAs/SM).
template <int M>
__host__ __device__ constexpr int tpf_of() { return M >= 512 ? 64 : 32; }

// Full transform over the TPF threads of a group; t = thread index in the
// group, bar = its named barrier (ignored for TPF = 32).  Data layout:
// thread t holds X[t + TPF*i].
template <int M, bool INV, int TPF = tpf_of<M>()>
__device__ __forceinline__ void fft(float2 (&x)[M / TPF], float2* __restrict__ sm, const float2* __restrict__ tw,
                                    int t, int bar) {
  group_sync<TPF>(bar);  // the row may still be read by threads finishing a previous use
  static_assert(M == 128 || M == 256 || M == 512, "unsupported FFT length");
  constexpr PassDesc p0 = fft_pass_desc(M, 0), p1 = fft_pass_desc(M, 1), p2 = fft_pass_desc(M, 2);
  constexpr int NP = fft_npasses(M);
  constexpr int X0 = exch_pad(M, 0), X1 = exch_pad(M, 1), X2 = exch_pad(M, 2);
  fft_pass<M, TPF, p0.R, p0.NS, true, false, INV, 0, X0, X0>(x, sm, tw, t, bar);
  fft_pass<M, TPF, p1.R, p1.NS, false, false, INV, tw_offset(M, 1), X0, X1>(x, sm, tw, t, bar);
  fft_pass<M, TPF, p2.R, p2.NS, false, NP == 3, INV, tw_offset(M, 2), X1, X2>(x, sm, tw, t, bar);
  if constexpr (NP == 4) {
    constexpr PassDesc p3 = fft_pass_desc(M, 3);
    fft_pass<M, TPF, p3.R, p3.NS, false, true, INV, tw_offset(M, 3), X2, X2>(x, sm, tw, t, bar);
  }
}

}  // namespace srk
