// conv_launch.cuh — launch sequences of the engine (both schedules) for one
// operator and storage type; included by conv_<type>.cu only.
#pragma once
#include "internal.h"
#include "hybrid_p1.cuh"
#include "hybrid_p1g.cuh"

namespace srk {

template <typename K>
srk_status set_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024)
    SRK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return SRK_OK;
}

// Three-pass schedule with the tensor-core row pass (SRK_SCHEDULE_TENSOR_ROWS):
// per chunk the column pass (-> FP16 planes, with each work tile's largest
// |Z|: the column DFT on the tensor cores, k_p1g, where its TMA boxes apply,
// else the column FFT, k_p1h) and its refit pass (the work tiles outside
// FP16's comfortable range again, scaled by a power of two), the row pass of
// hybrid.cu (-> S2), P3; two slots of chunks on two streams.
template <int OP, typename T>
srk_status launch_tensor_rows(srk_plan_s* p, const OpArgs& a, const Geom& g, int nwt, cudaStream_t s) {
  constexpr int M = kHybM;
  constexpr int LPU = lpu_of<M>();
  const size_t per = wt_elems<M, OP>(g.S);
  const size_t s1 = s1_elems<M, OP>();
  const size_t plane_wt = (size_t)2 * M * M;  // halves per work tile
  const size_t cap = std::min<size_t>(p->scratch_bytes / sizeof(float2) / per, p->hyb_s1_bytes / sizeof(__half) / plane_wt);
  const size_t smp1 = p1h_smem_bytes();
  const size_t sm3 = phase_smem_bytes<M>() + (p3_async_window<OP, T>() ? sizeof(float) * p3_window_floats<M>() : 0);
  SRK_TRY(set_smem(k_p1h<OP, T>, smp1));
  SRK_TRY(set_smem(k_p3<M, OP, T, kHybS2Layout>, sm3));
  SRK_TRY(set_smem(k_p1h_refit<OP, T>, smp1));
  static_assert(OpTraits<OP>::PAIRS, "the tensor-row schedule serves the pair ops");
  // k_p1g (column DFT on the tensor cores): a uniform batch, N % 8 == 0
  // (16-byte image rows), tile origins on 8-row boundaries (TMA's innermost
  // coordinate), a 16-byte aligned image array; else the column FFT, k_p1h
  const int nimg = g.TT > 0 ? g.U / g.TT : 0;
  const bool dft = p->p1g_tab && !g.rtile && g.N % 8 == 0 && (g.TT == 1 || g.S % 8 == 0) &&
                   (reinterpret_cast<uintptr_t>(a.E) & 15) == 0;
  CUtensorMap tmapg, smapg;
  if (dft) {
    SRK_TRY(set_smem(p1g::k_p1g<T>, p1g::smem_bytes()));
    SRK_TRY(tensor_rows_p1g_maps(p, a.E, g.N, nimg, &tmapg, &smapg));
  }
  int chunk = 0;  // work tiles per slot (two slots in the pipelined form)
  // largest |Z| of the work tiles of the chunk in slot k & 1 (their planes' scales)
  auto max_of = [&](int k) { return p->hyb_mx + (size_t)(k & 1) * chunk; };
  auto p1 = [&](int k, int w0, int c, __half* planes, cudaStream_t st) -> srk_status {
    CUtensorMap pmap;
    SRK_TRY(tensor_rows_plane_map(planes, c, kP1hCols, 1, kP1hBox, &pmap));
    SRK_CUDA(cudaMemsetAsync(max_of(k), 0, (size_t)c * sizeof(unsigned int), st));
    if (dft) {
      CUtensorMap pmapg;  // 128 ky rows of one parity x 2 parts x 64 columns, 128-byte swizzle
      SRK_TRY(tensor_rows_p1g_store_map(planes, c, &pmapg));
      p1g::Args ga;
      ga.planes = planes;
      ga.zmax = max_of(k);
      ga.err = p->direct_err;
      ga.spin_limit = 1ull << 22;
      ga.g = g;
      ga.w0 = w0;
      ga.c = c;
      ga.nimg = nimg;
      const int items = c * (p1g::M / p1g::XB) * 2;
      p1g::k_p1g<T><<<std::min(items, std::max(p->nsm, 1)), p1g::kThreadsG, p1g::smem_bytes(), st>>>(
          tmapg, smapg, pmapg, ga);
    } else {
      k_p1h<OP, T><<<dim3(M / kP1hCols, c), kThreads, smp1, st>>>(pmap, a, g, p->tw, w0, p->nsm, max_of(k),
                                                                   p->direct_err);
    }
    k_p1h_refit<OP, T><<<std::max(p->nsm, 1) * 2, kThreads, smp1, st>>>(pmap, a, g, p->tw, w0, c, max_of(k),
                                                                        p->direct_err);
    return SRK_OK;
  };
  auto p3 = [&](int w0, int c, float2* base, cudaStream_t st) {
    k_p3<M, OP, T, kHybS2Layout><<<dim3((g.S + LPU - 1) / LPU, c), kThreads, sm3, st>>>(base, a, g, p->tw, w0, p->nsm);
  };
  const int whole = (int)std::min<size_t>(std::max<size_t>(cap, 1), 65535);
  int launches = 0;
  if (nwt < 256 || !p->overlap || !p->ps1 || cap < 2) {
    for (int w0 = 0; w0 < nwt; w0 += whole, launches += 4) {
      const int c = std::min(whole, nwt - w0);
      SRK_TRY(p1(0, w0, c, p->hyb_s1, s));
      SRK_TRY(tensor_rows_p2(p, p->hyb_s1, max_of(0), c, p->scratch, per, s1, g.S, s2_pitch(g.S), s));
      p3(w0, c, p->scratch, s);
    }
  } else {
    // Two slots of chunks.  The persistent row pass occupies every SM, so it
    // runs alone: P2h(k) (caller's stream) waits for P1h(k) and follows
    // P3(k-1) in stream order; P1h(k+1) (plan stream) starts after P2h(k) and
    // runs beside P3(k).  Slot reuse: P1h(k+1) rewrites the planes P2h(k-1)
    // read (it waits for P2h(k)); P2h(k) rewrites the S2 P3(k-2) read
    // (earlier on the same stream).
    // at least four chunks where the slots allow (the overlap is between chunks)
    chunk = (int)std::min<size_t>({cap / 2, (size_t)std::max(128, (nwt + 3) / 4), (size_t)65535});
    const int nch = (nwt + chunk - 1) / chunk;
    auto planes_of = [&](int k) { return p->hyb_s1 + (size_t)(k & 1) * chunk * plane_wt; };
    auto base_of = [&](int k) { return p->scratch + (size_t)(k & 1) * chunk * per; };
    auto count_of = [&](int k) { return std::min(chunk, nwt - k * chunk); };
    SRK_CUDA(cudaEventRecord(p->ev_fork, s));
    SRK_CUDA(cudaStreamWaitEvent(p->ps1, p->ev_fork, 0));
    SRK_TRY(p1(0, 0, count_of(0), planes_of(0), p->ps1));
    SRK_CUDA(cudaEventRecord(p->ev1[0], p->ps1));
    for (int k = 0; k < nch; ++k, launches += 4) {
      SRK_CUDA(cudaStreamWaitEvent(s, p->ev1[k & 1], 0));
      SRK_TRY(tensor_rows_p2(p, planes_of(k), max_of(k), count_of(k), base_of(k), per, s1, g.S, s2_pitch(g.S), s));
      if (k + 1 < nch) {
        // the max words of slot (k+1) & 1 were last read by P2h(k-1), before P2h(k)
        SRK_CUDA(cudaEventRecord(p->ev2[k & 1], s));
        SRK_CUDA(cudaStreamWaitEvent(p->ps1, p->ev2[k & 1], 0));
        SRK_TRY(p1(k + 1, (k + 1) * chunk, count_of(k + 1), planes_of(k + 1), p->ps1));
        SRK_CUDA(cudaEventRecord(p->ev1[(k + 1) & 1], p->ps1));
      }
      p3(k * chunk, count_of(k), base_of(k), s);
    }
    // every plan-stream launch is followed by a row pass on the caller's stream: joined
  }
  p->last_launches = launches;
  return cuda_status(cudaGetLastError(), "tensor-row launch");
}

template <int M, int OP, typename T>
srk_status launch_conv_m(srk_plan_s* p, const OpArgs& a, const Geom& g, int nwt, bool conjG, cudaStream_t s) {
  // the tensor-core row pass serves the pair ops (forward, VJP); a tangent
  // field packed beside its primal in one complex column loses too much to
  // the FP16 planes (measured past the per-pixel tolerance on the
  // tangent-adjoint at N = 1024, KW = 121), so JVP and tangent-adjoint run
  // the FFT schedule on such a plan
  if constexpr (M == kHybM && OpTraits<OP>::K == 1 && OpTraits<OP>::PAIRS && !std::is_same<T, float>::value) {
    if (p->schedule == SRK_SCHEDULE_TENSOR_ROWS && p->hyb_ready) return launch_tensor_rows<OP, T>(p, a, g, nwt, s);
  }
  const size_t sm1 = phase_smem_bytes<M>();
  const size_t sm2 = sm1 + p2_tile_bytes<M>(g.S);
  const size_t sm3 = sm1 + (p3_async_window<OP, T>() ? sizeof(float) * p3_window_floats<M>() : 0);
  const size_t per = wt_elems<M, OP>(g.S);
  const size_t cap = p->scratch_bytes / sizeof(float2) / per;  // WTs that fit the scratch
  if (p->schedule == SRK_SCHEDULE_PERSISTENT && cap >= 3) {
    SRK_TRY(set_smem(k_persist<M, OP, T>, sm2));
    int dev = 0, nsm = 0, per_sm = 0;
    SRK_CUDA(cudaGetDevice(&dev));
    SRK_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    SRK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_persist<M, OP, T>, kThreads, sm2));
    if (per_sm < 1) return fail(SRK_ERR_UNSUPPORTED, "persistent kernel does not fit an SM (smem %zu)", sm2);
    const int round = M / lpu_of<M>() * 2 + (g.S + lpu_of<M>() - 1) / lpu_of<M>();
    int grid = nsm * per_sm;
    if (p->persist_grid > 0) grid = std::min(grid, p->persist_grid);
    // Tickets in flight ~ grid (x2 with prefetch): the lag between the phases
    // of a WT must exceed that window so a unit rarely finds its
    // dependency unmet; the ring must hold 2*lag+2 WTs for the same reason.
    const int window = grid * (p->persist_prefetch ? 2 : 1);
    PersistParams pp;
    pp.lag = p->persist_lag > 0 ? p->persist_lag : (window + round - 1) / round + 1;
    pp.nslot = 2 * pp.lag + 2;
    pp.prefetch = p->persist_prefetch;
    pp.pad = 0;
    pp.spin_limit = p->spin_limit;
    if (pp.nslot > (int)std::min<size_t>(cap, kMaxSlots)) {
      pp.nslot = (int)std::min<size_t>(cap, kMaxSlots);
      pp.lag = std::min(pp.lag, pp.nslot - 1);
    }
    const long long tickets = (long long)(nwt + 2 * pp.lag) * round;
    grid = (int)std::min<long long>(grid, tickets);
    SRK_CUDA(cudaMemsetAsync(p->ctl, 0, sizeof(Ctl), s));
    k_persist<M, OP, T><<<grid, kThreads, sm2, s>>>(a, g, p->G[0], p->G[1], conjG ? 1 : 0, p->tw, p->scratch, nwt,
                                                   p->ctl, pp);
    SRK_CUDA(cudaGetLastError());
    SRK_CUDA(cudaMemcpyAsync(p->mailbox, &p->ctl->abort, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    SRK_CUDA(cudaMemcpyAsync(p->mailbox_spins, &p->ctl->spins, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             s));
    if (stream_capturing(s)) {
      p->graph_mailbox = true;  // checked by srk_plan_sync after a replay
    } else {
      SRK_CUDA(cudaEventRecord(p->mailbox_ev, s));
      p->mailbox_pending = true;
    }
    p->last_grid = grid;
    p->last_launches = 1;
    p->last_lag = pp.lag;
    p->last_nslot = pp.nslot;
    return SRK_OK;
  }
  const size_t smp1 = p1_smem_bytes<M, OP>();
  SRK_TRY(set_smem(k_p1<M, OP, T>, smp1));
  const bool tan = OP == OP_ADJ && a.dI != nullptr;  // the tangent-adjoint's adjoint-type pass
  if (tan) SRK_TRY(set_smem(k_p1<M, OP, T, true>, smp1));
  SRK_TRY(set_smem(k_p2<M, OP>, sm2));
  SRK_TRY(set_smem(k_p3<M, OP, T>, sm3));
  constexpr int LPU = lpu_of<M>();
  auto launch3 = [&](int w0, int c, float2* base, cudaStream_t s1, cudaStream_t s2, cudaStream_t s3,
                     cudaEvent_t e1, cudaEvent_t e2) -> srk_status {
    const dim3 g1(M / LPU / p1_units<M, OP>(), c);
    if (tan)
      k_p1<M, OP, T, true><<<g1, kThreads, smp1, s1>>>(a, g, p->tw, w0, base, g.S, p->nsm);
    else
      k_p1<M, OP, T><<<g1, kThreads, smp1, s1>>>(a, g, p->tw, w0, base, g.S, p->nsm);
    if (e1) {
      SRK_CUDA(cudaEventRecord(e1, s1));
      SRK_CUDA(cudaStreamWaitEvent(s2, e1, 0));
    }
    k_p2<M, OP><<<dim3(M / LPU, c), kThreads, sm2, s2>>>(base, p->G[0], p->G[1], conjG ? 1 : 0, g, p->tw);
    if (e2) {
      SRK_CUDA(cudaEventRecord(e2, s2));
      SRK_CUDA(cudaStreamWaitEvent(s3, e2, 0));
    }
    k_p3<M, OP, T><<<dim3((g.S + LPU - 1) / LPU, c), kThreads, sm3, s3>>>(base, a, g, p->tw, w0, p->nsm);
    return SRK_OK;
  };
  const int whole = (int)std::min<size_t>(std::max<size_t>(cap, 1), 65535);
  int launches = 0;
  constexpr int R = srk_plan_s::kRing;
  if (nwt <= whole || !p->overlap || !p->ps1 || cap < (size_t)R) {
    // one chunk at a time on the caller's stream
    for (int w0 = 0; w0 < nwt; w0 += whole, launches += 3)
      SRK_TRY(launch3(w0, std::min(whole, nwt - w0), p->scratch, s, s, s, nullptr, nullptr));
  } else {
    // A ring of R scratch slots of `chunk` WTs: P1 (own stream) of chunk k
    // waits for P2 of chunk k-R (the last reader of the slot's S1), P2 (the
    // caller's stream) for P1 of chunk k and P3 of chunk k-R (the last reader
    // of its S2), P3 (own stream) for P2 of chunk k.  The phases of up to
    // three chunks run side by side; both streams fork from and join back
    // into the caller's stream.
    const int chunk = (int)std::min<size_t>(cap / R, 65535);
    const size_t per_slot = (size_t)chunk * per;
    SRK_CUDA(cudaEventRecord(p->ev_fork, s));
    SRK_CUDA(cudaStreamWaitEvent(p->ps1, p->ev_fork, 0));
    SRK_CUDA(cudaStreamWaitEvent(p->ps3, p->ev_fork, 0));
    int k = 0;
    for (int w0 = 0; w0 < nwt; w0 += chunk, ++k, launches += 3) {
      const int r = k % R;
      if (k >= R) {
        SRK_CUDA(cudaStreamWaitEvent(p->ps1, p->ev2[r], 0));
        SRK_CUDA(cudaStreamWaitEvent(s, p->ev3[r], 0));
      }
      SRK_TRY(launch3(w0, std::min(chunk, nwt - w0), p->scratch + r * per_slot, p->ps1, s, p->ps3, p->ev1[r],
                      p->ev2[r]));
      SRK_CUDA(cudaEventRecord(p->ev3[r], p->ps3));
    }
    SRK_CUDA(cudaStreamWaitEvent(s, p->ev3[(k - 1) % R], 0));  // joins P3; P1 joined through P2
  }
  p->last_launches = launches;
  return cuda_status(cudaGetLastError(), "conv launch");
}

template <int OP, typename T>
srk_status launch_conv(srk_plan_s* p, const OpArgs& a, const Geom& g, bool conjG, cudaStream_t s) {
  const int nwt = OpTraits<OP>::PAIRS ? (g.U + 1) / 2 : g.U;
  if (nwt <= 0) return SRK_OK;
  switch (p->M) {
    case 128: return launch_conv_m<128, OP, T>(p, a, g, nwt, conjG, s);
    case 256: return launch_conv_m<256, OP, T>(p, a, g, nwt, conjG, s);
    case 512: return launch_conv_m<512, OP, T>(p, a, g, nwt, conjG, s);
    default: return fail(SRK_ERR_UNSUPPORTED, "tile size %d not built", p->M);
  }
}

}  // namespace srk

#define SRK_INSTANTIATE_CONV(T)                                                                        \
  template srk_status srk::launch_conv<srk::OP_FWD, T>(srk_plan_s*, const srk::OpArgs&, const srk::Geom&, bool, cudaStream_t);      \
  template srk_status srk::launch_conv<srk::OP_VJP_F, T>(srk_plan_s*, const srk::OpArgs&, const srk::Geom&, bool, cudaStream_t);    \
  template srk_status srk::launch_conv<srk::OP_JVP, T>(srk_plan_s*, const srk::OpArgs&, const srk::Geom&, bool, cudaStream_t);      \
  template srk_status srk::launch_conv<srk::OP_TANADJ_F, T>(srk_plan_s*, const srk::OpArgs&, const srk::Geom&, bool, cudaStream_t); \
  template srk_status srk::launch_conv<srk::OP_ADJ, T>(srk_plan_s*, const srk::OpArgs&, const srk::Geom&, bool, cudaStream_t);
