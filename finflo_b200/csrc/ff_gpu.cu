// libfinflo_gpu.so: the C-ABI of the sm_100a FINFLO hot path.
//
// A context owns one CUDA stream and the device copies of the blocks; all
// stage calls are asynchronous on that stream.  The per-cycle sequence of the
// reference's CYCLES (ns3c.f:1354) for one grid level is available both as
// separate stage calls (drop-in replacements of STATIM/RESIDU/IMPS/FIN/BOUNDI)
// and as ff_cycles(), which captures one cycle in a CUDA graph and replays it.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>
#include "ff_kernels.cuh"
#include "ff_grid.cuh"
#include "../../include/finflo_gpu.h"

using namespace ff;

namespace {

struct BlockCtx {
  int imax = 0, jmax = 0, kmax = 0, ntot = 0, npatch = 0;
  double* base = nullptr;       // FF_NSLOTS slots of ntot doubles
  size_t slot_stride = 0;
  ff_patch* d_patch = nullptr;
  std::vector<ff_patch> h_patch;
  ff_params prm{};
  // LU-SGS data in the sweep layout (SW_N x ns) of the upper (sw) and the
  // lower (swl) sweep, and the increments in it (7 x ns), FP64 or FP32 as
  // the block's lusgs_fp32 asks.  sw_static: the metric-only part of both
  // layouts is filled (1 FP64, 2 FP32; 0 after the metrics change).
  double* sw = nullptr;
  double* swl = nullptr;
  double* dwp = nullptr;
  int sw_static = 0;
  // a second stream of the block: the second sweep's coefficient pass runs
  // on it beside the first sweep (fork / join events)
  cudaStream_t aux = nullptr;
  cudaEvent_t aux_fork = nullptr, aux_join = nullptr;
  // DDADI kernel form per direction (index 1..3 = i, j, k): index into
  // DD_CFG, or -1 for one thread per line; the tuner's time of the chosen
  // form per direction
  int dd_cfg[4] = {0, 0, 0, 0};
  float dd_ms[4] = {0.f, 0.f, 0.f, 0.f};
  float* sw32 = nullptr;
  float* swl32 = nullptr;
  float* dwp32 = nullptr;
  size_t ns = 0;
  unsigned long long* d_red = nullptr;   // per-block reduction word (FUN1KO CDMAX)
  int coop_threads = 128;       // threads per CTA of the hyperplane sweep (tune_sweep)
  int use_lines = 0;            // 1: cluster line-wavefront LU-SGS
  int can_lines = 0;            // the line sweep fits one cluster
  int can_pipe = 0, use_pipe = 0;   // pipelined tile wavefront possible / chosen
  int pipe_tk = 0;              // its tile height along k (8, 16 or 32 lines)
  bool pipe_stage = false;
  PipeGeom pg{};
  float pipe_ms = 0.f;          // measured upper sweep of the pipelined kernel
  int tuned = 0;                // sweep kind chosen by tune_sweep
  int res_shape = 0;            // residual tile shape (RES_SHAPES), chosen by tune_residual
  int res_tuned = 0;
  float sweep_ms[2] = {0.f, 0.f};   // measured upper sweep: lines, best hyperplane
  LineGeom lg{};
  bool lines_stage = false;     // the staged line sweep fits (one tile per thread group)
  DevBlock db{};
  cudaGraphExec_t graph = nullptr;
  int graph_fp32 = -1;
  int cycle_launches = 0;       // kernel launches in one captured cycle
  BlockCtx* coarse = nullptr;   // next multigrid level (MGRID > 1)
  int level = 1;
};

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<BlockCtx*> blocks;
  unsigned* d_bar = nullptr;            // grid barrier {count, generation}
  int* d_err = nullptr;                 // sweep time-out flag
  double* d_resi = nullptr;             // 5 sums of squares
  unsigned long long* d_dromax = nullptr;
  double* d_hist = nullptr;             // per-cycle {resi[5], dromax}
  int* d_hist_pos = nullptr;
  int hist_cap = 0;
  int sm_count = 0;
  int smem_optin = 0;                   // shared memory a CTA may opt in to
  int coop_occ[2][2][3] = {};           // CTAs per SM of k_lusgs_sweep<f64|f32, 5|7> at 64/128/256 threads
  char errmsg[256] = {0};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  long nlaunch = 0;                     // kernel launches issued so far
  bool side_by_side = false;            // inside fork_join's concurrent chains
  // multi-block: per-block streams for the concurrent chains inside a
  // captured cycle, the device block table and the connection work-list
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> side_ev;
  cudaEvent_t fork_ev = nullptr;
  std::vector<BlockCtx*> tops;          // level-1 blocks (a multigrid block's coarse levels hang off them)
  DevBlock* d_blocks = nullptr;
  ConnItem* d_conn = nullptr;
  int nconn = 0, maxconn = 1, conn_blocks = -1;
  cudaGraphExec_t mb_graph = nullptr;
  int mb_graph_n = -1;
  int mb_launches = 0;
  // halo exchange with blocks on other GPUs
  HaloItem* d_halo = nullptr;
  int nhalo = 0, halo_maxn = 1;
  bool halo_pack = false, halo_unpack = false;
  double *halo_send = nullptr, *halo_recv = nullptr;
  cudaGraphExec_t phase_graph[2] = {nullptr, nullptr};
};

int fail(Ctx* c, int code, const char* what, cudaError_t e = cudaSuccess) {
  if (c) snprintf(c->errmsg, sizeof(c->errmsg), "%s%s%s", what, e != cudaSuccess ? ": " : "",
                  e != cudaSuccess ? cudaGetErrorString(e) : "");
  return code;
}
#define CK(call)                                                   \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return fail(c, FF_ERR_CUDA, #call, e_); \
  } while (0)

inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

BlockCtx* getb(Ctx* c, int blk) {
  if (!c || blk < 0 || blk >= (int)c->blocks.size()) return nullptr;
  return c->blocks[blk];
}

// __global__ helpers for the cycle history
__global__ void k_reset_acc(double* resi, unsigned long long* dm) {
  if (threadIdx.x < 5) resi[threadIdx.x] = 0.;
  if (threadIdx.x == 0) *dm = 0ull;
}
__global__ void k_record(const double* resi, const unsigned long long* dm, double* hist, int* pos, int cap) {
  int p = *pos;
  if (p < cap) {
    for (int v = 0; v < 5; v++) hist[6 * p + v] = resi[v];
    hist[6 * p + 5] = __longlong_as_double((long long)*dm);
  }
  *pos = p + 1;
}

int launch_patch(Ctx* c, BlockCtx* b, void (*kern)(DevBlock, ff_params, int), int arg) {
  if (b->npatch == 0) return 0;
  int maxn = 1;
  for (auto& p : b->h_patch) maxn = max(maxn, (p.r1b - p.r1a + 1) * (p.r2b - p.r2a + 1));
  dim3 g(nblk(maxn, 128), b->npatch);
  kern<<<g, 128, 0, c->stream>>>(b->db, b->prm, arg);
  c->nlaunch++;
  return 0;
}

// ---- stages -----------------------------------------------------------------
// STATIM: equation of state and REFLEC; npass = 2 repeats them on the patch
// ghosts (BOUNDI calls STATIM twice, ns3c.f:10896, 10905).
int st_statim(Ctx* c, BlockCtx* b, int npass = 2) {
  k_state<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db, b->prm);
  c->nlaunch++;
  launch_patch(c, b, k_reflec, 0);
  if (npass > 1) launch_patch(c, b, k_reflec, 1);
  return 0;
}

int st_boundi(Ctx* c, BlockCtx* b) {
  k_refcor<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db);
  c->nlaunch++;
  if (b->npatch) {
    int maxn = 1;
    for (auto& p : b->h_patch) maxn = max(maxn, (p.r1b - p.r1a + 1) * (p.r2b - p.r2a + 1));
    k_mir<<<dim3(nblk(maxn, 128), b->npatch), 128, 0, c->stream>>>(b->db);
    c->nlaunch++;
  }
  return st_statim(c, b);
}

// TURBEQ res3c.f:5845 (level 1 at the start of the cycle, m2 = 1) and
// RESIKE res3c.f:3423 (k-omega SST) on a level; for m2 >= 2 RESIKE
// recomputes the velocity gradients of the level itself.
// Threads per CTA of the residual kernels: the same 32x4x4 tile and
// arithmetic.  Measured on B200 with one face work list per tile (128 /
// 256 / 512 threads): SST 0.798 / 0.514 / 0.403 ms on 128x64x64 cells,
// laminar 0.136 / 0.073 / 0.047 ms on 64x32x32; with one barrier per
// direction (FINFLO_RES_FUSED=0) SST 0.571 / 0.457 / 0.500 ms.
// FINFLO_RES_THREADS overrides.
int res_threads(bool sst) {
  static const int env = [] {
    const char* e = getenv("FINFLO_RES_THREADS");
    const int v = e ? atoi(e) : 0;
    return (v == 128 || v == 256 || v == 512) ? v : 0;
  }();
  (void)sst;
  return env ? env : 512;
}

template <int NT>
void launch_residual_t(cudaStream_t st, dim3 g, const BlockCtx* b, int level, bool sst) {
  // face buffer + running sums of the 32x4x4 tile, NV values each
  const size_t sm = (size_t)(sst ? 7 : 5) * (TI * (TJ + 1) * TK + TI * TJ * TK) * sizeof(double);
  if (sst) {
    cudaFuncSetAttribute(k_residual_sst<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_residual_sst<NT><<<g, NT, sm, st>>>(b->db, b->prm, level);
  } else {
    cudaFuncSetAttribute(k_residual<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_residual<NT><<<g, NT, sm, st>>>(b->db, b->prm, level);
  }
}

// One face work list per tile (k_residual_fused) unless FINFLO_RES_FUSED=0.
bool res_fused() {
  static const bool f = [] { const char* e = getenv("FINFLO_RES_FUSED"); return !(e && !strcmp(e, "0")); }();
  return f;
}

template <int NV, int NT, int I_, int J_, int K_, bool ST = false, typename FT = double, bool ALT = false>
void launch_residual_fused_s(cudaStream_t st, const BlockCtx* b, int level) {
  dim3 g(nblk(b->imax, I_), nblk(b->jmax, J_), nblk(b->kmax, K_));
  const size_t sm = residual_fused_smem(NV, I_, J_, K_, ST);
  cudaFuncSetAttribute(k_residual_fused<NV, NT, I_, J_, K_, ST, FT, ALT>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_residual_fused<NV, NT, I_, J_, K_, ST, FT, ALT><<<g, NT, sm, st>>>(b->db, b->prm, level);
}

template <int NV, int NT>
void launch_residual_fused_t(cudaStream_t st, dim3 g, const BlockCtx* b, int level) {
  (void)g;
  // the form the autotuner chose for this block (512 threads only): tile
  // shape, and the stencil staged in shared memory or not
  const int sh = NT == 512 ? b->res_shape : 0;
  // another IFLUX scheme, XXTRAA or JAMESON: the kernel with those variants
  // compiled in, in the default 32x4x4 unstaged form
  if (residual_alt(b->prm, level)) return launch_residual_fused_s<NV, NT, 32, 4, 4, false, double, true>(st, b, level);
  // a coarse level's face fluxes in FP32 (unstaged tiles; Roe with XXTRAP)
  if (level > 1 && b->prm.res_fp32) {
    const int s3 = sh % RES_NSHAPE;
    if (s3 == 1) return launch_residual_fused_s<NV, NT, 16, 8, 4, false, float>(st, b, level);
    if (s3 == 2) return launch_residual_fused_s<NV, NT, 8, 8, 8, false, float>(st, b, level);
    return launch_residual_fused_s<NV, NT, 32, 4, 4, false, float>(st, b, level);
  }
  if constexpr (NT == 512) {
    if (sh == 3) return launch_residual_fused_s<NV, NT, 32, 4, 4, true>(st, b, level);
    if (sh == 4) return launch_residual_fused_s<NV, NT, 16, 8, 4, true>(st, b, level);
    if (sh == 5) return launch_residual_fused_s<NV, NT, 8, 8, 8, true>(st, b, level);
  }
  if (sh == 1) return launch_residual_fused_s<NV, NT, 16, 8, 4>(st, b, level);
  if (sh == 2) return launch_residual_fused_s<NV, NT, 8, 8, 8>(st, b, level);
  launch_residual_fused_s<NV, NT, 32, 4, 4>(st, b, level);
}

void launch_residual(cudaStream_t st, const BlockCtx* b, int level) {
  dim3 g(nblk(b->imax, TI), nblk(b->jmax, TJ), nblk(b->kmax, TK));
  const bool sst = b->prm.iturb >= 3;
  if (res_fused()) {
    switch (res_threads(sst)) {
      case 128: sst ? launch_residual_fused_t<7, 128>(st, g, b, level) : launch_residual_fused_t<5, 128>(st, g, b, level); break;
      case 512: sst ? launch_residual_fused_t<7, 512>(st, g, b, level) : launch_residual_fused_t<5, 512>(st, g, b, level); break;
      default: sst ? launch_residual_fused_t<7, 256>(st, g, b, level) : launch_residual_fused_t<5, 256>(st, g, b, level);
    }
    return;
  }
  switch (res_threads(sst)) {
    case 128: launch_residual_t<128>(st, g, b, level, sst); break;
    case 512: launch_residual_t<512>(st, g, b, level, sst); break;
    default: launch_residual_t<256>(st, g, b, level, sst);
  }
}

// part: 0 the whole stage, 1 the kernels before the residual's face pass
// (gradients, sources, ghost updates), 2 the kernels after it -- so that a
// multi-block cycle can run the face pass of all blocks in one launch.
// SCALARD res3c.f:146, 3599: the JAMESON scale, first in the stage, before
// the inlet/outlet ghost update (finest level, RJK2 or RJK4 > 0).
static void launch_scalard(Ctx* c, BlockCtx* b, int level) {
  if (level != 1 || !(b->prm.rjk2 > 0. || b->prm.rjk4 > 0.)) return;
  const long n = (long)(b->imax + 2) * (b->jmax + 2) * (b->kmax + 2);
  k_scalard<<<nblk(n, 256), 256, 0, c->stream>>>(b->db);
  c->nlaunch++;
}

int st_residu_sst(Ctx* c, BlockCtx* b, int level, int m2, int icycle, int part = 0) {
  if (part == 2) goto post;
  {
  launch_scalard(c, b, level);
  const int ncell = b->imax * b->jmax * b->kmax;
  int gg = level == 1 ? 2 : 0;
  long ng = (long)(b->imax + gg) * (b->jmax + gg) * (b->kmax + gg);
  if (m2 >= 2 || level == 1) {   // DERFUN (+ TEMDER of T) of this level
    k_grad<<<nblk(ng, 128), 128, 0, c->stream>>>(b->db, level);
    c->nlaunch++;
  }
  if (level == 1 && m2 == 1) {
    k_eps2ko<<<nblk(ncell, 128), 128, 0, c->stream>>>(b->db, b->prm);
    c->nlaunch++;
  }
  k_crosko<<<nblk(ncell, 128), 128, 0, c->stream>>>(b->db);
  k_rk_roundtrip<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db);
  CK(cudaMemsetAsync(b->d_red, 0, sizeof(unsigned long long), c->stream));
  k_cdmax<<<min(nblk(b->ntot, 256), 4 * c->sm_count), 256, 0, c->stream>>>(b->db, b->d_red);
  k_fun1ko<<<nblk(ncell, 128), 128, 0, c->stream>>>(b->db, b->prm, b->d_red);
  c->nlaunch += 4;
  if (b->npatch && level == 1) {
    int maxn = 1;
    for (auto& p : b->h_patch) maxn = max(maxn, (p.r1b - p.r1a + 1) * (p.r2b - p.r2a + 1));
    k_refcen<<<dim3(nblk(maxn, 128), b->npatch), 128, 0, c->stream>>>(b->db, b->prm);
    c->nlaunch++;
  }
  k_prodke<<<nblk((long)b->jmax * b->db.is * b->kmax, 128), 128, 0, c->stream>>>(b->db);
  c->nlaunch++;
  if (b->prm.fullns) {
    long nt3 = (long)(b->imax + gg) * (b->jmax + gg) * ((level == 1 && b->kmax > 1) ? b->kmax + 2 : b->kmax);
    k_temder_ke<<<nblk(nt3, 128), 128, 0, c->stream>>>(b->db, level);
    c->nlaunch++;
  }
  if (level == 1) launch_patch(c, b, k_inlet_outlet, icycle);
  }
  if (part == 1) return 0;
  if (part == 0) {
    launch_residual(c->stream, b, level);
    c->nlaunch++;
  }
post:
  const int ncell = b->imax * b->jmax * b->kmax;
  k_sourko_addske<<<nblk(ncell, 128), 128, 0, c->stream>>>(b->db);
  c->nlaunch++;
  if (b->prm.timel && level == 1) {   // TIMDER + TIMDKE after ADDSKE (res3c.f:5097)
    k_timder<7><<<nblk(ncell, 256), 256, 0, c->stream>>>(b->db, b->prm);
    c->nlaunch++;
  }
  return 0;
}

int st_residu(Ctx* c, BlockCtx* b, int level, int icycle, int m2 = 1, int part = 0) {
  if (b->prm.iturb >= 3) return st_residu_sst(c, b, level, m2, icycle, part);
  if (part != 2) {
    launch_scalard(c, b, level);
    if (level == 1) {
      if (b->npatch) {
        int maxn = 1;
        for (auto& p : b->h_patch) maxn = max(maxn, (p.r1b - p.r1a + 1) * (p.r2b - p.r2a + 1));
        k_refcen<<<dim3(nblk(maxn, 128), b->npatch), 128, 0, c->stream>>>(b->db, b->prm);
        c->nlaunch++;
      }
    }
    if (b->prm.fullns && level == 1) {
      long ng = (long)(b->imax + 2) * (b->jmax + 2) * (b->kmax + 2);
      k_grad<<<nblk(ng, 128), 128, 0, c->stream>>>(b->db, level);
      c->nlaunch++;
    }
    if (level == 1) launch_patch(c, b, k_inlet_outlet, icycle);
    if (part == 1) return 0;
    launch_residual(c->stream, b, level);
    c->nlaunch++;
  }
  if (b->prm.timel && level == 1) {   // TIMDER after SWEEP (res3c.f:705)
    k_timder<5><<<nblk((long)b->imax * b->jmax * b->kmax, 256), 256, 0, c->stream>>>(b->db, b->prm);
    c->nlaunch++;
  }
  return 0;
}

// The residual face pass of several level-1 blocks in one launch over their
// tiles (k_residual_batch, RB_MAX blocks per launch); every block must have
// the same equation count.  The tile shape is the first block's.
template <int NV, int I_, int J_, int K_, bool ST = false>
void launch_residual_batch_t(cudaStream_t st, const ResBatch& rb, int level) {
  const size_t sm = residual_fused_smem(NV, I_, J_, K_, ST);
  cudaFuncSetAttribute(k_residual_batch<NV, 512, I_, J_, K_, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sm);
  k_residual_batch<NV, 512, I_, J_, K_, ST><<<rb.tile0[rb.nblk], 512, sm, st>>>(rb, level);
}

int launch_residual_batch(Ctx* c, const std::vector<BlockCtx*>& blks, int level) {
  const int shape = blks[0]->res_shape;
  const bool sst = blks[0]->prm.iturb >= 3;
  const int ti = RES_SHAPES[shape % RES_NSHAPE][0], tj = RES_SHAPES[shape % RES_NSHAPE][1],
            tk = RES_SHAPES[shape % RES_NSHAPE][2];
  for (size_t s0 = 0; s0 < blks.size(); s0 += RB_MAX) {
    static ResBatch rb;   // ~19 KB: kept off the host stack
    rb = ResBatch{};
    rb.nblk = (int)min(blks.size() - s0, (size_t)RB_MAX);
    rb.tile0[0] = 0;
    for (int n = 0; n < rb.nblk; n++) {
      const BlockCtx* b = blks[s0 + n];
      if ((b->prm.iturb >= 3) != sst) return fail(c, FF_ERR_ARG, "batched residual: mixed equation counts");
      rb.ntx[n] = nblk(b->imax, ti);
      rb.nty[n] = nblk(b->jmax, tj);
      rb.tile0[n + 1] = rb.tile0[n] + rb.ntx[n] * rb.nty[n] * nblk(b->kmax, tk);
      rb.b[n] = b->db;
      rb.p[n] = b->prm;
    }
    switch (shape) {
      case 1: sst ? launch_residual_batch_t<7, 16, 8, 4>(c->stream, rb, level)
                  : launch_residual_batch_t<5, 16, 8, 4>(c->stream, rb, level); break;
      case 2: sst ? launch_residual_batch_t<7, 8, 8, 8>(c->stream, rb, level)
                  : launch_residual_batch_t<5, 8, 8, 8>(c->stream, rb, level); break;
      case 3: sst ? launch_residual_batch_t<7, 32, 4, 4, true>(c->stream, rb, level)
                  : launch_residual_batch_t<5, 32, 4, 4, true>(c->stream, rb, level); break;
      case 4: sst ? launch_residual_batch_t<7, 16, 8, 4, true>(c->stream, rb, level)
                  : launch_residual_batch_t<5, 16, 8, 4, true>(c->stream, rb, level); break;
      case 5: sst ? launch_residual_batch_t<7, 8, 8, 8, true>(c->stream, rb, level)
                  : launch_residual_batch_t<5, 8, 8, 8, true>(c->stream, rb, level); break;
      default: sst ? launch_residual_batch_t<7, 32, 4, 4>(c->stream, rb, level)
                   : launch_residual_batch_t<5, 32, 4, 4>(c->stream, rb, level);
    }
    c->nlaunch++;
  }
  CK(cudaGetLastError());
  return 0;
}

// Batched face pass in the multi-block cycles unless FINFLO_RES_BATCH=0;
// only with the fused 512-thread residual and one equation count.
bool res_batch_ok(Ctx* c) {
  static const bool env = [] { const char* e = getenv("FINFLO_RES_BATCH"); return !(e && !strcmp(e, "0")); }();
  if (!env || !res_fused() || c->tops.size() < 2) return false;
  const bool sst = c->tops[0]->prm.iturb >= 3;
  if (res_threads(sst) != 512) return false;
  for (auto* b : c->tops)
    if ((b->prm.iturb >= 3) != sst || residual_alt(b->prm, 1)) return false;
  return true;
}

// The sweep-layout buffer of one sweep (upper = 1: the first, CORRGS
// order; 0: PREDGS), FP64 or FP32.
inline double* swd(const BlockCtx* b, int upper) { return upper ? b->sw : b->swl; }
inline float* swf(const BlockCtx* b, int upper) { return upper ? b->sw32 : b->swl32; }

// Sweep-layout buffers in the block's LU-SGS precision (the other
// precision's are freed).
int alloc_sweep(Ctx* c, BlockCtx* b) {
  const size_t ns = b->ns;
  b->sw_static = 0;
  if (b->prm.lusgs_fp32) {
    cudaFree(b->sw); cudaFree(b->swl); cudaFree(b->dwp);
    b->sw = nullptr; b->swl = nullptr; b->dwp = nullptr;
    if (!b->sw32) CK(cudaMalloc(&b->sw32, sizeof(float) * SW_N * ns));
    if (!b->swl32) CK(cudaMalloc(&b->swl32, sizeof(float) * SW_N * ns));
    if (!b->dwp32) CK(cudaMalloc(&b->dwp32, sizeof(float) * 7 * ns));
  } else {
    cudaFree(b->sw32); cudaFree(b->swl32); cudaFree(b->dwp32);
    b->sw32 = nullptr; b->swl32 = nullptr; b->dwp32 = nullptr;
    if (!b->sw) CK(cudaMalloc(&b->sw, sizeof(double) * SW_N * ns));
    if (!b->swl) CK(cudaMalloc(&b->swl, sizeof(double) * SW_N * ns));
    if (!b->dwp) CK(cudaMalloc(&b->dwp, sizeof(double) * 7 * ns));
  }
  return 0;
}

// Grid of the cooperative hyperplane sweep: enough threads for the widest
// plane (JMAX x KMAX cells), at most what can be co-resident.
int coop_grid(Ctx* c, BlockCtx* b, bool fp32, int threads) {
  int ti = threads == 64 ? 0 : (threads == 128 ? 1 : 2);
  long per_sm = c->coop_occ[fp32 ? 1 : 0][b->prm.iturb >= 3 ? 1 : 0][ti];
  long widest = (long)b->jmax * b->kmax;
  return (int)min(per_sm * c->sm_count, max(1L, (widest + threads - 1) / threads));
}

int coop_sweep_n(Ctx* c, BlockCtx* b, int upper, bool fp32, int threads) {
  int nb = coop_grid(c, b, fp32, threads);
  if (nb < 1) return fail(c, FF_ERR_CUDA, "no cooperative occupancy");
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nb);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e;
  const bool ke = b->prm.iturb >= 3;   // seven equations (k-omega)
  if (!fp32) {
    e = ke ? cudaLaunchKernelEx(&cfg, k_lusgs_sweep<double, 7>, b->db, (const double*)swd(b, upper), b->dwp,
                                upper, c->d_bar, c->d_err)
           : cudaLaunchKernelEx(&cfg, k_lusgs_sweep<double, 5>, b->db, (const double*)swd(b, upper), b->dwp,
                                upper, c->d_bar, c->d_err);
  } else {
    e = ke ? cudaLaunchKernelEx(&cfg, k_lusgs_sweep<float, 7>, b->db, (const float*)swf(b, upper), b->dwp32,
                                upper, c->d_bar, c->d_err)
           : cudaLaunchKernelEx(&cfg, k_lusgs_sweep<float, 5>, b->db, (const float*)swf(b, upper), b->dwp32,
                                upper, c->d_bar, c->d_err);
  }
  if (e != cudaSuccess) return fail(c, FF_ERR_CUDA, "cooperative sweep launch", e);
  c->nlaunch++;
  return 0;
}

int coop_sweep(Ctx* c, BlockCtx* b, int upper, bool fp32) {
  return coop_sweep_n(c, b, upper, fp32, b->coop_threads);
}

template <typename CT, int NV>
cudaError_t launch_lines(cudaLaunchConfig_t* cfg, BlockCtx* b, const CT* sw, CT* dwp, int upper, bool stage) {
  return stage ? cudaLaunchKernelEx(cfg, k_lusgs_lines<CT, NV, true>, b->db, sw, dwp, upper, b->lg)
               : cudaLaunchKernelEx(cfg, k_lusgs_lines<CT, NV, false>, b->db, sw, dwp, upper, b->lg);
}

// The staged line sweep for a block swept alone; the unstaged one when
// several blocks' sweeps run side by side (fork_join).
int lines_sweep(Ctx* c, BlockCtx* b, int upper, bool fp32) {
  const bool stage = b->lines_stage && !c->side_by_side;
  const int nv = b->prm.iturb >= 3 ? 7 : 5;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(b->lg.cs);
  cfg.blockDim = dim3(LTHREADS * b->lg.ng);
  cfg.dynamicSmemBytes = lines_smem_bytes(nv, b->lg.tpc, fp32 ? sizeof(float) : sizeof(double), stage);
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = b->lg.cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  static const int prio = [] {
    const char* e = getenv("FINFLO_SWEEP_PRIO");
    int lo = 0, hi = 0;
    if (!e || !strcmp(e, "0") || cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess) return 1;
    return hi;
  }();
  if (c->side_by_side && prio <= 0) {   // side by side: the sweeps' CTAs first
    attr[1].id = cudaLaunchAttributePriority;
    attr[1].val.priority = prio;
    cfg.numAttrs = 2;
  }
  cudaError_t e;
  if (nv == 7)
    e = fp32 ? launch_lines<float, 7>(&cfg, b, swf(b, upper), b->dwp32, upper, stage)
             : launch_lines<double, 7>(&cfg, b, swd(b, upper), b->dwp, upper, stage);
  else
    e = fp32 ? launch_lines<float, 5>(&cfg, b, swf(b, upper), b->dwp32, upper, stage)
             : launch_lines<double, 5>(&cfg, b, swd(b, upper), b->dwp, upper, stage);
  if (e != cudaSuccess) return fail(c, FF_ERR_CUDA, "cluster sweep launch", e);
  c->nlaunch++;
  return 0;
}

constexpr int kMaxDev = 64;
int g_lines_smem[kMaxDev][4];   // dynamic shared memory granted to k_lusgs_lines<f64|f32, 5|7, *>

template <typename CT, int NV>
int lines_attr_set(Ctx* c, size_t smem) {
  CK(cudaFuncSetAttribute(k_lusgs_lines<CT, NV, true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  CK(cudaFuncSetAttribute(k_lusgs_lines<CT, NV, false>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  CK(cudaFuncSetAttribute(k_lusgs_lines<CT, NV, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CK(cudaFuncSetAttribute(k_lusgs_lines<CT, NV, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return 0;
}

// Kernel attributes are per device, shared by all blocks: only raise them.
template <int NV>
int lines_attrs(Ctx* c, size_t sm64, size_t sm32) {
  int* g = g_lines_smem[c->device] + (NV == 7 ? 2 : 0);
  if ((int)sm64 > g[0]) {
    int rc = lines_attr_set<double, NV>(c, sm64);
    if (rc) return rc;
    g[0] = (int)sm64;
  }
  if ((int)sm32 > g[1]) {
    int rc = lines_attr_set<float, NV>(c, sm32);
    if (rc) return rc;
    g[1] = (int)sm32;
  }
  return 0;
}

// Choose the LU-SGS sweep kernel of a block: the cluster line wavefront
// when the (j,k) line tiles fit one cluster, else the cooperative hyperplane
// kernel.  The largest cluster that fits is taken; a smaller cluster only
// means more tiles per CTA.
int setup_lines(Ctx* c, BlockCtx* b) {
  LineGeom lg{};
  lg.ntj = (b->jmax + LTJ - 1) / LTJ;
  lg.ntk = (b->kmax + LTK - 1) / LTK;
  lg.ntiles = lg.ntj * lg.ntk;
  const int nv = b->prm.iturb >= 3 ? 7 : 5;
  if (c->device < 0 || c->device >= kMaxDev) return fail(c, FF_ERR_ARG, "device id");
  // FINFLO_LINES_CS caps the cluster size (16 by default): smaller clusters
  // let more blocks' sweeps run side by side in a multi-block cycle
  static const int cs_max = [] {
    const char* e = getenv("FINFLO_LINES_CS");
    const int v = e ? atoi(e) : 16;
    return (v == 1 || v == 2 || v == 4 || v == 8) ? v : 16;
  }();
  for (int cs = cs_max; cs >= 1; cs /= 2) {
    int csz = min(cs, lg.ntiles);
    int tpc = (lg.ntiles + csz - 1) / csz;
    int ng = min(tpc, LMAX_TPC);
    // staging needs one tile per thread group and room for the stage
    bool stage = tpc == ng && tpc <= LMAX_TPC_STAGE &&
                 lines_smem_bytes(nv, tpc, sizeof(double), true) <= (size_t)c->smem_optin;
    size_t sm64 = lines_smem_bytes(nv, tpc, sizeof(double), stage);
    size_t sm32 = lines_smem_bytes(nv, tpc, sizeof(float), stage);
    if (sm64 > (size_t)c->smem_optin) continue;
    int rc = nv == 7 ? lines_attrs<7>(c, sm64, sm32) : lines_attrs<5>(c, sm64, sm32);
    if (rc) return rc;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(csz);
    cfg.blockDim = dim3(LTHREADS * ng);
    cfg.dynamicSmemBytes = sm64;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csz; attr[0].val.clusterDim.y = 1; attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    cudaError_t e;
    if (nv == 7)
      e = stage ? cudaOccupancyMaxActiveClusters(&nclusters, k_lusgs_lines<double, 7, true>, &cfg)
                : cudaOccupancyMaxActiveClusters(&nclusters, k_lusgs_lines<double, 7, false>, &cfg);
    else
      e = stage ? cudaOccupancyMaxActiveClusters(&nclusters, k_lusgs_lines<double, 5, true>, &cfg)
                : cudaOccupancyMaxActiveClusters(&nclusters, k_lusgs_lines<double, 5, false>, &cfg);
    if (e != cudaSuccess || nclusters < 1) {
      cudaGetLastError();
      continue;
    }
    lg.cs = csz;
    lg.tpc = tpc;
    lg.ng = ng;
    b->lg = lg;
    b->lines_stage = stage;
    b->use_lines = 1;
    b->can_lines = 1;
    return 0;
  }
  b->use_lines = 0;
  b->can_lines = 0;
  return 0;
}
// ---- all blocks' line sweeps in one launch ----------------------------------
// The blocks of one multigrid level, swept together by k_lusgs_lines_batch:
// one cluster per block, every cluster of the launch the same size (the
// smallest of the blocks' own), so a block with a larger own cluster gets
// more tiles per CTA.  Returns false when a block cannot be swept this way.
struct LinesBatchShape {
  int cs = 0, threads = 0;
  size_t smem = 0;
};

bool lines_batch_shape(Ctx* c, const std::vector<BlockCtx*>& v, size_t elem, LinesBatchShape& sh,
                       std::vector<LineGeom>* geoms = nullptr) {
  sh = LinesBatchShape{};
  int cs = 16;
  for (auto* b : v) {
    if (!b->can_lines || b->prm.ddadi) return false;
    cs = min(cs, b->lg.cs);
  }
  if (geoms) geoms->clear();
  int ng_max = 1;
  for (auto* b : v) {
    LineGeom g = b->lg;
    if (g.cs != cs) {
      g.cs = cs;
      g.tpc = (g.ntiles + cs - 1) / cs;
      g.ng = min(g.tpc, LMAX_TPC);
    }
    const int nv = b->prm.iturb >= 3 ? 7 : 5;
    sh.smem = max(sh.smem, lines_smem_bytes(nv, g.tpc, elem, false));
    ng_max = max(ng_max, g.ng);
    if (geoms) geoms->push_back(g);
  }
  sh.cs = cs;
  sh.threads = LTHREADS * ng_max;
  return sh.smem <= (size_t)c->smem_optin;
}

int g_lb_smem[kMaxDev][4];   // dynamic shared memory granted to k_lusgs_lines_batch<f64|f32, 5|7>

template <typename CT, int NV>
int lines_batch_launch(Ctx* c, const std::vector<BlockCtx*>& v, int upper) {
  const bool fp32 = sizeof(CT) == 4;
  for (size_t s0 = 0; s0 < v.size(); s0 += LB_MAX) {
    std::vector<BlockCtx*> part(v.begin() + s0, v.begin() + min(v.size(), s0 + LB_MAX));
    LinesBatchShape sh;
    std::vector<LineGeom> geoms;
    if (!lines_batch_shape(c, part, sizeof(CT), sh, &geoms))
      return fail(c, FF_ERR_ARG, "batched line sweep: a block does not fit");
    int& granted = g_lb_smem[c->device][(fp32 ? 1 : 0) + (NV == 7 ? 2 : 0)];
    if ((int)sh.smem > granted) {
      CK(cudaFuncSetAttribute(k_lusgs_lines_batch<CT, NV>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
      CK(cudaFuncSetAttribute(k_lusgs_lines_batch<CT, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sh.smem));
      granted = (int)sh.smem;
    }
    static LinesBatch lb;   // ~15 KB: kept off the host stack
    lb = LinesBatch{};
    lb.n = (int)part.size();
    for (int n = 0; n < lb.n; n++) {
      BlockCtx* b = part[n];
      lb.upper[n] = upper ? (b->prm.predgs_full ? 3 : 1) : 0;
      lb.lg[n] = geoms[n];
      lb.sw[n] = fp32 ? (const void*)swf(b, upper) : (const void*)swd(b, upper);
      lb.dwp[n] = fp32 ? (void*)b->dwp32 : (void*)b->dwp;
      lb.b[n] = b->db;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(lb.n * sh.cs);
    cfg.blockDim = dim3(sh.threads);
    cfg.dynamicSmemBytes = sh.smem;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = sh.cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_lusgs_lines_batch<CT, NV>, lb);
    if (e != cudaSuccess) return fail(c, FF_ERR_CUDA, "batched line sweep launch", e);
    c->nlaunch++;
  }
  return 0;
}

// One sweep (upper = 1: PREDGS order, 0: CORRGS) of every block of v, one
// launch per equation count and precision.
int lines_batch(Ctx* c, const std::vector<BlockCtx*>& v, int upper) {
  for (int nv : {5, 7})
    for (int fp32 : {0, 1}) {
      std::vector<BlockCtx*> g;
      for (auto* b : v)
        if ((b->prm.iturb >= 3 ? 7 : 5) == nv && (b->prm.lusgs_fp32 != 0) == (fp32 != 0)) g.push_back(b);
      if (g.empty()) continue;
      int rc = nv == 7 ? (fp32 ? lines_batch_launch<float, 7>(c, g, upper) : lines_batch_launch<double, 7>(c, g, upper))
                       : (fp32 ? lines_batch_launch<float, 5>(c, g, upper) : lines_batch_launch<double, 5>(c, g, upper));
      if (rc) return rc;
    }
  return 0;
}

// ---- pipelined tile wavefront (k_lusgs_pipe) ------------------------------
template <typename CT, int NV, int TK, bool ST>
cudaError_t pipe_launch(cudaLaunchConfig_t* cfg, BlockCtx* b, const CT* sw, CT* dwp, int upper, int* err) {
  return cudaLaunchKernelEx(cfg, k_lusgs_pipe<CT, NV, TK, ST>, b->db, sw, dwp, upper, b->pg, err);
}

template <typename CT, int NV, int TK>
cudaError_t pipe_launch_st(cudaLaunchConfig_t* cfg, BlockCtx* b, const CT* sw, CT* dwp, int upper, int* err,
                           bool st) {
  return st ? pipe_launch<CT, NV, TK, true>(cfg, b, sw, dwp, upper, err)
            : pipe_launch<CT, NV, TK, false>(cfg, b, sw, dwp, upper, err);
}

template <typename CT, int NV>
cudaError_t pipe_launch_tk(cudaLaunchConfig_t* cfg, BlockCtx* b, const CT* sw, CT* dwp, int upper, int* err) {
  switch (b->pipe_tk) {
    case 8: return pipe_launch_st<CT, NV, 8>(cfg, b, sw, dwp, upper, err, b->pipe_stage);
    case 16: return pipe_launch_st<CT, NV, 16>(cfg, b, sw, dwp, upper, err, b->pipe_stage);
    default: return pipe_launch_st<CT, NV, 32>(cfg, b, sw, dwp, upper, err, b->pipe_stage);
  }
}

int pipe_sweep(Ctx* c, BlockCtx* b, int upper, bool fp32) {
  const int nv = b->prm.iturb >= 3 ? 7 : 5;
  const int ntiles = b->pg.ntj * b->pg.ntk;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ntiles);
  cfg.blockDim = dim3(PTJ * b->pipe_tk);
  cfg.dynamicSmemBytes = pipe_smem_bytes(nv, b->pipe_tk, fp32 ? sizeof(float) : sizeof(double), b->pipe_stage);
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = ntiles;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e;
  if (nv == 7)
    e = fp32 ? pipe_launch_tk<float, 7>(&cfg, b, swf(b, upper), b->dwp32, upper, c->d_err)
             : pipe_launch_tk<double, 7>(&cfg, b, swd(b, upper), b->dwp, upper, c->d_err);
  else
    e = fp32 ? pipe_launch_tk<float, 5>(&cfg, b, swf(b, upper), b->dwp32, upper, c->d_err)
             : pipe_launch_tk<double, 5>(&cfg, b, swd(b, upper), b->dwp, upper, c->d_err);
  if (e != cudaSuccess) return fail(c, FF_ERR_CUDA, "pipelined sweep launch", e);
  c->nlaunch++;
  return 0;
}

int g_pipe_smem[kMaxDev][2][2][3][2];   // granted dynamic shared memory per device and instantiation

template <typename CT, int NV, int TK, bool ST>
int pipe_attr(Ctx* c, size_t smem) {
  int& g = g_pipe_smem[c->device][sizeof(CT) == 4][NV == 7][TK == 8 ? 0 : (TK == 16 ? 1 : 2)][ST];
  if ((int)smem <= g) return 0;
  CK(cudaFuncSetAttribute(k_lusgs_pipe<CT, NV, TK, ST>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  CK(cudaFuncSetAttribute(k_lusgs_pipe<CT, NV, TK, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  g = (int)smem;
  return 0;
}

template <typename CT, int NV, int TK, bool ST>
int pipe_fits(Ctx* c, int ntiles, size_t smem, bool* ok) {
  *ok = false;
  int rc = pipe_attr<CT, NV, TK, ST>(c, smem);
  if (rc) return rc;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ntiles);
  cfg.blockDim = dim3(PTJ * TK);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = ntiles; attr[0].val.clusterDim.y = 1; attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  cudaError_t e = cudaOccupancyMaxActiveClusters(&n, k_lusgs_pipe<CT, NV, TK, ST>, &cfg);
  if (e != cudaSuccess) { cudaGetLastError(); return 0; }
  *ok = n >= 1;
  return 0;
}

template <typename CT, int NV, int TK>
int pipe_try(Ctx* c, BlockCtx* b, int ntiles, bool* found) {
  const size_t st_b = pipe_smem_bytes(NV, TK, sizeof(CT), true), un_b = pipe_smem_bytes(NV, TK, sizeof(CT), false);
  bool ok = false;
  int rc;
  *found = false;
  if (st_b <= (size_t)c->smem_optin) {
    if ((rc = pipe_fits<CT, NV, TK, true>(c, ntiles, st_b, &ok))) return rc;
    if (ok) { b->pipe_stage = true; *found = true; return 0; }
  }
  if (un_b <= (size_t)c->smem_optin) {
    if ((rc = pipe_fits<CT, NV, TK, false>(c, ntiles, un_b, &ok))) return rc;
    if (ok) { b->pipe_stage = false; *found = true; }
  }
  return 0;
}

template <int TK>
int pipe_try_tk(Ctx* c, BlockCtx* b, int ntiles, bool* found) {
  const bool fp32 = b->prm.lusgs_fp32 != 0, ke = b->prm.iturb >= 3;
  if (fp32) return ke ? pipe_try<float, 7, TK>(c, b, ntiles, found) : pipe_try<float, 5, TK>(c, b, ntiles, found);
  return ke ? pipe_try<double, 7, TK>(c, b, ntiles, found) : pipe_try<double, 5, TK>(c, b, ntiles, found);
}

// The pipelined tile wavefront fits when the (j,k) lines make at most 16
// tiles of 16 x TK (the smallest TK of 8, 16, 32 that does; more tiles, more
// SMs) and one cluster of them can be resident.
int setup_pipe(Ctx* c, BlockCtx* b) {
  b->can_pipe = 0;
  const int tks[3] = {8, 16, 32};
  for (int q = 0; q < 3; q++) {
    const int tk = tks[q];
    PipeGeom pg;
    pg.ntj = (b->jmax + PTJ - 1) / PTJ;
    pg.ntk = (b->kmax + tk - 1) / tk;
    if (pg.ntj * pg.ntk > 16) continue;
    bool found = false;
    const int nt = pg.ntj * pg.ntk;
    int rc = tk == 8 ? pipe_try_tk<8>(c, b, nt, &found)
                     : (tk == 16 ? pipe_try_tk<16>(c, b, nt, &found) : pipe_try_tk<32>(c, b, nt, &found));
    if (rc) return rc;
    if (found) {
      b->pg = pg;
      b->pipe_tk = tk;
      b->can_pipe = 1;
      return 0;
    }
  }
  return 0;
}

// The metric-only part of both sweep layouts (k_sweep_static), once per
// block and precision and again after the metrics change.  Inside a stream
// capture the fill goes into the graph and the layouts stay marked unfilled.
void sweep_static(Ctx* c, BlockCtx* b, bool fp32) {
  const int want = fp32 ? 2 : 1;
  if (b->sw_static == want) return;
  for (int up = 0; up < 2; up++) {
    if (fp32) k_sweep_static<float><<<nblk((long)b->ns, 128), 128, 0, c->stream>>>(b->db, swf(b, up), up);
    else k_sweep_static<double><<<nblk((long)b->ns, 128), 128, 0, c->stream>>>(b->db, swd(b, up), up);
    c->nlaunch++;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(c->stream, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) b->sw_static = want;
}

// The metrics of a block changed: its sweep layouts' static part is stale,
// and so is every captured graph that skipped refilling it.
void metrics_changed(Ctx* c, BlockCtx* b) {
  b->sw_static = 0;
  for (auto* x : c->blocks)
    if (x->graph) { cudaGraphExecDestroy(x->graph); x->graph = nullptr; }
  for (auto& g : c->phase_graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  if (c->mb_graph) { cudaGraphExecDestroy(c->mb_graph); c->mb_graph = nullptr; }
}

// Sweep data of one sweep in the sweep layout (and, for upper = 1, the
// right-hand side copied into it).
void sweep_coef(Ctx* c, BlockCtx* b, int upper, bool fp32) {
  sweep_static(c, b, fp32);
  if (fp32)
    k_sweep_coef<float><<<nblk((long)b->ns, 128), 128, 0, c->stream>>>(b->db, b->prm, swf(b, upper), b->dwp32, upper);
  else
    k_sweep_coef<double><<<nblk((long)b->ns, 128), 128, 0, c->stream>>>(b->db, b->prm, swd(b, upper), b->dwp, upper);
  c->nlaunch++;
}

// Sweep autotuner.  Candidates: the pipelined tile wavefront and the cluster
// line sweep (each in one cluster of at most 16 CTAs), and the cooperative
// hyperplane sweep over the whole GPU at 64/128/256 threads per CTA.  Which
// is fastest depends on the block's shape.  Each candidate is timed (upper
// sweep in the block's precision, on its current state, in the block's own
// sweep buffers, which hold nothing between implicit stages) and the
// fastest is kept.  FINFLO_LUSGS=pipe|lines|hyperplane restricts the choice.
// Blocks that run side by side in a multi-block cycle use cluster sweeps
// (see fork_join).
// DDADI kernel shapes: the prefetch depth and CTA size of the one thread
// per line kernels, and the (lines per CTA, cells per chunk) of the
// producer/consumer kernels the autotuner chooses from.
constexpr int DD_PD = 4, DD_TPB = 32;
// (lines per CTA, cells per chunk) of the producer/consumer kernels the
// autotuner chooses from
constexpr int DD_NCFG = 4;
[[maybe_unused]] constexpr int DD_CFG[DD_NCFG][2] = {{32, 4}, {16, 4}, {16, 8}, {8, 8}};

// The autotuner's choice per device, block shape, equation count and
// precision, kept for the life of the process: a later context with a block
// of the same shape takes it without timing again.
struct TuneKey {
  int dev, imax, jmax, kmax, nv, fp32, ddadi;
  bool operator<(const TuneKey& o) const {
    return std::tie(dev, imax, jmax, kmax, nv, fp32, ddadi) <
           std::tie(o.dev, o.imax, o.jmax, o.kmax, o.nv, o.fp32, o.ddadi);
  }
};
struct TuneVal {
  int use_pipe, use_lines, coop_threads, dd_cfg;
  float pipe_ms, lines_ms, hyp_ms;
};
std::map<TuneKey, TuneVal> g_tune_cache;
std::mutex g_tune_mu;

int ddadi_sweeps(Ctx* c, BlockCtx* b, int only_dir = 0);

// DDADI: time the producer/consumer forms (lines per CTA, cells per chunk)
// per direction -- the i lines are fewer and longer than the j and k lines
// -- and keep the fastest.  FINFLO_DDADI=simple selects the one thread per
// line kernels, FINFLO_DDADI=<index> one form everywhere without timing.
int tune_ddadi(Ctx* c, BlockCtx* b, const TuneKey& key) {
  const char* env = getenv("FINFLO_DDADI");
  if (env) {
    const int k = !strcmp(env, "simple") ? -1 : max(0, min(DD_NCFG - 1, atoi(env)));
    for (int d = 1; d <= 3; d++) b->dd_cfg[d] = k;
    return 0;
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      const int packed = it->second.dd_cfg;
      b->dd_cfg[1] = packed / 100; b->dd_cfg[2] = (packed / 10) % 10; b->dd_cfg[3] = packed % 10;
      b->dd_ms[1] = it->second.pipe_ms; b->dd_ms[2] = it->second.lines_ms; b->dd_ms[3] = it->second.hyp_ms;
      return 0;
    }
  }
  for (int d = 1; d <= 3; d++) {
    int best = 0;
    float best_ms = 0.f;
    for (int k = 0; k < DD_NCFG; k++) {
      b->dd_cfg[d] = k;
      float bt = 0.f;
      for (int rep = 0; rep < 3; rep++) {   // rep 0 warms up
        CK(cudaEventRecord(c->ev0, c->stream));
        int rc = ddadi_sweeps(c, b, d);
        if (rc) return rc;
        CK(cudaEventRecord(c->ev1, c->stream));
        CK(cudaEventSynchronize(c->ev1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        if (rep > 0) bt = rep == 1 ? ms : fminf(bt, ms);
      }
      if (k == 0 || bt < best_ms) { best = k; best_ms = bt; }
    }
    b->dd_cfg[d] = best;
    b->dd_ms[d] = best_ms;
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = TuneVal{0, 0, 0, b->dd_cfg[1] * 100 + b->dd_cfg[2] * 10 + b->dd_cfg[3],
                              b->dd_ms[1], b->dd_ms[2], b->dd_ms[3]};
  return 0;
}

// Residual form of a block: each tile shape of RES_SHAPES, with and without
// the staged stencil, timed on the block's own level (CUDA events, after
// one untimed launch), the fastest kept; cached per device, block shape and
// equation count.  FINFLO_RES_SHAPE (0..5) fixes it.
std::map<TuneKey, int> g_res_cache;

int tune_residual(Ctx* c, BlockCtx* b) {
  if (b->res_tuned) return 0;
  b->res_tuned = 1;
  const char* e = getenv("FINFLO_RES_SHAPE");
  const int env = e ? atoi(e) : -1;
  if (env >= 0 && env < RES_NFORM) { b->res_shape = env; return 0; }
  if (!res_fused() || res_threads(b->prm.iturb >= 3) != 512) return 0;
  const TuneKey key{c->device, b->imax, b->jmax, b->kmax, (b->prm.iturb >= 3 ? 7 : 5) + 10 * b->level, 0, 0};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_res_cache.find(key);
    if (it != g_res_cache.end()) { b->res_shape = it->second; return 0; }
  }
  float best = 1e30f;
  int pick = 0;
  for (int s = 0; s < RES_NFORM; s++) {
    b->res_shape = s;
    launch_residual(c->stream, b, b->level);
    CK(cudaEventRecord(c->ev0, c->stream));
    for (int r = 0; r < 3; r++) launch_residual(c->stream, b, b->level);
    CK(cudaEventRecord(c->ev1, c->stream));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    if (ms < best) { best = ms; pick = s; }
  }
  b->res_shape = pick;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_res_cache[key] = pick;
  return 0;
}

int tune_sweep(Ctx* c, BlockCtx* b) {
  {
    int rc = tune_residual(c, b);
    if (rc) return rc;
  }
  if (b->tuned) return 0;
  b->tuned = 1;
  const TuneKey key{c->device, b->imax, b->jmax, b->kmax, b->prm.iturb >= 3 ? 7 : 5, b->prm.lusgs_fp32 != 0,
                    b->prm.ddadi != 0};
  if (b->prm.ddadi) return tune_ddadi(c, b, key);
  const char* env = getenv("FINFLO_LUSGS");
  if (!env) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end() && (!it->second.use_pipe || b->can_pipe) && (!it->second.use_lines || b->can_lines)) {
      const TuneVal& v = it->second;
      b->use_pipe = v.use_pipe; b->use_lines = v.use_lines; b->coop_threads = v.coop_threads;
      b->pipe_ms = v.pipe_ms; b->sweep_ms[0] = v.lines_ms; b->sweep_ms[1] = v.hyp_ms;
      return 0;
    }
  }
  const bool fp32 = b->prm.lusgs_fp32 != 0;
  const int threads[3] = {64, 128, 256};
  const bool only = env && (!strcmp(env, "pipe") || !strcmp(env, "lines") || !strcmp(env, "hyperplane"));
  const bool try_pipe = b->can_pipe && (!only || !strcmp(env, "pipe"));
  const bool try_lines = b->can_lines && (!only || !strcmp(env, "lines"));
  bool try_hyp = !only || !strcmp(env, "hyperplane");
  if (!try_pipe && !try_lines) try_hyp = true;   // nothing else fits
  sweep_coef(c, b, 1, fp32);
  float best_k[3] = {0.f, 0.f, 0.f};   // pipe, lines, hyperplane
  int best_t = b->coop_threads;
  int rc = 0;
  b->use_pipe = 0;
  for (int kind = 0; kind < 5 && !rc; kind++) {
    if (kind == 0 && !try_pipe) continue;
    if (kind == 1 && !try_lines) continue;
    if (kind > 1 && !try_hyp) continue;
    float best = 0.f;
    for (int rep = 0; rep < 4 && !rc; rep++) {   // rep 0 warms up
      cudaEventRecord(c->ev0, c->stream);
      rc = kind == 0 ? pipe_sweep(c, b, 1, fp32)
                     : (kind == 1 ? lines_sweep(c, b, 1, fp32) : coop_sweep_n(c, b, 1, fp32, threads[kind - 2]));
      if (rc) break;
      cudaEventRecord(c->ev1, c->stream);
      cudaError_t s2 = cudaEventSynchronize(c->ev1);
      if (s2 != cudaSuccess) { rc = fail(c, FF_ERR_CUDA, "sweep autotune", s2); break; }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, c->ev0, c->ev1);
      if (rep > 0) best = rep == 1 ? ms : fminf(best, ms);
    }
    if (kind < 2) best_k[kind] = best;
    else if (best_k[2] == 0.f || best < best_k[2]) { best_k[2] = best; best_t = threads[kind - 2]; }
  }
  if (rc) return rc;
  int herr = 0;
  CK(cudaMemcpy(&herr, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (herr) return fail(c, FF_ERR_TIMEOUT, "sweep autotune: a bounded wait gave up");
  b->pipe_ms = best_k[0];
  b->sweep_ms[0] = best_k[1];
  b->sweep_ms[1] = best_k[2];
  b->coop_threads = best_t;
  // the fastest measured candidate
  int pick = -1;
  float bt = 0.f;
  for (int k = 0; k < 3; k++)
    if (best_k[k] > 0.f && (pick < 0 || best_k[k] < bt)) { pick = k; bt = best_k[k]; }
  b->use_pipe = pick == 0;
  b->use_lines = pick == 1 ? 1 : 0;
  if (pick == 0) b->use_lines = 0;
  if (!env) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = TuneVal{b->use_pipe, b->use_lines, b->coop_threads, 0, b->pipe_ms, b->sweep_ms[0], b->sweep_ms[1]};
  }
  return 0;
}

int sweep(Ctx* c, BlockCtx* b, int upper, bool fp32) {
  // bit 2 of the lower (PREDGS) sweep's flag keeps the row-JMAX i+1 coupling
  if (upper && b->prm.predgs_full) upper |= 2;
  if (b->use_pipe) return pipe_sweep(c, b, upper, fp32);
  return b->use_lines ? lines_sweep(c, b, upper, fp32) : coop_sweep(c, b, upper, fp32);
}

// DDADI (LUSGS=0): the k, i and j lines in turn (imps3.f:320-356), each a
// PRED+DIAG launch and a CORR launch.  Default: 32 lines per CTA with
// producer warps (k_ddadi_pc); FINFLO_DDADI=simple selects one thread per
// line with a cp.async prefetch ring (k_ddadi_pred/k_ddadi_corr).

template <typename CT, int NV, int LPC, int CH>
void ddadi_pc_launch_t(cudaStream_t st, const DevBlock& db, const ff_params& prm, int dir, int lines) {
  auto kp = k_ddadi_pc<CT, NV, LPC, CH, false>;
  auto kc = k_ddadi_pc<CT, NV, LPC, CH, true>;
  const size_t sp = ddadi_pc_smem_bytes<CT>(NV, LPC, CH, false), sc = ddadi_pc_smem_bytes<CT>(NV, LPC, CH, true);
  cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp);
  cudaFuncSetAttribute(kc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sc);
  kp<<<nblk(lines, LPC), 32 + LPC * CH, sp, st>>>(db, prm, dir);
  kc<<<nblk(lines, LPC), 32 + LPC * CH, sc, st>>>(db, prm, dir);
}

template <typename CT, int NV>
void ddadi_pc_launch(cudaStream_t st, const DevBlock& db, const ff_params& prm, int dir, int lines, int cfg) {
  switch (cfg) {
    case 1: ddadi_pc_launch_t<CT, NV, 16, 4>(st, db, prm, dir, lines); break;
    case 2: ddadi_pc_launch_t<CT, NV, 16, 8>(st, db, prm, dir, lines); break;
    case 3: ddadi_pc_launch_t<CT, NV, 8, 8>(st, db, prm, dir, lines); break;
    default: ddadi_pc_launch_t<CT, NV, 32, 4>(st, db, prm, dir, lines); break;
  }
}

template <typename CT, int NV>
void ddadi_launch(Ctx* c, BlockCtx* b, int dir, int lines) {
  if (b->dd_cfg[dir] < 0) {   // FINFLO_DDADI=simple
    const size_t sm = ddadi_smem_bytes(NV, DD_PD, DD_TPB);
    k_ddadi_pred<CT, NV, DD_PD, DD_TPB><<<nblk(lines, DD_TPB), DD_TPB, sm, c->stream>>>(b->db, b->prm, dir);
    k_ddadi_corr<CT, NV, DD_PD, DD_TPB><<<nblk(lines, DD_TPB), DD_TPB, sm, c->stream>>>(b->db, b->prm, dir);
  } else {
    ddadi_pc_launch<CT, NV>(c->stream, b->db, b->prm, dir, lines, b->dd_cfg[dir]);
  }
  c->nlaunch += 2;
}

int ddadi_sweeps(Ctx* c, BlockCtx* b, int only_dir) {
  const bool fp32 = b->prm.lusgs_fp32 != 0, ke = b->prm.iturb >= 3;
  const int dirs[3] = {3, 1, 2};
  for (int d : dirs) {
    if (only_dir && d != only_dir) continue;
    const int n = d == 1 ? b->imax : (d == 2 ? b->jmax : b->kmax);
    if (n <= 1) continue;   // IMPSWE skips a direction one cell deep (imps3.f:601)
    const int lines = b->imax * b->jmax * b->kmax / n;
    if (fp32) {
      if (ke) ddadi_launch<float, 7>(c, b, d, lines); else ddadi_launch<float, 5>(c, b, d, lines);
    } else {
      if (ke) ddadi_launch<double, 7>(c, b, d, lines); else ddadi_launch<double, 5>(c, b, d, lines);
    }
  }
  CK(cudaGetLastError());
  return 0;
}

// IMPS (imps3.f:6) in three parts: the time step and COPR before the
// sweeps, the sweeps, and the increments out of the sweep layout (plus
// DRO/CP for a standalone IMPS) after them.
void st_imps_pre(Ctx* c, BlockCtx* b, int level) {
  int ncell = b->imax * b->jmax * b->kmax;
  double cfl = level == 1 ? b->prm.cfl : b->prm.cfll;
  if (b->prm.iturb >= 3) {   // TIME3, then LOCDTK + IMSOKO + COPRKE
    k_time3_copr<<<nblk(ncell, 128), 128, 0, c->stream>>>(b->db, b->prm, cfl, 1);
    k_locdtk_imsoko_coprke<<<nblk(ncell, 128), 128, 0, c->stream>>>(b->db, b->prm);
    c->nlaunch += 2;
  } else {
    k_time3_copr<<<nblk(ncell, 128), 128, 0, c->stream>>>(b->db, b->prm, cfl);
    c->nlaunch++;
  }
}

void st_sweep_out(Ctx* c, BlockCtx* b) {
  int ncell = b->imax * b->jmax * b->kmax;
  if (b->prm.lusgs_fp32)
    k_sweep_out<float><<<nblk(ncell, 128), 128, 0, c->stream>>>(b->db, b->dwp32, b->prm.iturb >= 3 ? 7 : 5);
  else
    k_sweep_out<double><<<nblk(ncell, 128), 128, 0, c->stream>>>(b->db, b->dwp, b->prm.iturb >= 3 ? 7 : 5);
  c->nlaunch++;
}

void st_imps_post(Ctx* c, BlockCtx* b, bool divide_cp) {
  if (divide_cp) {
    // standalone IMPS: finish with DRO/CP (imps3.f:483); the fused cycle
    // folds this division into the FIN kernel instead
    k_fin_divide<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db, b->prm.iturb >= 3);
    c->nlaunch++;
  }
}

int st_imps(Ctx* c, BlockCtx* b, int level, bool divide_cp) {
  st_imps_pre(c, b, level);
  bool fp32 = b->prm.lusgs_fp32 != 0;
  int rc;
  if (b->prm.ddadi) {
    if ((rc = ddadi_sweeps(c, b))) return rc;
  } else {
    sweep_coef(c, b, 1, fp32);
    if (b->use_lines || b->use_pipe) {
      // the second sweep's coefficients (their own layout buffer; they read
      // the state, which the first sweep does not change) beside the first
      // sweep, whose one cluster leaves most SMs free.  Not beside the
      // cooperative hyperplane sweep, which needs every CTA resident.
      if (!b->aux) {
        CK(cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&b->aux_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&b->aux_join, cudaEventDisableTiming));
      }
      cudaStream_t main = c->stream;
      CK(cudaEventRecord(b->aux_fork, main));
      CK(cudaStreamWaitEvent(b->aux, b->aux_fork, 0));
      c->stream = b->aux;
      sweep_coef(c, b, 0, fp32);
      c->stream = main;
      CK(cudaEventRecord(b->aux_join, b->aux));
      if ((rc = sweep(c, b, 1, fp32))) return rc;
      CK(cudaStreamWaitEvent(main, b->aux_join, 0));
    } else {
      if ((rc = sweep(c, b, 1, fp32))) return rc;
      sweep_coef(c, b, 0, fp32);
    }
    if ((rc = sweep(c, b, 0, fp32))) return rc;
    st_sweep_out(c, b);
  }
  st_imps_post(c, b, divide_cp);
  return 0;
}

int st_fin(Ctx* c, BlockCtx* b, int divide_cp) {
  k_fin<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db, b->prm, c->d_dromax, divide_cp);
  c->nlaunch++;
  return 0;
}

int one_cycle(Ctx* c, BlockCtx* b, int icycle) {
  int rc;
  const bool sst = b->prm.iturb >= 3;
  k_reset_acc<<<1, 32, 0, c->stream>>>(c->d_resi, c->d_dromax);
  c->nlaunch++;
  // STATIM at the start of CYCLES: after the previous BOUNDI it only matters
  // where SUBIN capped k (E includes k)
  if (sst && (rc = st_statim(c, b, 1))) return rc;
  if ((rc = st_residu(c, b, 1, icycle))) return rc;
  int ncell = b->imax * b->jmax * b->kmax;
  k_resl2<<<min(nblk(ncell, 256), 4 * c->sm_count), 256, 0, c->stream>>>(b->db, c->d_resi);
  c->nlaunch++;
  if ((rc = st_imps(c, b, 1, false))) return rc;
  if ((rc = st_fin(c, b, 1))) return rc;
  if ((rc = st_boundi(c, b))) return rc;
  if (sst) {   // SUBIN: k cap, RKOLD / EPSOLD
    k_subin_sst<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db, b->prm);
    c->nlaunch++;
  }
  k_record<<<1, 1, 0, c->stream>>>(c->d_resi, c->d_dromax, c->d_hist, c->d_hist_pos, c->hist_cap);
  c->nlaunch++;
  return 0;
}

// The per-block part of a multigrid cycle of CYCLES (ns3c.f:1400-2130):
// fine-level update, then for each coarser level STATIM/RESIDI of the finer
// level, TRANSF, STATIM, RESIDI, FORCFU, ADDRES, IMPSDI, FIN; then INTERP
// back up and REFLEC.  RESL2 of the level-1 residual after the fine update
// is added to the context's sums; `own` (a single block) resets them here.
// part: 0 all of it; 1 up to the level-1 residual's face pass (not
// included); 2 from after that face pass on (launch_residual_batch runs the
// face pass of all blocks in between).
int mg_body(Ctx* c, BlockCtx* b, int icycle, bool own, int part = 0) {
  int rc;
  const int sst = b->prm.iturb >= 3;
  if (part != 2) {
    if (own) {
      k_reset_acc<<<1, 32, 0, c->stream>>>(c->d_resi, c->d_dromax);
      c->nlaunch++;
    }
    if (sst && (rc = st_statim(c, b, 1))) return rc;
  }
  if ((rc = st_residu(c, b, 1, icycle, 1, part))) return rc;
  if (part == 1) return 0;
  if ((rc = st_imps(c, b, 1, false))) return rc;
  if ((rc = st_fin(c, b, 1))) return rc;
  std::vector<BlockCtx*> lv;
  for (BlockCtx* x = b; x; x = x->coarse) lv.push_back(x);
  for (size_t m = 1; m < lv.size(); m++) {
    BlockCtx *f = lv[m - 1], *cc = lv[m];
    st_statim(c, f, 1);
    if ((rc = st_residu(c, f, (int)m, icycle, (int)m + 1))) return rc;
    if (m == 1) {   // RESL2 of the level-1 residual after the fine update
      if (own) {
        k_reset_acc<<<1, 32, 0, c->stream>>>(c->d_resi, c->d_dromax);
        c->nlaunch++;
      }
      int ncell = f->imax * f->jmax * f->kmax;
      k_resl2<<<min(nblk(ncell, 256), 4 * c->sm_count), 256, 0, c->stream>>>(f->db, c->d_resi);
      c->nlaunch++;
    } else {
      k_forcing<<<nblk(f->ntot, 256), 256, 0, c->stream>>>(f->db, 1, sst);
      c->nlaunch++;
    }
    long nc = (long)(cc->imax + 2) * (cc->jmax + 2) * (cc->kmax + 2);
    k_transf<<<nblk(nc, 128), 128, 0, c->stream>>>(f->db, cc->db, sst);
    c->nlaunch++;
    k_transf_ring<<<nblk(cc->ntot, 256), 256, 0, c->stream>>>(cc->db, sst);
    c->nlaunch++;
    st_statim(c, cc, 1);
    if ((rc = st_residu(c, cc, (int)m + 1, icycle, (int)m + 1))) return rc;
    k_forcing<<<nblk(cc->ntot, 256), 256, 0, c->stream>>>(cc->db, 0, sst);
    c->nlaunch++;
    k_forcing<<<nblk(cc->ntot, 256), 256, 0, c->stream>>>(cc->db, 1, sst);
    c->nlaunch++;
    if ((rc = st_imps(c, cc, (int)m + 1, true))) return rc;
    k_fin_coarse<<<nblk(cc->ntot, 256), 256, 0, c->stream>>>(cc->db, cc->prm, 1);
    c->nlaunch++;
  }
  for (size_t m = lv.size() - 1; m >= 1; m--) {
    BlockCtx *f = lv[m - 1], *cc = lv[m];
    int nf = f->imax * f->jmax * f->kmax;
    k_interp<<<nblk(nf, 256), 256, 0, c->stream>>>(cc->db, f->db);
    c->nlaunch++;
    if (sst) {
      k_intert<<<nblk(nf, 256), 256, 0, c->stream>>>(cc->db, f->db, f->prm);
      c->nlaunch++;
    }
    k_fin_coarse<<<nblk(f->ntot, 256), 256, 0, c->stream>>>(f->db, f->prm, 0);
    c->nlaunch++;
  }
  launch_patch(c, b, k_reflec, 0);
  return 0;
}

// One multigrid cycle of one block: mg_body, BOUNDI, SUBIN.
int mg_cycle(Ctx* c, BlockCtx* b, int icycle) {
  int rc;
  const int sst = b->prm.iturb >= 3;
  if ((rc = mg_body(c, b, icycle, true))) return rc;
  if ((rc = st_boundi(c, b))) return rc;
  // SUBIN's *OLD copies (INTERP changed the level-1 state after FIN)
  k_subin_copy<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db);
  c->nlaunch++;
  if (sst) {   // SUBIN: k cap, RKOLD / EPSOLD
    k_subin_sst<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db, b->prm);
    c->nlaunch++;
  }
  // SUBIN's max|DE| sees the level-1 residual of the second RESIDI
  k_reset_acc<<<1, 32, 0, c->stream>>>(c->d_resi + 6, c->d_dromax);
  c->nlaunch++;
  int ncell = b->imax * b->jmax * b->kmax;
  k_maxabs_de<<<min(nblk(ncell, 256), 4 * c->sm_count), 256, 0, c->stream>>>(b->db, c->d_dromax);
  c->nlaunch++;
  k_record<<<1, 1, 0, c->stream>>>(c->d_resi, c->d_dromax, c->d_hist, c->d_hist_pos, c->hist_cap);
  c->nlaunch++;
  return 0;
}

void drop_phase_graphs(Ctx* c);

// Device block table and connection work-list of all blocks of the context.
int ensure_conn(Ctx* c) {
  int nb = (int)c->blocks.size();
  if (c->conn_blocks == nb) return 0;
  drop_phase_graphs(c);
  std::vector<DevBlock> tab(nb);
  std::vector<ConnItem> items;
  int maxn = 1;
  c->tops.clear();
  for (int n = 0; n < nb; n++) {
    tab[n] = c->blocks[n]->db;
    // 1:1 ghosts are exchanged on level 1 only (BOUNDI(M) of the coarse
    // levels is commented out in the reference, ns3c.f:1618 / 1843): coarse
    // ghosts come from TRANSF
    if (c->blocks[n]->level != 1) continue;
    c->tops.push_back(c->blocks[n]);
    for (auto& pa : c->blocks[n]->h_patch) {
      if (pa.ityp != FF_BC_CON || pa.ibtype < 0) continue;   // negative: remote source
      if (pa.ibtype >= nb || c->blocks[pa.ibtype]->level != 1)
        return fail(c, FF_ERR_ARG, "connection to an unknown block (the source must be a level-1 block id)");
      ConnItem it;
      it.dst = n; it.src = pa.ibtype; it.pa = pa;
      items.push_back(it);
      maxn = max(maxn, (pa.r1b - pa.r1a + 1) * (pa.r2b - pa.r2a + 1));
    }
  }
  if (c->d_blocks) cudaFree(c->d_blocks);
  if (c->d_conn) cudaFree(c->d_conn);
  c->d_blocks = nullptr; c->d_conn = nullptr;
  CK(cudaMalloc(&c->d_blocks, sizeof(DevBlock) * max(1, nb)));
  CK(cudaMemcpy(c->d_blocks, tab.data(), sizeof(DevBlock) * nb, cudaMemcpyHostToDevice));
  c->nconn = (int)items.size();
  c->maxconn = maxn;
  if (c->nconn) {
    CK(cudaMalloc(&c->d_conn, sizeof(ConnItem) * c->nconn));
    CK(cudaMemcpy(c->d_conn, items.data(), sizeof(ConnItem) * c->nconn, cudaMemcpyHostToDevice));
  }
  while (c->side.size() < c->tops.size()) {
    cudaStream_t s; cudaEvent_t e;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    c->side.push_back(s); c->side_ev.push_back(e);
  }
  if (!c->fork_ev) CK(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
  c->conn_blocks = nb;
  return 0;
}

int st_connec(Ctx* c) {
  if (!c->nconn) return 0;
  k_connec<<<dim3(nblk(c->maxconn, 128), c->nconn), 128, 0, c->stream>>>(c->d_blocks, c->d_conn);
  c->nlaunch++;
  return 0;
}

// Run fn(n) for every level-1 block c->tops[n] on its own stream, forked
// from and joined back into the context stream (captured as parallel graph
// branches).
// Blocks whose sweep is the cooperative hyperplane kernel share the context's
// grid barrier and need the whole GPU, so their chains run one after another.
template <typename F>
int fork_join(Ctx* c, int nb, F fn) {
  bool concurrent = nb > 1;
  for (int n = 0; n < nb; n++)
    for (BlockCtx* x = c->tops[n]; x; x = x->coarse) concurrent = concurrent && (x->use_lines || x->use_pipe);
  if (!concurrent) {
    for (int n = 0; n < nb; n++) {
      int rc = fn(n);
      if (rc) return rc;
    }
    return 0;
  }
  cudaStream_t main = c->stream;
  CK(cudaEventRecord(c->fork_ev, main));
  int rc = 0;
  c->side_by_side = true;
  for (int n = 0; n < nb && !rc; n++) {
    CK(cudaStreamWaitEvent(c->side[n], c->fork_ev, 0));
    c->stream = c->side[n];
    rc = fn(n);
    c->stream = main;
    CK(cudaEventRecord(c->side_ev[n], c->side[n]));
  }
  c->side_by_side = false;
  c->stream = main;
  for (int n = 0; n < nb; n++) CK(cudaStreamWaitEvent(main, c->side_ev[n], 0));
  return rc;
}

// fn(n) for n < cnt on side streams, forked from and joined back into the
// context stream, with no sweep inside (the lockstep cycle's per-block
// stages between its batched sweeps).
template <typename F>
int fork_n(Ctx* c, int cnt, F fn) {
  if (cnt <= 1) return cnt == 1 ? fn(0) : 0;
  cudaStream_t main = c->stream;
  CK(cudaEventRecord(c->fork_ev, main));
  int rc = 0;
  c->side_by_side = true;
  for (int n = 0; n < cnt && !rc; n++) {
    CK(cudaStreamWaitEvent(c->side[n], c->fork_ev, 0));
    c->stream = c->side[n];
    rc = fn(n);
    c->stream = main;
    CK(cudaEventRecord(c->side_ev[n], c->side[n]));
  }
  c->side_by_side = false;
  c->stream = main;
  for (int n = 0; n < cnt; n++) CK(cudaStreamWaitEvent(main, c->side_ev[n], 0));
  return rc;
}

// Multi-block cycles in lockstep (the reference's order: each stage of
// CYCLES over all blocks, ns3c.f:1400-2130) with every level's LU-SGS sweeps
// as one batched launch, with FINFLO_MB_LOCKSTEP=1.  Needs the cluster line
// sweep on every block and level.  Not the default: the per-block branches
// overlap one block's latency-bound sweeps (16 SMs each) with the other
// blocks' residual work, which lockstep cannot (8-block SST case,
// 512x256x128 cells: 64.2 ms per V-cycle as branches, 71.8 ms in lockstep).
bool ls_ok(Ctx* c) {
  const char* env = getenv("FINFLO_MB_LOCKSTEP");
  const char* kind = getenv("FINFLO_LUSGS");
  if (!env || strcmp(env, "1") || (kind && strcmp(kind, "lines")) || c->tops.size() < 2) return false;
  std::vector<std::vector<BlockCtx*>> lv;
  for (auto* t : c->tops) {
    size_t m = 0;
    for (BlockCtx* x = t; x; x = x->coarse, m++) {
      if (lv.size() <= m) lv.resize(m + 1);
      lv[m].push_back(x);
    }
  }
  for (auto& v : lv) {
    LinesBatchShape sh;
    for (size_t s0 = 0; s0 < v.size(); s0 += LB_MAX) {
      std::vector<BlockCtx*> part(v.begin() + s0, v.begin() + min(v.size(), s0 + LB_MAX));
      if (!lines_batch_shape(c, part, sizeof(double), sh)) return false;
    }
  }
  return true;
}

// IMPS of the blocks v (one level) in lockstep: both sweeps batched.
int ls_imps(Ctx* c, const std::vector<BlockCtx*>& v, int level, bool divide_cp) {
  const int n = (int)v.size();
  int rc = fork_n(c, n, [&](int i) {
    st_imps_pre(c, v[i], level);
    sweep_coef(c, v[i], 1, v[i]->prm.lusgs_fp32 != 0);
    return 0;
  });
  if (rc || (rc = lines_batch(c, v, 1))) return rc;
  rc = fork_n(c, n, [&](int i) {
    sweep_coef(c, v[i], 0, v[i]->prm.lusgs_fp32 != 0);
    return 0;
  });
  if (rc || (rc = lines_batch(c, v, 0))) return rc;
  return fork_n(c, n, [&](int i) {
    st_sweep_out(c, v[i]);
    st_imps_post(c, v[i], divide_cp);
    return 0;
  });
}

// mg_body of every level-1 block in lockstep, stage by stage in mg_body's
// order within each block.
int mb_mg_body_ls(Ctx* c, int icycle) {
  std::vector<BlockCtx*>& tops = c->tops;
  const int nb = (int)tops.size();
  const bool rbatch = res_batch_ok(c);
  int rc = fork_n(c, nb, [&](int n) {
    BlockCtx* b = tops[n];
    int r;
    if (b->prm.iturb >= 3 && (r = st_statim(c, b, 1))) return r;
    return st_residu(c, b, 1, icycle, 1, rbatch ? 1 : 0);
  });
  if (rc) return rc;
  if (rbatch && (rc = launch_residual_batch(c, tops, 1))) return rc;
  if (rbatch && (rc = fork_n(c, nb, [&](int n) { return st_residu(c, tops[n], 1, icycle, 1, 2); }))) return rc;
  if ((rc = ls_imps(c, tops, 1, false))) return rc;
  if ((rc = fork_n(c, nb, [&](int n) { return st_fin(c, tops[n], 1); }))) return rc;
  std::vector<std::vector<BlockCtx*>> chain(nb);
  size_t nlev = 0;
  for (int n = 0; n < nb; n++) {
    for (BlockCtx* x = tops[n]; x; x = x->coarse) chain[n].push_back(x);
    nlev = max(nlev, chain[n].size());
  }
  for (size_t m = 1; m < nlev; m++) {
    std::vector<BlockCtx*> fs, cs;
    for (int n = 0; n < nb; n++)
      if (chain[n].size() > m) { fs.push_back(chain[n][m - 1]); cs.push_back(chain[n][m]); }
    rc = fork_n(c, (int)fs.size(), [&](int n) {
      BlockCtx *f = fs[n], *cc = cs[n];
      const int sst = f->prm.iturb >= 3;
      int r;
      st_statim(c, f, 1);
      if ((r = st_residu(c, f, (int)m, icycle, (int)m + 1))) return r;
      if (m == 1) {   // RESL2 of the level-1 residual after the fine update
        int ncell = f->imax * f->jmax * f->kmax;
        k_resl2<<<min(nblk(ncell, 256), 4 * c->sm_count), 256, 0, c->stream>>>(f->db, c->d_resi);
        c->nlaunch++;
      } else {
        k_forcing<<<nblk(f->ntot, 256), 256, 0, c->stream>>>(f->db, 1, sst);
        c->nlaunch++;
      }
      long nc = (long)(cc->imax + 2) * (cc->jmax + 2) * (cc->kmax + 2);
      k_transf<<<nblk(nc, 128), 128, 0, c->stream>>>(f->db, cc->db, sst);
      k_transf_ring<<<nblk(cc->ntot, 256), 256, 0, c->stream>>>(cc->db, sst);
      c->nlaunch += 2;
      st_statim(c, cc, 1);
      if ((r = st_residu(c, cc, (int)m + 1, icycle, (int)m + 1))) return r;
      k_forcing<<<nblk(cc->ntot, 256), 256, 0, c->stream>>>(cc->db, 0, sst);
      k_forcing<<<nblk(cc->ntot, 256), 256, 0, c->stream>>>(cc->db, 1, sst);
      c->nlaunch += 2;
      return 0;
    });
    if (rc || (rc = ls_imps(c, cs, (int)m + 1, true))) return rc;
    rc = fork_n(c, (int)cs.size(), [&](int n) {
      k_fin_coarse<<<nblk(cs[n]->ntot, 256), 256, 0, c->stream>>>(cs[n]->db, cs[n]->prm, 1);
      c->nlaunch++;
      return 0;
    });
    if (rc) return rc;
  }
  return fork_n(c, nb, [&](int n) {
    auto& lv = chain[n];
    for (size_t m = lv.size() - 1; m >= 1; m--) {
      BlockCtx *f = lv[m - 1], *cc = lv[m];
      int nf = f->imax * f->jmax * f->kmax;
      k_interp<<<nblk(nf, 256), 256, 0, c->stream>>>(cc->db, f->db);
      c->nlaunch++;
      if (f->prm.iturb >= 3) {
        k_intert<<<nblk(nf, 256), 256, 0, c->stream>>>(cc->db, f->db, f->prm);
        c->nlaunch++;
      }
      k_fin_coarse<<<nblk(f->ntot, 256), 256, 0, c->stream>>>(f->db, f->prm, 0);
      c->nlaunch++;
    }
    launch_patch(c, tops[n], k_reflec, 0);
    return 0;
  });
}

// BOUNDI ns3c.f:10608 over all blocks: REFCOR, MIR and STATIM per block,
// CONNEC of every 1:1 patch in one launch, STATIM again.
int mb_boundi(Ctx* c) {
  int nb = (int)c->tops.size(), rc;
  rc = fork_join(c, nb, [&](int n) {
    BlockCtx* b = c->tops[n];
    k_refcor<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db);
    c->nlaunch++;
    if (b->npatch) {
      int maxn = 1;
      for (auto& p : b->h_patch) maxn = max(maxn, (p.r1b - p.r1a + 1) * (p.r2b - p.r2a + 1));
      k_mir<<<dim3(nblk(maxn, 128), b->npatch), 128, 0, c->stream>>>(b->db);
      c->nlaunch++;
    }
    return st_statim(c, b, 1);
  });
  if (rc) return rc;
  if ((rc = st_connec(c))) return rc;
  return fork_join(c, nb, [&](int n) { return st_statim(c, c->tops[n], 1); });
}

// One NS3D cycle over all single-grid blocks: CYCLES per block (concurrent
// branches), then the all-block BOUNDI and SUBIN.
int mb_mg_cycle(Ctx* c, int icycle);

int mb_cycle(Ctx* c, int icycle) {
  int nb = (int)c->tops.size(), rc;
  for (auto* b : c->tops)
    if (b->coarse) return mb_mg_cycle(c, icycle);
  k_reset_acc<<<1, 32, 0, c->stream>>>(c->d_resi, c->d_dromax);
  c->nlaunch++;
  const bool batch = res_batch_ok(c), lockstep = ls_ok(c);
  if (lockstep) {   // lockstep: RESIDI, RESL2, IMPSDI (batched sweeps), FIN
    rc = fork_n(c, nb, [&](int n) {
      BlockCtx* b = c->tops[n];
      int r;
      if (b->prm.iturb >= 3 && (r = st_statim(c, b, 1))) return r;
      return st_residu(c, b, 1, icycle, 1, batch ? 1 : 0);
    });
    if (rc) return rc;
    if (batch && (rc = launch_residual_batch(c, c->tops, 1))) return rc;
    rc = fork_n(c, nb, [&](int n) {
      BlockCtx* b = c->tops[n];
      int r;
      if (batch && (r = st_residu(c, b, 1, icycle, 1, 2))) return r;
      int ncell = b->imax * b->jmax * b->kmax;
      k_resl2<<<min(nblk(ncell, 256), 4 * c->sm_count), 256, 0, c->stream>>>(b->db, c->d_resi);
      c->nlaunch++;
      return 0;
    });
    if (rc || (rc = ls_imps(c, c->tops, 1, false))) return rc;
    if ((rc = fork_n(c, nb, [&](int n) { return st_fin(c, c->tops[n], 1); }))) return rc;
  } else if (batch) {   // the face pass of all blocks in one launch
    rc = fork_join(c, nb, [&](int n) {
      BlockCtx* b = c->tops[n];
      int r;
      if (b->prm.iturb >= 3 && (r = st_statim(c, b, 1))) return r;
      return st_residu(c, b, 1, icycle, 1, 1);
    });
    if (rc) return rc;
    if ((rc = launch_residual_batch(c, c->tops, 1))) return rc;
  }
  if (!lockstep) {
    rc = fork_join(c, nb, [&](int n) {
      BlockCtx* b = c->tops[n];
      int r;
      if (!batch && b->prm.iturb >= 3 && (r = st_statim(c, b, 1))) return r;
      if ((r = st_residu(c, b, 1, icycle, 1, batch ? 2 : 0))) return r;
      int ncell = b->imax * b->jmax * b->kmax;
      k_resl2<<<min(nblk(ncell, 256), 4 * c->sm_count), 256, 0, c->stream>>>(b->db, c->d_resi);
      c->nlaunch++;
      if ((r = st_imps(c, b, 1, false))) return r;
      return st_fin(c, b, 1);
    });
    if (rc) return rc;
  }
  if ((rc = mb_boundi(c))) return rc;
  for (auto* b : c->tops)
    if (b->prm.iturb >= 3) {
      k_subin_sst<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db, b->prm);
      c->nlaunch++;
    }
  k_record<<<1, 1, 0, c->stream>>>(c->d_resi, c->d_dromax, c->d_hist, c->d_hist_pos, c->hist_cap);
  c->nlaunch++;
  return 0;
}

// One multigrid cycle of all blocks: every block's mg_body (concurrent
// branches), BOUNDI over the level-1 blocks (1:1 ghosts on level 1 only),
// SUBIN per block, then the monitor (RESL2 sums of all blocks, max|DE|).
int mb_mg_cycle(Ctx* c, int icycle) {
  int nb = (int)c->tops.size(), rc;
  k_reset_acc<<<1, 32, 0, c->stream>>>(c->d_resi, c->d_dromax);
  c->nlaunch++;
  if (ls_ok(c)) {
    rc = mb_mg_body_ls(c, icycle);
  } else if (res_batch_ok(c)) {   // the level-1 face pass of all blocks in one launch
    rc = fork_join(c, nb, [&](int n) { return mg_body(c, c->tops[n], icycle, false, 1); });
    if (rc) return rc;
    if ((rc = launch_residual_batch(c, c->tops, 1))) return rc;
    rc = fork_join(c, nb, [&](int n) { return mg_body(c, c->tops[n], icycle, false, 2); });
  } else {
    rc = fork_join(c, nb, [&](int n) { return mg_body(c, c->tops[n], icycle, false); });
  }
  if (rc) return rc;
  if ((rc = mb_boundi(c))) return rc;
  rc = fork_join(c, nb, [&](int n) {
    BlockCtx* b = c->tops[n];
    k_subin_copy<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db);
    c->nlaunch++;
    if (b->prm.iturb >= 3) {
      k_subin_sst<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db, b->prm);
      c->nlaunch++;
    }
    return 0;
  });
  if (rc) return rc;
  k_reset_acc<<<1, 32, 0, c->stream>>>(c->d_resi + 6, c->d_dromax);
  c->nlaunch++;
  rc = fork_join(c, nb, [&](int n) {
    BlockCtx* b = c->tops[n];
    int ncell = b->imax * b->jmax * b->kmax;
    k_maxabs_de<<<min(nblk(ncell, 256), 4 * c->sm_count), 256, 0, c->stream>>>(b->db, c->d_dromax);
    c->nlaunch++;
    return 0;
  });
  if (rc) return rc;
  k_record<<<1, 1, 0, c->stream>>>(c->d_resi, c->d_dromax, c->d_hist, c->d_hist_pos, c->hist_cap);
  c->nlaunch++;
  return 0;
}

int st_halo(Ctx* c, int mode) {
  if (!c->nhalo || !(mode == 0 ? c->halo_pack : c->halo_unpack)) return 0;
  k_halo<<<dim3(nblk(c->halo_maxn, 128), c->nhalo), 128, 0, c->stream>>>(c->d_blocks, c->d_halo, mode,
                                                                          c->halo_send, c->halo_recv);
  c->nlaunch++;
  return 0;
}

// Multi-GPU phases (see ff_mb_phase in the header).
int mb_phase(Ctx* c, int phase, int icycle) {
  int nb = (int)c->tops.size(), rc;
  if (phase == FF_PHASE_CYCLE_A) {
    k_reset_acc<<<1, 32, 0, c->stream>>>(c->d_resi, c->d_dromax);
    c->nlaunch++;
    rc = fork_join(c, nb, [&](int n) {
      BlockCtx* b = c->tops[n];
      int r;
      if ((r = st_residu(c, b, 1, icycle))) return r;
      int ncell = b->imax * b->jmax * b->kmax;
      k_resl2<<<min(nblk(ncell, 256), 4 * c->sm_count), 256, 0, c->stream>>>(b->db, c->d_resi);
      c->nlaunch++;
      if ((r = st_imps(c, b, 1, false))) return r;
      return st_fin(c, b, 1);
    });
    if (rc) return rc;
  }
  if (phase == FF_PHASE_CYCLE_A || phase == FF_PHASE_BOUNDI_A) {
    rc = fork_join(c, nb, [&](int n) {
      BlockCtx* b = c->tops[n];
      k_refcor<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db);
      c->nlaunch++;
      if (b->npatch) {
        int maxn = 1;
        for (auto& p : b->h_patch) maxn = max(maxn, (p.r1b - p.r1a + 1) * (p.r2b - p.r2a + 1));
        k_mir<<<dim3(nblk(maxn, 128), b->npatch), 128, 0, c->stream>>>(b->db);
        c->nlaunch++;
      }
      return st_statim(c, b, 1);
    });
    if (rc) return rc;
    if ((rc = st_connec(c))) return rc;
    return st_halo(c, 0);
  }
  if (phase == FF_PHASE_B) {
    if ((rc = st_halo(c, 1))) return rc;
    return fork_join(c, nb, [&](int n) { return st_statim(c, c->tops[n], 1); });
  }
  if (phase == FF_PHASE_RECORD) {
    k_record<<<1, 1, 0, c->stream>>>(c->d_resi, c->d_dromax, c->d_hist, c->d_hist_pos, c->hist_cap);
    c->nlaunch++;
    return 0;
  }
  return fail(c, FF_ERR_ARG, "ff_mb_phase: unknown phase");
}

void drop_phase_graphs(Ctx* c) {
  for (auto& g : c->phase_graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  if (c->mb_graph) { cudaGraphExecDestroy(c->mb_graph); c->mb_graph = nullptr; }
}

int run_cycle(Ctx* c, BlockCtx* b, int icycle) {
  return b->coarse ? mg_cycle(c, b, icycle) : one_cycle(c, b, icycle);
}

int ensure_hist(Ctx* c, int n) {
  if (n <= c->hist_cap) return 0;
  if (c->d_hist) cudaFree(c->d_hist);
  CK(cudaMalloc(&c->d_hist, sizeof(double) * 6 * n));
  c->hist_cap = n;
  for (auto* b : c->blocks)
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
  drop_phase_graphs(c);
  return 0;
}

}  // namespace


// ============================================================================
extern "C" {

int ff_abi_version(void) { return FF_ABI_VERSION; }

const char* ff_last_error(void* ctx) { return ctx ? ((Ctx*)ctx)->errmsg : "no context"; }

int ff_create(void** out, int device) {
  Ctx* c = new Ctx();
  c->device = device;
  *out = nullptr;
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CK(cudaMalloc(&c->d_bar, 2 * sizeof(unsigned)));
  CK(cudaMemset(c->d_bar, 0, 2 * sizeof(unsigned)));
  CK(cudaMalloc(&c->d_err, sizeof(int)));
  CK(cudaMemset(c->d_err, 0, sizeof(int)));
  CK(cudaMalloc(&c->d_resi, 16 * sizeof(double)));
  CK(cudaMalloc(&c->d_dromax, sizeof(unsigned long long)));
  CK(cudaMalloc(&c->d_hist_pos, sizeof(int)));
  CK(cudaMemset(c->d_hist_pos, 0, sizeof(int)));
  CK(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
  CK(cudaDeviceGetAttribute(&c->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  {   // co-resident CTAs of the cooperative sweep per SM, per instantiation and CTA size
    const int th[3] = {64, 128, 256};
    for (int t = 0; t < 3; t++) {
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->coop_occ[0][0][t], k_lusgs_sweep<double, 5>, th[t], 0));
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->coop_occ[0][1][t], k_lusgs_sweep<double, 7>, th[t], 0));
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->coop_occ[1][0][t], k_lusgs_sweep<float, 5>, th[t], 0));
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->coop_occ[1][1][t], k_lusgs_sweep<float, 7>, th[t], 0));
    }
  }
  CK(cudaEventCreate(&c->ev0));
  CK(cudaEventCreate(&c->ev1));
  *out = c;
  return 0;
}

int ff_destroy(void* ctx) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return FF_ERR_ARG;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (auto* b : c->blocks) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    cudaFree(b->base); cudaFree(b->d_patch);
    cudaFree(b->sw); cudaFree(b->swl); cudaFree(b->dwp); cudaFree(b->sw32); cudaFree(b->swl32); cudaFree(b->dwp32);
    cudaFree(b->d_red);
    if (b->aux) { cudaStreamDestroy(b->aux); cudaEventDestroy(b->aux_fork); cudaEventDestroy(b->aux_join); }
    delete b;
  }
  drop_phase_graphs(c);
  cudaFree(c->d_halo);
  for (size_t n = 0; n < c->side.size(); n++) { cudaStreamDestroy(c->side[n]); cudaEventDestroy(c->side_ev[n]); }
  if (c->fork_ev) cudaEventDestroy(c->fork_ev);
  cudaFree(c->d_blocks); cudaFree(c->d_conn);
  cudaFree(c->d_bar); cudaFree(c->d_err); cudaFree(c->d_resi); cudaFree(c->d_dromax);
  cudaFree(c->d_hist); cudaFree(c->d_hist_pos);
  cudaEventDestroy(c->ev0); cudaEventDestroy(c->ev1);
  cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

// ff_params.flux: a known scheme, and for a k-omega block one that RESIKE
// offers (van Leer, WPS and AUSM are laminar only: res3c.f:6946-7041).
static const char* flux_check(const ff_params* prm) {
  const int f = prm->flux;
  if (f != FF_FLUX_ROE && f != FF_FLUX_VANLEER && f != FF_FLUX_WPS && f != FF_FLUX_AUSM && f != FF_FLUX_KT &&
      f != FF_FLUX_HCUSP)
    return "ff_params.flux: unknown scheme";
  if (prm->iturb >= 3 && (f == FF_FLUX_VANLEER || f == FF_FLUX_WPS || f == FF_FLUX_AUSM))
    return "ff_params.flux: van Leer, WPS and AUSM (IFLUX=0, 2, 3) are laminar only";
  return nullptr;
}

// The body of ff_block_add: 0 and the new block's id in *id, or an error code.
static int block_add(Ctx* c, int imax, int jmax, int kmax, int npatch, const ff_patch* patches,
                     const ff_params* prm, int* id) {
  if (!c || imax < 2 || jmax < 2 || kmax < 1 || npatch < 0 || !prm) return fail(c, FF_ERR_ARG, "ff_block_add: bad dims");
  if (const char* why = flux_check(prm)) return fail(c, FF_ERR_ARG, why);
  BlockCtx* b = new BlockCtx();
  b->imax = imax; b->jmax = jmax; b->kmax = kmax;
  b->ntot = (imax + 4) * (jmax + 4) * (kmax + 4);
  b->slot_stride = (size_t)b->ntot;   // DRO..DE stay contiguous (5 x ntot)
  b->prm = *prm;
  b->npatch = npatch;
  b->h_patch.assign(patches, patches + npatch);
  for (auto& p : b->h_patch) {
    if (p.iface < 1 || p.iface > 6 || p.r1a < 1 || p.r2a < 1 || p.r1b < p.r1a || p.r2b < p.r2a) {
      delete b;
      return fail(c, FF_ERR_ARG, "ff_block_add: bad patch range");
    }
  }
  CK(cudaMalloc(&b->base, sizeof(double) * b->slot_stride * FF_NSLOTS));
  CK(cudaMemsetAsync(b->base, 0, sizeof(double) * b->slot_stride * FF_NSLOTS, c->stream));
  if (npatch) {
    CK(cudaMalloc(&b->d_patch, sizeof(ff_patch) * npatch));
    CK(cudaMemcpyAsync(b->d_patch, patches, sizeof(ff_patch) * npatch, cudaMemcpyHostToDevice, c->stream));
  }
  b->ns = sw_size(imax, jmax, kmax);
  { int rc = alloc_sweep(c, b); if (rc) return rc; }
  CK(cudaMalloc(&b->d_red, sizeof(unsigned long long) * 2));
  b->db.imax = imax; b->db.jmax = jmax; b->db.kmax = kmax;
  b->db.is = imax + 4; b->db.il = (imax + 4) * (jmax + 4); b->db.ntot = b->ntot;
  b->db.npatch = npatch; b->db.patch = b->d_patch;
  for (int s = 0; s < FF_NSLOTS; s++) b->db.a[s] = b->base + (size_t)s * b->slot_stride;
  {
    int rc = setup_lines(c, b);
    if (rc) return rc;
    if ((rc = setup_pipe(c, b))) return rc;
    const char* env = getenv("FINFLO_LUSGS");
    if (env && strcmp(env, "hyperplane") == 0) b->use_lines = 0;
    if (env && strcmp(env, "pipe") == 0 && b->can_pipe) { b->use_pipe = 1; b->use_lines = 0; }
  }
  b->tuned = 0;
  c->blocks.push_back(b);
  *id = (int)c->blocks.size() - 1;
  return FF_OK;
}

int ff_block_add(void* ctx, int imax, int jmax, int kmax, int npatch, const ff_patch* patches,
                 const ff_params* prm) {
  int id = -1;
  const int rc = block_add((Ctx*)ctx, imax, jmax, kmax, npatch, patches, prm, &id);
  return rc ? -rc : id;
}

int ff_mg_link(void* ctx, int fine, int coarse) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx *f = getb(c, fine), *cc = getb(c, coarse);
  if (!f || !cc || f == cc || f->imax != 2 * cc->imax || f->jmax != 2 * cc->jmax || f->kmax != 2 * cc->kmax)
    return fail(c, FF_ERR_ARG, "ff_mg_link: the coarse block must halve every dimension");
  f->coarse = cc;
  cc->level = f->level + 1;
  c->conn_blocks = -1;   // the level-1 block list changes
  if (f->graph) { cudaGraphExecDestroy(f->graph); f->graph = nullptr; }
  return 0;
}

int ff_block_params(void* ctx, int blk, const ff_params* prm) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || !prm) return fail(c, FF_ERR_ARG, "ff_block_params");
  if (const char* why = flux_check(prm)) return fail(c, FF_ERR_ARG, why);
  bool nv_changed = (b->prm.iturb >= 3) != (prm->iturb >= 3);
  bool fp_changed = (b->prm.lusgs_fp32 != 0) != (prm->lusgs_fp32 != 0);
  if ((b->prm.ddadi != 0) != (prm->ddadi != 0)) b->tuned = 0;
  b->prm = *prm;
  if (nv_changed) {   // the line sweep's shared memory depends on the equation count
    int rc = setup_lines(c, b);
    if (rc) return rc;
  }
  if (fp_changed) {
    int rc = alloc_sweep(c, b);
    if (rc) return rc;
  }
  if (nv_changed || fp_changed) {   // the pipelined sweep's instantiation and shared memory
    int rc = setup_pipe(c, b);
    if (rc) return rc;
    if (!b->can_pipe) b->use_pipe = 0;
  }
  if (nv_changed || fp_changed) b->tuned = 0;
  // captured cycles of any block may include this one (multigrid levels)
  for (auto* x : c->blocks)
    if (x->graph) { cudaGraphExecDestroy(x->graph); x->graph = nullptr; }
  drop_phase_graphs(c);
  return 0;
}

int ff_upload(void* ctx, int blk, int slot, const double* host) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || slot < 0 || slot >= FF_NSLOTS || !host) return fail(c, FF_ERR_ARG, "ff_upload");
  CK(cudaMemcpyAsync(b->db.a[slot], host, sizeof(double) * b->ntot, cudaMemcpyHostToDevice, c->stream));
  if (slot >= FF_A1 && slot <= FF_VOL && b->sw_static) metrics_changed(c, b);
  return 0;
}

int ff_host_register(void* ctx, void* host, size_t bytes) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !host || !bytes) return fail(c, FF_ERR_ARG, "ff_host_register");
  CK(cudaHostRegister(host, bytes, cudaHostRegisterDefault));
  return 0;
}

int ff_host_unregister(void* ctx, void* host) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !host) return fail(c, FF_ERR_ARG, "ff_host_unregister");
  CK(cudaHostUnregister(host));
  return 0;
}

int ff_download(void* ctx, int blk, int slot, double* host) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || slot < 0 || slot >= FF_NSLOTS || !host) return fail(c, FF_ERR_ARG, "ff_download");
  CK(cudaMemcpyAsync(host, b->db.a[slot], sizeof(double) * b->ntot, cudaMemcpyDeviceToHost, c->stream));
  return 0;
}

void* ff_device_ptr(void* ctx, int blk, int slot) {
  BlockCtx* b = getb((Ctx*)ctx, blk);
  if (!b || slot < 0 || slot >= FF_NSLOTS) return nullptr;
  return b->db.a[slot];
}

void* ff_stream(void* ctx) { return ctx ? (void*)((Ctx*)ctx)->stream : nullptr; }

int ff_synchronize(void* ctx) {
  Ctx* c = (Ctx*)ctx;
  if (!c) return FF_ERR_ARG;
  CK(cudaStreamSynchronize(c->stream));
  int err = 0;
  CK(cudaMemcpy(&err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemset(c->d_err, 0, sizeof(int));
    cudaMemset(c->d_bar, 0, 2 * sizeof(unsigned));
    return fail(c, FF_ERR_TIMEOUT, "LU-SGS grid barrier timed out");
  }
  return 0;
}

int ff_statim(void* ctx, int blk) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b) return fail(c, FF_ERR_ARG, "ff_statim");
  st_statim(c, b, 1);   // one STATIM call: equation of state + REFLEC
  CK(cudaGetLastError());
  return 0;
}

int ff_boundi(void* ctx, int blk) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b) return fail(c, FF_ERR_ARG, "ff_boundi");
  st_boundi(c, b);
  CK(cudaGetLastError());
  return 0;
}

int ff_residu(void* ctx, int blk, int level, int icycle) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || level != b->level) return fail(c, FF_ERR_ARG, "ff_residu: level is not the block's multigrid level");
  st_residu(c, b, level, icycle, level);
  CK(cudaGetLastError());
  return 0;
}

int ff_residi(void* ctx, int blk, int m2, int icycle) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || m2 < b->level || m2 > b->level + 1) return fail(c, FF_ERR_ARG, "ff_residi: M2 must be M or M+1");
  st_residu(c, b, b->level, icycle, m2);
  CK(cudaGetLastError());
  return 0;
}

int ff_transf(void* ctx, int fine, int coarse) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx *f = getb(c, fine), *cc = getb(c, coarse);
  if (!f || !cc || f->coarse != cc) return fail(c, FF_ERR_ARG, "ff_transf: blocks are not linked levels");
  const int sst = f->prm.iturb >= 3;
  long nc = (long)(cc->imax + 2) * (cc->jmax + 2) * (cc->kmax + 2);
  k_transf<<<nblk(nc, 128), 128, 0, c->stream>>>(f->db, cc->db, sst);
  k_transf_ring<<<nblk(cc->ntot, 256), 256, 0, c->stream>>>(cc->db, sst);
  c->nlaunch += 2;
  CK(cudaGetLastError());
  return 0;
}

int ff_forcfu(void* ctx, int blk) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b) return fail(c, FF_ERR_ARG, "ff_forcfu");
  k_forcing<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db, 0, b->prm.iturb >= 3);
  c->nlaunch++;
  CK(cudaGetLastError());
  return 0;
}

int ff_addres(void* ctx, int blk) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b) return fail(c, FF_ERR_ARG, "ff_addres");
  k_forcing<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db, 1, b->prm.iturb >= 3);
  c->nlaunch++;
  CK(cudaGetLastError());
  return 0;
}

int ff_interp(void* ctx, int coarse, int fine) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx *f = getb(c, fine), *cc = getb(c, coarse);
  if (!f || !cc || f->coarse != cc) return fail(c, FF_ERR_ARG, "ff_interp: blocks are not linked levels");
  int nf = f->imax * f->jmax * f->kmax;
  k_interp<<<nblk(nf, 256), 256, 0, c->stream>>>(cc->db, f->db);
  c->nlaunch++;
  if (f->prm.iturb >= 3) {
    k_intert<<<nblk(nf, 256), 256, 0, c->stream>>>(cc->db, f->db, f->prm);
    c->nlaunch++;
  }
  k_fin_coarse<<<nblk(f->ntot, 256), 256, 0, c->stream>>>(f->db, f->prm, 0);
  c->nlaunch++;
  CK(cudaGetLastError());
  return 0;
}

int ff_resl2(void* ctx, int blk, double* out5) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || !out5) return fail(c, FF_ERR_ARG, "ff_resl2");
  k_reset_acc<<<1, 32, 0, c->stream>>>(c->d_resi, c->d_dromax);
  c->nlaunch++;
  int ncell = b->imax * b->jmax * b->kmax;
  k_resl2<<<min(nblk(ncell, 256), 4 * c->sm_count), 256, 0, c->stream>>>(b->db, c->d_resi);
  c->nlaunch++;
  CK(cudaMemcpyAsync(out5, c->d_resi, 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int ff_block_metrics(void* ctx, int blk, const double* xyz) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || !xyz) return fail(c, FF_ERR_ARG, "ff_block_metrics");
  metrics_changed(c, b);
  const GridDims g{b->imax + 1, b->jmax + 1, b->kmax + 1};
  const size_t nn = (size_t)g.ni * g.nj * g.nk, ne = (size_t)(g.ni + 4) * (g.nj + 4) * (g.nk + 4);
  double *dn = nullptr, *de = nullptr;
  CK(cudaMalloc(&dn, 3 * nn * sizeof(double)));
  if (cudaMalloc(&de, 3 * ne * sizeof(double)) != cudaSuccess) { cudaFree(dn); return fail(c, FF_ERR_CUDA, "ff_block_metrics"); }
  cudaError_t e = cudaMemcpyAsync(dn, xyz, 3 * nn * sizeof(double), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) {
    k_extend_nodes<<<nblk((long)ne, 256), 256, 0, c->stream>>>(dn, de, g);
    k_cell_metrics<<<nblk((long)b->ntot, 256), 256, 0, c->stream>>>(b->db, de);
    c->nlaunch += 2;
    e = cudaStreamSynchronize(c->stream);
  }
  cudaFree(dn);
  cudaFree(de);
  if (e != cudaSuccess) return fail(c, FF_ERR_CUDA, "ff_block_metrics", e);
  CK(cudaGetLastError());
  return 0;
}

int ff_block_metrics_levels(void* ctx, int blk, int nlev, const double* xyz) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || !xyz || nlev < 1) return fail(c, FF_ERR_ARG, "ff_block_metrics_levels");
  std::vector<BlockCtx*> lv;
  for (BlockCtx* x = b; x && (int)lv.size() < nlev; x = x->coarse) lv.push_back(x);
  if ((int)lv.size() != nlev) return fail(c, FF_ERR_ARG, "ff_block_metrics_levels: fewer linked levels than nlev");
  for (BlockCtx* x : lv) metrics_changed(c, x);
  const int ng = 2 << (nlev - 1);
  const GridDims g{b->imax + 1, b->jmax + 1, b->kmax + 1};
  const size_t nn = (size_t)g.ni * g.nj * g.nk;
  RawDims r{b->imax + 2 * ng, b->jmax + 2 * ng, b->kmax + 2 * ng};
  const size_t ne = (size_t)(r.ci + 1) * (r.cj + 1) * (r.ck + 1);
  double *dn = nullptr, *de = nullptr, *raw = nullptr, *raw2 = nullptr;
  auto cleanup = [&]() { cudaFree(dn); cudaFree(de); cudaFree(raw); cudaFree(raw2); };
  if (cudaMalloc(&dn, 3 * nn * sizeof(double)) != cudaSuccess || cudaMalloc(&de, 3 * ne * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&raw, RW_N * r.n() * sizeof(double)) != cudaSuccess) {
    cleanup();
    return fail(c, FF_ERR_CUDA, "ff_block_metrics_levels: device memory");
  }
  cudaError_t e = cudaMemcpyAsync(dn, xyz, 3 * nn * sizeof(double), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) {
    k_extend_nodes<<<nblk((long)ne, 256), 256, 0, c->stream>>>(dn, de, g, ng);
    k_raw_metrics<<<nblk((long)r.n(), 256), 256, 0, c->stream>>>(de, raw, r);
    c->nlaunch += 2;
    int lng = ng;
    for (int l = 0; l < nlev && e == cudaSuccess; l++) {
      BlockCtx* x = lv[l];
      k_finish_metrics<<<nblk((long)x->ntot, 256), 256, 0, c->stream>>>(x->db, raw, r, lng);
      c->nlaunch++;
      if (l + 1 < nlev) {
        RawDims rc{r.ci / 2, r.cj / 2, r.ck / 2};
        if (lv[l + 1]->imax + 2 * (lng / 2) != rc.ci || lv[l + 1]->jmax + 2 * (lng / 2) != rc.cj ||
            lv[l + 1]->kmax + 2 * (lng / 2) != rc.ck) {
          cleanup();
          return fail(c, FF_ERR_ARG, "ff_block_metrics_levels: a coarse level does not halve the finer one");
        }
        if (cudaMalloc(&raw2, RW_N * rc.n() * sizeof(double)) != cudaSuccess) { e = cudaErrorMemoryAllocation; break; }
        k_lump<<<nblk((long)rc.n(), 256), 256, 0, c->stream>>>(raw, r, raw2, rc);
        c->nlaunch++;
        e = cudaStreamSynchronize(c->stream);
        cudaFree(raw);
        raw = raw2;
        raw2 = nullptr;
        r = rc;
        lng /= 2;
      }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  }
  cleanup();
  if (e != cudaSuccess) return fail(c, FF_ERR_CUDA, "ff_block_metrics_levels", e);
  CK(cudaGetLastError());
  return 0;
}

int ff_wall_distance(void* ctx, int blk, const double* pts, int npts) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || npts < 0 || (npts > 0 && !pts)) return fail(c, FF_ERR_ARG, "ff_wall_distance");
  double* dp = nullptr;
  if (npts > 0) CK(cudaMalloc(&dp, (size_t)npts * 3 * sizeof(double)));
  cudaError_t e = npts > 0 ? cudaMemcpyAsync(dp, pts, (size_t)npts * 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream)
                           : cudaSuccess;
  // the block, then each coarser level: every cell's nearest point, and
  // the interior cells again as the mean of their children (LUMP_DIST)
  BlockCtx* fine = nullptr;
  for (BlockCtx* x = b; x && e == cudaSuccess; fine = x, x = x->coarse) {
    k_wall_distance<<<nblk((long)x->ntot, WD_THREADS), WD_THREADS, 0, c->stream>>>(x->db, dp, npts);
    c->nlaunch++;
    if (fine) {
      k_lump_distw<<<nblk((long)x->imax * x->jmax * x->kmax, 256), 256, 0, c->stream>>>(fine->db, x->db);
      c->nlaunch++;
    }
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (dp) cudaFree(dp);
  if (e != cudaSuccess) return fail(c, FF_ERR_CUDA, "ff_wall_distance", e);
  return 0;
}

int ff_time_levels(void* ctx, int blk, int mode) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || (mode != 0 && mode != 1)) return fail(c, FF_ERR_ARG, "ff_time_levels");
  const long n = mode == 0 ? (long)b->ntot : (long)b->imax * b->jmax * b->kmax;
  k_time_levels<<<nblk(n, 256), 256, 0, c->stream>>>(b->db, b->prm.iturb >= 3 ? 7 : 5, mode);
  c->nlaunch++;
  CK(cudaGetLastError());
  return 0;
}

int ff_imps(void* ctx, int blk, int level) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || level != b->level) return fail(c, FF_ERR_ARG, "ff_imps: level is not the block's multigrid level");
  int rc = st_imps(c, b, level, true);
  if (rc) return rc;
  CK(cudaGetLastError());
  return 0;
}

int ff_fin(void* ctx, int blk, double* dromax) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b) return fail(c, FF_ERR_ARG, "ff_fin");
  k_reset_acc<<<1, 32, 0, c->stream>>>(c->d_resi, c->d_dromax);
  c->nlaunch++;
  if (b->level > 1) {   // coarse level: FIN with the coarse limits (ns3c.f:1935-1990)
    k_fin_coarse<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db, b->prm, 1);
    c->nlaunch++;
    if (dromax) *dromax = 0.0;
    CK(cudaGetLastError());
    return 0;
  }
  st_fin(c, b, 0);
  if (dromax) {
    unsigned long long bits;
    CK(cudaMemcpyAsync(&bits, c->d_dromax, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    memcpy(dromax, &bits, sizeof(double));
  }
  CK(cudaGetLastError());
  return 0;
}

int ff_cycles(void* ctx, int blk, int ncycles, int icycle0, double* hist, int use_graph) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || ncycles < 0) return fail(c, FF_ERR_ARG, "ff_cycles");
  int rc;
  for (BlockCtx* x = b; x; x = x->coarse) {
    if (!x->tuned) {
      if ((rc = tune_sweep(c, x))) return rc;
      if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    }
  }
  if ((rc = ensure_hist(c, max(ncycles, 1)))) return rc;
  CK(cudaMemsetAsync(c->d_hist_pos, 0, sizeof(int), c->stream));
  int it = 0;
  // the first cycle of a run (ICYCLE = 1) differs (INLET density), run it eagerly
  while (it < ncycles && (icycle0 + it == 1 || !use_graph)) {
    if ((rc = run_cycle(c, b, icycle0 + it))) return rc;
    it++;
  }
  if (it < ncycles) {
    int want = b->prm.lusgs_fp32 ? 1 : 0;
    if (!b->graph || b->graph_fp32 != want) {
      if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      long n0 = c->nlaunch;
      rc = run_cycle(c, b, 2);
      b->cycle_launches = (int)(c->nlaunch - n0);
      cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      if (rc) return rc;
      if (e != cudaSuccess) return fail(c, FF_ERR_CUDA, "cycle capture", e);
      CK(cudaGraphInstantiate(&b->graph, g, 0));
      cudaGraphDestroy(g);
      b->graph_fp32 = want;
    }
    for (; it < ncycles; it++) CK(cudaGraphLaunch(b->graph, c->stream));
  }
  CK(cudaGetLastError());
  if (hist) {
    CK(cudaMemcpyAsync(hist, c->d_hist, sizeof(double) * 6 * ncycles, cudaMemcpyDeviceToHost, c->stream));
    rc = ff_synchronize(ctx);
    if (rc) return rc;
  }
  return 0;
}

int ff_sweep_tuning(void* ctx, int blk, float* ms2) {
  BlockCtx* b = getb((Ctx*)ctx, blk);
  if (!b || !ms2) return FF_ERR_ARG;
  ms2[0] = b->sweep_ms[0];
  ms2[1] = b->sweep_ms[1];
  return 0;
}

int ff_sweep_times(void* ctx, int blk, float* ms3) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || !ms3) return fail(c, FF_ERR_ARG, "ff_sweep_times");
  if (b->prm.ddadi) {   // DDADI: the chosen form's time per direction {k, i, j}
    ms3[0] = b->dd_ms[3]; ms3[1] = b->dd_ms[1]; ms3[2] = b->dd_ms[2];
    return 0;
  }
  ms3[0] = b->pipe_ms;
  ms3[1] = b->sweep_ms[0];
  ms3[2] = b->sweep_ms[1];
  return 0;
}

int ff_lusgs_kind(void* ctx, int blk) {
  BlockCtx* b = getb((Ctx*)ctx, blk);
  if (!b) return -FF_ERR_ARG;
  if (b->prm.ddadi)
    return b->dd_cfg[1] < 0 ? 4 : 4 + 100 * (1000 + 100 * b->dd_cfg[3] + 10 * b->dd_cfg[1] + b->dd_cfg[2]);
  if (b->use_pipe) return 3 + 100 * b->pg.ntj * b->pg.ntk;
  return b->use_lines ? 1 + b->lg.cs * 100 : 2 + b->coop_threads * 100;
}

int ff_residual_shape(void* ctx, int blk) {
  BlockCtx* b = getb((Ctx*)ctx, blk);
  if (!b) return -FF_ERR_ARG;
  return b->res_shape;
}

int ff_cycle_launches(void* ctx, int blk) {
  BlockCtx* b = getb((Ctx*)ctx, blk);
  return b ? b->cycle_launches : -FF_ERR_ARG;
}

int ff_halo_plan(void* ctx, int nitems, const ff_halo_item* items, double* send_buf, double* recv_buf) {
  Ctx* c = (Ctx*)ctx;
  if (!c || nitems < 0 || (nitems && !items)) return fail(c, FF_ERR_ARG, "ff_halo_plan");
  int nb = (int)c->blocks.size();
  std::vector<HaloItem> h(nitems);
  bool pk = false, up = false;
  int maxn = 1;
  for (int i = 0; i < nitems; i++) {
    const ff_halo_item& it = items[i];
    if (it.blk < 0 || it.blk >= nb || (it.mode != 0 && it.mode != 1) || it.offset < 0)
      return fail(c, FF_ERR_ARG, "ff_halo_plan: bad item");
    BlockCtx* b = c->blocks[it.blk];
    const ff_patch& pa = it.pa;
    int face = it.mode == 0 ? pa.nface : pa.iface;
    int n1 = pa.r1b - pa.r1a + 1, n2 = pa.r2b - pa.r2a + 1;
    int d = (face - 1) % 3;
    int e1 = d == 0 ? b->jmax : b->imax, e2 = d == 2 ? b->jmax : b->kmax;
    int s1 = it.mode == 0 ? pa.n1a : pa.r1a, s2 = it.mode == 0 ? pa.n2a : pa.r2a;
    if (face < 1 || face > 6 || n1 < 1 || n2 < 1 || s1 < 1 || s2 < 1 || s1 + n1 - 1 > e1 || s2 + n2 - 1 > e2)
      return fail(c, FF_ERR_ARG, "ff_halo_plan: patch range outside the block");
    if (it.mode == 0 ? !send_buf : !recv_buf) return fail(c, FF_ERR_ARG, "ff_halo_plan: missing buffer");
    h[i].blk = it.blk; h[i].mode = it.mode; h[i].offset = it.offset; h[i].pa = pa;
    pk = pk || it.mode == 0; up = up || it.mode == 1;
    maxn = max(maxn, n1 * n2);
  }
  int rc;
  if ((rc = ensure_conn(c))) return rc;
  if (c->d_halo) cudaFree(c->d_halo);
  c->d_halo = nullptr;
  if (nitems) {
    CK(cudaMalloc(&c->d_halo, sizeof(HaloItem) * nitems));
    CK(cudaMemcpy(c->d_halo, h.data(), sizeof(HaloItem) * nitems, cudaMemcpyHostToDevice));
  }
  c->nhalo = nitems; c->halo_maxn = maxn; c->halo_pack = pk; c->halo_unpack = up;
  c->halo_send = send_buf; c->halo_recv = recv_buf;
  drop_phase_graphs(c);
  return 0;
}

int ff_mb_phase(void* ctx, int phase, int icycle, int use_graph) {
  Ctx* c = (Ctx*)ctx;
  if (!c || c->blocks.empty()) return fail(c, FF_ERR_ARG, "ff_mb_phase");
  for (auto* b : c->blocks)
    if (b->coarse || b->level != 1) return fail(c, FF_ERR_ARG, "ff_mb_phase: single-grid blocks only");
  int rc;
  if ((rc = ensure_conn(c))) return rc;
  if (phase == FF_PHASE_RECORD && (rc = ensure_hist(c, 1))) return rc;
  int gi = phase == FF_PHASE_CYCLE_A ? 0 : (phase == FF_PHASE_B ? 1 : -1);
  if (!use_graph || icycle <= 1 || gi < 0) {
    if ((rc = mb_phase(c, phase, icycle))) return rc;
  } else {
    if (!c->phase_graph[gi]) {
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      rc = mb_phase(c, phase, 2);
      cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      if (rc) return rc;
      if (e != cudaSuccess) return fail(c, FF_ERR_CUDA, "phase capture", e);
      CK(cudaGraphInstantiate(&c->phase_graph[gi], g, 0));
      cudaGraphDestroy(g);
    }
    CK(cudaGraphLaunch(c->phase_graph[gi], c->stream));
  }
  CK(cudaGetLastError());
  return 0;
}

int ff_history(void* ctx, int n, double* hist, int reset) {
  Ctx* c = (Ctx*)ctx;
  if (!c || n < 0) return fail(c, FF_ERR_ARG, "ff_history");
  if (!hist) {
    int rc = ensure_hist(c, max(n, 1));
    if (rc) return rc;
    if (reset) CK(cudaMemsetAsync(c->d_hist_pos, 0, sizeof(int), c->stream));
    return 0;
  }
  if (n > c->hist_cap) return fail(c, FF_ERR_ARG, "ff_history: more rows than recorded");
  if (n) CK(cudaMemcpyAsync(hist, c->d_hist, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, c->stream));
  if (reset && c->d_hist_pos) CK(cudaMemsetAsync(c->d_hist_pos, 0, sizeof(int), c->stream));
  return ff_synchronize(ctx);
}

int ff_boundi_all(void* ctx) {
  Ctx* c = (Ctx*)ctx;
  if (!c || c->blocks.empty()) return fail(c, FF_ERR_ARG, "ff_boundi_all");
  int rc;
  if ((rc = ensure_conn(c))) return rc;   // BOUNDI over the level-1 blocks
  if ((rc = mb_boundi(c))) return rc;
  CK(cudaGetLastError());
  return 0;
}

int ff_cycles_all(void* ctx, int ncycles, int icycle0, double* hist, int use_graph) {
  Ctx* c = (Ctx*)ctx;
  if (!c || ncycles < 0 || c->blocks.empty()) return fail(c, FF_ERR_ARG, "ff_cycles_all");
  int rc;
  if ((rc = ensure_conn(c))) return rc;
  if ((rc = ensure_hist(c, max(ncycles, 1)))) return rc;
  CK(cudaMemsetAsync(c->d_hist_pos, 0, sizeof(int), c->stream));
  int it = 0;
  while (it < ncycles && (icycle0 + it == 1 || !use_graph)) {
    if ((rc = mb_cycle(c, icycle0 + it))) return rc;
    it++;
  }
  if (it < ncycles) {
    int nb = (int)c->tops.size();
    if (!c->mb_graph || c->mb_graph_n != nb) {
      if (c->mb_graph) { cudaGraphExecDestroy(c->mb_graph); c->mb_graph = nullptr; }
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      long n0 = c->nlaunch;
      rc = mb_cycle(c, 2);
      c->mb_launches = (int)(c->nlaunch - n0);
      cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      if (rc) return rc;
      if (e != cudaSuccess) return fail(c, FF_ERR_CUDA, "multi-block cycle capture", e);
      CK(cudaGraphInstantiate(&c->mb_graph, g, 0));
      cudaGraphDestroy(g);
      c->mb_graph_n = nb;
    }
    for (; it < ncycles; it++) CK(cudaGraphLaunch(c->mb_graph, c->stream));
  }
  CK(cudaGetLastError());
  if (hist) {
    CK(cudaMemcpyAsync(hist, c->d_hist, sizeof(double) * 6 * ncycles, cudaMemcpyDeviceToHost, c->stream));
    rc = ff_synchronize(ctx);
    if (rc) return rc;
  }
  return 0;
}

int ff_time_cycles_all(void* ctx, int ncycles, float* ms, int* launches_per_cycle) {
  Ctx* c = (Ctx*)ctx;
  if (!c || !ms) return fail(c, FF_ERR_ARG, "ff_time_cycles_all");
  CK(cudaEventRecord(c->ev0, c->stream));
  int rc = ff_cycles_all(ctx, ncycles, 2, nullptr, 1);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  CK(cudaEventElapsedTime(ms, c->ev0, c->ev1));
  if (launches_per_cycle) *launches_per_cycle = c->mb_launches;
  return ff_synchronize(ctx);
}

int ff_time_cycles(void* ctx, int blk, int ncycles, float* ms) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || !ms) return fail(c, FF_ERR_ARG, "ff_time_cycles");
  CK(cudaEventRecord(c->ev0, c->stream));
  int rc = ff_cycles(ctx, blk, ncycles, 2, nullptr, 1);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  CK(cudaEventElapsedTime(ms, c->ev0, c->ev1));
  return ff_synchronize(ctx);
}

int ff_time_stage(void* ctx, int blk, int stage, int reps, float* ms) {
  Ctx* c = (Ctx*)ctx;
  BlockCtx* b = getb(c, blk);
  if (!b || !ms || reps < 1) return fail(c, FF_ERR_ARG, "ff_time_stage");
  if (stage == FF_STAGE_SWEEP) {   // the sweep's kernel choice and (LU-SGS) its data in the sweep layout
    int rc = tune_sweep(c, b);
    if (rc) return rc;
    if (!b->prm.ddadi) sweep_coef(c, b, 1, b->prm.lusgs_fp32 != 0);
  }
  CK(cudaEventRecord(c->ev0, c->stream));
  for (int r = 0; r < reps; r++) {
    if (stage == FF_STAGE_RESIDUAL) {
      launch_residual(c->stream, b, 1);
      c->nlaunch++;
    } else if (stage == FF_STAGE_SWEEP) {   // LU-SGS: the lower sweep; DDADI: all three directions
      int rc = b->prm.ddadi ? ddadi_sweeps(c, b) : sweep(c, b, 1, b->prm.lusgs_fp32 != 0);
      if (rc) return rc;
    } else if (stage == FF_STAGE_GRAD) {
      long ng = (long)(b->imax + 2) * (b->jmax + 2) * (b->kmax + 2);
      k_grad<<<nblk(ng, 128), 128, 0, c->stream>>>(b->db, 1);
      c->nlaunch++;
    } else if (stage == FF_STAGE_STATE) {
      k_state<<<nblk(b->ntot, 256), 256, 0, c->stream>>>(b->db, b->prm);
      c->nlaunch++;
    } else {
      return fail(c, FF_ERR_ARG, "ff_time_stage: unknown stage");
    }
  }
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  CK(cudaEventElapsedTime(ms, c->ev0, c->ev1));
  *ms /= reps;
  return 0;
}

}  // extern "C"

// The allocation-free implicit stage shares this translation unit's kernels.
#include "ff_noalloc.cu"
// The Fortran call-site wrappers (statim_, residi_, impsdi_, fin_, boundi_).
#include "ff_fortran.cu"
