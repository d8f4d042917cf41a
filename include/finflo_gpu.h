/*
 * libfinflo_gpu.so -- C-ABI of the sm_100a FINFLO per-iteration hot path.
 *
 * One context = one CUDA device + one stream.  Blocks are stored on the
 * device in the reference's own layout (finflo_types.h): every per-cell array
 * is FP64, NTOT = (IMAX+4)*(JMAX+4)*(KMAX+4), i fastest, two ghost layers.
 * Stage calls are asynchronous on the context's stream; ff_synchronize()
 * waits and reports device-side time-outs.  Every function returns 0 on
 * success or one of the FF_ERR_* codes (ff_last_error() has the message); no
 * function aborts the process (the reference STOPs, e.g. ns3c.f:2209-2217).
 *
 * Reference interfaces replaced (Fortran, every argument by reference):
 *   ff_statim    STATIM  ns3c.f:10318  (PDTOP, STATE/PERFGA, CONSVA, REFLEC)
 *   ff_residu    RESIDI  ns3c.f:2355 -> RESIDU res3c.f:6 (level 1, laminar)
 *   ff_resl2     RESL2   res3c.f:8920
 *   ff_imps      IMPSDI  ns3c.f:2683 -> IMPS imps3.f:6 (LUSGS = 1: PREDGS,
 *                DIAGGS, CORRGS; prm->ddadi = 1 selects LUSGS = 0: IMPSWE
 *                imps3.f:578 per direction, PRED/DIAG/CORR imps4.f:671-971)
 *   ff_fin       FIN     res3c.f:1077 + the limits of CYCLES ns3c.f:1553-1596
 *   ff_boundi    BOUNDI  ns3c.f:10608 (REFCOR, MIR, STATIM; single block)
 *   ff_cycles    CYCLES  ns3c.f:1354 + BOUNDI + SUBIN per cycle, graph-replayed
 *   ff_residi    RESIDI  ns3c.f:2355 on any multigrid level (M2 as passed)
 *   ff_transf    TRANSF  multi.f:156 (+ TRANKE multi.f:434 for k-omega)
 *   ff_forcfu    FORCFU  multi.f:1609    ff_addres  ADDRES multi.f:1686
 *   ff_interp    INTERP  multi.f:1763 (+ INTERT multi.f:2051) and the limits
 *                after it (ns3c.f:2059-2125)
 * and, for a Fortran host, the call-site wrappers statim_, residi_, impsdi_,
 * fin_ and boundi_ (gfortran names; declared at the end of this header).
 */
#ifndef FINFLO_GPU_H
#define FINFLO_GPU_H
#include "finflo_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define FF_ABI_VERSION 7   /* 7: ff_params.xxtral, rjk2, rjk4 and the FF_SCALEJ slot; 6: ff_params.flux (ff_flux) replaces vanleer */

enum { FF_OK = 0, FF_ERR_CUDA = 1, FF_ERR_ARG = 2, FF_ERR_TIMEOUT = 3, FF_ERR_SIZE = 4 };
enum { FF_STAGE_RESIDUAL = 1, FF_STAGE_GRAD = 2, FF_STAGE_STATE = 3, FF_STAGE_SWEEP = 4 };

int ff_abi_version(void);
const char *ff_last_error(void *ctx);

int ff_create(void **ctx, int device);
int ff_destroy(void *ctx);

/* Add a block (one multigrid level); returns the block id (>= 0) or -code. */
int ff_block_add(void *ctx, int imax, int jmax, int kmax, int npatch,
                 const ff_patch *patches, const ff_params *prm);
int ff_block_params(void *ctx, int blk, const ff_params *prm);
/* Make `coarse` the next multigrid level of `fine` (every dimension halved;
 * MGRID levels, main.f:4613-4630).  ff_cycles on the finest block then runs
 * the FAS V-cycle of CYCLES (ns3c.f:1607-2170) over the chain. */
int ff_mg_link(void *ctx, int fine, int coarse);

/* Host <-> device copy of one per-cell array slot (enum ff_slot), NTOT doubles. */
int ff_upload(void *ctx, int blk, int slot, const double *host);
int ff_download(void *ctx, int blk, int slot, double *host);
/* Page-lock (and release) a host array that ff_upload / ff_download use
 * every cycle, so the copies run as direct DMA at full PCIe/NVLink-C2C rate
 * instead of through a staging buffer.  Nothing is allocated on the device;
 * the host memory stays the caller's.  No reference counterpart (the
 * reference's arrays never leave the host). */
int ff_host_register(void *ctx, void *host, size_t bytes);
int ff_host_unregister(void *ctx, void *host);
void *ff_device_ptr(void *ctx, int blk, int slot);
void *ff_stream(void *ctx);
int ff_synchronize(void *ctx);

/* Stages (drop-in replacements of the reference routines listed above). */
int ff_statim(void *ctx, int blk);
int ff_boundi(void *ctx, int blk);
int ff_residu(void *ctx, int blk, int level, int icycle);
int ff_resl2(void *ctx, int blk, double *out5);
int ff_imps(void *ctx, int blk, int level);
int ff_fin(void *ctx, int blk, double *dromax);
/* ff_residu, ff_imps and ff_fin also run on a coarse multigrid level: level
 * must be the block's own level (1 + its depth in the ff_mg_link chain); on
 * a coarse level ff_residu is RESIDI(M, N, M) (first-order Roe, FLUXDO),
 * ff_fin applies the coarse-level limits (ns3c.f:1935-1990) and returns
 * dromax = 0. */

/* RESIDI(M, N, M2) ns3c.f:2355 on the block's own level M: M2 = M, or
 * M2 = M + 1 for the finer level's residual that TRANSF restricts next (the
 * k-omega gradients are then recomputed, ns3c.f:1626).  ICYCLE as passed. */
int ff_residi(void *ctx, int blk, int m2, int icycle);

/* Multigrid stages of CYCLES (ns3c.f:1607-2170) for a host that drives the
 * V-cycle itself; `fine` and `coarse` must be linked by ff_mg_link.
 * ff_transf  TRANSF multi.f:156 (TRANKE multi.f:434 with k-omega): volume-
 *            weighted restriction of TEMP, U, V, W, PDIFF, EPS2, VIST (RK,
 *            REPS) and of the fine residual into the coarse P2H, the coarse
 *            *OLD copies and ghost rings (ns3c.f:1687);
 * ff_forcfu  FORCFU multi.f:1609: P2H = P2H - R(coarse) (ns3c.f:1859);
 * ff_addres  ADDRES multi.f:1686: R = P2H + R (ns3c.f:1677, 1877);
 * ff_interp  INTERP multi.f:1763 (INTERT multi.f:2051 with k-omega): the
 *            coarse correction injected into the fine level, then the limits
 *            CYCLES applies after it (ns3c.f:2017-2125). */
int ff_transf(void *ctx, int fine, int coarse);
int ff_forcfu(void *ctx, int blk);
int ff_addres(void *ctx, int blk);
int ff_interp(void *ctx, int coarse, int fine);

/* Time-accurate runs (ff_params.timel = 1, physical step ff_params.dt):
 * ff_residu adds TIMDER res3c.f:3014 (and TIMDKE res3c.f:3062) on level 1
 * and TIME3 takes the dual time step (base3c.f:206-215).  The old time
 * levels live in slots FF_ROLE2..FF_EPSLE3.  mode 0 = STARTI res3c.f:3175
 * (both old levels = the current state, once before the first physical
 * step), mode 1 = NEWTIM ns3c.f:9420 (shift the levels at the start of
 * every later physical step), asynchronous. */
int ff_time_levels(void *ctx, int blk, int mode);

/* Block set-up on the device (no counterpart call in the reference, which
 * computes its metrics in GRIVAL/GRID1B ns3c.f:5636, gluebm.f:1265 and its
 * wall distance in DISTANCES gluebm.f:9136 on the host).
 * ff_block_metrics: xyz = the block's nodes, X then Y then Z, each
 * (KMAX+1)(JMAX+1)(IMAX+1) values with i fastest; fills A1..A3ZA, VOL,
 * XC..ZC and D1..D3 of every cell, ghosts included: GRID1B's construction
 * (gluebm.f:1265; GRIDEX ghost nodes 1029, AREVC1 1586, D1D2D3 2326), the
 * further ghost layers from continued mirror reflection of the nodes.
 * ff_wall_distance: pts = npts wall points of 3 values (PICK_XYZ
 * gluebm.f:9452: halfway between the first interior and ghost cell centres
 * of the solid patches, of every block); fills DISTW of every cell of the
 * block with the distance of its centre to the nearest point (WALL_DIST
 * 9533; 1e4 when npts = 0), and of its linked coarse levels the same, their
 * interior cells then the mean of their eight children (LUMP_DIST 9562).
 * Both synchronous. */
int ff_block_metrics(void *ctx, int blk, const double *xyz);
/* The same for a block and its nlev - 1 linked coarse levels (ff_mg_link):
 * the fine cells with 2 * 2^(nlev-1) ghost layers, each coarse level lumped
 * from the finer one (LUMPA1 gluebm.f:2194 for the faces, LUMPVS 2256 for
 * volumes and centres). */
int ff_block_metrics_levels(void *ctx, int blk, int nlev, const double *xyz);
int ff_wall_distance(void *ctx, int blk, const double *pts, int npts);

/* With ff_params.iturb = 6 (k-omega SST) ff_residu is
 * TURBEQ res3c.f:5845 + RESIKE res3c.f:3423, ff_imps the seven-equation
 * IMPS (LOCDTK, IMSOKO, COPRKE, PRKEGS/DIKEGS/COKEGS) and ff_fin also
 * updates RK, REPS; ff_cycles adds the cycle-start STATIM and the k cap of
 * SUBIN; linked multigrid levels run TRANKE, the k-omega forcing, the
 * coarse-level RESIKE (FLUDKE, first-order Roe) and INTERT. */

/* ncycles full cycles (RESIDU, RESL2, IMPS, FIN, BOUNDI, SUBIN); hist
 * (nullable) receives ncycles x {RESI(31..35) sums of squares, DROMAX}. */
int ff_cycles(void *ctx, int blk, int ncycles, int icycle0, double *hist, int use_graph);

/* Allocation-free implicit stage.  No counterpart in the reference: it is the
 * ff_imps stage (TIME3, LOCDT, COPR, PREDGS, DIAGGS, CORRGS, DRO/CP) for
 * callers that cannot call cudaMalloc while they run -- for example a host
 * code whose device memory is all owned by its own pool, or one running
 * under a fixed memory cap.  No context is created and nothing is allocated:
 * slots[] holds the caller's device pointers (enum ff_slot; the five
 * increment arrays DRO..DE must be contiguous, NTOT apart), and the LU-SGS
 * coefficients and barrier words live in a file-scope device array that
 * every GPU loading the library keeps (~10 MB) until the process exits.
 * Limit: NTOT = (IMAX+4)(JMAX+4)(KMAX+4) <= FF_NOALLOC_MAX_NTOT, else
 * FF_ERR_SIZE with nothing queued.  The first call on a device resolves the
 * array's device address; make that first call before any stream capture.
 * Calls share the array, so calls that overlap on the GPU race: serialise
 * them (one stream, or events).  With prm->ddadi = 1 it runs the DDADI line
 * sweeps instead, which use no scratch.  Laminar (five-equation) blocks only:
 * prm->iturb >= 3 gives FF_ERR_ARG.  The LU-SGS sweeps here are FP64 only:
 * prm->lusgs_fp32 = 1 without ddadi gives FF_ERR_ARG.  Asynchronous on
 * `stream` (a cudaStream_t), so a sweep whose bounded grid barrier timed out
 * cannot report it from the call that queued it: the flag stays set on the
 * device until the caller asks.  level = 0 is that status query (the other
 * arguments are ignored): it waits for `stream` and returns FF_ERR_TIMEOUT if
 * any call since the last query timed out (and clears the flag), else 0. */
#define FF_NOALLOC_MAX_NTOT 98304
int ff_imps_noalloc(int imax, int jmax, int kmax, const ff_params *prm,
                    double *const *slots, int level, void *stream);

/* ncycles cycles of NS3D over every (single-grid) block of the context:
 * CYCLES per block as concurrent graph branches, then BOUNDI with the 1:1
 * connections (CONNEC ns3c.f:8605) of all blocks in one launch, and SUBIN.
 * Connection patches have ityp = FF_BC_CON, ibtype = source block id,
 * nface = source face, n1a/n2a = source range start (aligned patches). */
int ff_cycles_all(void *ctx, int ncycles, int icycle0, double *hist, int use_graph);
/* BOUNDI(1) ns3c.f:10608 over every block, 1:1 connections included. */
int ff_boundi_all(void *ctx);

/* Blocks spread over several GPUs (one context per GPU).  A 1:1 patch whose
 * source block lives on another GPU keeps ityp = FF_BC_CON with a negative
 * ibtype in this context; the host moves its ghost data between contexts
 * (e.g. NCCL send/recv) as packed halo buffers.  One item per remote patch:
 * mode 0 packs the two interior layers of local block `blk` behind the
 * source face pa.nface (pa is the destination block's patch), mode 1 unpacks
 * them into the ghost layers of local block `blk` behind pa.iface.  Packed
 * layout at `offset` (doubles): [layer 0..1][var 0..9][cell of the patch],
 * vars TEMP,U,V,W,E,EPS2,VIST,CH,P,PDIFF, cells in r1-fastest order
 * (EXPTOT/IMPVO2 gluebm.f:6819/6964 send the same ten variables). */
typedef struct {
  int blk;
  int mode;
  long long offset;
  ff_patch pa;
} ff_halo_item;
int ff_halo_plan(void *ctx, int nitems, const ff_halo_item *items, double *send_buf,
                 double *recv_buf);

/* A multi-GPU cycle, in phases with the host's exchange in between:
 *   FF_PHASE_CYCLE_A   CYCLES of every local block, then BOUNDI part one
 *                      (REFCOR, MIR, STATIM), local CONNEC and the halo pack;
 *   FF_PHASE_BOUNDI_A  BOUNDI part one, local CONNEC and the pack only;
 *   FF_PHASE_B         halo unpack and the second STATIM of every block;
 *   FF_PHASE_RECORD    append this context's {sum of squares[5], max|dp|}
 *                      to the history (sums add, maxima max over GPUs).
 * Cycle phases A and B are replayed as CUDA graphs when use_graph is set
 * and icycle > 1. */
#define FF_PHASE_CYCLE_A 0
#define FF_PHASE_BOUNDI_A 1
#define FF_PHASE_B 2
#define FF_PHASE_RECORD 3
int ff_mb_phase(void *ctx, int phase, int icycle, int use_graph);
/* Copy the first n history rows (6 doubles each) to the host; with
 * hist == NULL reserve room for n rows instead.  reset != 0 restarts the
 * history at row 0. */
int ff_history(void *ctx, int n, double *hist, int reset);
int ff_time_cycles_all(void *ctx, int ncycles, float *ms, int *launches_per_cycle);

/* Timing helpers (CUDA events on the context stream); ff_cycle_launches is
 * the number of kernel launches in one graph-captured cycle. */
int ff_cycle_launches(void *ctx, int blk);
/* LU-SGS sweep kernel of a block: 1 + 100*cluster_size = cluster line
 * wavefront, 2 + 100*threads_per_CTA = cooperative hyperplane kernel. */
/* The autotuner's measured upper-sweep times in ms {cluster lines, fastest
 * cooperative hyperplane} of a block (zeros until its first ff_cycles call
 * or sweep stage timing; lines 0 where the lines do not fit a cluster). */
int ff_sweep_tuning(void *ctx, int blk, float *ms2);
/* The autotuner's measured upper-sweep times in ms {pipelined tile
 * wavefront, cluster lines, fastest cooperative hyperplane} (zero where not
 * tried).  LU-SGS kind 3 + 100*tiles = the pipelined tile wavefront.
 * DDADI blocks (prm->ddadi = 1): the tuned PRED+CORR time per direction
 * {k, i, j}, and kind 4 + 100*(1000 + 100*fk + 10*fi + fj) with f the
 * chosen producer/consumer form per direction (0: 32 lines x 4 cells per
 * CTA chunk, 1: 16 x 4, 2: 16 x 8, 3: 8 x 8), or 4 alone for one thread per
 * line. */
int ff_sweep_times(void *ctx, int blk, float *ms3);
/* The residual form the autotuner chose for a block (its first
 * ff_cycles / ff_cycles_all call times each): 0 = 32x4x4, 1 = 16x8x4,
 * 2 = 8x8x8 cells per CTA (i, j, k); 3, 4, 5 the same tiles with the face
 * stencils staged in shared memory. */
int ff_residual_shape(void *ctx, int blk);
int ff_lusgs_kind(void *ctx, int blk);
int ff_time_cycles(void *ctx, int blk, int ncycles, float *ms);
int ff_time_stage(void *ctx, int blk, int stage, int reps, float *ms);

/* ---- Fortran call sites ------------------------------------------------
 * External subroutines with the reference's names and argument lists, for a
 * FINFLO host built with gfortran (lower case, trailing underscore, every
 * argument by reference), linked in place of the CPU routines CYCLES calls:
 *   statim_  STATIM(M, N, INN, REFLEL)  ns3c.f:10318 (call ns3c.f:1450)
 *   residi_  RESIDI(M, N, M2, IPR)      ns3c.f:2355  (call ns3c.f:1484)
 *   impsdi_  IMPSDI(M, N, M2, AMGDIVL)  ns3c.f:2683  (call ns3c.f:1497)
 *   fin_     FIN(TEMP, ..., NGL, ICYCLE) res3c.f:1077 (call ns3c.f:1517)
 *   boundi_  BOUNDI(M)                  ns3c.f:10608 (call ns3c.f:556)
 * They act on one module-level context: ff_fortran_bind names it,
 * ff_fortran_block maps the host's level M, block N and global block number
 * NGL to a block id, ff_fortran_cycle sets the cycle number RESIDI passes
 * on.  A subroutine returns no status: ff_fortran_ierr returns (and clears)
 * the first failing stage's FF_ERR_* code since it was last called.  FIN's
 * host arrays are not read (the state is on the device), and fin_ includes
 * the limits CYCLES applies right after FIN (ns3c.f:1553-1596), which the
 * host then skips. */
int ff_fortran_bind(void *ctx);
int ff_fortran_block(int m, int n, int ngl, int blk);
int ff_fortran_cycle(int icycle);
int ff_fortran_ierr(void);
void statim_(const int *m, const int *n, const int *inn, const int *reflel);
void residi_(const int *m, const int *n, const int *m2, const int *ipr);
void impsdi_(const int *m, const int *n, const int *m2, const double *amgdivl);
void fin_(void *temp, void *u, void *v, void *w, void *pdiff, void *dtemp, void *du, void *dv, void *dw,
          void *dp, void *told, void *uold, void *vold, void *wold, void *pold, void *rk, void *reps,
          void *drk, void *deps, void *rkold, void *epsold, const double *rklim, const double *epslim,
          void *pro, void *var, void *fi, void *dfi, void *fiold, void *rlolim, void *upplim,
          const int *imax, const int *jmax, const int *kmax, const int *maxsb, const int *nscal,
          const int *nsca2, const int *iturb, const int *ipresc, const double *turlim, void *vis,
          const int *transl, void *trm, void *blks, const int *ngl, const int *icycle);
void boundi_(const int *m);

#ifdef __cplusplus
}
#endif
#endif
