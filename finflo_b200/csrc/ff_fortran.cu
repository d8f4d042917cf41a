// Fortran call-site wrappers: external subroutines with the reference's own
// names and by-reference integer arguments, so that a FINFLO host compiled
// with gfortran (lower case + trailing underscore) links them in place of
// the CPU routines its CYCLES (ns3c.f:1354) calls.
//
//   statim_(M, N, INN, REFLEL)   STATIM  ns3c.f:10318, called at ns3c.f:1450
//   residi_(M, N, M2, IPR)       RESIDI  ns3c.f:2355,  called at ns3c.f:1484
//   impsdi_(M, N, M2, AMGDIVL)   IMPSDI  ns3c.f:2683,  called at ns3c.f:1497
//   fin_(TEMP, ..., NGL, ICYCLE) FIN     res3c.f:1077, called at ns3c.f:1517 (45 args)
//   boundi_(M)                   BOUNDI  ns3c.f:10608, called at ns3c.f:556
//
// The reference's routines find their arrays through the MAIN_ARRAYS module
// (charac.f:391) and the block offsets IG(M,N); here the arrays stay
// resident in one library context, and a module-level table maps the
// host's (level M, block N) and global block number NGL to the context's
// block ids.  The host fills it once, after ff_block_add / ff_mg_link:
//
//   ff_fortran_bind(ctx)                 the context the wrappers use
//   ff_fortran_block(M, N, NGL, blk)     (M, N) and NGL -> block id
//   ff_fortran_cycle(ICYCLE)             the cycle number RESIDI passes on
//   ff_fortran_ierr()                    last status of a wrapper (cleared)
//
// A Fortran subroutine returns no status, so each wrapper keeps the code of
// its stage call (0 or FF_ERR_*) for ff_fortran_ierr; the first failure
// sticks until it is read.  The host arrays named in FIN's argument list are
// not read: the state they hold lives on the device (ff_download copies it
// back for output or a restart).
//
// This file is compiled as part of ff_gpu.cu's translation unit (included at
// its end); it calls the library's entry points and reads its block table
// (dimensions and patch types) to check the arguments.

#include <map>
#include <mutex>
#include <utility>

namespace {

struct FortranTable {
  void* ctx = nullptr;
  std::map<std::pair<int, int>, int> by_mn;   // (M, N) -> block id
  std::map<int, int> by_ngl;                  // NGL -> block id of level 1
  int icycle = 1;
  int ierr = 0;
};
FortranTable g_ftn;
std::mutex g_ftn_mu;

void ftn_status(int rc) {
  if (rc && !g_ftn.ierr) g_ftn.ierr = rc;
}

int ftn_block(int m, int n) {
  auto it = g_ftn.by_mn.find({m, n});
  return it == g_ftn.by_mn.end() ? -1 : it->second;
}

}  // namespace

extern "C" {

int ff_fortran_bind(void* ctx) {
  std::lock_guard<std::mutex> lk(g_ftn_mu);
  g_ftn = FortranTable{};
  g_ftn.ctx = ctx;
  return ctx ? 0 : FF_ERR_ARG;
}

int ff_fortran_block(int m, int n, int ngl, int blk) {
  std::lock_guard<std::mutex> lk(g_ftn_mu);
  if (!g_ftn.ctx || m < 1 || n < 1 || blk < 0) return FF_ERR_ARG;
  g_ftn.by_mn[{m, n}] = blk;
  if (m == 1) g_ftn.by_ngl[ngl] = blk;
  return 0;
}

int ff_fortran_cycle(int icycle) {
  std::lock_guard<std::mutex> lk(g_ftn_mu);
  g_ftn.icycle = icycle;
  return 0;
}

int ff_fortran_ierr(void) {
  std::lock_guard<std::mutex> lk(g_ftn_mu);
  int e = g_ftn.ierr;
  g_ftn.ierr = 0;
  return e;
}

// STATIM(M, N, INN, REFLEL): the equation of state over the block and, with
// REFLEL = .TRUE., the ghost reflection REFLEC.  The device stage always
// includes REFLEC, so REFLEL = .FALSE. is refused (FF_ERR_ARG).
void statim_(const int* m, const int* n, const int* inn, const int* reflel) {
  std::lock_guard<std::mutex> lk(g_ftn_mu);
  (void)inn;
  const int b = ftn_block(*m, *n);
  if (b < 0 || !*reflel) { ftn_status(FF_ERR_ARG); return; }
  ftn_status(ff_statim(g_ftn.ctx, b));
}

// RESIDI(M, N, M2, IPR): the residual of block N on level M (M2 = M, or
// M + 1 when a finer level's residual is about to be restricted).  IPR only
// selects printing in the reference.
void residi_(const int* m, const int* n, const int* m2, const int* ipr) {
  std::lock_guard<std::mutex> lk(g_ftn_mu);
  (void)ipr;
  const int b = ftn_block(*m, *n);
  if (b < 0) { ftn_status(FF_ERR_ARG); return; }
  ftn_status(ff_residi(g_ftn.ctx, b, *m2, g_ftn.icycle));
}

// IMPSDI(M, N, M2, AMGDIVL): the implicit stage of block N on level M.
// AMGDIVL (a multigrid divergence monitor of the reference) is not used.
void impsdi_(const int* m, const int* n, const int* m2, const double* amgdivl) {
  std::lock_guard<std::mutex> lk(g_ftn_mu);
  (void)m2;
  (void)amgdivl;
  const int b = ftn_block(*m, *n);
  if (b < 0) { ftn_status(FF_ERR_ARG); return; }
  ftn_status(ff_imps(g_ftn.ctx, b, *m));
}

// FIN res3c.f:1077 with its 45 arguments in the reference's order; the
// block is the level-1 block of global number NGL (argument 44).
void fin_(void* temp, void* u, void* v, void* w, void* pdiff, void* dtemp, void* du, void* dv, void* dw,
          void* dp, void* told, void* uold, void* vold, void* wold, void* pold, void* rk, void* reps, void* drk,
          void* deps, void* rkold, void* epsold, const double* rklim, const double* epslim, void* pro, void* var,
          void* fi, void* dfi, void* fiold, void* rlolim, void* upplim, const int* imax, const int* jmax,
          const int* kmax, const int* maxsb, const int* nscal, const int* nsca2, const int* iturb,
          const int* ipresc, const double* turlim, void* vis, const int* transl, void* trm, void* blks,
          const int* ngl, const int* icycle) {
  std::lock_guard<std::mutex> lk(g_ftn_mu);
  (void)temp; (void)u; (void)v; (void)w; (void)pdiff; (void)dtemp; (void)du; (void)dv; (void)dw; (void)dp;
  (void)told; (void)uold; (void)vold; (void)wold; (void)pold; (void)rk; (void)reps; (void)drk; (void)deps;
  (void)rkold; (void)epsold; (void)rklim; (void)epslim; (void)pro; (void)var; (void)fi; (void)dfi;
  (void)fiold; (void)rlolim; (void)upplim; (void)maxsb; (void)nscal; (void)nsca2; (void)iturb; (void)ipresc;
  (void)turlim; (void)vis; (void)transl; (void)trm; (void)blks; (void)icycle;
  auto it = g_ftn.by_ngl.find(*ngl);
  if (it == g_ftn.by_ngl.end()) { ftn_status(FF_ERR_ARG); return; }
  Ctx* c = (Ctx*)g_ftn.ctx;
  BlockCtx* b = getb(c, it->second);
  if (!b || b->imax != *imax || b->jmax != *jmax || b->kmax != *kmax) { ftn_status(FF_ERR_ARG); return; }
  ftn_status(ff_fin(g_ftn.ctx, it->second, nullptr));
}

// BOUNDI(M): ghost updates of every block of level M; with 1:1 connection
// patches in the context, level 1 runs the multi-block BOUNDI (CONNEC of
// all blocks in one launch).
void boundi_(const int* m) {
  std::lock_guard<std::mutex> lk(g_ftn_mu);
  Ctx* c = (Ctx*)g_ftn.ctx;
  if (!c) { ftn_status(FF_ERR_ARG); return; }
  bool conn = false;
  for (auto& kv : g_ftn.by_mn) {
    BlockCtx* b = getb(c, kv.second);
    if (!b || kv.first.first != *m) continue;
    for (auto& p : b->h_patch) conn = conn || p.ityp == FF_BC_CON;
  }
  if (conn && *m == 1) { ftn_status(ff_boundi_all(g_ftn.ctx)); return; }
  for (auto& kv : g_ftn.by_mn)
    if (kv.first.first == *m) ftn_status(ff_boundi(g_ftn.ctx, kv.second));
}

}  // extern "C"
