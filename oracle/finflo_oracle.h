/*
 * CPU oracle for the FINFLO per-iteration hot path (test infrastructure only).
 *
 * A restatement in C, FP64, of the reference Fortran routines on the path,
 * in their loop and accumulation order.  It is the checker for the sm_100a
 * library: only the tests, the smoke check and the bench's CPU-baseline leg
 * call it.  PARITY UNPINNED: the reference has no tests, fixtures or golden
 * vectors and no Fortran compiler exists on these machines, so the oracle is
 * pinned only by the analytic invariants in tests/ (free-stream preservation,
 * Roe consistency, rotational invariance, conservation).
 */
#ifndef FINFLO_ORACLE_H
#define FINFLO_ORACLE_H
#include "../include/finflo_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_block {
  int imax, jmax, kmax, npatch;
  const ff_patch *patch;
  double *a[FF_NSLOTS];
} orc_block;

int  orc_version(void);
void orc_statim(orc_block *b, const ff_params *p);
void orc_adjuin_laminar(orc_block *b);
void orc_refcen(orc_block *b, const ff_params *p);
void orc_gradients(orc_block *b, int level);
void orc_inlet_outlet(orc_block *b, const ff_params *p, int dir, int icycle);
void orc_flux_dir(orc_block *b, const ff_params *p, int dir, int level);
void orc_sweep(orc_block *b, int dir, int ido);
void orc_residu(orc_block *b, const ff_params *p, int level, int icycle);
void orc_resl2(const orc_block *b, double *resi5);
void orc_time3(orc_block *b, const ff_params *p, double cfl);
void orc_locdt_copr(orc_block *b);
void orc_predgs(orc_block *b, const ff_params *p);
void orc_diaggs(orc_block *b, const ff_params *p);
void orc_corrgs(orc_block *b, const ff_params *p);
void orc_imps(orc_block *b, const ff_params *p, int level);
void orc_ddadi(orc_block *b, const ff_params *p);
void orc_timder(orc_block *b, const ff_params *p, int nv);
void orc_time_levels(orc_block *b, int nv, int mode);
void orc_fin_limits(orc_block *b, const ff_params *p);
void orc_refcor(orc_block *b);
void orc_mir(orc_block *b);
void orc_subin(orc_block *b, double *dromax);
void orc_boundi(orc_block *b, const ff_params *p);
void orc_cycle(orc_block *b, const ff_params *p, int icycle, double *resi5, double *dromax);
void orc_transf(orc_block *f, orc_block *c);
void orc_forcfu(orc_block *c);
void orc_addres(orc_block *c);
void orc_interp(orc_block *c, orc_block *f);
void orc_fin_coarse(orc_block *b, const ff_params *p);
void orc_interp_limits(orc_block *c, orc_block *f, const ff_params *pf);
void orc_connec_patch(orc_block *dst, const ff_patch *pa, const orc_block *src);
void orc_connec(orc_block **blk, int nblk);
/* k-omega SST (ITURB=6), single grid level: finflo_oracle_sst.c */
void orc_turbeq_sst(orc_block *b, const ff_params *p);
void orc_residu_sst(orc_block *b, const ff_params *p, int icycle);
void orc_flux_dir_sst(orc_block *b, const ff_params *p, int dir);
void orc_imps_sst(orc_block *b, const ff_params *p);
void orc_fin_limits_sst(orc_block *b, const ff_params *p);
void orc_subin_sst(orc_block *b, const ff_params *p, double *dromax);
void orc_residu_sst_lev(orc_block *b, const ff_params *p, int lev, int m2, int icycle);
void orc_imps_sst_lev(orc_block *b, const ff_params *p, int lev);
void orc_tranke(orc_block *f, orc_block *c);
void orc_forcfu_ke(orc_block *c);
void orc_addres_ke(orc_block *c);
void orc_intert(orc_block *c, orc_block *f, const ff_params *pf);
void orc_fin_coarse_sst(orc_block *b, const ff_params *p);
void orc_mg_cycle_sst(orc_block **lv, int nlev, const ff_params *prm, int icycle, double *resi5, double *dromax);
void orc_cycle_sst(orc_block *b, const ff_params *p, int icycle, double *resi5, double *dromax);
void orc_halo_pack(const orc_block *src, const ff_patch *pa, double *out);
void orc_halo_unpack(orc_block *dst, const ff_patch *pa, const double *in);
void orc_mb_boundi(orc_block **blk, int nblk, const ff_params *prm);
void orc_mb_cycle(orc_block **blk, int nblk, const ff_params *prm, int icycle, double *resi5, double *dromax);
void orc_mg_cycle(orc_block **lv, int nlev, const ff_params *prm, int icycle, double *resi5, double *dromax);

/* single-face kernels exposed for the invariant tests */
void orc_roe_face(const double *qr, const double *ql, const double *qrr, const double *qll,
                  const double *nrm, double area, int intem, const ff_params *p,
                  const double *cell_r, const double *cell_l, int kquirk, double *f5);

/* SCALARD base3c.f:6: the JAMESON dissipation scale SCALEJ of cells 0..MAX+1 */
void orc_scalard(orc_block *b);

/* the reference's block set-up (finflo_oracle_grid.c) */
void orc_grid_metrics(orc_block *b, const double *X, const double *Y, const double *Z);
void orc_grid_lump(const orc_block *f, orc_block *c);
int orc_wall_points(orc_block **blk, int nblk, double *xyz);
void orc_wall_distance(orc_block *b, const double *xyz, int np);

#ifdef __cplusplus
}
#endif
#endif
