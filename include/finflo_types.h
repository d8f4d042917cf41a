/*
 * Shared plain-C types for the FINFLO hot-path boundary.
 *
 * These structs carry the scalars and the boundary-patch table that the
 * reference passes as individual by-reference arguments to its block
 * routines (RESIDU res3c.f:6, IMPS imps3.f:6, FIN res3c.f:1077, ...).  Both the
 * sm_100a library (libfinflo_gpu.so) and the CPU oracle use them, so one
 * parameter block describes the same case to both.
 *
 * Storage convention (identical to the reference): every per-cell array of a
 * block is one FP64 array of NTOT = (IMAX+4)*(JMAX+4)*(KMAX+4) entries,
 * i fastest, two ghost layers per side (IN=JN=KN=2, charac.f:179).
 */
#ifndef FINFLO_TYPES_H
#define FINFLO_TYPES_H

#ifdef __cplusplus
extern "C" {
#endif

/* ICON(1) boundary types used by the configs (gluebm.f:2737-2797). */
enum { FF_BC_CON = 1, FF_BC_INL = 3, FF_BC_MIR = 4, FF_BC_OUT = 5, FF_BC_SOL = 8 };

/* One boundary patch; mirrors the ICON(IC9,L) columns the hot path reads
 * (charac.f:182, meaning of the columns at res3c.f:7730-7740). */
typedef struct ff_patch {
  int ityp;      /* ICON(1,L): 3 INL, 4 MIR, 5 OUT, 8 SOL, 1 CON             */
  int iface;     /* ICON(3,L): 1..3 low i/j/k face, 4..6 high i/j/k face      */
  int r1a, r1b;  /* ICON(4,L),ICON(5,L): range of the first in-face index     */
  int r2a, r2b;  /* ICON(6,L),ICON(7,L): range of the second in-face index    */
  int ibtype;    /* ICON(8,L): inlet/outlet sub-type (INLOUT), or the         */
                 /*            neighbour block for CON patches                */
  int iheat;     /* ICON(20,L): wall heat condition (0 = adiabatic)           */
  int nface;     /* ICON(9,L): face number in the neighbour block (CON)       */
  int iori;      /* ICON(14,L): orientation index for CON (0 = aligned)       */
  int n1a, n2a;  /* start of the matching range in the neighbour face (CON)   */
  /* BOUNR/BOUNU/BOUNV/BOUNW/BOUNT/BOUNP/BOUNPD, uniform over the patch       */
  double bounr, bounu, bounv, bounw, bount, bounp, bounpd;
  /* BOUNRK/BOUNEP: inlet rho*k and rho*omega (two-equation models)          */
  double bounrk, bounep;
} ff_patch;

/* ff_params.flux: the inviscid face flux (IFLUX, FLUXME multi.f:3567).
 * Zero is the reference's default, Roe; the others carry IFLUX's own number,
 * except van Leer (IFLUX = 0), which takes the 1 that Roe leaves free.
 * Van Leer, WPS and AUSM have no two-equation form (FLUCYC res3c.f:7890-7960
 * calls them, RESIKE res3c.f:6946-7030 does not). */
enum ff_flux {
  FF_FLUX_ROE = 0,       /* IFLUX = 1: FLUXKE base3c.f:4753           */
  FF_FLUX_VANLEER = 1,   /* IFLUX = 0: FLUXVL base3c.f:1733, laminar  */
  FF_FLUX_WPS = 2,       /* IFLUX = 2: FLUXWP base3c.f:1967, laminar  */
  FF_FLUX_AUSM = 3,      /* IFLUX = 3: FLUXAU base3c.f:2201, laminar  */
  FF_FLUX_KT = 7,        /* IFLUX = 7: FLUXKT base3c.f:4403           */
  FF_FLUX_HCUSP = 8      /* IFLUX = 8: FLUCUSP base3c.f:5133          */
};

/* Flow, gas and solver constants (defaults: main.f:5234-5440, 3499, 3827). */
typedef struct ff_params {
  double gamma, rgas, pr, prt;          /* 1.4, 287.05287, 0.72, 0.9          */
  double visu0, expsu, tsu0;            /* Sutherland 1.458e-6, 1.5, 110.4    */
  double e0ref, t0ref;                  /* 0, 0                                */
  double frsden, frspre, frsvel, frsvis, frstem;
  double cfl, cfll;                     /* fine / coarse-level CFL            */
  double theta;                         /* THETA = 1.5 (main.f:3499)          */
  double cdiff;                         /* CDIFF = 2 (main.f)                 */
  double pvisc;                         /* PVISC = 1.8 (imps3.f:110)          */
  double tlolim, tuplim;                /* 0.05*FRSTEM, 6*FRSTEM              */
  double cmgk, cmgeps;                  /* 0.1, 0.2 (main.f:5343-5344)        */
  /* two-equation (k-omega SST) constants, main.f:3770-3830, 5338-5346      */
  double rklim, epslim;                 /* free-stream rho*k, rho*omega        */
  double turlim;                        /* mu_t / mu cap (5000)               */
  double csimps;                        /* point-implicit source factor (5)   */
  double re;                            /* Reynolds number (FUN1KO DISLIM)    */
  int interi, interj, interk;           /* XXTRAP INTEM per direction         */
  int entropy_fix;                      /* ENTROPY_FIX (0 default)            */
  int iturb;                            /* 0 laminar, 6 k-omega SST (KOVER=0) */
  int fullns;                           /* 1: FLUXBL on level 1, else FLUXDO  */
  int idi1, idi2, idi3;                 /* viscous extents IDI1..3 (nodes)    */
  int coarse_inter;                     /* INTEM on coarse levels (55)        */
  int lusgs_fp32;                       /* 1: implicit operator in FP32       */
  int ddadi;                            /* 1: DDADI (LUSGS=0, imps3.f:320),    */
                                        /* 0: LU-SGS (LUSGS=1, imps3.f:378)    */
  int timel;                            /* 1: time-accurate dual time stepping */
                                        /* (TIMEL, level 1 of the block only)  */
  int flux;                             /* inviscid face flux, ff_flux below   */
                                        /* (IFLUX of the reference)            */
  double dt;                            /* physical time step DT (TIMEL)       */
  int predgs_full;                      /* 1: the LU-SGS lower sweep (PREDGS)  */
                                        /* keeps the i+1 coupling in row JMAX  */
                                        /* that imps4.f:1460-1466 drops (its   */
                                        /* shift loop starts one index late);  */
                                        /* 0: the reference's sweep            */
  int res_fp32;                         /* 1 on a coarse level: its Roe face  */
                                        /* fluxes in FP32 (sums, update and   */
                                        /* norms FP64); ignored on level 1    */
  int xxtral;                           /* XXTRAL: MUSCL weighted by the cell */
                                        /* extents D1..D3 (XXTRAA) for Roe,   */
                                        /* KT and H-CUSP                      */
  double rjk2, rjk4;                    /* RJK2, RJK4: JAMESON's second- and  */
                                        /* fourth-difference dissipation with */
                                        /* Roe on the finest level (0, 0 off; */
                                        /* main.f:5289-5290)                  */
} ff_params;

/* Per-cell array slots of one block (names are the reference's MAIN_ARRAYS,
 * charac.f:391).  Every slot is an FP64 array of NTOT entries in the
 * storage convention above. */
enum ff_slot {
  /* flow state (STATIM outputs, charac.f:391) */
  FF_RO, FF_RM, FF_RN, FF_RW, FF_E, FF_P, FF_PDIFF, FF_U, FF_V, FF_W, FF_C,
  FF_TEMP, FF_VIS, FF_CH, FF_CP, FF_DRDP, FF_DRDH, FF_EPS2, FF_VIST,
  /* residual / increments (RESIDU -> IMPS -> FIN) and local time step */
  FF_DRO, FF_DM, FF_DN, FF_DW, FF_DE, FF_DRK, FF_DEPS, FF_DTL,
  /* values at the start of the cycle (SUBIN ns3c.f:9742) */
  FF_TOLD, FF_UOLD, FF_VOLD, FF_WOLD, FF_POLD,
  /* metrics */
  FF_A1, FF_A1XA, FF_A1YA, FF_A1ZA, FF_A2, FF_A2XA, FF_A2YA, FF_A2ZA,
  FF_A3, FF_A3XA, FF_A3YA, FF_A3ZA, FF_VOL, FF_XC, FF_YC, FF_ZC,
  FF_D1, FF_D2, FF_D3,
  /* velocity / temperature gradients (DERFUN turb3.f:2476, TEMDER 3456) */
  FF_W12, FF_W13, FF_W23, FF_S11, FF_S12, FF_S13, FF_S22, FF_S23, FF_S33,
  FF_DTDX, FF_DTDY, FF_DTDZ, FF_OHMI, FF_STRAIN,
  /* face fluxes of one direction (F1R..F1E, res3c.f:7705-7710) */
  FF_F1R, FF_F1RM, FF_F1RN, FF_F1RW, FF_F1E,
  /* multigrid forcing P2H (TRANSF/FORCFU, multi.f:156, 1609) */
  FF_ROP2H, FF_RMP2H, FF_RNP2H, FF_RWP2H, FF_EP2H,
  /* two-equation model: rho*k, rho*omega, wall distance (DISTW), blending
   * F1 (FUN1), sources SRK/SEPS, production PTUR, gradients of k and omega
   * (GRADK/GREPS), their start-of-cycle copies and face fluxes (F1RK,
   * F1EPS), multigrid forcing of k and omega */
  FF_RK, FF_REPS, FF_DISTW, FF_FUN1, FF_SRK, FF_SEPS, FF_PTUR,
  FF_DKDX, FF_DKDY, FF_DKDZ, FF_DEDX, FF_DEDY, FF_DEDZ,
  FF_RKOLD, FF_EPSOLD, FF_F1RK, FF_F1EPS, FF_RKP2H, FF_EPP2H,
  /* the two previous physical time levels of the conservative variables
   * (TIMEL: ROLE2..EPSLE2 = level n, ROLE3..EPSLE3 = level n-1; STARTI
   * res3c.f:3175, NEWTIM ns3c.f:9420) */
  FF_ROLE2, FF_RMLE2, FF_RNLE2, FF_RWLE2, FF_ELE2, FF_RKLE2, FF_EPSLE2,
  FF_ROLE3, FF_RMLE3, FF_RNLE3, FF_RWLE3, FF_ELE3, FF_RKLE3, FF_EPSLE3,
  /* SCALEJ: the spectral-radius scale of JAMESON's dissipation (SCALARD
   * base3c.f:6; the finest level, when RJK2 or RJK4 > 0) */
  FF_SCALEJ,
  FF_NSLOTS
};

#ifdef __cplusplus
}
#endif
#endif
