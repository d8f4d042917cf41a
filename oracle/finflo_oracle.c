/*
 * CPU oracle for the FINFLO per-iteration hot path.  TEST INFRASTRUCTURE ONLY:
 * it is the checker for libfinflo_gpu.so and is called from tests/, the smoke
 * check and bench.py's CPU-baseline leg, never from the product path.
 *
 * Restatement in C99/FP64 of the reference Fortran routines, keeping their
 * loop order, accumulation order and constants (compile with
 * -ffp-contract=off so no FMA is introduced).  Only the branches the configs
 * select are restated: perfect gas (ISTATE=1), Roe FDS (IFLUX=1), LU-SGS
 * (LUSGS=1), laminar (ITURB=0), full Navier-Stokes on level 1 (FULLNC='YES'),
 * IDIFF=1, IDERI=1, no rotation/gravity/chimera/free surface.
 *
 * PARITY UNPINNED: the reference ships no tests or golden vectors and cannot be
 * compiled here (no Fortran compiler); see the invariant tests in tests/.
 *
 * Indexing: I,J,K are the reference's 1-based cell indices; ghosts are
 * 0, -1 and MAX+1, MAX+2.  IX() gives the 0-based storage index.
 */
#include "finflo_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXD(a, b) ((a) > (b) ? (a) : (b))
#define MIND(a, b) ((a) < (b) ? (a) : (b))

typedef struct {
  int imax, jmax, kmax, is, il, ntot;
} dims_t;

static dims_t dims_of(const orc_block *b) {
  dims_t d;
  d.imax = b->imax; d.jmax = b->jmax; d.kmax = b->kmax;
  d.is = b->imax + 4;
  d.il = d.is * (b->jmax + 4);
  d.ntot = d.il * (b->kmax + 4);
  return d;
}
#define IX(d, I, J, K) ((size_t)((K) + 1) * (d).il + (size_t)((J) + 1) * (d).is + (size_t)((I) + 1))

int orc_version(void) { return 1; }

/* ---------------------------------------------------------------------- */
/* STATIM (ns3c.f:10318): PDTOP state.f:1690, PERFGA state.f:159 (EXPSU=1.5 */
/* branch, IUPPTL=0), CONSVA base3c.f:489 (ITURB<3 and two-equation), REFLEC*/
/* turb3.f:5294 (solid walls and the inlet-pressure extrapolation).         */
/* ---------------------------------------------------------------------- */
static void state_cells(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  double *P = b->a[FF_P], *PD = b->a[FF_PDIFF], *T = b->a[FF_TEMP], *RO = b->a[FF_RO];
  double *E = b->a[FF_E], *VIS = b->a[FF_VIS], *CH = b->a[FF_CH], *CP = b->a[FF_CP];
  double *DRDP = b->a[FF_DRDP], *DRDH = b->a[FF_DRDH], *C = b->a[FF_C];
  double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W];
  double *RM = b->a[FF_RM], *RN = b->a[FF_RN], *RW = b->a[FF_RW];
  const double *RK = b->a[FF_RK];
  const double gm1 = p->gamma - 1.0, cp2 = p->gamma / gm1 * p->rgas;
  for (int n = 0; n < d.ntot; n++) {
    P[n] = PD[n] + p->frspre;                      /* PDTOP, g = 0 */
    double trgs = T[n] * p->rgas;                   /* PERFGA */
    DRDP[n] = 1.0 / trgs;
    RO[n] = P[n] * DRDP[n];
    VIS[n] = p->visu0 * T[n] * 1.0 * sqrt(T[n]) / (T[n] + p->tsu0);
    E[n] = trgs / gm1;
    DRDH[n] = -RO[n] / E[n] / p->gamma;
    CP[n] = cp2;
    CH[n] = VIS[n] * cp2 / p->pr;
    double rkin = (U[n] * U[n] + V[n] * V[n] + W[n] * W[n]) * .5;   /* CONSVA */
    if (p->iturb < 3) {
      C[n] = sqrt(MAXD(1.0 / (DRDH[n] / RO[n] + DRDP[n]), 1.0));
      E[n] = (E[n] + rkin + 0.0) * RO[n];
    } else {                                        /* two-equation branch */
      double ypro = 1. / RO[n];
      double xturb = 1. + (2. / 3.) * RK[n] * ypro * DRDP[n];
      C[n] = sqrt(MAXD(xturb / (DRDH[n] * ypro + DRDP[n]), 1.0));
      E[n] = (E[n] + rkin + 0.0) * RO[n] + RK[n];
    }
    RM[n] = RO[n] * U[n];
    RN[n] = RO[n] * V[n];
    RW[n] = RO[n] * W[n];
  }
}

/* Face geometry helper: for face number iface (1..6) return the direction
 * (1 i, 2 j, 3 k), the normal-direction stride, the in-face strides for the
 * ICON(4..5)/(6..7) ranges, and the interior layer index (1 or MAX). */
typedef struct { int dir, idir, s, s1, s2, layer; } face_t;

static face_t face_geom(const dims_t *d, int iface) {
  face_t f;
  f.dir = (iface - 1) % 3 + 1;
  f.idir = iface <= 3 ? 1 : -1;
  if (f.dir == 1) { f.s = 1; f.s1 = d->is; f.s2 = d->il; f.layer = iface <= 3 ? 1 : d->imax; }
  else if (f.dir == 2) { f.s = d->is; f.s1 = 1; f.s2 = d->il; f.layer = iface <= 3 ? 1 : d->jmax; }
  else { f.s = d->il; f.s1 = 1; f.s2 = d->is; f.layer = iface <= 3 ? 1 : d->kmax; }
  return f;
}

/* storage index of the interior cell next to the face at in-face (a,b) */
static size_t face_cell(const dims_t *d, const face_t *f, int a, int bb) {
  if (f->dir == 1) return IX(*d, f->layer, a, bb);
  if (f->dir == 2) return IX(*d, a, f->layer, bb);
  return IX(*d, a, bb, f->layer);
}

static void reflec(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *T = b->a[FF_TEMP];
  double *RO = b->a[FF_RO], *P = b->a[FF_P], *PD = b->a[FF_PDIFF];
  double *RM = b->a[FF_RM], *RN = b->a[FF_RN], *RW = b->a[FF_RW], *E = b->a[FF_E];
  double *VIS = b->a[FF_VIS], *CH = b->a[FF_CH], *C = b->a[FF_C];
  double *DRDP = b->a[FF_DRDP], *DRDH = b->a[FF_DRDH], *EPS2 = b->a[FF_EPS2], *VIST = b->a[FF_VIST];
  for (int ip = 0; ip < b->npatch; ip++) {
    const ff_patch *pa = &b->patch[ip];
    face_t f = face_geom(&d, pa->iface);
    int ls = f.idir * f.s;
    if (pa->ityp == FF_BC_INL) {               /* turb3.f:5437-5455 */
      for (int bb = pa->r2a; bb <= pa->r2b; bb++)
        for (int a = pa->r1a; a <= pa->r1b; a++) {
          size_t L = face_cell(&d, &f, a, bb);
          size_t LB = L - ls, LC = L - 2 * ls;
          P[LB] = P[L]; PD[LB] = PD[L]; P[LC] = P[L]; PD[LC] = PD[L];
        }
    }
    if (pa->ityp < 7 || pa->ityp > 10) continue;
    /* heat condition: IHEAT = ICON(20); 1 gives a wall temperature */
    int ihfl = pa->iheat == 1 ? 1 : 0;
    double tsurf = pa->iheat == 1 ? pa->bount : 0.0;
    for (int bb = pa->r2a; bb <= pa->r2b; bb++)
      for (int a = pa->r1a; a <= pa->r1b; a++) {
        size_t L = face_cell(&d, &f, a, bb);
        size_t LB = L - ls, LT = L + ls, LC = L - 2 * ls;
        /* turb3.f:5460-5478 */
        T[LB] = (1 - ihfl) * (1. * T[L] - 0. * T[LT]) + ihfl * (2. * tsurf - T[L]);
        T[LB] = MIND(T[LB], p->tuplim);
        T[LB] = MAXD(T[LB], p->tlolim);
        T[LC] = T[LB];
        VIS[LB] = VIS[L]; CH[LB] = CH[L]; C[LB] = C[L];
        DRDP[LB] = DRDP[L]; DRDH[LB] = DRDH[L];
        /* viscous surface, REFLECL false (turb3.f:5520-5530); wall at rest */
        U[LB] = -U[L] + 2. * 0.0; V[LB] = -V[L] + 2. * 0.0; W[LB] = -W[L] + 2. * 0.0;
        U[LC] = U[LB]; V[LC] = V[LB]; W[LC] = W[LB];
        RO[LB] = MAXD(0.001 * p->frsden, 1. * RO[L] - 0. * RO[LT]);
        P[LB] = MAXD(0.001 * p->frspre, 2. * P[L] - P[LT]);
        PD[LB] = MAXD(-0.999 * p->frspre, 2. * PD[L] - PD[LT]);
        EPS2[LB] = 1.; VIST[LB] = 0.;
        RM[LB] = RO[LB] * U[LB]; RN[LB] = RO[LB] * V[LB]; RW[LB] = RO[LB] * W[LB];
        E[LB] = E[L];
        RM[LC] = RM[LB]; RN[LC] = RN[LB]; RW[LC] = RW[LB]; E[LC] = E[LB];
        EPS2[LC] = EPS2[LB]; VIST[LC] = VIST[LB]; PD[LC] = PD[LB]; P[LC] = P[LB]; RO[LC] = RO[LB];
        if (p->iturb >= 3) {                        /* turb3.f:5646-5658, ITURB=6 */
          double *RK = b->a[FF_RK], *REPS = b->a[FF_REPS];
          RK[LB] = -RK[L];
          REPS[LB] = MAXD(0., 2. * REPS[L] - REPS[LT]);
        }
      }
  }
}

/* One STATIM call: equation of state on every cell, then REFLEC. */
void orc_statim(orc_block *b, const ff_params *p) {
  state_cells(b, p);
  reflec(b, p);
}

/* TURBDI laminar branch: ADJUIN EPS2=1, VIST=0 on internal cells (res3c.f:9447). */
void orc_adjuin_laminar(orc_block *b) {
  dims_t d = dims_of(b);
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t L = IX(d, I, J, K);
        b->a[FF_EPS2][L] = 1.0;
        b->a[FF_VIST][L] = 0.0;
      }
}

/* REFCEN turb3.f:5881: linear extrapolation into the first ghost of walls. */
void orc_refcen(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  double *RO = b->a[FF_RO], *P = b->a[FF_P], *PD = b->a[FF_PDIFF], *E = b->a[FF_E];
  double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W];
  double *RM = b->a[FF_RM], *RN = b->a[FF_RN], *RW = b->a[FF_RW];
  for (int ip = 0; ip < b->npatch; ip++) {
    const ff_patch *pa = &b->patch[ip];
    if (pa->ityp < 7 || pa->ityp > 10) continue;
    face_t f = face_geom(&d, pa->iface);
    int ls = f.idir * f.s;
    for (int bb = pa->r2a; bb <= pa->r2b; bb++)
      for (int a = pa->r1a; a <= pa->r1b; a++) {
        size_t L = face_cell(&d, &f, a, bb), LB = L - ls, LT = L + ls;
        RO[LB] = MAXD(0.001 * p->frsden, 2. * RO[L] - RO[LT]);
        P[LB] = MAXD(0.001 * p->frspre, 2. * P[L] - P[LT]);
        PD[LB] = MAXD(-0.999 * p->frspre, 2. * PD[L] - PD[LT]);
        E[LB] = 2. * E[L] - E[LT];
        U[LB] = 2. * U[L] - U[LT];
        V[LB] = 2. * V[L] - V[LT];
        W[LB] = 2. * W[L] - W[LT];
        RM[LB] = 2. * RM[L] - RM[LT];
        RN[LB] = 2. * RN[L] - RN[LT];
        RW[LB] = 2. * RW[L] - RW[LT];
      }
    if (p->iturb >= 3) {                            /* turb3.f:6013-6027 */
      double *RK = b->a[FF_RK], *REPS = b->a[FF_REPS];
      for (int bb = pa->r2a; bb <= pa->r2b; bb++)
        for (int a = pa->r1a; a <= pa->r1b; a++) {
          size_t L = face_cell(&d, &f, a, bb), LB = L - ls, LT = L + ls;
          RK[LB] = MAXD(p->rklim, 2. * RK[L] - 1. * RK[LT]);
          REPS[LB] = MAXD(p->epslim, 2. * REPS[L] - 1. * REPS[LT]);
        }
    }
  }
}

/* DERFUN turb3.f:2476 and TEMDER turb3.f:3456, IDERI=1 (distance-weighted
 * Gauss).  On level 1 the first ghost layer is included. */
void orc_gradients(orc_block *b, int level) {
  dims_t d = dims_of(b);
  const int IS = d.is, IL = d.il;
  const double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *T = b->a[FF_TEMP];
  const double *A1 = b->a[FF_A1], *A2 = b->a[FF_A2], *A3 = b->a[FF_A3], *VOL = b->a[FF_VOL];
  const double *A1X = b->a[FF_A1XA], *A1Y = b->a[FF_A1YA], *A1Z = b->a[FF_A1ZA];
  const double *A2X = b->a[FF_A2XA], *A2Y = b->a[FF_A2YA], *A2Z = b->a[FF_A2ZA];
  const double *A3X = b->a[FF_A3XA], *A3Y = b->a[FF_A3YA], *A3Z = b->a[FF_A3ZA];
  const double *D1 = b->a[FF_D1], *D2 = b->a[FF_D2], *D3 = b->a[FF_D3];
  int lo = level == 1 ? 0 : 1, hi = level == 1 ? 1 : 0;
  for (int K = lo; K <= d.kmax + hi; K++)
    for (int J = lo; J <= d.jmax + hi; J++)
      for (int I = lo; I <= d.imax + hi; I++) {
        size_t L = IX(d, I, J, K);
        double w1, w2;
        w1 = 2.0 * (D1[L] / (D1[L] + D1[L - 1])); w2 = 2.0 - w1;
        double u1m = A1[L] * (w2 * U[L] + w1 * U[L - 1]);
        double v1m = A1[L] * (w2 * V[L] + w1 * V[L - 1]);
        double x1m = A1[L] * (w2 * W[L] + w1 * W[L - 1]);
        w1 = 2.0 * (D1[L] / (D1[L] + D1[L + 1])); w2 = 2.0 - w1;
        double u1p = A1[L + 1] * (w2 * U[L] + w1 * U[L + 1]);
        double v1p = A1[L + 1] * (w2 * V[L] + w1 * V[L + 1]);
        double x1p = A1[L + 1] * (w2 * W[L] + w1 * W[L + 1]);
        w1 = 2.0 * (D2[L] / (D2[L] + D2[L - IS])); w2 = 2.0 - w1;
        double u2m = A2[L] * (w2 * U[L] + w1 * U[L - IS]);
        double v2m = A2[L] * (w2 * V[L] + w1 * V[L - IS]);
        double x2m = A2[L] * (w2 * W[L] + w1 * W[L - IS]);
        w1 = 2.0 * (D2[L] / (D2[L] + D2[L + IS])); w2 = 2.0 - w1;
        double u2p = A2[L + IS] * (w2 * U[L] + w1 * U[L + IS]);
        double v2p = A2[L + IS] * (w2 * V[L] + w1 * V[L + IS]);
        double x2p = A2[L + IS] * (w2 * W[L] + w1 * W[L + IS]);
        w1 = 2.0 * (D3[L] / (D3[L] + D3[L - IL])); w2 = 2.0 - w1;
        double u3m = A3[L] * (w2 * U[L] + w1 * U[L - IL]);
        double v3m = A3[L] * (w2 * V[L] + w1 * V[L - IL]);
        double x3m = A3[L] * (w2 * W[L] + w1 * W[L - IL]);
        w1 = 2.0 * (D3[L] / (D3[L] + D3[L + IL])); w2 = 2.0 - w1;
        double u3p = A3[L + IL] * (w2 * U[L] + w1 * U[L + IL]);
        double v3p = A3[L + IL] * (w2 * V[L] + w1 * V[L + IL]);
        double x3p = A3[L + IL] * (w2 * W[L] + w1 * W[L + IL]);
        double pvol = .5 / VOL[L];
#define GSUM(P1, P2, P3, q3p, q3m, q2p, q2m, q1p, q1m) \
  (pvol * (P3[L + IL] * q3p - P3[L] * q3m + P2[L + IS] * q2p - P2[L] * q2m + P1[L + 1] * q1p - P1[L] * q1m))
        double dudx = GSUM(A1X, A2X, A3X, u3p, u3m, u2p, u2m, u1p, u1m);
        double dudy = GSUM(A1Y, A2Y, A3Y, u3p, u3m, u2p, u2m, u1p, u1m);
        double dudz = GSUM(A1Z, A2Z, A3Z, u3p, u3m, u2p, u2m, u1p, u1m);
        double dvdx = GSUM(A1X, A2X, A3X, v3p, v3m, v2p, v2m, v1p, v1m);
        double dvdy = GSUM(A1Y, A2Y, A3Y, v3p, v3m, v2p, v2m, v1p, v1m);
        double dvdz = GSUM(A1Z, A2Z, A3Z, v3p, v3m, v2p, v2m, v1p, v1m);
        double dwdx = GSUM(A1X, A2X, A3X, x3p, x3m, x2p, x2m, x1p, x1m);
        double dwdy = GSUM(A1Y, A2Y, A3Y, x3p, x3m, x2p, x2m, x1p, x1m);
        double dwdz = GSUM(A1Z, A2Z, A3Z, x3p, x3m, x2p, x2m, x1p, x1m);
#undef GSUM
        double w12 = .5 * (dudy - dvdx), w13 = .5 * (dudz - dwdx), w23 = .5 * (dvdz - dwdy);
        b->a[FF_W12][L] = w12; b->a[FF_W13][L] = w13; b->a[FF_W23][L] = w23;
        b->a[FF_OHMI][L] = 2. * sqrt(w12 * w12 + w13 * w13 + w23 * w23);
        double s11 = .5 * (dudx + dudx), s22 = .5 * (dvdy + dvdy), s33 = .5 * (dwdz + dwdz);
        double s12 = .5 * (dudy + dvdx), s13 = .5 * (dudz + dwdx), s23 = .5 * (dvdz + dwdy);
        double st = s11 * s11 + s12 * s12 + s13 * s13 + s12 * s12 + s22 * s22 + s23 * s23
                  + s13 * s13 + s23 * s23 + s33 * s33;
        b->a[FF_STRAIN][L] = sqrt(2. * st);
        b->a[FF_S11][L] = s11; b->a[FF_S12][L] = s12; b->a[FF_S13][L] = s13;
        b->a[FF_S22][L] = s22; b->a[FF_S23][L] = s23; b->a[FF_S33][L] = s33;
      }
  /* TEMDER: the k-range includes the ghost layer only when KMAX > 1 */
  int klo = (level == 1 && d.kmax > 1) ? 0 : 1, khi = (level == 1 && d.kmax > 1) ? 1 : 0;
  for (int K = klo; K <= d.kmax + khi; K++)
    for (int J = lo; J <= d.jmax + hi; J++)
      for (int I = lo; I <= d.imax + hi; I++) {
        size_t L = IX(d, I, J, K);
        double w1, w2;
        w1 = 2.0 * (D1[L] / (D1[L] + D1[L - 1])); w2 = 2.0 - w1;
        double t1m = w2 * T[L] + w1 * T[L - 1];
        w1 = 2.0 * (D1[L] / (D1[L] + D1[L + 1])); w2 = 2.0 - w1;
        double t1p = w2 * T[L] + w1 * T[L + 1];
        w1 = 2.0 * (D2[L] / (D2[L] + D2[L - IS])); w2 = 2.0 - w1;
        double t2m = w2 * T[L] + w1 * T[L - IS];
        w1 = 2.0 * (D2[L] / (D2[L] + D2[L + IS])); w2 = 2.0 - w1;
        double t2p = w2 * T[L] + w1 * T[L + IS];
        w1 = 2.0 * (D3[L] / (D3[L] + D3[L - IL])); w2 = 2.0 - w1;
        double t3m = w2 * T[L] + w1 * T[L - IL];
        w1 = 2.0 * (D3[L] / (D3[L] + D3[L + IL])); w2 = 2.0 - w1;
        double t3p = w2 * T[L] + w1 * T[L + IL];
        double pvol = .5 / VOL[L];
        b->a[FF_DTDX][L] = pvol * (A3[L + IL] * A3X[L + IL] * t3p - A3[L] * A3X[L] * t3m
                                   + A2[L + IS] * A2X[L + IS] * t2p - A2[L] * A2X[L] * t2m
                                   + A1[L + 1] * A1X[L + 1] * t1p - A1[L] * A1X[L] * t1m);
        b->a[FF_DTDY][L] = pvol * (A3[L + IL] * A3Y[L + IL] * t3p - A3[L] * A3Y[L] * t3m
                                   + A2[L + IS] * A2Y[L + IS] * t2p - A2[L] * A2Y[L] * t2m
                                   + A1[L + 1] * A1Y[L + 1] * t1p - A1[L] * A1Y[L] * t1m);
        b->a[FF_DTDZ][L] = pvol * (A3[L + IL] * A3Z[L + IL] * t3p - A3[L] * A3Z[L] * t3m
                                   + A2[L + IS] * A2Z[L + IS] * t2p - A2[L] * A2Z[L] * t2m
                                   + A1[L + 1] * A1Z[L + 1] * t1p - A1[L] * A1Z[L] * t1m);
      }
}

/* INLET base3c.f:9223 (INLOUT=4) and OUTLET base3c.f:9595 (INLOUT=3), the
 * ghost updates FLUCYC applies on level 1 before the fluxes of a direction
 * (res3c.f:7730-7834).  TURLIM is FLUCYC's local 1e-6 (res3c.f:7750). */
static void surfvects(double a11, double a12, double a13, double *a21, double *a22,
                      double *a23, double *a31, double *a32, double *a33);

void orc_inlet_outlet(orc_block *b, const ff_params *p, int dir, int icycle) {
  dims_t d = dims_of(b);
  double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *T = b->a[FF_TEMP];
  double *RO = b->a[FF_RO], *P = b->a[FF_P], *PD = b->a[FF_PDIFF], *E = b->a[FF_E];
  double *RM = b->a[FF_RM], *RN = b->a[FF_RN], *RW = b->a[FF_RW];
  double *EPS2 = b->a[FF_EPS2], *VIST = b->a[FF_VIST], *VIS = b->a[FF_VIS];
  double *RK = b->a[FF_RK], *REPS = b->a[FF_REPS];
  /* FLUCYC's local TURLIM (res3c.f:7750); FLXCYC passes the real one */
  const double turlim = p->iturb >= 3 ? p->turlim : 1.e-6;
  for (int ip = 0; ip < b->npatch; ip++) {
    const ff_patch *pa = &b->patch[ip];
    face_t f = face_geom(&d, pa->iface);
    if (f.dir != dir) continue;
    int inl = pa->ityp == FF_BC_INL && pa->ibtype <= 6;
    int out = pa->ityp == FF_BC_OUT && pa->ibtype <= 5;
    if (!inl && !out) continue;
    int ls = f.idir * f.s;
    const double *AX = b->a[FF_A1XA + 4 * (dir - 1)], *AY = b->a[FF_A1YA + 4 * (dir - 1)],
                 *AZ = b->a[FF_A1ZA + 4 * (dir - 1)];
    for (int bb = pa->r2a; bb <= pa->r2b; bb++)
      for (int a = pa->r1a; a <= pa->r1b; a++) {
        size_t II = face_cell(&d, &f, a, bb);
        size_t II2 = II + ls, IM1 = II - ls, IM2 = IM1 - ls;
        size_t IF1 = f.idir == 1 ? II : II + f.s;
        if (inl && pa->ibtype == 4) {
          double dpkoe = 1.0 * (1. * P[II] + 0. * P[II2]) + (1. - 1.0) * P[IM1];
          double dpdif = 1.0 * (1. * PD[II] + 0. * PD[II2]) + (1. - 1.0) * PD[IM1];
          EPS2[IM1] = 1. * EPS2[II] + 0. * EPS2[II2]; EPS2[IM2] = EPS2[IM1];
          VIST[IM1] = 1. * VIST[II] + 0. * VIST[II2]; VIST[IM2] = VIST[IM1];
          RM[IM1] = pa->bounu * pa->bounr;
          RN[IM1] = pa->bounv * pa->bounr;
          RW[IM1] = pa->bounw * pa->bounr;
          if (icycle == 1) RO[IM1] = pa->bounr;
          T[IM1] = pa->bount; T[IM2] = T[IM1];
          /* grid-velocity correction RM += A*WROT*(RO-BOUNR) vanishes (WROT=0) */
          RM[IM2] = RM[IM1]; RN[IM2] = RN[IM1]; RW[IM2] = RW[IM1];
          P[IM1] = dpkoe; P[IM2] = P[IM1];
          PD[IM1] = dpdif; PD[IM2] = PD[IM1];
          E[IM1] = p->rgas / (p->gamma - 1.) * T[IM1];    /* EFPT state.f:876 */
          E[IM2] = E[IM1];
          U[IM1] = RM[IM1] / RO[IM1]; U[IM2] = RM[IM2] / RO[IM2];
          V[IM1] = RN[IM1] / RO[IM1]; V[IM2] = RN[IM2] / RO[IM2];
          W[IM1] = RW[IM1] / RO[IM1]; W[IM2] = RW[IM2] / RO[IM2];
          E[IM1] = RO[IM1] * (E[IM1] + .5 * (U[IM1] * U[IM1] + V[IM1] * V[IM1] + W[IM1] * W[IM1]));
          E[IM2] = RO[IM2] * (E[IM2] + .5 * (U[IM2] * U[IM2] + V[IM2] * V[IM2] + W[IM2] * W[IM2]));
          if (p->iturb >= 3) {                      /* base3c.f:9534-9541 */
            RK[IM1] = pa->bounrk; RK[IM2] = RK[IM1];
            REPS[IM1] = pa->bounep; REPS[IM2] = REPS[IM1];
            E[IM1] = E[IM1] + RK[IM1];
            E[IM2] = E[IM2] + RK[IM2];
          }
        } else if (out && (pa->ibtype == 2 || pa->ibtype == 3)) {
          double rk3 = pa->ibtype == 2 ? 0.7 : 1.0, rk4 = pa->ibtype == 2 ? 0.3 : 0.0;
          double a11 = AX[IF1], a12 = AY[IF1], a13 = AZ[IF1], a21, a22, a23, a31, a32, a33;
          surfvects(a11, a12, a13, &a21, &a22, &a23, &a31, &a32, &a33);
          double uim1 = pa->bounu, vim1 = pa->bounv, wim1 = pa->bounw;
          double veloc = .5 * (a11 * (U[II] + uim1) + a12 * (V[II] + vim1) + a13 * (W[II] + wim1));
          P[IM1] = 1. * (pa->bounp - 0.) + 0. * (pa->bounp - 0.); P[IM2] = P[IM1];
          PD[IM1] = 1. * (pa->bounpd - 0.) + 0. * (pa->bounpd - 0.); PD[IM2] = PD[IM1];
          if (-veloc * f.idir > 0.) {
            U[IM1] = (1. * RO[II] * U[II] + 0. * RO[II2] * U[II2]) / RO[IM1]; U[IM2] = U[IM1];
            V[IM1] = 1. * V[II] + 0. * V[II2]; V[IM2] = V[IM1];
            W[IM1] = 1. * W[II] + 0. * W[II2]; W[IM2] = W[IM1];
            EPS2[IM2] = 1. * EPS2[II] + 0. * EPS2[II2];
            VIST[IM2] = 1. * VIST[II] + 0. * VIST[II2];
            EPS2[IM2] = MIND(EPS2[IM2], turlim);
            VIST[IM2] = MIND(VIST[IM2], turlim * VIS[IM2]);
            EPS2[IM1] = EPS2[IM2]; VIST[IM1] = VIST[IM2];
            T[IM1] = 1. * T[II] + 0. * T[II2]; T[IM2] = T[IM1];
            RM[IM1] = RO[IM1] * U[IM1]; RM[IM2] = RO[IM2] * U[IM2];
            RN[IM1] = RO[IM1] * V[IM1]; RN[IM2] = RO[IM2] * V[IM2];
            RW[IM1] = RO[IM1] * W[IM1]; RW[IM2] = RO[IM2] * W[IM2];
          } else {
            double ukm1 = 1. * U[II] + 0. * U[II2], vkm1 = 1. * V[II] + 0. * V[II2], wkm1 = 1. * W[II] + 0. * W[II2];
            double velc1 = a11 * ukm1 + a12 * vkm1 + a13 * wkm1;
            double ukp1 = pa->bounu, vkp1 = pa->bounv, wkp1 = pa->bounw;
            double velc2 = a21 * ukp1 + a22 * vkp1 + a23 * wkp1;
            double velc3 = a31 * ukp1 + a32 * vkp1 + a33 * wkp1;
            double uu = a11 * velc1 + a21 * velc2 + a31 * velc3;
            double vv = a12 * velc1 + a22 * velc2 + a32 * velc3;
            double ww = a13 * velc1 + a23 * velc2 + a33 * velc3;
            U[IM1] = rk3 * U[IM1] + rk4 * uu; U[IM2] = U[IM1];
            V[IM1] = rk3 * V[IM1] + rk4 * vv; V[IM2] = V[IM1];
            W[IM1] = rk3 * W[IM1] + rk4 * ww; W[IM2] = W[IM1];
            EPS2[IM2] = 1. * EPS2[II] + 0. * EPS2[II2];
            VIST[IM2] = 1. * VIST[II] + 0. * VIST[II2];
            EPS2[IM2] = MIND(EPS2[IM2], turlim);
            VIST[IM2] = MIND(VIST[IM2], turlim * VIS[IM2]);
            EPS2[IM1] = EPS2[IM2]; VIST[IM1] = VIST[IM2];
            T[IM1] = pa->bount; T[IM2] = T[IM1];
            RO[IM1] = pa->bounr; RO[IM2] = RO[IM1];
          }
          if (p->iturb >= 3 && -veloc * f.idir > 0.) {   /* base3c.f:10134-10146 */
            RK[IM1] = 1. * RK[II] + 0. * RK[II2]; RK[IM2] = RK[IM1];
            REPS[IM1] = 1. * REPS[II] + 0. * REPS[II2]; REPS[IM2] = REPS[IM1];
            E[IM1] = E[IM1] + RK[IM1];
            E[IM2] = E[IM2] + RK[IM2];
          }
        }
      }
  }
}

/* SURFVECTS base3c.f:12245 */
static void surfvects(double a11, double a12, double a13, double *a21, double *a22,
                      double *a23, double *a31, double *a32, double *a33) {
  double am = fabs(a11);
  int idir = 1;
  if (fabs(a12) < am) { am = fabs(a12); idir = 2; }
  if (fabs(a13) < am) idir = 3;
  double b1, b2, b3;
  if (idir == 1) { b1 = 0.0; b2 = -a13; b3 = a12; }
  else if (idir == 2) { b1 = a13; b2 = 0.0; b3 = -a11; }
  else { b1 = -a12; b2 = a11; b3 = 0.0; }
  double palpo = 1. / sqrt(b1 * b1 + b2 * b2 + b3 * b3);
  b1 = b1 * palpo; b2 = b2 * palpo; b3 = b3 * palpo;
  *a21 = b1; *a22 = b2; *a23 = b3;
  *a31 = a12 * b3 - a13 * b2;
  *a32 = a13 * b1 - a11 * b3;
  *a33 = a11 * b2 - a12 * b1;
}

/* XXTRAP base3c.f:750 (INCHIML false).  r0..r3 = RO(I-KL),RO(I-IL),RO(I),RO(I+IL). */
static void xxtrap(double r0, double r1, double r2, double r3, int intem, double *rip, double *rim) {
  static const double rkk1[5] = {0., 1., 1.3333333, 2., 1.5};
  int inter = abs(intem);
  int inte2 = inter < 1 ? 1 : (inter > 5 ? 5 : inter);
  double rk1 = rkk1[inte2 - 1], rk2 = 2. - rk1;
  double R1 = .25 * rk1, R2 = .25 * rk2, eps = 1.e-10;
  double diff0 = r1 - r0, diff1 = r2 - r1, diff2 = r3 - r2;
  if (intem <= 0 && intem >= -5) {
    *rip = r2 - (diff1 * R1 + diff2 * R2);
    *rim = r1 + (diff1 * R1 + diff0 * R2);
  } else if (inter <= 4) {
    double diff12 = diff1 * diff1 + eps;
    double phibi = (diff12 + diff1 * diff0) / (diff12 + diff0 * diff0);
    double phifi = (diff12 + diff1 * diff2) / (diff12 + diff2 * diff2);
    *rip = r2 - phifi * (diff1 * R1 + diff2 * R2);
    *rim = r1 + phibi * (diff1 * R1 + diff0 * R2);
  } else {
    *rip = r2;
    *rim = r1;
  }
}

/* XXTRAA base3c.f:1444-1570 (INCHIML false): XXTRAP with the cells' extents
 * along the face normal, d0..d3 = D(I-KL), D(I-IL), D(I), D(I+IL) (D1/D2/D3
 * of the direction): the differences become slopes over the centre
 * distances and the half extents scale the extrapolation.  FLUXKE, FLUXKT
 * and FLUCUSP call it in place of XXTRAP when XXTRAL is set. */
static void xxtraa(double r0, double r1, double r2, double r3, double d0, double d1, double d2, double d3,
                   int intem, double *rip, double *rim) {
  static const double rkk1[5] = {0., 1., 1.3333333, 2., 1.5};
  const double eps = 1.e-10;
  int inter = abs(intem);
  int inte2 = inter < 1 ? 1 : (inter > 5 ? 5 : inter);
  double rk1 = rkk1[inte2 - 1], rk2 = 2. - rk1;
  if (intem <= 0 && intem >= -5) {
    double dxl = .5 * d1, dxr = .5 * d2;
    double dx0 = 1. / (d0 + d1 + eps), dx1 = 1. / (d1 + d2 + eps), dx2 = 1. / (d2 + d3 + eps);
    *rip = r2 - dxr * (dx1 * (r2 - r1) * rk1 + dx2 * (r3 - r2) * rk2);
    *rim = r1 + dxl * (dx1 * (r2 - r1) * rk1 + dx0 * (r1 - r0) * rk2);
  } else if (inter <= 4) {
    double dxl = .5 * d1, dxr = .5 * d2;
    double dx0 = 1. / (d0 + d1 + eps), dx1 = 1. / (d1 + d2 + eps), dx2 = 1. / (d2 + d3 + eps);
    double diff0 = dx0 * (r1 - r0), diff1 = dx1 * (r2 - r1), diff2 = dx2 * (r3 - r2);
    double diff12 = diff1 * diff1 + eps;
    double phibi = (diff12 + diff1 * diff0) / (diff12 + diff0 * diff0);
    double phifi = (diff12 + diff1 * diff2) / (diff12 + diff2 * diff2);
    *rip = r2 - dxr * phifi * (diff1 * rk1 + diff2 * rk2);
    *rim = r1 + dxl * phibi * (diff1 * rk1 + diff0 * rk2);
  } else {
    *rip = r2;
    *rim = r1;
  }
}

/* The MUSCL pair of one variable, q[0..3] = cells I-2S..I+S: XXTRAP, or
 * XXTRAA with the cells' extents dd[0..3] when dd is given (XXTRAL). */
static void xxm(const double *q, const double *dd, int intem, double *ip, double *im) {
  if (dd) xxtraa(q[0], q[1], q[2], q[3], dd[0], dd[1], dd[2], dd[3], intem, ip, im);
  else xxtrap(q[0], q[1], q[2], q[3], intem, ip, im);
}

/* One face of FLUXKE base3c.f:4753-5120 (laminar: k = eps = 0, UROT = 0),
 * with EFPRO state.f:620 (perfect gas) and DERIV base3c.f:707.
 * q[v][m]: v = ro,u,v,w,p ; m = 0..3 -> cells I-2S, I-S, I, I+S.
 * cr/cl = {C, DRDP, DRDH, RO, P} of cell I and of cell I2 (DERIV).
 * dd: the cells' extents for XXTRAA (XXTRAL), or NULL for XXTRAP.
 * Adds the 5 flux components to f5[]. */
static void roe_face_core(const double q[5][4], const double *nrm, double area, int intem,
                          const ff_params *p, double c_r, double c_l, const double *cr,
                          const double *cl2, const double *dd, double *f5) {
  double roip, roim, rmip, rmim, rnip, rnim, rwip, rwim, ppi, pmi;
  xxm(q[0], dd, intem, &roip, &roim);
  xxm(q[1], dd, intem, &rmip, &rmim);
  xxm(q[2], dd, intem, &rnip, &rnim);
  xxm(q[3], dd, intem, &rwip, &rwim);
  xxm(q[4], dd, intem, &ppi, &pmi);
  roip = MAXD(0.001 * p->frsden, roip);
  ppi = MAXD(0.001 * p->frspre, ppi);
  roim = MAXD(0.001 * p->frsden, roim);
  pmi = MAXD(0.001 * p->frspre, pmi);
  const double gm1 = p->gamma - 1.;
  double eip = (ppi + 0.) / (gm1 * roip) - p->e0ref;
  double eim = (pmi + 0.) / (gm1 * roim) - p->e0ref;
  double elr = (ppi + 0.) / (gm1 * roim) - p->e0ref;
  double erl = (pmi + 0.) / (gm1 * roip) - p->e0ref;
  /* DERIV */
  double ypro1 = 1. / cr[3], ypro2 = 1. / cl2[3];
  double dedp1 = -cr[1] / cr[2] - ypro1;
  double dedp2 = -cl2[1] / cl2[2] - ypro2;
  double dedph = 0.5 * (dedp1 + dedp2);
  double dedr1 = 1. / cr[2] + cr[4] * (ypro1 * ypro1);
  double dedr2 = 1. / cl2[2] + cl2[4] * (ypro2 * ypro2);
  double dedrh = 0.5 * (dedr1 + dedr2);
  {
    double dpp = 2. * (ppi - pmi), drr = 2. * (roip - roim);
    if (fabs(dpp) >= 1.e-2 * (ppi + pmi)) dedph = (eip + elr - eim - erl) / dpp;
    if (fabs(drr) >= 1.e-2 * (roip + roim)) dedrh = (eip + erl - eim - elr) / drr;
  }
  double a11 = nrm[0], a12 = nrm[1], a13 = nrm[2], a21, a22, a23, a31, a32, a33;
  surfvects(a11, a12, a13, &a21, &a22, &a23, &a31, &a32, &a33);
  double ur = a11 * rmip + a12 * rnip + a13 * rwip;
  double vr = a21 * rmip + a22 * rnip + a23 * rwip;
  double wr = a31 * rmip + a32 * rnip + a33 * rwip;
  double ul = a11 * rmim + a12 * rnim + a13 * rwim;
  double vl = a21 * rmim + a22 * rnim + a23 * rwim;
  double wl = a31 * rmim + a32 * rnim + a33 * rwim;
  const double rkipi = 0., reipi = 0., rkimi = 0., reimi = 0.;   /* MAX(0.001*0, 0) */
  double ypror = 1. / roip, rkr = rkipi * ypror;
  double yprol = 1. / roim, rkl = rkimi * yprol;
  double eir = eip + .5 * (ur * ur + vr * vr + wr * wr) + rkr;
  double eil = eim + .5 * (ul * ul + vl * vl + wl * wl) + rkl;
  double pr = ppi, pkr = .6667 * rkipi, epsr = reipi * ypror, hr = eir + pr * ypror, er = eip;
  double rohat = sqrt(roip * roim), yproh = 1. / rohat;
  double pl = pmi, pkl = .6667 * rkimi, epsl = reimi * yprol, hl = eil + yprol * pl, el = eim;
  double sqrl = 1. / (roim + rohat), cql = roim * sqrl, cqr = 1. - cql;
  double uhat = cqr * ur + cql * ul, vhat = cqr * vr + cql * vl, what = cqr * wr + cql * wl;
  double hhat = cqr * hr + cql * hl, ehat = cqr * er + cql * el;
  double rkhat = cqr * rkr + cql * rkl, epshat = cqr * epsr + cql * epsl;
  double phat = rohat * (hhat - ehat - .5 * (uhat * uhat + vhat * vhat + what * what) - rkhat);
  double pmin = MIND(pr, pl), pmax = MAXD(pr, pl);
  phat = MIND(pmax, phat);
  phat = MAXD(pmin, phat);
  double drdhh = 1. / (dedrh - phat * (yproh * yproh));
  double drdph = -drdhh * (dedph + yproh);
  double xturb = 1. + .6667 * rkhat * yproh * drdph;
  double chat2 = xturb / (drdhh * yproh + drdph);
  double cmin = MIND(c_r, c_l), cmax = MAXD(c_r, c_l);
  chat2 = MIND(cmax * cmax, chat2);
  chat2 = MAXD(cmin * cmin, chat2);
  double chat = sqrt(chat2);
  double pdpde = dedph;
  double dro = roip - roim, du = ur - ul, dk = rkr - rkl;
  double dp = pr - pl + .6667 * (rkhat * dro + rohat * dk);
  double pchat2 = 1. / (chat * chat);
  double alfa1 = .5 * (dp + rohat * chat * du) * pchat2;
  double alfa2 = .5 * (dp - rohat * chat * du) * pchat2;
  double alfa3 = dro - dp * pchat2;
  double alfa4 = rohat * (vr - vl), alfa5 = rohat * (wr - wl), alfa6 = rohat * dk;
  (void)epshat;
  const double uc = 0.;
  double rl1h = uhat - uc + chat, rl2h = uhat - uc - chat, rl3h = uhat - uc;
  double rl1 = fabs(rl1h), rl2 = fabs(rl2h), rl3 = fabs(rl3h);
  if (p->entropy_fix) {
    double rl1r = ur - uc + c_r, rl2r = ur - uc - c_r, rl3r = ur - uc;
    double rl1l = ul - uc + c_l, rl2l = ul - uc - c_l, rl3l = ul - uc;
    double e22;
    e22 = 4. * MAXD(MAXD(1.e-10, rl1h - rl1l), rl1r - rl1h);
    if (rl1 <= e22) rl1 = .5 * (rl1h * rl1h + e22 * e22) / e22;
    e22 = 4. * MAXD(MAXD(1.e-10, rl2h - rl2l), rl2r - rl2h);
    if (rl2 <= e22) rl2 = .5 * (rl2h * rl2h + e22 * e22) / e22;
    e22 = 4. * MAXD(MAXD(1.e-10, rl3h - rl3l), rl3r - rl3h);
    if (rl3 <= e22) rl3 = .5 * (rl3h * rl3h + e22 * e22) / e22;
  }
  double rl4 = rl3, rl5 = rl3, rl6 = rl3;
  double roucr = roip * (ur - uc), roucl = roim * (ul - uc);
  double damp = rl1 * alfa1 + rl2 * alfa2 + rl3 * alfa3;
  double f1 = .5 * area * (roucr + roucl - damp);
  double f2 = .5 * area * (roucr * ur + pr + pkr + roucl * ul + pl + pkl
                           - (damp * uhat + (rl1 * alfa1 - rl2 * alfa2) * chat));
  double f3 = .5 * area * (roucr * vr + roucl * vl - damp * vhat - rl4 * alfa4);
  double f4 = .5 * area * (roucr * wr + roucl * wl - damp * what - rl5 * alfa5);
  double f5v = .5 * area * (roucr * (hr + pkr * ypror) + roucl * (hl + pkl * yprol)
                            + uc * (pr + pkr + pl + pkl)
                            - damp * hhat - ((rl1 * alfa1 - rl2 * alfa2) * uhat * chat
                            - rl3 * alfa3 * rohat * (chat * chat) * pdpde + rl4 * alfa4 * vhat
                            + rl5 * alfa5 * what) + rl6 * alfa6 * (1. - .6667 * rohat * pdpde));
  double f2pm = a11 * f2 + a21 * f3 + a31 * f4;
  double f3pm = a12 * f2 + a22 * f3 + a32 * f4;
  double f4pm = a13 * f2 + a23 * f3 + a33 * f4;
  f5[0] = f1 + f5[0];
  f5[1] = f2pm + f5[1];
  f5[2] = f3pm + f5[2];
  f5[3] = f4pm + f5[3];
  f5[4] = f5v + f5[4];
}

void orc_roe_face(const double *qr, const double *ql, const double *qrr, const double *qll,
                  const double *nrm, double area, int intem, const ff_params *p,
                  const double *cell_r, const double *cell_l, int kquirk, double *f5) {
  double q[5][4];
  for (int v = 0; v < 5; v++) { q[v][0] = qll[v]; q[v][1] = ql[v]; q[v][2] = qr[v]; q[v][3] = qrr[v]; }
  roe_face_core(q, nrm, area, intem, p, cell_r[0], cell_l[0], cell_r, kquirk ? cell_r : cell_l, NULL, f5);
}

/* FLUXBL base3c.f:4085 (IDIFF=1) for the face between L-S and L. */
static void fluxbl_face(const orc_block *b, const ff_params *p, size_t L, int S, int dir, double *F) {
  const double *A = b->a[FF_A1 + 4 * (dir - 1)], *NX = b->a[FF_A1XA + 4 * (dir - 1)];
  const double *NY = b->a[FF_A1YA + 4 * (dir - 1)], *NZ = b->a[FF_A1ZA + 4 * (dir - 1)];
  const double *D = b->a[FF_D1 + (dir - 1)];
  const double *S11 = b->a[FF_S11], *S12 = b->a[FF_S12], *S13 = b->a[FF_S13];
  const double *S22 = b->a[FF_S22], *S23 = b->a[FF_S23], *S33 = b->a[FF_S33];
  const double *W12 = b->a[FF_W12], *W13 = b->a[FF_W13], *W23 = b->a[FF_W23];
  const double *DTX = b->a[FF_DTDX], *DTY = b->a[FF_DTDY], *DTZ = b->a[FF_DTDZ];
  const double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *T = b->a[FF_TEMP];
  const double *XC = b->a[FF_XC], *YC = b->a[FF_YC], *ZC = b->a[FF_ZC];
  const double *VIS = b->a[FF_VIS], *EPS2 = b->a[FF_EPS2], *VIST = b->a[FF_VIST];
  const double *CP = b->a[FF_CP], *CH = b->a[FF_CH];
  size_t M = L - S;
  const double R23 = .6666667;
  double w1 = 2.0 * (D[L] / (D[L] + D[M])), w2 = 2.0 - w1, w1p = .5 * w1, w2p = .5 * w2;
  double dudx = w2p * S11[L] + w1p * S11[M];
  double dvdy = w2p * S22[L] + w1p * S22[M];
  double dwdz = w2p * S33[L] + w1p * S33[M];
  double dudy = w2p * (S12[L] + W12[L]) + w1p * (S12[M] + W12[M]);
  double dudz = w2p * (S13[L] + W13[L]) + w1p * (S13[M] + W13[M]);
  double dvdx = w2p * (S12[L] - W12[L]) + w1p * (S12[M] - W12[M]);
  double dvdz = w2p * (S23[L] + W23[L]) + w1p * (S23[M] + W23[M]);
  double dwdx = w2p * (S13[L] - W13[L]) + w1p * (S13[M] - W13[M]);
  double dwdy = w2p * (S23[L] - W23[L]) + w1p * (S23[M] - W23[M]);
  double s11i = w2 * S11[L] + w1 * S11[M], s12i = w2 * S12[L] + w1 * S12[M];
  double s13i = w2 * S13[L] + w1 * S13[M], s22i = w2 * S22[L] + w1 * S22[M];
  double s23i = w2 * S23[L] + w1 * S23[M], s33i = w2 * S33[L] + w1 * S33[M];
  double dtdxi = w2p * DTX[L] + w1p * DTX[M];
  double dtdyi = w2p * DTY[L] + w1p * DTY[M];
  double dtdzi = w2p * DTZ[L] + w1p * DTZ[M];
  double sxi = XC[L] - XC[M], syi = YC[L] - YC[M], szi = ZC[L] - ZC[M];
  double slen = sqrt(sxi * sxi + syi * syi + szi * szi) + 1.e-21;
  sxi = sxi / slen; syi = syi / slen; szi = szi / slen;
  double nx = NX[L], ny = NY[L], nz = NZ[L];
  double alfa = sxi * nx + syi * ny + szi * nz;
  double surf = 0.5 * A[L] * (EPS2[L] * VIS[L] + EPS2[M] * VIS[M]);
  double surfe = 0.5 * A[L] * (CP[L] * VIST[L] / p->prt + CH[L] + CP[M] * VIST[M] / p->prt + CH[M]);
  double dudxsj = dudx * sxi + dudy * syi + dudz * szi;
  double dvdxsj = dvdx * sxi + dvdy * syi + dvdz * szi;
  double dwdxsj = dwdx * sxi + dwdy * syi + dwdz * szi;
  double duvwsj = nx * dudxsj + ny * dvdxsj + nz * dwdxsj;
  double sdotdu = sxi * dudx + syi * dudy + szi * dudz;
  double sdotdv = sxi * dvdx + syi * dvdy + szi * dvdz;
  double sdotdw = sxi * dwdx + syi * dwdy + szi * dwdz;
  double adotu = (nx * (U[L] - U[M]) + ny * (V[L] - V[M]) + nz * (W[L] - W[M]));
  double f2 = nx * s11i + ny * s12i + nz * s13i;
  double f3 = nx * s12i + ny * s22i + nz * s23i;
  double f4 = nx * s13i + ny * s23i + nz * s33i;
  if (alfa > 0.) {
    f2 = alfa * ((U[L] - U[M]) / slen - sdotdu) + sxi * (adotu / slen - duvwsj) + f2;
    f3 = alfa * ((V[L] - V[M]) / slen - sdotdv) + syi * (adotu / slen - duvwsj) + f3;
    f4 = alfa * ((W[L] - W[M]) / slen - sdotdw) + szi * (adotu / slen - duvwsj) + f4;
  }
  f2 = f2 - R23 * nx * (dudx + dvdy + dwdz);
  f3 = f3 - R23 * ny * (dudx + dvdy + dwdz);
  f4 = f4 - R23 * nz * (dudx + dvdy + dwdz);
  f2 = surf * f2; f3 = surf * f3; f4 = surf * f4;
  double f5 = .5 * ((U[L] + U[M]) * f2 + (V[L] + V[M]) * f3 + (W[L] + W[M]) * f4)
            + surfe * (dtdxi * nx + dtdyi * ny + dtdzi * nz);
  if (alfa > 0.)
    f5 = surfe * alfa * ((T[L] - T[M]) / slen - sxi * dtdxi - syi * dtdyi - szi * dtdzi) + f5;
  F[0] = 0.; F[1] = -f2; F[2] = -f3; F[3] = -f4; F[4] = 0. - f5;
}

static void fluxdo_face_fe(const orc_block *b, const ff_params *p, size_t L, int S, int dir, double fe0,
                           double *F);

/* FLUXDO base3c.f:3677 (thin layer, IDIFF=1): the viscous flux on coarse
 * levels and whenever FULLNS is off. */
static void fluxdo_face(const orc_block *b, const ff_params *p, size_t L, int S, int dir, double *F) {
  fluxdo_face_fe(b, p, L, S, dir, 0., F);
}

/* FLUXDO with the energy flux already holding fe0 (FLUDKE's k diffusion on
 * two-equation coarse levels): FE = fe0 + F5VIG + SURFE*(T(I)-T(I-IL)). */
static void fluxdo_face_fe(const orc_block *b, const ff_params *p, size_t L, int S, int dir, double fe0,
                           double *F) {
  const double *A = b->a[FF_A1 + 4 * (dir - 1)], *NX = b->a[FF_A1XA + 4 * (dir - 1)];
  const double *NY = b->a[FF_A1YA + 4 * (dir - 1)], *NZ = b->a[FF_A1ZA + 4 * (dir - 1)];
  const double *VOL = b->a[FF_VOL], *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *T = b->a[FF_TEMP];
  const double *VIS = b->a[FF_VIS], *EPS2 = b->a[FF_EPS2], *VIST = b->a[FF_VIST];
  const double *CP = b->a[FF_CP], *CH = b->a[FF_CH];
  size_t M = L - S;
  double ypd2 = A[L] / (VOL[L] + VOL[M]);
  double surg = -A[L] * ypd2;
  double surf = surg * (EPS2[L] * VIS[L] + EPS2[M] * VIS[M]);
  double surfe = surg * (CP[L] * VIST[L] / p->prt + CH[L] + CP[M] * VIST[M] / p->prt + CH[M]);
  double duc = .333333 * (NX[L] * (U[L] - U[M]) + NY[L] * (V[L] - V[M]) + NZ[L] * (W[L] - W[M]));
  double f2 = surf * (U[L] - U[M] + NX[L] * duc);
  double f3 = surf * (V[L] - V[M] + NY[L] * duc);
  double f4 = surf * (W[L] - W[M] + NZ[L] * duc);
  double f5 = .5 * ((U[L] + U[M]) * f2 + (V[L] + V[M]) * f3 + (W[L] + W[M]) * f4);
  F[0] = 0.; F[1] = f2; F[2] = f3; F[3] = f4;
  F[4] = fe0 + f5 + surfe * (T[L] - T[M]);
}

/* BOTSKE base3c.f:6147-6760: solid-wall face flux on level 1, laminar,
 * TURCOR=.FALSE. (the value FLUCYC passes, res3c.f:8107), wall at rest. */
static void botske_face(const orc_block *b, const ff_params *p, size_t II, int S, int idir,
                        int dir, int iheat, int intem, double *F) {
  const double *A = b->a[FF_A1 + 4 * (dir - 1)], *NX = b->a[FF_A1XA + 4 * (dir - 1)];
  const double *NY = b->a[FF_A1YA + 4 * (dir - 1)], *NZ = b->a[FF_A1ZA + 4 * (dir - 1)];
  const double *VOL = b->a[FF_VOL], *VIS = b->a[FF_VIS], *CH = b->a[FF_CH], *P = b->a[FF_P];
  const double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *T = b->a[FF_TEMP];
  double rc1 = 1.5, rc2 = rc1 - 1.;
  if (intem == 6) { rc1 = 1.; rc2 = 0.; }
  const double prs = p->pr / p->prt, ymr = .166666667, eps = 1.e-3;
  int lstrid = S * idir;
  size_t II2 = II + lstrid;
  size_t IF1 = idir == 1 ? II : II + S;
  int ihfl = (iheat == 2 || iheat >= 12) ? 1 : 0;
  int iht = (iheat == 0 || iheat == 15) ? 0 : 1;
  double vislim = 0.01 * p->frsvis;
  double dist = (A[IF1] + A[IF1 + lstrid]) / VOL[II];
  double surg = -dist * ymr;
  double eps2b = 1., vistb = 0.;
  double visb = MAXD(vislim, rc1 * VIS[II] - rc2 * VIS[II2]);
  double chsb = MAXD(eps, rc1 * CH[II] - rc2 * CH[II2]);
  double pb1 = MAXD(0.01 * p->frspre, rc1 * P[II] - rc2 * P[II2]);
  double surf = surg * eps2b * visb;
  double surfe = surg * (prs * vistb / visb + 1.) * chsb;
  double tempb = MAXD(0.01 * p->frstem, rc1 * T[II] - rc2 * T[II2]);
  double tsurf = iheat == 1 ? p->frstem : p->frstem;   /* T0; TWALL for IHEAT=1 */
  if (iheat == 3) tsurf = tempb;
  const double usurf = 0., vsurf = 0., wsurf = 0.;
  double temp1 = T[II], temp2 = T[II + lstrid];
  double cvi2 = iht * idir * (9.000 * temp1 - 1.000 * temp2 - 8. * tsurf);
  double uvi2 = idir * (9.000 * U[II] - 1.000 * U[II2] - 8. * usurf);
  double vvi2 = idir * (9.000 * V[II] - 1.000 * V[II2] - 8. * vsurf);
  double wvi2 = idir * (9.000 * W[II] - 1.000 * W[II2] - 8. * wsurf);
  double cvi1 = iht * idir * (temp1 - tsurf);
  double uvi1 = idir * (U[II] - usurf) * 6.;
  double vvi1 = idir * (V[II] - vsurf) * 6.;
  double wvi1 = idir * (W[II] - wsurf) * 6.;
  double pb4 = MAXD(-.99 * p->frspre, rc1 * b->a[FF_PDIFF][II] - rc2 * b->a[FF_PDIFF][II2]);
  /* YP1, YP4 (base3c.f:6304-6315): the pressure difference for KT (IFLUX=7) */
  const double yp1 = p->flux == FF_FLUX_KT ? 0. : 1., yp4 = 1. - yp1;
  double pb = yp1 * pb1 + yp4 * pb4;
  double alpha = 1.;
  double cvii = (1. - alpha) * cvi1 + alpha * cvi2;
  double uvii = (1. - alpha) * uvi1 + alpha * uvi2;
  double vvii = (1. - alpha) * vvi1 + alpha * vvi2;
  double wvii = (1. - alpha) * wvi1 + alpha * wvi2;
  double ax = NX[IF1], ay = NY[IF1], az = NZ[IF1];
  double duc = .33333 * (ay * vvii + az * wvii + ax * uvii);
  double f2v = surf * (uvii + ax * duc);
  double f3v = surf * (vvii + ay * duc);
  double f4v = surf * (wvii + az * duc);
  double f5vf = usurf * f2v + vsurf * f3v + wsurf * f4v;
  double f5vq = (1 - ihfl) * surfe * cvii + ihfl * 0.0;
  double f5v = f5vf + f5vq;
  double f6v = 0.;
  F[0] = 0.;
  F[1] = A[IF1] * (ax * pb + f2v);
  F[2] = A[IF1] * (ay * pb + f3v);
  F[3] = A[IF1] * (az * pb + f4v);
  F[4] = A[IF1] * (0. * pb1 + f5v + f6v);
}

/* FLUCYC res3c.f:7572 for one direction: zero the face fluxes, inlet/outlet
 * ghosts (done by the caller), viscous flux, Roe flux, wall faces. */
/* FLUXVL base3c.f:1733-1961 (IFLUX=0) for one face: van Leer flux-vector
 * splitting of the MUSCL-extrapolated conservative variables (cells
 * I-2S..I+S in qc[v][m], v = RO, RM, RN, RW, E), added to f (perfect gas).
 * wps = 1: FLUXWP base3c.f:1967-2195 (IFLUX=2), the same routine with the
 * wave/particle split of the subsonic momentum and energy fluxes
 * (base3c.f:2118-2125, 2156-2163). */
static void vl_face(const double qc[5][4], const double *nrm, double area, int intem, const ff_params *p,
                    int wps, double *f) {
  const double gamma = p->gamma, gm1 = gamma - 1., ygm = 1. / gamma;
  double ip[5], im[5];
  for (int v = 0; v < 5; v++) xxtrap(qc[v][0], qc[v][1], qc[v][2], qc[v][3], intem, &ip[v], &im[v]);
  double ppi = (gamma - 1.) * (ip[4] - .5 / ip[0] * (ip[1] * ip[1] + ip[2] * ip[2] + ip[3] * ip[3]));
  double pmi = (gamma - 1.) * (im[4] - .5 / im[0] * (im[1] * im[1] + im[2] * im[2] + im[3] * im[3]));
  ip[0] = MAXD(0.001 * p->frsden, ip[0]);
  ppi = MAXD(0.001 * p->frspre, ppi);
  im[0] = MAXD(0.001 * p->frsden, im[0]);
  pmi = MAXD(0.001 * p->frspre, pmi);
  const double a11 = nrm[0], a12 = nrm[1], a13 = nrm[2];
  double a21, a22, a23, a31, a32, a33;
  surfvects(a11, a12, a13, &a21, &a22, &a23, &a31, &a32, &a33);
  double rip[3] = {a11 * ip[1] + a12 * ip[2] + a13 * ip[3], a21 * ip[1] + a22 * ip[2] + a23 * ip[3],
                   a31 * ip[1] + a32 * ip[2] + a33 * ip[3]};
  double rim[3] = {a11 * im[1] + a12 * im[2] + a13 * im[3], a21 * im[1] + a22 * im[2] + a23 * im[3],
                   a31 * im[1] + a32 * im[2] + a33 * im[3]};
  double fm[5], fp[5];
  { /* F- from the right state (IP) */
    double ypro = 1. / ip[0], u = ypro * rip[0], v = ypro * rip[1], w = ypro * rip[2];
    double pp = MAXD(0.01, ppi), c = sqrt(gamma * pp * ypro), rma = u / c;
    if (rma < -1.) {
      fm[0] = area * rip[0]; fm[1] = area * (rip[0] * u + pp); fm[2] = area * rip[0] * v;
      fm[3] = area * rip[0] * w; fm[4] = area * u * (ip[4] + pp);
    } else if (rma < 1.) {
      double h = .5 * (rma - 1.);
      double f1 = -area * ip[0] * c * (h * h);
      fm[0] = f1; fm[2] = f1 * v; fm[3] = f1 * w;
      if (wps) {
        double rma2 = .25 * ((rma - 1.) * (rma - 1.)) * (2. + rma);
        fm[1] = f1 * u + area * pp * rma2;
        fm[4] = f1 * ip[4] * ypro + area * u * pp * rma2;
      } else {
        fm[1] = f1 * (gm1 * u - 2. * c) * ygm;
        fm[4] = f1 * (ip[4] + pp) * ypro;
      }
    } else {
      fm[0] = fm[1] = fm[2] = fm[3] = fm[4] = 0.;
    }
  }
  { /* F+ from the left state (IM) */
    double ypro = 1. / im[0], u = ypro * rim[0], v = ypro * rim[1], w = ypro * rim[2];
    double pm = MAXD(0.01, pmi), c = sqrt(gamma * pm * ypro), rma = u / c;
    if (rma > 1.) {
      fp[0] = area * rim[0]; fp[1] = area * (rim[0] * u + pm); fp[2] = area * rim[0] * v;
      fp[3] = area * rim[0] * w; fp[4] = area * u * (im[4] + pm);
    } else if (rma > -1.) {
      double h = .5 * (rma + 1.);
      double f1 = +area * im[0] * c * (h * h);
      fp[0] = f1; fp[2] = f1 * v; fp[3] = f1 * w;
      if (wps) {
        double rma2 = .25 * ((rma + 1.) * (rma + 1.)) * (2. - rma);
        fp[1] = f1 * u + area * pm * rma2;
        fp[4] = f1 * im[4] * ypro + area * u * pm * rma2;
      } else {
        fp[1] = f1 * (gm1 * u + 2. * c) * ygm;
        fp[4] = f1 * (im[4] + pm) * ypro;
      }
    } else {
      fp[0] = fp[1] = fp[2] = fp[3] = fp[4] = 0.;
    }
  }
  double f2 = fp[1] + fm[1], f3 = fp[2] + fm[2], f4 = fp[3] + fm[3];
  f[0] = fm[0] + fp[0] + f[0];
  f[1] = a11 * f2 + a21 * f3 + a31 * f4 + f[1];
  f[2] = a12 * f2 + a22 * f3 + a32 * f4 + f[2];
  f[3] = a13 * f2 + a23 * f3 + a33 * f4 + f[3];
  f[4] = fm[4] + fp[4] + f[4];
}

#include "finflo_oracle_flux.c"

void orc_flux_dir(orc_block *b, const ff_params *p, int dir, int level) {
  dims_t d = dims_of(b);
  int S = dir == 1 ? 1 : (dir == 2 ? d.is : d.il);
  int nmax = dir == 1 ? d.imax : (dir == 2 ? d.jmax : d.kmax);
  int intem = dir == 1 ? p->interi : (dir == 2 ? p->interj : p->interk);
  if (level > 1) intem = p->coarse_inter;
  double *F[5] = {b->a[FF_F1R], b->a[FF_F1RM], b->a[FF_F1RN], b->a[FF_F1RW], b->a[FF_F1E]};
  for (int v = 0; v < 5; v++) memset(F[v], 0, sizeof(double) * d.ntot);
  const double *A = b->a[FF_A1 + 4 * (dir - 1)], *NX = b->a[FF_A1XA + 4 * (dir - 1)];
  const double *NY = b->a[FF_A1YA + 4 * (dir - 1)], *NZ = b->a[FF_A1ZA + 4 * (dir - 1)];
  const double *RO = b->a[FF_RO], *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W];
  const double *P = b->a[FF_P], *C = b->a[FF_C], *DRDP = b->a[FF_DRDP], *DRDH = b->a[FF_DRDH];
  /* faces bounding interior cells: normal index 1..nmax+1, transverse interior */
  int t1max = dir == 1 ? d.jmax : d.imax, t2max = dir == 3 ? d.jmax : d.kmax;
  for (int t2 = 1; t2 <= t2max; t2++)
    for (int t1 = 1; t1 <= t1max; t1++)
      for (int m = 1; m <= nmax + 1; m++) {
        size_t L = dir == 1 ? IX(d, m, t1, t2) : (dir == 2 ? IX(d, t1, m, t2) : IX(d, t1, t2, m));
        double f[5] = {0, 0, 0, 0, 0};
        int idi = dir == 1 ? p->idi1 : (dir == 2 ? p->idi2 : p->idi3);
        if (m <= MIND(idi, nmax + 1)) {          /* SINVIS: viscous faces */
          if (level == 1 && p->fullns) fluxbl_face(b, p, L, S, dir, f);
          else fluxdo_face(b, p, L, S, dir, f);
        }
        double q[5][4];
        const double *arr[5] = {RO, U, V, W, P};
        for (int v = 0; v < 5; v++) {
          q[v][0] = arr[v][L - 2 * S]; q[v][1] = arr[v][L - S];
          q[v][2] = arr[v][L]; q[v][3] = arr[v][L + S];
        }
        double nrm[3] = {NX[L], NY[L], NZ[L]};
        double cr[5] = {C[L], DRDP[L], DRDH[L], RO[L], P[L]};
        size_t L2 = dir == 3 ? L : L - S;      /* DERIV I2 = I-IL, or I itself */
        double cl[5] = {C[L2], DRDP[L2], DRDH[L2], RO[L2], P[L2]};
        if (p->flux != FF_FLUX_ROE) {   /* the other IFLUX schemes */
          alt_face(b, p, dir, L, S, intem, 1, 5, f);
        } else {
          double dd[4];
          roe_face_core(q, nrm, A[L], intem, p, C[L], C[L - S], cr, cl, stencil_d(b, p, dir, L, S, dd), f);
          if (level == 1 && (p->rjk2 > 0. || p->rjk4 > 0.)) jst_face(b, p, L, S, f);
        }
        for (int v = 0; v < 5; v++) F[v][L] = f[v];
      }
  /* wall faces: BOTSKE overwrites (res3c.f:8092, only where IDIM > KBOT) */
  {
    for (int ip = 0; ip < b->npatch; ip++) {
      const ff_patch *pa = &b->patch[ip];
      if (pa->ityp < 8 || pa->ityp > 10) continue;
      face_t f = face_geom(&d, pa->iface);
      if (f.dir != dir) continue;
      for (int bb = pa->r2a; bb <= pa->r2b; bb++)
        for (int a = pa->r1a; a <= pa->r1b; a++) {
          size_t II = face_cell(&d, &f, a, bb);
          double fw[5];
          botske_face(b, p, II, S, f.idir, dir, pa->iheat, intem, fw);
          size_t IF1 = f.idir == 1 ? II : II + S;
          for (int v = 0; v < 5; v++) F[v][IF1] = fw[v];
        }
    }
  }
}

/* SWEEP res3c.f:992: D -= F(n+S)-F(n); the last direction (IDO=1) also
 * multiplies by 1/VOL. */
void orc_sweep(orc_block *b, int dir, int ido) {
  dims_t d = dims_of(b);
  int S = dir == 1 ? 1 : (dir == 2 ? d.is : d.il);
  double *D[5] = {b->a[FF_DRO], b->a[FF_DM], b->a[FF_DN], b->a[FF_DW], b->a[FF_DE]};
  double *F[5] = {b->a[FF_F1R], b->a[FF_F1RM], b->a[FF_F1RN], b->a[FF_F1RW], b->a[FF_F1E]};
  const double *VOL = b->a[FF_VOL];
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t n = IX(d, I, J, K);
        if (ido == 0) {
          for (int v = 0; v < 5; v++) D[v][n] = D[v][n] - (F[v][n + S] - F[v][n]);
        } else {
          double dt1 = 1. / VOL[n];
          for (int v = 0; v < 5; v++) D[v][n] = (D[v][n] - (F[v][n + S] - F[v][n])) * dt1;
        }
      }
}

/* RESIDU res3c.f:6 (laminar): zero D, REFCEN, gradients, k, i, j fluxes. */
/* TIMDER res3c.f:3014 (and TIMDKE res3c.f:3062 for nv = 7): the second
 * order physical-time derivative added to the residual of the interior
 * cells, PDT * (-1.5 VOL (Q - Q2) + 0.5 VOL (Q2 - Q3)), PDT = 1/(VOL DT). */
void orc_timder(orc_block *b, const ff_params *p, int nv) {
  dims_t d = dims_of(b);
  const int sq[7] = {FF_RO, FF_RM, FF_RN, FF_RW, FF_E, FF_RK, FF_REPS};
  const int s2[7] = {FF_ROLE2, FF_RMLE2, FF_RNLE2, FF_RWLE2, FF_ELE2, FF_RKLE2, FF_EPSLE2};
  const int s3[7] = {FF_ROLE3, FF_RMLE3, FF_RNLE3, FF_RWLE3, FF_ELE3, FF_RKLE3, FF_EPSLE3};
  const double *VOL = b->a[FF_VOL];
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t n = IX(d, I, J, K);
        double pdt = 1. / (VOL[n] * p->dt);
        for (int v = 0; v < nv; v++) {
          const double q = b->a[sq[v]][n], q2 = b->a[s2[v]][n], q3 = b->a[s3[v]][n];
          b->a[FF_DRO + v][n] = b->a[FF_DRO + v][n] + pdt * (-1.5 * VOL[n] * (q - q2) + 0.5 * VOL[n] * (q2 - q3));
        }
      }
}

/* STARTI res3c.f:3175 (mode 0: both old levels = the current state, every
 * cell) and NEWTIM ns3c.f:9420 with R1 = 1, R2 = R3 = 0 (mode 1: level n-1
 * <- level n, level n <- the current state, interior cells). */
void orc_time_levels(orc_block *b, int nv, int mode) {
  dims_t d = dims_of(b);
  const int sq[7] = {FF_RO, FF_RM, FF_RN, FF_RW, FF_E, FF_RK, FF_REPS};
  const int s2[7] = {FF_ROLE2, FF_RMLE2, FF_RNLE2, FF_RWLE2, FF_ELE2, FF_RKLE2, FF_EPSLE2};
  const int s3[7] = {FF_ROLE3, FF_RMLE3, FF_RNLE3, FF_RWLE3, FF_ELE3, FF_RKLE3, FF_EPSLE3};
  for (int v = 0; v < nv; v++) {
    double *Q = b->a[sq[v]], *Q2 = b->a[s2[v]], *Q3 = b->a[s3[v]];
    if (mode == 0) {
      for (int n = 0; n < d.ntot; n++) { Q3[n] = Q[n]; Q2[n] = Q[n]; }
    } else {
      for (int K = 1; K <= d.kmax; K++)
        for (int J = 1; J <= d.jmax; J++)
          for (int I = 1; I <= d.imax; I++) {
            size_t n = IX(d, I, J, K);
            Q3[n] = Q2[n];
            Q2[n] = Q[n];
          }
    }
  }
}

void orc_residu(orc_block *b, const ff_params *p, int level, int icycle) {
  dims_t d = dims_of(b);
  for (int s = FF_DRO; s <= FF_DE; s++) memset(b->a[s], 0, sizeof(double) * d.ntot);
  for (int s = FF_W12; s <= FF_W23; s++) memset(b->a[s], 0, sizeof(double) * d.ntot);
  for (int s = FF_DTDX; s <= FF_DTDZ; s++) memset(b->a[s], 0, sizeof(double) * d.ntot);
  if (level == 1 && (p->rjk2 > 0. || p->rjk4 > 0.)) orc_scalard(b);   /* res3c.f:146 */
  if (level == 1) orc_refcen(b, p);
  if (p->fullns && level == 1) orc_gradients(b, level);
  const int order[3] = {3, 1, 2};
  for (int o = 0; o < 3; o++) {
    int dir = order[o];
    if (level == 1) orc_inlet_outlet(b, p, dir, icycle);
    orc_flux_dir(b, p, dir, level);
    orc_sweep(b, dir, dir == 2);
  }
  if (p->timel && level == 1) orc_timder(b, p, 5);   /* res3c.f:705 */
}

/* RESL2 res3c.f:8920: sums of squares of the explicit residuals. */
void orc_resl2(const orc_block *b, double *resi) {
  dims_t d = dims_of(b);
  for (int v = 0; v < 5; v++) resi[v] = 0.;
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t n = IX(d, I, J, K);
        for (int v = 0; v < 5; v++) resi[v] = resi[v] + b->a[FF_DRO + v][n] * b->a[FF_DRO + v][n];
      }
}

/* TIME3 base3c.f:79 (IVISC=1, TIMEL false, UROT=VROT=WROT=0). */
void orc_time3(orc_block *b, const ff_params *p, double cfl) {
  dims_t d = dims_of(b);
  const int IS = d.is, IL = d.il;
  const double *A1 = b->a[FF_A1], *A2 = b->a[FF_A2], *A3 = b->a[FF_A3], *VOL = b->a[FF_VOL];
  const double *A1X = b->a[FF_A1XA], *A1Y = b->a[FF_A1YA], *A1Z = b->a[FF_A1ZA];
  const double *A2X = b->a[FF_A2XA], *A2Y = b->a[FF_A2YA], *A2Z = b->a[FF_A2ZA];
  const double *A3X = b->a[FF_A3XA], *A3Y = b->a[FF_A3YA], *A3Z = b->a[FF_A3ZA];
  const double *RO = b->a[FF_RO], *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W];
  const double *C = b->a[FF_C], *P = b->a[FF_P], *VIS = b->a[FF_VIS], *VIST = b->a[FF_VIST];
  double *DTL = b->a[FF_DTL];
  const double eps = 1.e-10, pcfl = 1. / cfl, prs = p->pr / p->prt;
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t kk = IX(d, I, J, K);
        /* ZZZ = max of the mean face areas over the viscous directions */
        double zz = 0.;
        if (p->idi1 != 0 && I <= MIND(p->idi1, d.imax)) zz = .5 * (A1[kk] + A1[kk + 1]);
        if (p->idi2 != 0 && J <= MIND(p->idi2, d.jmax)) zz = MAXD(.5 * (A2[kk] + A2[kk + IS]), zz);
        if (p->idi3 != 0 && K <= MIND(p->idi3, d.kmax)) zz = MAXD(.5 * (A3[kk] + A3[kk + IL]), zz);
        double pvol = 1. / VOL[kk], ypro = 1. / (RO[kk] + eps);
        double a1k = .5 * (A1[kk] + A1[kk + 1]);
        double a2k = .5 * (A2[kk] + A2[kk + IS]);
        double a3k = .5 * (A3[kk] + A3[kk + IL]);
        double a1xk = .5 * (A1X[kk] * A1[kk] + A1X[kk + 1] * A1[kk + 1]);
        double a1yk = .5 * (A1Y[kk] * A1[kk] + A1Y[kk + 1] * A1[kk + 1]);
        double a1zk = .5 * (A1Z[kk] * A1[kk] + A1Z[kk + 1] * A1[kk + 1]);
        double a2xk = .5 * (A2X[kk] * A2[kk] + A2X[kk + IS] * A2[kk + IS]);
        double a2yk = .5 * (A2Y[kk] * A2[kk] + A2Y[kk + IS] * A2[kk + IS]);
        double a2zk = .5 * (A2Z[kk] * A2[kk] + A2Z[kk + IS] * A2[kk + IS]);
        double a3xk = .5 * (A3X[kk] * A3[kk] + A3X[kk + IL] * A3[kk + IL]);
        double a3yk = .5 * (A3Y[kk] * A3[kk] + A3Y[kk + IL] * A3[kk + IL]);
        double a3zk = .5 * (A3Z[kk] * A3[kk] + A3Z[kk + IL] * A3[kk + IL]);
        double ucrot = .5 * (A1[kk] * 0. + A1[kk + 1] * 0.);
        double vcrot = .5 * (A2[kk] * 0. + A2[kk + IS] * 0.);
        double wcrot = .5 * (A3[kk] * 0. + A3[kk + IL] * 0.);
        double ucii = a1xk * U[kk] + a1yk * V[kk] + a1zk * W[kk] - ucrot;
        double vcii = a2xk * U[kk] + a2yk * V[kk] + a2zk * W[kk] - vcrot;
        double wcii = a3xk * U[kk] + a3yk * V[kk] + a3zk * W[kk] - wcrot;
        double b1 = pvol * (fabs(ucii) + fabs(vcii) + fabs(wcii)
                            + C[kk] * sqrt(a1k * a1k + a2k * a2k + a3k * a3k)) * pcfl;
        double rnum = zz * zz * (pvol * pvol) * ypro;
        double t = rnum * (VIS[kk] + prs * VIST[kk]) / p->cdiff;
        double b2 = 2. * t * p->pvisc;
        double b11 = MAXD(b1, b2);
        double denlow = (1. + MAXD(0., (p->frspre - 2. * P[kk]) / P[kk]));
        double denmax = (1. + MAXD(0., (RO[kk] - 2. * p->frsden) * ypro) * 5.);
        denlow = MAXD(denlow, denmax);
        DTL[kk] = 1. / (b11 * denlow);
        /* TIMEL: the dual time step, base3c.f:206-215 */
        if (p->timel) DTL[kk] = DTL[kk] * p->dt / (1.5 * DTL[kk] + p->dt);
      }
}

/* LOCDT imps3.f:784 and COPR imps3.f:891 on the interior cells (the ghost
 * residuals are zero in the reference and stay zero). */
void orc_locdt_copr(orc_block *b) {
  dims_t d = dims_of(b);
  double *DRO = b->a[FF_DRO], *DM = b->a[FF_DM], *DN = b->a[FF_DN], *DW = b->a[FF_DW], *DE = b->a[FF_DE];
  const double *DTL = b->a[FF_DTL], *RO = b->a[FF_RO], *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W];
  const double *E = b->a[FF_E], *P = b->a[FF_P], *C = b->a[FF_C], *DRDP = b->a[FF_DRDP], *DRDH = b->a[FF_DRDH];
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t i = IX(d, I, J, K);
        double dt1 = DTL[i];
        DRO[i] = dt1 * DRO[i]; DM[i] = dt1 * DM[i]; DN[i] = dt1 * DN[i];
        DW[i] = dt1 * DW[i]; DE[i] = dt1 * DE[i];
        double vel2 = (U[i] * U[i] + V[i] * V[i] + W[i] * W[i]);
        double beta = .5 * vel2;
        double drodh = DRDH[i], drodp = DRDP[i], ypro = 1. / RO[i];
        double dri = DRO[i], dmi = DM[i], dni = DN[i], dwi = DW[i], dre = DE[i];
        double dkin = U[i] * dmi + V[i] * dni + W[i] * dwi;
        DM[i] = ypro * (-U[i] * dri + dmi);
        DN[i] = ypro * (-V[i] * dri + dni);
        DW[i] = ypro * (-W[i] * dri + dwi);
        double hi = ypro * (E[i] + P[i]);
        double dei = dre - (hi - 2 * beta) * dri - dkin;
        double dpi = C[i] * C[i] * (dri - drodh * ypro * dei);
        double dhi = (dri - drodp * dpi) / drodh;
        DRO[i] = dhi;
        DE[i] = dpi;
      }
}

/* SYI / SYM1I imps4.f:10/46: primitive <-> characteristic increments. */
static void syi(double *w, const double *x, double c, double ro, double a2x, double a2y,
                double a2z, double *a2) {
  double z1i = x[0], z5i = x[4];
  double a21, a22, a23, a31, a32, a33;
  surfvects(a2x, a2y, a2z, &a21, &a22, &a23, &a31, &a32, &a33);
  a2[0] = a21; a2[1] = a22; a2[2] = a23; a2[3] = a31; a2[4] = a32; a2[5] = a33;
  double z2i = a2x * x[1] + a2y * x[2] + a2z * x[3];
  double z3i = a21 * x[1] + a22 * x[2] + a23 * x[3];
  double z4i = a31 * x[1] + a32 * x[2] + a33 * x[3];
  double roc = ro * c;
  w[0] = z1i - z5i / ro;
  w[1] = roc * z2i + z5i;
  w[2] = z3i;
  w[3] = z4i;
  w[4] = -roc * z2i + z5i;
}

static void sym1i(double *x, const double *w, double c, double ro, double a2x, double a2y,
                  double a2z, const double *a2) {
  double ypro = 1. / ro, pc2 = .5 * ypro, proc = pc2 / c;
  x[0] = w[0] + pc2 * (w[1] + w[4]);
  double x2i = proc * (w[1] - w[4]), x3i = w[2], x4i = w[3];
  x[4] = .5 * (w[1] + w[4]);
  x[1] = a2x * x2i + a2[0] * x3i + a2[3] * x4i;
  x[2] = a2y * x2i + a2[1] * x3i + a2[4] * x4i;
  x[3] = a2z * x2i + a2[2] * x3i + a2[5] * x4i;
}

/* The product M(face) * dW of one neighbour: SYM1I(diag(l1,l2,l1,l1,l5) SYI(dW)). */
static void jac_product(double *out, const double *dw, double c, double ro, double nx, double ny,
                        double nz, double l1, double l2, double l5) {
  double w[5], a2[6];
  syi(w, dw, c, ro, nx, ny, nz, a2);
  w[0] = l1 * w[0]; w[1] = l2 * w[1]; w[2] = l1 * w[2]; w[3] = l1 * w[3]; w[4] = l5 * w[4];
  sym1i(out, w, c, ro, nx, ny, nz, a2);
}

/* PREDGS imps4.f:345-600, in the reference's own order: k descending, and in
 * each k-slab the i+j hyperplanes descending with the YDROI/BDRO row buffers
 * (including their shift at imps4.f:547-559). */
void orc_predgs(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  const int IS = d.is, IL = d.il, IMAX = d.imax, JMAX = d.jmax, KMAX = d.kmax;
  double *D[5] = {b->a[FF_DRO], b->a[FF_DM], b->a[FF_DN], b->a[FF_DW], b->a[FF_DE]};
  const double *VOL = b->a[FF_VOL], *DTL = b->a[FF_DTL];
  const double *A1 = b->a[FF_A1], *A2 = b->a[FF_A2], *A3 = b->a[FF_A3];
  const double *A1X = b->a[FF_A1XA], *A1Y = b->a[FF_A1YA], *A1Z = b->a[FF_A1ZA];
  const double *A2X = b->a[FF_A2XA], *A2Y = b->a[FF_A2YA], *A2Z = b->a[FF_A2ZA];
  const double *A3X = b->a[FF_A3XA], *A3Y = b->a[FF_A3YA], *A3Z = b->a[FF_A3ZA];
  const double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *C = b->a[FF_C], *RO = b->a[FF_RO];
  const double *VIS = b->a[FF_VIS], *VIST = b->a[FF_VIST];
  const int maw = JMAX * IS + 8;
  double *cd = calloc((size_t)5 * maw, sizeof(double));
  double *xi = calloc((size_t)3 * maw, sizeof(double)), *xj = calloc((size_t)3 * maw, sizeof(double));
  double *xk = calloc((size_t)3 * maw, sizeof(double)), *dt = calloc((size_t)maw, sizeof(double));
  double *scinv = calloc((size_t)maw, sizeof(double)), *scinp = calloc((size_t)maw, sizeof(double));
  double *yd = calloc((size_t)5 * (IMAX + 2), sizeof(double)), *bd = calloc((size_t)5 * (IMAX + 2), sizeof(double));
  const double cdiff = 2.;
  for (int l = 0; l < 5 * maw; l++) cd[l] = 0.;
  for (int K = KMAX; K >= 1; K--) {
    size_t kk = (size_t)(2 + K - 1) * IL;
    double ffk = 2.;
    if (K == 1) ffk = 4.;
    if (K > p->idi3) ffk = 0.;
    double cdiffk = ffk * cdiff;
    for (int J = 1; J <= JMAX; J++) {
      double ffj = 2.;
      if (J == 1) ffj = 4.;
      if (J > p->idi2) ffj = 0.;
      double cdiffj = cdiff * ffj;
      for (int I = 1; I <= IMAX; I++) {
        size_t N = kk + (size_t)(J + 1) * IS + (I + 1);
        int L = (J - 1) * IS + 2 + I;
        double ffi = 2.;
        if (I == 1) ffi = 4.;
        if (I > p->idi1) ffi = 0.;
        double cdiffi = ffi * cdiff;
        double rl1 = A1X[N] * U[N] + A1Y[N] * V[N] + A1Z[N] * W[N] - 0.;
        double rl2 = rl1 + C[N], rl5 = rl1 - C[N];
        double rnum = (VOL[N] + VOL[N - 1]) * (RO[N] + RO[N - 1]);
        double t = cdiffi * A1[N] / rnum * (VIST[N] + VIS[N] + VIST[N - 1] + VIS[N - 1]);
        double rimax = 1.00 * (fabs(rl1) + C[N]);
        xi[3 * L + 0] = (rl1 - rimax) * .5 - t;
        xi[3 * L + 1] = (rl2 - rimax) * .5 - t;
        xi[3 * L + 2] = (rl5 - rimax) * .5 - t;
        double xia = rimax + t;
        rl1 = A2X[N] * U[N] + A2Y[N] * V[N] + A2Z[N] * W[N] - 0.;
        rl2 = rl1 + C[N]; rl5 = rl1 - C[N];
        rnum = (VOL[N] + VOL[N - IS]) * (RO[N] + RO[N - IS]);
        t = cdiffj * A2[N] / rnum * (VIST[N] + VIS[N] + VIST[N - IS] + VIS[N - IS]);
        double rjmax = 1.00 * (fabs(rl1) + C[N]);
        xj[3 * L + 0] = (rl1 - rjmax) * .5 - t;
        xj[3 * L + 1] = (rl2 - rjmax) * .5 - t;
        xj[3 * L + 2] = (rl5 - rjmax) * .5 - t;
        double xja = rjmax + t;
        rl1 = A3X[N] * U[N] + A3Y[N] * V[N] + A3Z[N] * W[N] - 0.;
        rl2 = rl1 + C[N]; rl5 = rl1 - C[N];
        rnum = (VOL[N] + VOL[N - IL]) * (RO[N] + RO[N - IL]);
        t = cdiffk * A3[N] / rnum * (VIST[N] + VIS[N] + VIST[N - IL] + VIS[N - IL]);
        double rkmax = 1.00 * (fabs(rl1) + C[N]);
        xk[3 * L + 0] = (rl1 - rkmax) * .5 - t;
        xk[3 * L + 1] = (rl2 - rkmax) * .5 - t;
        xk[3 * L + 2] = (rl5 - rkmax) * .5 - t;
        double xka = rkmax + t;
        double dt1 = p->theta * DTL[N];
        dt[L] = dt1;
        for (int v = 0; v < 5; v++) cd[5 * L + v] = -dt1 * A3[N + IL] * cd[5 * L + v] + VOL[N] * D[v][N];
        scinv[L] = 1. / (VOL[N] + dt1 * (xia * A1[N] + xja * A2[N] + xka * A3[N]) + VOL[N] * 0.);
        scinp[L] = 1. / (VOL[N] + dt1 * (rimax * A1[N] + rjmax * A2[N] + rkmax * A3[N]) + VOL[N] * 0.);
      }
    }
    for (int l = 0; l < 5 * (IMAX + 2); l++) { yd[l] = 0.; bd[l] = 0.; }
    for (int M = IMAX + JMAX; M >= 2; M--) {
      int ialku = MAXD(1, M - JMAX), iloppu = MIND(IMAX, M - 1);
      for (int I = ialku; I <= iloppu; I++) {
        int J = M - I;
        size_t N = kk + (size_t)(J + 1) * IS + (I + 1);
        int L = (J - 1) * IS + 2 + I;
        double dt1 = dt[L];
        for (int v = 0; v < 5; v++)
          cd[5 * L + v] = cd[5 * L + v] - dt1 * (A1[N + 1] * yd[5 * I + v] + A2[N + IS] * bd[5 * I + v]);
        for (int v = 0; v < 4; v++) cd[5 * L + v] = cd[5 * L + v] * scinv[L];
        cd[5 * L + 4] = cd[5 * L + 4] * scinp[L];
        double dw[5];
        for (int v = 0; v < 5; v++) { D[v][N] = cd[5 * L + v]; dw[v] = cd[5 * L + v]; }
        double out[5];
        jac_product(out, dw, C[N], RO[N], A1X[N], A1Y[N], A1Z[N], xi[3 * L], xi[3 * L + 1], xi[3 * L + 2]);
        for (int v = 0; v < 5; v++) yd[5 * I + v] = out[v];
        jac_product(out, dw, C[N], RO[N], A2X[N], A2Y[N], A2Z[N], xj[3 * L], xj[3 * L + 1], xj[3 * L + 2]);
        for (int v = 0; v < 5; v++) bd[5 * I + v] = out[v];
      }
      /* imps4.f:1460 starts the shift at IALKU, so cell (IALKU-1, JMAX) of the
       * next hyperplane never receives the i+1 product of (IALKU, JMAX);
       * predgs_full starts it one index earlier */
      for (int I = (p->predgs_full && ialku > 1) ? ialku - 1 : ialku; I <= iloppu - 1; I++)
        for (int v = 0; v < 5; v++) yd[5 * I + v] = yd[5 * (I + 1) + v];
      for (int v = 0; v < 5; v++) yd[5 * iloppu + v] = 0.;
    }
    for (int l = 1; l <= JMAX * IS; l++) {
      size_t N = kk + l + 2 * IS - 1;
      double dw[5], out[5];
      for (int v = 0; v < 5; v++) dw[v] = D[v][N];
      jac_product(out, dw, C[N], RO[N], A3X[N], A3Y[N], A3Z[N], xk[3 * l], xk[3 * l + 1], xk[3 * l + 2]);
      for (int v = 0; v < 5; v++) cd[5 * l + v] = out[v];
    }
  }
  free(cd); free(xi); free(xj); free(xk); free(dt); free(scinv); free(scinp); free(yd); free(bd);
}

/* DIAGGS imps4.f:604 on the interior cells. */
void orc_diaggs(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  const int IS = d.is, IL = d.il;
  double *D[5] = {b->a[FF_DRO], b->a[FF_DM], b->a[FF_DN], b->a[FF_DW], b->a[FF_DE]};
  const double *VOL = b->a[FF_VOL], *DTL = b->a[FF_DTL];
  const double *A1 = b->a[FF_A1], *A2 = b->a[FF_A2], *A3 = b->a[FF_A3];
  const double *A1X = b->a[FF_A1XA], *A1Y = b->a[FF_A1YA], *A1Z = b->a[FF_A1ZA];
  const double *A2X = b->a[FF_A2XA], *A2Y = b->a[FF_A2YA], *A2Z = b->a[FF_A2ZA];
  const double *A3X = b->a[FF_A3XA], *A3Y = b->a[FF_A3YA], *A3Z = b->a[FF_A3ZA];
  const double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *C = b->a[FF_C];
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t N = IX(d, I, J, K);
        double ucn = A1X[N + 1] * U[N] + A1Y[N + 1] * V[N] + A1Z[N + 1] * W[N] - 0.;
        double r1n = 1.00 * (fabs(ucn) + C[N]);
        double ucp = A1X[N] * U[N] + A1Y[N] * V[N] + A1Z[N] * W[N] - 0.;
        double r1p = 1.00 * (fabs(ucp) + C[N]);
        ucn = A2X[N + IS] * U[N] + A2Y[N + IS] * V[N] + A2Z[N + IS] * W[N] - 0.;
        double r2n = 1.00 * (fabs(ucn) + C[N]);
        ucp = A2X[N] * U[N] + A2Y[N] * V[N] + A2Z[N] * W[N] - 0.;
        double r2p = 1.00 * (fabs(ucp) + C[N]);
        ucn = A3X[N + IL] * U[N] + A3Y[N + IL] * V[N] + A3Z[N + IL] * W[N] - 0.;
        double r3n = 1.00 * (fabs(ucn) + C[N]);
        ucp = A3X[N] * U[N] + A3Y[N] * V[N] + A3Z[N] * W[N] - 0.;
        double r3p = 1.00 * (fabs(ucp) + C[N]);
        double dt1 = p->theta * DTL[N] / VOL[N];
        double scinv = .5 * (A1[N] * r1p + A1[N + 1] * r1n + A2[N] * r2p + A2[N + IS] * r2n
                             + A3[N] * r3p + A3[N + IL] * r3n);
        for (int v = 0; v < 5; v++) D[v][N] = D[v][N] * (1. + dt1 * scinv + 0.);
      }
}

/* CORRGS imps4.f:76-343: k ascending, i+j hyperplanes ascending. */
void orc_corrgs(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  const int IS = d.is, IL = d.il, IMAX = d.imax, JMAX = d.jmax, KMAX = d.kmax;
  double *D[5] = {b->a[FF_DRO], b->a[FF_DM], b->a[FF_DN], b->a[FF_DW], b->a[FF_DE]};
  const double *VOL = b->a[FF_VOL], *DTL = b->a[FF_DTL];
  const double *A1 = b->a[FF_A1], *A2 = b->a[FF_A2], *A3 = b->a[FF_A3];
  const double *A1X = b->a[FF_A1XA], *A1Y = b->a[FF_A1YA], *A1Z = b->a[FF_A1ZA];
  const double *A2X = b->a[FF_A2XA], *A2Y = b->a[FF_A2YA], *A2Z = b->a[FF_A2ZA];
  const double *A3X = b->a[FF_A3XA], *A3Y = b->a[FF_A3YA], *A3Z = b->a[FF_A3ZA];
  const double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *C = b->a[FF_C], *RO = b->a[FF_RO];
  const double *VIS = b->a[FF_VIS], *VIST = b->a[FF_VIST];
  const int maw = JMAX * IS + 8;
  double *cd = calloc((size_t)5 * maw, sizeof(double));
  double *xi = calloc((size_t)3 * maw, sizeof(double)), *xj = calloc((size_t)3 * maw, sizeof(double));
  double *xk = calloc((size_t)3 * maw, sizeof(double)), *dt = calloc((size_t)maw, sizeof(double));
  double *scinv = calloc((size_t)maw, sizeof(double)), *scinp = calloc((size_t)maw, sizeof(double));
  double *yd = calloc((size_t)5 * (IMAX + 3), sizeof(double)), *bd = calloc((size_t)5 * (IMAX + 3), sizeof(double));
  const double cdiff = 2.;
  for (int K = 1; K <= KMAX; K++) {
    size_t kk = (size_t)(K + 1) * IL;
    double ffk = 2.;
    if (K > p->idi3) ffk = 0.;
    double cdiffk = ffk * cdiff;
    for (int J = 1; J <= JMAX; J++) {
      double ffj = 2.;
      if (J > p->idi2) ffj = 0.;
      double cdiffj = cdiff * ffj;
      for (int I = 1; I <= IMAX; I++) {
        size_t N = kk + (size_t)(J + 1) * IS + (I + 1);
        int L = (J - 1) * IS + 2 + I;
        double ffi = 2.;
        if (I > p->idi1) ffi = 0.;
        double cdiffi = ffi * cdiff;
        double rl1 = A1X[N + 1] * U[N] + A1Y[N + 1] * V[N] + A1Z[N + 1] * W[N] - 0.;
        double rl2 = rl1 + C[N], rl5 = rl1 - C[N];
        double rnum = (VOL[N] + VOL[N + 1]) * (RO[N] + RO[N + 1]);
        double t = cdiffi * A1[N] / rnum * (VIST[N] + VIS[N] + VIST[N + 1] + VIS[N + 1]);
        double rimax = 1.00 * (fabs(rl1) + C[N]);
        xi[3 * L + 0] = (rl1 + rimax) * .5 + t;
        xi[3 * L + 1] = (rl2 + rimax) * .5 + t;
        xi[3 * L + 2] = (rl5 + rimax) * .5 + t;
        double xia = rimax + t;
        rl1 = A2X[N + IS] * U[N] + A2Y[N + IS] * V[N] + A2Z[N + IS] * W[N] - 0.;
        rl2 = rl1 + C[N]; rl5 = rl1 - C[N];
        rnum = (VOL[N] + VOL[N + IS]) * (RO[N] + RO[N + IS]);
        t = cdiffj * A2[N] / rnum * (VIST[N] + VIS[N] + VIST[N + IS] + VIS[N + IS]);
        double rjmax = 1.00 * (fabs(rl1) + C[N]);
        xj[3 * L + 0] = (rl1 + rjmax) * .5 + t;
        xj[3 * L + 1] = (rl2 + rjmax) * .5 + t;
        xj[3 * L + 2] = (rl5 + rjmax) * .5 + t;
        double xja = rjmax + t;
        rl1 = A3X[N + IL] * U[N] + A3Y[N + IL] * V[N] + A3Z[N + IL] * W[N] - 0.;
        rl2 = rl1 + C[N]; rl5 = rl1 - C[N];
        rnum = (VOL[N] + VOL[N + IL]) * (RO[N] + RO[N + IL]);
        t = cdiffk * A3[N] / rnum * (VIST[N] + VIS[N] + VIST[N + IL] + VIS[N + IL]);
        double rkmax = 1.00 * (fabs(rl1) + C[N]);
        xk[3 * L + 0] = (rl1 + rkmax) * .5 + t;
        xk[3 * L + 1] = (rl2 + rkmax) * .5 + t;
        xk[3 * L + 2] = (rl5 + rkmax) * .5 + t;
        double xka = rkmax + t;
        double dt1 = p->theta * DTL[N];
        dt[L] = dt1;
        for (int v = 0; v < 5; v++) cd[5 * L + v] = dt1 * A3[N] * cd[5 * L + v] + VOL[N] * D[v][N];
        scinv[L] = 1. / (VOL[N] + dt1 * (xia * A1[N + 1] + xja * A2[N + IS] + xka * A3[N + IL]) + VOL[N] * 0.);
        scinp[L] = 1. / (VOL[N] + dt1 * (rimax * A1[N] + rjmax * A2[N] + rkmax * A3[N]) + VOL[N] * 0.);
      }
    }
    for (int l = 0; l < 5 * (IMAX + 3); l++) { yd[l] = 0.; bd[l] = 0.; }
    for (int M = 2; M <= IMAX + JMAX; M++) {
      int ialku = MAXD(1, M - JMAX), iloppu = MIND(IMAX, M - 1);
      for (int I = ialku; I <= iloppu; I++) {
        int J = M - I;
        size_t N = kk + (size_t)(J + 1) * IS + (I + 1);
        int L = (J - 1) * IS + 2 + I;
        double dt1 = dt[L];
        for (int v = 0; v < 5; v++)
          cd[5 * L + v] = cd[5 * L + v] + dt1 * (A1[N] * yd[5 * I + v] + A2[N] * bd[5 * I + v]);
        for (int v = 0; v < 4; v++) cd[5 * L + v] = cd[5 * L + v] * scinv[L];
        cd[5 * L + 4] = cd[5 * L + 4] * scinp[L];
        double dw[5], out[5];
        for (int v = 0; v < 5; v++) { D[v][N] = cd[5 * L + v]; dw[v] = cd[5 * L + v]; }
        jac_product(out, dw, C[N], RO[N], A1X[N + 1], A1Y[N + 1], A1Z[N + 1], xi[3 * L], xi[3 * L + 1], xi[3 * L + 2]);
        for (int v = 0; v < 5; v++) yd[5 * I + v] = out[v];
        jac_product(out, dw, C[N], RO[N], A2X[N + IS], A2Y[N + IS], A2Z[N + IS], xj[3 * L], xj[3 * L + 1], xj[3 * L + 2]);
        for (int v = 0; v < 5; v++) bd[5 * I + v] = out[v];
      }
      for (int I = iloppu + 1; I >= MAXD(ialku + 1, 2); I--)
        for (int v = 0; v < 5; v++) yd[5 * I + v] = yd[5 * (I - 1) + v];
      for (int v = 0; v < 5; v++) yd[5 * ialku + v] = 0.;
    }
    for (int l = 1; l <= JMAX * IS; l++) {
      size_t N = kk + l + 2 * IS - 1;
      double dw[5], out[5];
      for (int v = 0; v < 5; v++) dw[v] = D[v][N];
      jac_product(out, dw, C[N], RO[N], A3X[N + IL], A3Y[N + IL], A3Z[N + IL], xk[3 * l], xk[3 * l + 1], xk[3 * l + 2]);
      for (int v = 0; v < 5; v++) cd[5 * l + v] = out[v];
    }
  }
  free(cd); free(xi); free(xj); free(xk); free(dt); free(scinv); free(scinp); free(yd); free(bd);
}

static void ddadi_sweeps(orc_block *b, const ff_params *p, int nv);

/* IMPS imps3.f:6 (laminar): TIME3, LOCDT, COPR, then PREDGS, DIAGGS, CORRGS
 * (LUSGS=1) or the DDADI line sweeps (LUSGS=0, imps3.f:320), then DRO/CP
 * (dh -> dT, imps3.f:483). */
void orc_imps(orc_block *b, const ff_params *p, int level) {
  dims_t d = dims_of(b);
  orc_time3(b, p, level == 1 ? p->cfl : p->cfll);
  orc_locdt_copr(b);
  if (p->ddadi) {
    ddadi_sweeps(b, p, 5);
  } else {
    orc_predgs(b, p);
    orc_diaggs(b, p);
    orc_corrgs(b, p);
  }
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t n = IX(d, I, J, K);
        b->a[FF_DRO][n] = b->a[FF_DRO][n] / b->a[FF_CP][n];
      }
}

/* FIN res3c.f:1077 (ITURB<=2 branch) and the limits CYCLES applies after it
 * (ns3c.f:1553-1596): UPLIM/LOLIM res3c.f:3314-3401, PDTOP, LOLIMP. */
void orc_fin_limits(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  double *T = b->a[FF_TEMP], *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *PD = b->a[FF_PDIFF];
  double *P = b->a[FF_P];
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t n = IX(d, I, J, K);
        T[n] = b->a[FF_TOLD][n] + b->a[FF_DRO][n];
        U[n] = b->a[FF_UOLD][n] + b->a[FF_DM][n];
        V[n] = b->a[FF_VOLD][n] + b->a[FF_DN][n];
        W[n] = b->a[FF_WOLD][n] + b->a[FF_DW][n];
        PD[n] = b->a[FF_POLD][n] + b->a[FF_DE][n];
      }
  /* UPLIM: interior k-planes, all rows/columns of them; LOLIM: every cell */
  for (int K = 1; K <= d.kmax; K++) {
    size_t ia = (size_t)(K + 1) * d.il + 2 * d.is;
    for (int i = 0; i < d.jmax * d.is; i++) T[ia + i] = MIND(T[ia + i], p->tuplim);
  }
  for (int n = 0; n < d.ntot; n++) T[n] = MAXD(T[n], p->tlolim);
  double *VV[3] = {U, V, W};
  for (int c = 0; c < 3; c++) {
    for (int K = 1; K <= d.kmax; K++) {
      size_t ia = (size_t)(K + 1) * d.il + 2 * d.is;
      for (int i = 0; i < d.jmax * d.is; i++) VV[c][ia + i] = MIND(VV[c][ia + i], 5000.);
    }
    for (int n = 0; n < d.ntot; n++) VV[c][n] = MAXD(VV[c][n], -5000.);
  }
  for (int n = 0; n < d.ntot; n++) P[n] = PD[n] + p->frspre;      /* PDTOP */
  for (int n = 0; n < d.ntot; n++) {                               /* LOLIMP */
    double prelim = MIND(0., P[n] - 0.01 * p->frspre);
    P[n] = P[n] - prelim;
    PD[n] = PD[n] - prelim;
  }
}

/* REFCOR turb3.f:6040 (REFVAR 6194, EXTCOR 6419): every ghost cell outside
 * the block's faces (two or three ghost indices) takes the values of the
 * interior edge/corner cell next to it. */
void orc_refcor(orc_block *b) {
  dims_t d = dims_of(b);
  static const int slots[] = {FF_RO, FF_RM, FF_RN, FF_RW, FF_E, FF_U, FF_V, FF_W, FF_P, FF_PDIFF,
                              FF_EPS2, FF_VIST, FF_TEMP, FF_VIS, FF_CH, FF_C, FF_DRDP, FF_DRDH,
                              FF_RK, FF_REPS};
  for (int K = -1; K <= d.kmax + 2; K++)
    for (int J = -1; J <= d.jmax + 2; J++)
      for (int I = -1; I <= d.imax + 2; I++) {
        int gi = I < 1 || I > d.imax, gj = J < 1 || J > d.jmax, gk = K < 1 || K > d.kmax;
        if (gi + gj + gk < 2) continue;
        int Ic = I < 1 ? 1 : (I > d.imax ? d.imax : I);
        int Jc = J < 1 ? 1 : (J > d.jmax ? d.jmax : J);
        int Kc = K < 1 ? 1 : (K > d.kmax ? d.kmax : K);
        size_t L = IX(d, I, J, K), LB = IX(d, Ic, Jc, Kc);
        for (size_t s = 0; s < sizeof(slots) / sizeof(slots[0]); s++) b->a[slots[s]][L] = b->a[slots[s]][LB];
      }
}

/* MIR ns3c.f:9003 -> MIRVOL gluebm.f:7510 -> MIRROR gluebm.f:3911 for the
 * symmetry patches (MIR is called with TEMP in the RO position). */
void orc_mir(orc_block *b) {
  dims_t d = dims_of(b);
  double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W];
  for (int ip = 0; ip < b->npatch; ip++) {
    const ff_patch *pa = &b->patch[ip];
    if (pa->ityp != FF_BC_MIR) continue;
    face_t f = face_geom(&d, pa->iface);
    const double *NX = b->a[FF_A1XA + 4 * (f.dir - 1)], *NY = b->a[FF_A1YA + 4 * (f.dir - 1)];
    const double *NZ = b->a[FF_A1ZA + 4 * (f.dir - 1)];
    int kdir = f.idir == 1 ? -1 : 1, koff = f.idir == 1 ? 0 : 1;
    for (int bb = pa->r2a; bb <= pa->r2b; bb++)
      for (int a = pa->r1a; a <= pa->r1b; a++) {
        size_t IC1 = face_cell(&d, &f, a, bb);
        size_t IT = IC1 + (size_t)koff * f.s;           /* wall face */
        size_t IT1 = IC1 + kdir * f.s, IT2 = IC1 + 2 * kdir * f.s, IC2 = IC1 - kdir * f.s;
        double nx = NX[IT], ny = NY[IT], nz = NZ[IT];
        double a11 = 1. * (-2. * nx * nx + 1.0), a12 = 1. * (-2. * nx * ny), a13 = 1. * (-2. * nx * nz);
        double a21 = 1. * (-2. * nx * ny), a22 = 1. * (-2. * ny * ny + 1.0), a23 = 1. * (-2. * ny * nz);
        double a31 = 1. * (-2. * nx * nz), a32 = 1. * (-2. * ny * nz), a33 = 1. * (-2. * nz * nz + 1.0);
        double u1 = U[IC1], v1 = V[IC1], w1 = W[IC1], u2 = U[IC2], v2 = V[IC2], w2 = W[IC2];
        U[IT1] = a11 * u1 + a12 * v1 + a13 * w1;
        V[IT1] = a21 * u1 + a22 * v1 + a23 * w1;
        W[IT1] = a31 * u1 + a32 * v1 + a33 * w1;
        U[IT2] = a11 * u2 + a12 * v2 + a13 * w2;
        V[IT2] = a21 * u2 + a22 * v2 + a23 * w2;
        W[IT2] = a31 * u2 + a32 * v2 + a33 * w2;
        static const int sc[] = {FF_TEMP, FF_E, FF_P, FF_PDIFF, FF_EPS2, FF_VIST, FF_RK, FF_REPS};
        for (int s = 0; s < 8; s++) {   /* RK, REPS: gluebm.f:4104-4125 */
          b->a[sc[s]][IT1] = b->a[sc[s]][IC1];
          b->a[sc[s]][IT2] = b->a[sc[s]][IC2];
        }
      }
  }
}

/* SUBIN ns3c.f:9742: max |dp| monitor (DROMXX, IDRXX=6) and the *OLD copies. */
void orc_subin(orc_block *b, double *dromax) {
  dims_t d = dims_of(b);
  double m = 0.;
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t n = IX(d, I, J, K);
        double a = fabs(b->a[FF_DE][n]);
        if (a > m) m = a;
      }
  *dromax = m;
  memcpy(b->a[FF_TOLD], b->a[FF_TEMP], sizeof(double) * d.ntot);
  memcpy(b->a[FF_UOLD], b->a[FF_U], sizeof(double) * d.ntot);
  memcpy(b->a[FF_VOLD], b->a[FF_V], sizeof(double) * d.ntot);
  memcpy(b->a[FF_WOLD], b->a[FF_W], sizeof(double) * d.ntot);
  memcpy(b->a[FF_POLD], b->a[FF_PDIFF], sizeof(double) * d.ntot);
}

/* BOUNDI ns3c.f:10608 for one block without 1:1 connections: REFCOR, MIR,
 * and STATIM before and after CONNEC (ns3c.f:10896, 10905); the second
 * STATIM sees the ghost pressures the first REFLEC wrote. */
void orc_boundi(orc_block *b, const ff_params *p) {
  orc_refcor(b);
  orc_mir(b);
  orc_statim(b, p);
  orc_statim(b, p);
}

/* One single-grid cycle of NS3D/CYCLES (ns3c.f:467-663, 1400-1600):
 * STATIM, TURBDI, RESIDU (+RESL2), IMPS, FIN + limits, BOUNDI, SUBIN. */
void orc_cycle(orc_block *b, const ff_params *p, int icycle, double *resi5, double *dromax) {
  orc_statim(b, p);
  orc_adjuin_laminar(b);
  orc_residu(b, p, 1, icycle);
  orc_resl2(b, resi5);
  orc_imps(b, p, 1);
  orc_fin_limits(b, p);
  orc_boundi(b, p);
  orc_subin(b, dromax);
}

/* ---------------------------------------------------------------------- */
/* Multigrid (FAS V-cycle of CYCLES ns3c.f:1607-2170)                      */
/* ---------------------------------------------------------------------- */

/* TRANSF multi.f:156: volume-weighted 8 -> 1 restriction of TEMP,U,V,W,PD,
 * EPS2,VIST and of the residuals into the coarse forcing P2H, the coarse
 * *OLD copies, and the coarse ghost rings (multi.f:250-432). */
void orc_transf(orc_block *f, orc_block *c) {
  dims_t df = dims_of(f), dc = dims_of(c);
  static const int vs[7] = {FF_TEMP, FF_U, FF_V, FF_W, FF_PDIFF, FF_EPS2, FF_VIST};
  static const int rs[5] = {FF_DRO, FF_DM, FF_DN, FF_DW, FF_DE};
  static const int ps[5] = {FF_ROP2H, FF_RMP2H, FF_RNP2H, FF_RWP2H, FF_EP2H};
  const double *VOL = f->a[FF_VOL], *VOL2 = c->a[FF_VOL];
  for (int K = 0; K <= dc.kmax + 1; K++)
    for (int J = 0; J <= dc.jmax + 1; J++)
      for (int I = 0; I <= dc.imax + 1; I++) {
        size_t N = IX(dc, I, J, K);
        size_t ijk = IX(df, 2 * I - 1, 2 * J - 1, 2 * K - 1);
        size_t ipjk = ijk + 1, ijpk = ijk + df.is, ipjpk = ijk + df.is + 1;
        size_t ijkp = ijk + df.il, ipjpkp = ipjpk + df.il, ijpkp = ijpk + df.il, ipjkp = ipjk + df.il;
        double pvol = 1. / VOL2[N];
#define R8(X) ((VOL[ipjpk] * X[ipjpk] + VOL[ijk] * X[ijk] + VOL[ipjk] * X[ipjk] + VOL[ijpk] * X[ijpk] + \
                VOL[ipjpkp] * X[ipjpkp] + VOL[ijkp] * X[ijkp] + VOL[ipjkp] * X[ipjkp] + VOL[ijpkp] * X[ijpkp]) * pvol)
        for (int v = 0; v < 7; v++) { const double *X = f->a[vs[v]]; c->a[vs[v]][N] = R8(X); }
        for (int v = 0; v < 5; v++) { const double *X = f->a[rs[v]]; c->a[ps[v]][N] = R8(X); }
#undef R8
      }
  for (int K = 1; K <= dc.kmax; K++)
    for (int J = 1; J <= dc.jmax; J++)
      for (int I = 1; I <= dc.imax; I++) {
        size_t N = IX(dc, I, J, K);
        c->a[FF_TOLD][N] = c->a[FF_TEMP][N];
        c->a[FF_UOLD][N] = c->a[FF_U][N];
        c->a[FF_VOLD][N] = c->a[FF_V][N];
        c->a[FF_WOLD][N] = c->a[FF_W][N];
        c->a[FF_POLD][N] = c->a[FF_PDIFF][N];
      }
  /* ghost rings: P2H zero on both ghost layers, state copied outward from
   * the first ghost layer (order of multi.f: low i, high i, high j, low j,
   * low k, high k) */
  #define RING(N0, OFF)                                                          \
    do {                                                                         \
      size_t n0 = (N0);                                                          \
      for (int v = 0; v < 5; v++) { c->a[ps[v]][n0] = 0.; c->a[ps[v]][n0 + (OFF)] = 0.; } \
      for (int v = 0; v < 7; v++) c->a[vs[v]][n0 + (OFF)] = c->a[vs[v]][n0];     \
    } while (0)
  for (int K = -1; K <= dc.kmax + 2; K++)
    for (int J = -1; J <= dc.jmax + 2; J++) RING(IX(dc, 0, J, K), -1);
  for (int K = -1; K <= dc.kmax + 2; K++)
    for (int J = -1; J <= dc.jmax + 2; J++) RING(IX(dc, dc.imax + 1, J, K), 1);
  for (int K = -1; K <= dc.kmax + 2; K++)
    for (int I = -1; I <= dc.imax + 2; I++) RING(IX(dc, I, dc.jmax + 1, K), dc.is);
  for (int K = -1; K <= dc.kmax + 2; K++)
    for (int I = -1; I <= dc.imax + 2; I++) RING(IX(dc, I, 0, K), -dc.is);
  for (int J = -1; J <= dc.jmax + 2; J++)
    for (int I = -1; I <= dc.imax + 2; I++) RING(IX(dc, I, J, 0), -dc.il);
  for (int J = -1; J <= dc.jmax + 2; J++)
    for (int I = -1; I <= dc.imax + 2; I++) RING(IX(dc, I, J, dc.kmax + 1), dc.il);
  #undef RING
}

/* FORCFU multi.f:1609: P2H -= R (every cell of the level). */
void orc_forcfu(orc_block *c) {
  dims_t d = dims_of(c);
  for (int v = 0; v < 5; v++)
    for (int n = 0; n < d.ntot; n++) c->a[FF_ROP2H + v][n] = c->a[FF_ROP2H + v][n] - c->a[FF_DRO + v][n];
}

/* ADDRES multi.f:1686: R = P2H + R. */
void orc_addres(orc_block *c) {
  dims_t d = dims_of(c);
  for (int v = 0; v < 5; v++)
    for (int n = 0; n < d.ntot; n++) c->a[FF_DRO + v][n] = c->a[FF_ROP2H + v][n] + c->a[FF_DRO + v][n];
}

/* INTERP multi.f:1763: inject the coarse correction into the 8 children. */
void orc_interp(orc_block *c, orc_block *f) {
  dims_t dc = dims_of(c), df = dims_of(f);
  for (int K = 1; K <= df.kmax; K++)
    for (int J = 1; J <= df.jmax; J++)
      for (int I = 1; I <= df.imax; I++) {
        size_t N = IX(dc, (I + 1) / 2, (J + 1) / 2, (K + 1) / 2), F = IX(df, I, J, K);
        double dto = c->a[FF_TEMP][N] - c->a[FF_TOLD][N];
        double du = c->a[FF_U][N] - c->a[FF_UOLD][N];
        double dv = c->a[FF_V][N] - c->a[FF_VOLD][N];
        double dw = c->a[FF_W][N] - c->a[FF_WOLD][N];
        double dp = c->a[FF_PDIFF][N] - c->a[FF_POLD][N];
        f->a[FF_TEMP][F] = f->a[FF_TEMP][F] + dto;
        f->a[FF_U][F] = f->a[FF_U][F] + du;
        f->a[FF_V][F] = f->a[FF_V][F] + dv;
        f->a[FF_W][F] = f->a[FF_W][F] + dw;
        f->a[FF_P][F] = f->a[FF_P][F] + dp;
        f->a[FF_PDIFF][F] = f->a[FF_PDIFF][F] + dp;
      }
}

/* FIN on a coarse level and the limits after it (ns3c.f:1935-1990) or after
 * INTERP (ns3c.f:2059-2125): UPLIM/LOLIM of TEMP and LOLIMP, without PDTOP. */
static void temp_p_limits(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  double *T = b->a[FF_TEMP], *P = b->a[FF_P], *PD = b->a[FF_PDIFF];
  for (int K = 1; K <= d.kmax; K++) {
    size_t ia = (size_t)(K + 1) * d.il + 2 * d.is;
    for (int i = 0; i < d.jmax * d.is; i++) T[ia + i] = MIND(T[ia + i], p->tuplim);
  }
  for (int n = 0; n < d.ntot; n++) T[n] = MAXD(T[n], p->tlolim);
  for (int n = 0; n < d.ntot; n++) {
    double prelim = MIND(0., P[n] - 0.01 * p->frspre);
    P[n] = P[n] - prelim;
    PD[n] = PD[n] - prelim;
  }
}

void orc_fin_coarse(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t n = IX(d, I, J, K);
        b->a[FF_TEMP][n] = b->a[FF_TOLD][n] + b->a[FF_DRO][n];
        b->a[FF_U][n] = b->a[FF_UOLD][n] + b->a[FF_DM][n];
        b->a[FF_V][n] = b->a[FF_VOLD][n] + b->a[FF_DN][n];
        b->a[FF_W][n] = b->a[FF_WOLD][n] + b->a[FF_DW][n];
        b->a[FF_PDIFF][n] = b->a[FF_POLD][n] + b->a[FF_DE][n];
      }
  temp_p_limits(b, p);
}

void orc_intert(orc_block *c, orc_block *f, const ff_params *pf);

/* After INTERP (ns3c.f:2016-2120): the two-equation branch limits T, RK,
 * REPS (UPLIM/LOLIM); LOLIMP always. */
void orc_interp_limits(orc_block *c, orc_block *f, const ff_params *pf) {
  orc_interp(c, f);
  dims_t d = dims_of(f);
  double *T = f->a[FF_TEMP], *P = f->a[FF_P], *PD = f->a[FF_PDIFF];
  if (pf->iturb >= 3) {
    orc_intert(c, f, pf);
    for (int K = 1; K <= d.kmax; K++) {
      size_t ia = (size_t)(K + 1) * d.il + 2 * d.is;
      for (int i = 0; i < d.jmax * d.is; i++) T[ia + i] = MIND(T[ia + i], pf->tuplim);
    }
    for (int n = 0; n < d.ntot; n++) T[n] = MAXD(T[n], pf->tlolim);
    for (int n = 0; n < d.ntot; n++) f->a[FF_RK][n] = MAXD(f->a[FF_RK][n], pf->rklim);
    for (int n = 0; n < d.ntot; n++) f->a[FF_REPS][n] = MAXD(f->a[FF_REPS][n], pf->epslim);
  }
  for (int n = 0; n < d.ntot; n++) {
    double prelim = MIND(0., P[n] - 0.01 * pf->frspre);
    P[n] = P[n] - prelim;
    PD[n] = PD[n] - prelim;
  }
}

/* One multigrid cycle of CYCLES (ns3c.f:1400-2170) with BOUNDI and SUBIN.
 * lv[0] is the fine level; prm[m] are the level's parameters (IDM1..3). */
/* The per-block part of a multigrid cycle (CYCLES ns3c.f:1400-2130): fine
 * update, the coarse levels down, INTERP back up, REFLEC.  resi5 gets the
 * RESL2 sums of the level-1 residual after the fine update. */
void orc_mg_body(orc_block **lv, int nlev, const ff_params *prm, int icycle, double *resi5) {
  orc_block *b = lv[0];
  orc_statim(b, &prm[0]);
  orc_adjuin_laminar(b);
  orc_residu(b, &prm[0], 1, icycle);
  orc_resl2(b, resi5);
  orc_imps(b, &prm[0], 1);
  orc_fin_limits(b, &prm[0]);
  for (int m = 1; m < nlev; m++) {          /* down: level m (0-based) */
    orc_block *f = lv[m - 1], *c = lv[m];
    orc_statim(f, &prm[m - 1]);
    orc_residu(f, &prm[m - 1], m, icycle);
    if (m == 1) orc_resl2(f, resi5);
    if (m > 1) orc_addres(f);
    orc_transf(f, c);
    orc_statim(c, &prm[m]);
    orc_residu(c, &prm[m], m + 1, icycle);
    orc_forcfu(c);
    orc_addres(c);
    orc_imps(c, &prm[m], m + 1);
    orc_fin_coarse(c, &prm[m]);
  }
  for (int m = nlev - 1; m >= 1; m--) orc_interp_limits(lv[m], lv[m - 1], &prm[m - 1]);
  reflec(b, &prm[0]);
}

void orc_mg_cycle(orc_block **lv, int nlev, const ff_params *prm, int icycle, double *resi5, double *dromax) {
  orc_mg_body(lv, nlev, prm, icycle, resi5);
  orc_boundi(lv[0], &prm[0]);
  orc_subin(lv[0], dromax);
}

/* ---------------------------------------------------------------------- */
/* Multi-block: 1:1 connections (CONNEC ns3c.f:8605 -> EXPTOT gluebm.f:6819 */
/* / IMPVO2 gluebm.f:6964) in the four orientations ICON(14) = 0..3.       */
/* ---------------------------------------------------------------------- */

/* The donor face cell (*ad, *cd) of receiver patch point (a, c).  The donor
 * exports its patch with the second in-face index running fastest on odd
 * faces and the first on even faces (EXPVOL gluebm.f:6115-6136, EXPORT
 * 5096); the receiver reads that sequence with its first index fastest on
 * odd faces and its second on even faces (IMPVO2 7040-7080, IMPORT 5174),
 * after PERMUT (4868: PERM1/2/3, a quarter, half or three-quarter turn of
 * the P x Q receiver sequence) by ICON(14). */
void orc_conn_donor(const ff_patch *pa, int a, int c, int *ad, int *cd) {
  const int n1 = pa->r1b - pa->r1a + 1, n2 = pa->r2b - pa->r2a + 1;
  const int rodd = pa->iface & 1, dodd = pa->nface & 1;
  const int P = rodd ? n1 : n2, Q = rodd ? n2 : n1;
  const int x = rodd ? a - pa->r1a + 1 : c - pa->r2a + 1;
  const int y = rodd ? c - pa->r2a + 1 : a - pa->r1a + 1;
  int u, v;
  switch (pa->iori & 3) {
    case 1: u = Q + 1 - y; v = x; break;     /* PERM1: I' = J, J' = ISTR - I + 1 */
    case 2: u = P + 1 - x; v = Q + 1 - y; break;
    case 3: u = y; v = P + 1 - x; break;     /* PERM3: I' = JSTR - J + 1, J' = I */
    default: u = x; v = y;
  }
  if (dodd) { *cd = pa->n2a + u - 1; *ad = pa->n1a + v - 1; }
  else { *ad = pa->n1a + u - 1; *cd = pa->n2a + v - 1; }
}

/* Copy the two interior layers next to the source face of block `src` into
 * the two ghost layers of patch `pa` of block `dst`.  BOUNDI passes TEMP in
 * the RO position and U,V,W in RM,RN,RW (ns3c.f:10900), so the exchanged
 * variables are TEMP,U,V,W,E,EPS2,VIST,CH,P,PDIFF. */
void orc_connec_patch(orc_block *dst, const ff_patch *pa, const orc_block *src) {
  static const int vs[12] = {FF_TEMP, FF_U, FF_V, FF_W, FF_E, FF_EPS2, FF_VIST, FF_CH, FF_P, FF_PDIFF,
                             FF_RK, FF_REPS};
  dims_t dd = dims_of(dst), ds = dims_of((orc_block *)src);
  face_t fd = face_geom(&dd, pa->iface), fs = face_geom(&ds, pa->nface);
  int lsd = fd.idir * fd.s, lss = fs.idir * fs.s;
  for (int bb = pa->r2a; bb <= pa->r2b; bb++)
    for (int a = pa->r1a; a <= pa->r1b; a++) {
      int ad, cd;
      orc_conn_donor(pa, a, bb, &ad, &cd);
      size_t L = face_cell(&dd, &fd, a, bb);
      size_t S = face_cell(&ds, &fs, ad, cd);
      for (int g = 1; g <= 2; g++) {
        size_t G = L - g * lsd, Q = S + (g - 1) * lss;
        for (int v = 0; v < 12; v++) dst->a[vs[v]][G] = src->a[vs[v]][Q];
      }
    }
}

void orc_connec(orc_block **blk, int nblk) {
  for (int n = 0; n < nblk; n++)
    for (int ip = 0; ip < blk[n]->npatch; ip++) {
      const ff_patch *pa = &blk[n]->patch[ip];
      if (pa->ityp != FF_BC_CON) continue;
      orc_connec_patch(blk[n], pa, blk[pa->ibtype]);
    }
}

/* BOUNDI ns3c.f:10608 for several blocks: REFCOR, MIR, STATIM per block
 * (ns3c.f:10660-10700), CONNEC of the 1:1 patches, STATIM again. */
void orc_mb_boundi(orc_block **blk, int nblk, const ff_params *prm) {
  for (int n = 0; n < nblk; n++) { orc_refcor(blk[n]); orc_mir(blk[n]); orc_statim(blk[n], &prm[n]); }
  orc_connec(blk, nblk);
  for (int n = 0; n < nblk; n++) orc_statim(blk[n], &prm[n]);
}

/* One cycle of NS3D for several single-grid blocks: CYCLES per block, then
 * BOUNDI over all blocks (REFCOR, MIR, STATIM, CONNEC, STATIM) and SUBIN. */
void orc_mb_cycle(orc_block **blk, int nblk, const ff_params *prm, int icycle, double *resi5, double *dromax) {
  for (int v = 0; v < 5; v++) resi5[v] = 0.;
  double dm = 0.;
  for (int n = 0; n < nblk; n++) {
    double r[5];
    orc_statim(blk[n], &prm[n]);
    orc_adjuin_laminar(blk[n]);
    orc_residu(blk[n], &prm[n], 1, icycle);
    orc_resl2(blk[n], r);
    for (int v = 0; v < 5; v++) resi5[v] += r[v];
    orc_imps(blk[n], &prm[n], 1);
    orc_fin_limits(blk[n], &prm[n]);
  }
  orc_mb_boundi(blk, nblk, prm);
  for (int n = 0; n < nblk; n++) {
    double d;
    orc_subin(blk[n], &d);
    if (d > dm) dm = d;
  }
  *dromax = dm;
}

void orc_mg_body_sst(orc_block **lv, int nlev, const ff_params *prm, int icycle, double *resi5);

/* Several blocks with nlev multigrid levels each (lv and prm hold block n's
 * levels at [n * nlev .. n * nlev + nlev - 1]): the multigrid part of CYCLES
 * per block, then BOUNDI over the level-1 blocks and SUBIN.  The reference
 * exchanges 1:1 ghosts on level 1 only (BOUNDI(M) on the coarse levels is
 * commented out, ns3c.f:1618 and 1843); coarse ghosts come from TRANSF.
 * Patch IBTYPE of a 1:1 patch is the source block's index n. */
void orc_mb_mg_cycle(orc_block **lv, int nblk, int nlev, const ff_params *prm, int icycle, double *resi5,
                     double *dromax) {
  for (int v = 0; v < 5; v++) resi5[v] = 0.;
  orc_block *fine[256];
  ff_params fprm[256] = {{0}};
  if (nblk > 256) return;
  const int sst = prm[0].iturb >= 3;
  for (int n = 0; n < nblk; n++) {
    double r[5];
    if (sst) orc_mg_body_sst(lv + n * nlev, nlev, prm + n * nlev, icycle, r);
    else orc_mg_body(lv + n * nlev, nlev, prm + n * nlev, icycle, r);
    for (int v = 0; v < 5; v++) resi5[v] += r[v];
    fine[n] = lv[n * nlev];
    fprm[n] = prm[n * nlev];
  }
  orc_mb_boundi(fine, nblk, fprm);
  double dm = 0.;
  for (int n = 0; n < nblk; n++) {
    double d;
    if (sst) orc_subin_sst(fine[n], &fprm[n], &d);
    else orc_subin(fine[n], &d);
    if (d > dm) dm = d;
  }
  *dromax = dm;
}

/* Remote 1:1 patch: the ten CONNEC variables of the two source layers
 * packed as [layer][var][cell, r1 fastest] (the library's halo layout), and
 * their unpacking into the destination ghosts; together they equal
 * orc_connec_patch. */
void orc_halo_pack(const orc_block *src, const ff_patch *pa, double *out) {
  static const int vs[12] = {FF_TEMP, FF_U, FF_V, FF_W, FF_E, FF_EPS2, FF_VIST, FF_CH, FF_P, FF_PDIFF,
                             FF_RK, FF_REPS};
  dims_t ds = dims_of((orc_block *)src);
  face_t fs = face_geom(&ds, pa->nface);
  int lss = fs.idir * fs.s;
  int n1 = pa->r1b - pa->r1a + 1, n2 = pa->r2b - pa->r2a + 1, n = n1 * n2;
  for (int c = 0; c < n2; c++)
    for (int a = 0; a < n1; a++) {
      int ad, cd;
      orc_conn_donor(pa, a + pa->r1a, c + pa->r2a, &ad, &cd);
      size_t S = face_cell(&ds, &fs, ad, cd);
      for (int g = 0; g < 2; g++)
        for (int v = 0; v < 12; v++) out[(size_t)(g * 12 + v) * n + c * n1 + a] = src->a[vs[v]][S + g * lss];
    }
}

void orc_halo_unpack(orc_block *dst, const ff_patch *pa, const double *in) {
  static const int vs[12] = {FF_TEMP, FF_U, FF_V, FF_W, FF_E, FF_EPS2, FF_VIST, FF_CH, FF_P, FF_PDIFF,
                             FF_RK, FF_REPS};
  dims_t dd = dims_of(dst);
  face_t fd = face_geom(&dd, pa->iface);
  int lsd = fd.idir * fd.s;
  int n1 = pa->r1b - pa->r1a + 1, n2 = pa->r2b - pa->r2a + 1, n = n1 * n2;
  for (int c = 0; c < n2; c++)
    for (int a = 0; a < n1; a++) {
      size_t L = face_cell(&dd, &fd, a + pa->r1a, c + pa->r2a);
      for (int g = 0; g < 2; g++)
        for (int v = 0; v < 12; v++) dst->a[vs[v]][L - (g + 1) * lsd] = in[(size_t)(g * 12 + v) * n + c * n1 + a];
    }
}

#include "finflo_oracle_sst.c"
#include "finflo_oracle_ddadi.c"
#include "finflo_oracle_grid.c"
