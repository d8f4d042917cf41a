/*
 * CPU oracle, k-omega SST part (ITURB=6, KOVER=0, IDIS=2, single grid level).
 * TEST INFRASTRUCTURE ONLY (see finflo_oracle.c).  Included at the end of
 * finflo_oracle.c so that it shares that file's static helpers.
 *
 * Restated routines, in the order CYCLES calls them:
 *   TURBEQ res3c.f:5845 (DERFUN, EPS2KO turb3.f:7454 with STRAIN, COEFKO 8068)
 *   RESIKE res3c.f:3423: CROSKO turb3.f:7790, FUN1KO 7385, MAKE_EPS 7905,
 *     PRODKE 4687 (Kato-Launder, the default KATOL), TEMDER of T, k, omega,
 *     FLXCYC res3c.f:6424 per direction (INLET/OUTLET k-omega ghosts,
 *     FLKEBL base3c.f:5727, SETV12, FLUXBL, FLUXKE base3c.f:4753 with k and
 *     omega, BOTSKE base3c.f:6147 with the omega wall value), SWEEPK 1342,
 *     SOURKO turb3.f:7624, ADDSKE res3c.f:1473
 *   IMPS imps3.f:6: TIME3, LOCDTK 807, IMSOKO 972, COPRKE 1113, PRKEGS
 *     imps4.f:1462, DIKEGS 1841, COKEGS 1078 (SYIKE/SYM1KE 982/1034), then
 *     DRO/CP and DRK,DEPS times RO (imps3.f:483-492)
 *   FIN res3c.f:1077 (damped k, omega update, LOLIM) and the CYCLES limits
 *   SUBIN ns3c.f:9742 (k cap, RKOLD/EPSOLD)
 * PARITY UNPINNED, like the rest of the oracle.
 */

/* COEFKO turb3.f:8068, ITURB=6 and KOVER<5 (SST) */
static const double SST_A1KLEB = 0.31, SST_BSTAR = 0.09, SST_CKAPPA = 0.41, SST_BETA1 = 0.075;
static const double SST_SIGRK1 = 0.85, SST_SIGOM1 = 0.5, SST_BETA2 = 0.0828, SST_SIGRK2 = 1.0,
                    SST_SIGOM2 = 0.856;

/* TEMDER turb3.f:3456 for one scalar field phi into (ox, oy, oz), the same
 * cell range as orc_gradients' temperature gradient. */
static void temder_field(orc_block *b, int level, const double *PH, double *OX, double *OY, double *OZ) {
  dims_t d = dims_of(b);
  const int IS = d.is, IL = d.il;
  const double *A1 = b->a[FF_A1], *A2 = b->a[FF_A2], *A3 = b->a[FF_A3], *VOL = b->a[FF_VOL];
  const double *A1X = b->a[FF_A1XA], *A1Y = b->a[FF_A1YA], *A1Z = b->a[FF_A1ZA];
  const double *A2X = b->a[FF_A2XA], *A2Y = b->a[FF_A2YA], *A2Z = b->a[FF_A2ZA];
  const double *A3X = b->a[FF_A3XA], *A3Y = b->a[FF_A3YA], *A3Z = b->a[FF_A3ZA];
  const double *D1 = b->a[FF_D1], *D2 = b->a[FF_D2], *D3 = b->a[FF_D3];
  int lo = level == 1 ? 0 : 1, hi = level == 1 ? 1 : 0;
  int klo = (level == 1 && d.kmax > 1) ? 0 : 1, khi = (level == 1 && d.kmax > 1) ? 1 : 0;
  for (int K = klo; K <= d.kmax + khi; K++)
    for (int J = lo; J <= d.jmax + hi; J++)
      for (int I = lo; I <= d.imax + hi; I++) {
        size_t L = IX(d, I, J, K);
        double w1, w2;
        w1 = 2.0 * (D1[L] / (D1[L] + D1[L - 1])); w2 = 2.0 - w1;
        double t1m = w2 * PH[L] + w1 * PH[L - 1];
        w1 = 2.0 * (D1[L] / (D1[L] + D1[L + 1])); w2 = 2.0 - w1;
        double t1p = w2 * PH[L] + w1 * PH[L + 1];
        w1 = 2.0 * (D2[L] / (D2[L] + D2[L - IS])); w2 = 2.0 - w1;
        double t2m = w2 * PH[L] + w1 * PH[L - IS];
        w1 = 2.0 * (D2[L] / (D2[L] + D2[L + IS])); w2 = 2.0 - w1;
        double t2p = w2 * PH[L] + w1 * PH[L + IS];
        w1 = 2.0 * (D3[L] / (D3[L] + D3[L - IL])); w2 = 2.0 - w1;
        double t3m = w2 * PH[L] + w1 * PH[L - IL];
        w1 = 2.0 * (D3[L] / (D3[L] + D3[L + IL])); w2 = 2.0 - w1;
        double t3p = w2 * PH[L] + w1 * PH[L + IL];
        double pvol = .5 / VOL[L];
        OX[L] = pvol * (A3[L + IL] * A3X[L + IL] * t3p - A3[L] * A3X[L] * t3m
                        + A2[L + IS] * A2X[L + IS] * t2p - A2[L] * A2X[L] * t2m
                        + A1[L + 1] * A1X[L + 1] * t1p - A1[L] * A1X[L] * t1m);
        OY[L] = pvol * (A3[L + IL] * A3Y[L + IL] * t3p - A3[L] * A3Y[L] * t3m
                        + A2[L + IS] * A2Y[L + IS] * t2p - A2[L] * A2Y[L] * t2m
                        + A1[L + 1] * A1Y[L + 1] * t1p - A1[L] * A1Y[L] * t1m);
        OZ[L] = pvol * (A3[L + IL] * A3Z[L + IL] * t3p - A3[L] * A3Z[L] * t3m
                        + A2[L + IS] * A2Z[L + IS] * t2p - A2[L] * A2Z[L] * t2m
                        + A1[L + 1] * A1Z[L + 1] * t1p - A1[L] * A1Z[L] * t1m);
      }
}

/* TURBEQ res3c.f:5845 for SST at level 1: DERFUN (velocity gradients, OHMI,
 * STRAIN), then EPS2KO turb3.f:7454 called with STRAIN in the OHMI slot
 * (KOVER=0, res3c.f:6338) and the local FRSMUT = 1e-3*FRSVIS. */
void orc_turbeq_sst(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  orc_gradients(b, 1);
  const double *VIS = b->a[FF_VIS], *ST = b->a[FF_STRAIN], *RO = b->a[FF_RO];
  const double *RK = b->a[FF_RK], *ROM = b->a[FF_REPS], *DW = b->a[FF_DISTW];
  double *EPS2 = b->a[FF_EPS2], *VIST = b->a[FF_VIST];
  const double frsmut = 1.e-3 * p->frsvis, eps = 1.e-20;
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t L = IX(d, I, J, K);
        double prol = 1. / RO[L];
        double rkl = MAXD(RK[L] * prol, 0.0);
        double oml = ROM[L] * prol;
        double dis2 = DW[L] * DW[L];
        double arg21 = 2. * sqrt(rkl) / (MAXD(eps, SST_BSTAR * oml * DW[L]));
        double auxvi = VIS[L] / (MAXD(eps, ROM[L] * dis2));
        double arg22 = 500. * auxvi;
        double arg2 = MAXD(arg21, arg22);
        double arg4 = 150. * auxvi;
        double fun2 = tanh(arg2 * arg2);
        double fun3 = 1. - tanh(arg4 * arg4 * arg4 * arg4);
        double rmubas = RK[L] / oml;
        double rmumen = SST_A1KLEB * RK[L] / (MAXD(eps, ST[L] * fun2 * fun3));
        double rmutrb = MIND(rmubas, rmumen);
        rmutrb = rmutrb * 1.0 + rmubas * 0.0;
        rmutrb = MAXD(rmutrb, frsmut);
        rmutrb = MIND(rmutrb, p->turlim * VIS[L]);
        VIST[L] = rmutrb;
        double rmutpv = rmutrb / VIS[L];
        EPS2[L] = 1.0 + rmutpv;
      }
}

/* CROSKO turb3.f:7790: cross diffusion into SEPS.  RK and REPS are divided
 * by RO in place and multiplied back afterwards, as the reference does. */
static void crosko(orc_block *b) {
  dims_t d = dims_of(b);
  const int IS = d.is, IL = d.il;
  double *RK = b->a[FF_RK], *ROM = b->a[FF_REPS], *CROSSD = b->a[FF_SEPS];
  const double *RO = b->a[FF_RO], *VOL = b->a[FF_VOL];
  const double *A1 = b->a[FF_A1], *A2 = b->a[FF_A2], *A3 = b->a[FF_A3];
  const double *A1X = b->a[FF_A1XA], *A1Y = b->a[FF_A1YA], *A1Z = b->a[FF_A1ZA];
  const double *A2X = b->a[FF_A2XA], *A2Y = b->a[FF_A2YA], *A2Z = b->a[FF_A2ZA];
  const double *A3X = b->a[FF_A3XA], *A3Y = b->a[FF_A3YA], *A3Z = b->a[FF_A3ZA];
  const double sigo22 = 2.0 * SST_SIGOM2;
  for (int L = 0; L < d.ntot; L++) {
    double prol = 1. / RO[L];
    RK[L] = RK[L] * prol;
    ROM[L] = ROM[L] * prol;
  }
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t L = IX(d, I, J, K);
        double rk1m = A1[L] * (RK[L] + RK[L - 1]), rk1p = A1[L + 1] * (RK[L] + RK[L + 1]);
        double om1m = A1[L] * (ROM[L] + ROM[L - 1]), om1p = A1[L + 1] * (ROM[L] + ROM[L + 1]);
        double rk2m = A2[L] * (RK[L] + RK[L - IS]), rk2p = A2[L + IS] * (RK[L] + RK[L + IS]);
        double om2m = A2[L] * (ROM[L] + ROM[L - IS]), om2p = A2[L + IS] * (ROM[L] + ROM[L + IS]);
        double rk3m = A3[L] * (RK[L] + RK[L - IL]), rk3p = A3[L + IL] * (RK[L] + RK[L + IL]);
        double om3m = A3[L] * (ROM[L] + ROM[L - IL]), om3p = A3[L + IL] * (ROM[L] + ROM[L + IL]);
        double pvol = 0.5 / VOL[L];
#define CSUM(X1, X2, X3, p3, m3, p2, m2, p1, m1) \
  (pvol * (X3[L + IL] * p3 - X3[L] * m3 + X2[L + IS] * p2 - X2[L] * m2 + X1[L + 1] * p1 - X1[L] * m1))
        double dkdx = CSUM(A1X, A2X, A3X, rk3p, rk3m, rk2p, rk2m, rk1p, rk1m);
        double dkdy = CSUM(A1Y, A2Y, A3Y, rk3p, rk3m, rk2p, rk2m, rk1p, rk1m);
        double dkdz = CSUM(A1Z, A2Z, A3Z, rk3p, rk3m, rk2p, rk2m, rk1p, rk1m);
        double dodx = CSUM(A1X, A2X, A3X, om3p, om3m, om2p, om2m, om1p, om1m);
        double dody = CSUM(A1Y, A2Y, A3Y, om3p, om3m, om2p, om2m, om1p, om1m);
        double dodz = CSUM(A1Z, A2Z, A3Z, om3p, om3m, om2p, om2m, om1p, om1m);
#undef CSUM
        double divdot = dkdx * dodx + dkdy * dody + dkdz * dodz;
        CROSSD[L] = sigo22 * RO[L] * divdot / ROM[L];
      }
  for (int L = 0; L < d.ntot; L++) {
    RK[L] = RK[L] * RO[L];
    ROM[L] = ROM[L] * RO[L];
  }
}

/* FUN1KO turb3.f:7385 (TRANSL false): blending function F1 on interior cells. */
static void fun1ko(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  const double *CROSSD = b->a[FF_SEPS], *VIS = b->a[FF_VIS], *RO = b->a[FF_RO];
  const double *RK = b->a[FF_RK], *ROM = b->a[FF_REPS], *DW = b->a[FF_DISTW];
  double *FUN1 = b->a[FF_FUN1];
  const double eps = 1.e-20, sigo24 = 4. * SST_SIGOM2;
  double cdmax = 0.0, sqrtre = sqrt(p->re);
  /* LBEG..LEND: a contiguous storage range from cell (1,1,1) to (IMAX,JMAX,KMAX) */
  size_t lbeg = IX(d, 1, 1, 1), lend = IX(d, d.imax, d.jmax, d.kmax);
  for (size_t L = lbeg; L <= lend; L++) cdmax = MAXD(CROSSD[L], cdmax);
  double cdmin = 1e-8 * cdmax;
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t L = IX(d, I, J, K);
        double prol = 1. / RO[L];
        double rkl = MAXD(RK[L] * prol, 0.0);
        double oml = ROM[L] * prol;
        double dis2 = DW[L] * DW[L];
        double cdkom = MAXD(CROSSD[L], cdmin);
        double arg11 = sqrt(rkl) / (MAXD(eps, SST_BSTAR * oml * DW[L]));
        double arg12 = 500. * VIS[L] / (MAXD(eps, ROM[L] * dis2));
        double arg13 = MAXD(arg11, arg12);
        double arg14 = sigo24 * RK[L] / (MAXD(eps, cdkom * dis2));
        double arg1 = MIND(arg13, arg14);
        FUN1[L] = tanh(arg1 * arg1 * arg1 * arg1);
        double dislim = .40559E-7 * sqrtre;
        if (DW[L] < dislim) FUN1[L] = 1.;
      }
}

/* MAKE_EPS turb3.f:7905 (ITURB=6) into eps_true, and PRODKE turb3.f:4687
 * with the Kato-Launder production (KATOL, the default), VTRAN = 1. */
static void prodke(orc_block *b, double *trueps) {
  dims_t d = dims_of(b);
  const double *RO = b->a[FF_RO], *RK = b->a[FF_RK], *REPS = b->a[FF_REPS];
  const double *S11 = b->a[FF_S11], *S12 = b->a[FF_S12], *S13 = b->a[FF_S13];
  const double *S22 = b->a[FF_S22], *S23 = b->a[FF_S23], *S33 = b->a[FF_S33];
  const double *OHMI = b->a[FF_OHMI], *EPS2 = b->a[FF_EPS2], *VIS = b->a[FF_VIS];
  double *PTUR = b->a[FF_PTUR];
  for (int L = 0; L < d.ntot; L++) trueps[L] = 0.09 * REPS[L] * RK[L] / RO[L];
  for (int K = 1; K <= d.kmax; K++) {
    size_t ia = (size_t)(K + 1) * d.il + 2 * d.is;
    for (int jj = 0; jj < d.jmax * d.is; jj++) {
      size_t L = ia + jj;
      double strain = S11[L] * S11[L] + S12[L] * S12[L] + S13[L] * S13[L]
                    + S12[L] * S12[L] + S22[L] * S22[L] + S23[L] * S23[L]
                    + S13[L] * S13[L] + S23[L] * S23[L] + S33[L] * S33[L];
      strain = sqrt(2. * strain);
      double visco = (EPS2[L] - 1. + 0.) * VIS[L];
      PTUR[L] = visco * strain * OHMI[L];
      PTUR[L] = MIND(PTUR[L], 20. * trueps[L]);
      PTUR[L] = PTUR[L] * 1.;
    }
  }
}

/* FLKEBL base3c.f:5727 for one face (IDIFF default, full NS): the k and omega
 * diffusion fluxes, F1-blended sigmas of the face's high-side cell. */
static void flkebl_face(const orc_block *b, size_t I, int S, int dir, double *frk, double *feps) {
  const double *A = b->a[FF_A1 + 4 * (dir - 1)], *NX = b->a[FF_A1XA + 4 * (dir - 1)];
  const double *NY = b->a[FF_A1YA + 4 * (dir - 1)], *NZ = b->a[FF_A1ZA + 4 * (dir - 1)];
  const double *D = b->a[FF_D1 + (dir - 1)];
  const double *FUN1 = b->a[FF_FUN1], *VIS = b->a[FF_VIS], *VIST = b->a[FF_VIST], *RO = b->a[FF_RO];
  const double *RK = b->a[FF_RK], *REPS = b->a[FF_REPS];
  const double *DKX = b->a[FF_DKDX], *DKY = b->a[FF_DKDY], *DKZ = b->a[FF_DKDZ];
  const double *DEX = b->a[FF_DEDX], *DEY = b->a[FF_DEDY], *DEZ = b->a[FF_DEDZ];
  const double *XC = b->a[FF_XC], *YC = b->a[FF_YC], *ZC = b->a[FF_ZC];
  size_t M = I - S;
  double onemf1 = MAXD(0.0, (1.0 - FUN1[I]));
  double psigk = FUN1[I] * SST_SIGRK1 + onemf1 * SST_SIGRK2;
  double psige = FUN1[I] * SST_SIGOM1 + onemf1 * SST_SIGOM2;
  double w1 = 2.0 * (D[I] / (D[I] + D[M])), w2 = 2.0 - w1;
  double dkdxi = 0.5 * (w2 * DKX[I] + w1 * DKX[M]);
  double dkdyi = 0.5 * (w2 * DKY[I] + w1 * DKY[M]);
  double dkdzi = 0.5 * (w2 * DKZ[I] + w1 * DKZ[M]);
  double dedxi = 0.5 * (w2 * DEX[I] + w1 * DEX[M]);
  double dedyi = 0.5 * (w2 * DEY[I] + w1 * DEY[M]);
  double dedzi = 0.5 * (w2 * DEZ[I] + w1 * DEZ[M]);
  double sxi = XC[I] - XC[M], syi = YC[I] - YC[M], szi = ZC[I] - ZC[M];
  double slen = sqrt(sxi * sxi + syi * syi + szi * szi) + 1.E-21;
  sxi = sxi / slen; syi = syi / slen; szi = szi / slen;
  double alfa = sxi * NX[I] + syi * NY[I] + szi * NZ[I];
  alfa = MAXD(alfa, 0.);
  double rmut2 = VIST[I] + VIST[M];
  double surfk = 0.5 * A[I] * (VIS[I] + VIS[M] + rmut2 * psigk);
  double surfep = 0.5 * A[I] * (VIS[I] + VIS[M] + rmut2 * psige);
  double ypro1 = 1. / RO[I], ypro2 = 1. / RO[M];
  *frk = -surfk * (alfa * (RK[I] * ypro1 - RK[M] * ypro2) / slen + dkdxi * (NX[I] - alfa * sxi)
                   + dkdyi * (NY[I] - alfa * syi) + dkdzi * (NZ[I] - alfa * szi));
  *feps = -surfep * (alfa * (REPS[I] * ypro1 - REPS[M] * ypro2) / slen + dedxi * (NX[I] - alfa * sxi)
                     + dedyi * (NY[I] - alfa * syi) + dedzi * (NZ[I] - alfa * szi));
}

/* One face of FLUXKE base3c.f:4753-5120 with k and omega (ITURB=6, UROT=0):
 * q[v][m]: v = ro,u,v,w,p,rk,reps; m = cells I-2S..I+S.  Adds 7 fluxes. */
static void roe_face_ke(const double q[7][4], const double *nrm, double area, int intem, int intet,
                        const ff_params *p, double c_r, double c_l, const double *cr,
                        const double *cl2, const double *dd, double *f7) {
  double roip, roim, rmip, rmim, rnip, rnim, rwip, rwim, ppi, pmi, rkip, rkim, reip, reim;
  xxm(q[0], dd, intem, &roip, &roim);
  xxm(q[1], dd, intem, &rmip, &rmim);
  xxm(q[2], dd, intem, &rnip, &rnim);
  xxm(q[3], dd, intem, &rwip, &rwim);
  xxm(q[4], dd, intem, &ppi, &pmi);
  /* XXTRAA takes INTEM for k and omega too (base3c.f:4861-4862) */
  xxm(q[5], dd, dd ? intem : intet, &rkip, &rkim);
  xxm(q[6], dd, dd ? intem : intet, &reip, &reim);
  roip = MAXD(0.001 * p->frsden, roip);
  ppi = MAXD(0.001 * p->frspre, ppi);
  roim = MAXD(0.001 * p->frsden, roim);
  pmi = MAXD(0.001 * p->frspre, pmi);
  const double gm1 = p->gamma - 1.;
  double eip = (ppi + 0.) / (gm1 * roip) - p->e0ref;
  double eim = (pmi + 0.) / (gm1 * roim) - p->e0ref;
  double elr = (ppi + 0.) / (gm1 * roim) - p->e0ref;
  double erl = (pmi + 0.) / (gm1 * roip) - p->e0ref;
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
  double rkipi = MAXD(0.001 * p->rklim, rkip), reipi = MAXD(0.001 * p->epslim, reip);
  double rkimi = MAXD(0.001 * p->rklim, rkim), reimi = MAXD(0.001 * p->epslim, reim);
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
  double alfa7 = rohat * (epsr - epsl);
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
  double rl4 = rl3, rl5 = rl3, rl6 = rl3, rl7 = rl3;
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
  double f6 = .5 * area * (roucr * rkr + roucl * rkl - damp * rkhat - rl6 * alfa6);
  double f7v = .5 * area * (roucr * epsr + roucl * epsl - damp * epshat - rl7 * alfa7);
  double f2pm = a11 * f2 + a21 * f3 + a31 * f4;
  double f3pm = a12 * f2 + a22 * f3 + a32 * f4;
  double f4pm = a13 * f2 + a23 * f3 + a33 * f4;
  f7[0] = f1 + f7[0];
  f7[1] = f2pm + f7[1];
  f7[2] = f3pm + f7[2];
  f7[3] = f4pm + f7[3];
  f7[4] = f5v + f7[4];
  f7[5] = f6 + f7[5];
  f7[6] = f7v + f7[6];
}

/* BOTSKE base3c.f:6147-6760 wall face with k and omega (IDIS=2: RM1=RC1,
 * PSIGK=PSIGK1, PSIGE=PSIGE1, ROMFAC=1, XAUX1=1; smooth wall RBK=0):
 * the laminar wall flux plus F6V (k) and F7V (omega, from the surface value
 * OMSURF), and F6V added to the energy flux. */
static void botske_face_ke(const orc_block *b, const ff_params *p, size_t II, int S, int idir,
                           int dir, int iheat, int intem, double *F) {
  const double *A = b->a[FF_A1 + 4 * (dir - 1)], *NX = b->a[FF_A1XA + 4 * (dir - 1)];
  const double *NY = b->a[FF_A1YA + 4 * (dir - 1)], *NZ = b->a[FF_A1ZA + 4 * (dir - 1)];
  const double *VOL = b->a[FF_VOL], *VIS = b->a[FF_VIS], *CH = b->a[FF_CH], *P = b->a[FF_P];
  const double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *T = b->a[FF_TEMP];
  const double *RO = b->a[FF_RO], *RK = b->a[FF_RK], *REPS = b->a[FF_REPS], *ST = b->a[FF_STRAIN];
  double rc1 = 1.5, rc2 = rc1 - 1.;
  if (intem == 6) { rc1 = 1.; rc2 = 0.; }
  const double prs = p->pr / p->prt, ymr = .166666667, eps = 1.e-3;
  int lstrid = S * idir;
  size_t II2 = II + lstrid;
  size_t IF1 = idir == 1 ? II : II + S;
  int ihfl = (iheat == 2 || iheat >= 12) ? 1 : 0;
  int iht = (iheat == 0 || iheat == 15) ? 0 : 1;
  double vislim = 0.01 * p->frsvis;
  double rolim = 0.001 * p->frsden;
  double dist = (A[IF1] + A[IF1 + lstrid]) / VOL[II];
  double surg = -dist * ymr;
  double eps2b = 1., vistb = 0.;
  double visb = MAXD(vislim, rc1 * VIS[II] - rc2 * VIS[II2]);
  double chsb = MAXD(eps, rc1 * CH[II] - rc2 * CH[II2]);
  double straib = MAXD(eps, rc1 * ST[II] - rc2 * ST[II2]);
  double pb1 = MAXD(0.01 * p->frspre, rc1 * P[II] - rc2 * P[II2]);
  double rob = MAXD(rolim, rc1 * RO[II] - rc2 * RO[II2]);
  double surf = surg * eps2b * visb;
  double surfe = surg * (prs * vistb / visb + 1.) * chsb;
  double rapub = MAXD(1.0E-20, eps2b - 1.0);
  double surfrk = surg * (1.0 + SST_SIGRK1 * rapub) * visb;
  double surfep = surg * (1.0 + SST_SIGOM1 * rapub) * visb;
  double ypro1 = 1. / RO[II], ypro2 = 1. / RO[II2];
  double rksurf = 0.0;
  /* surface value of omega (smooth wall: SKPLUS = SKPMIN) */
  double rnub = visb / rob;
  double utau2 = rnub * straib;
  double plusfc = sqrt(utau2) / rnub;
  double yplus1 = 2.0 * plusfc / dist;
  double skpmin = MIND(2.4 * pow(yplus1, 0.85), 8.0);
  skpmin = MAXD(skpmin, 1.e-3);
  double skplus = MAXD(0.0 * plusfc, skpmin);
  double pskp = 1.0 / skplus;
  double sr1 = 2500.0 * pskp * pskp, sr2 = 100.0 * pskp;
  double srcoef = MAXD(sr1, sr2);
  double omsurf = straib * srcoef;
  double epsurf = 1.0 * omsurf + 0.0 * 0.0;
  double tempb = MAXD(0.01 * p->frstem, rc1 * T[II] - rc2 * T[II2]);
  double tsurf = p->frstem;
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
  double evii = idir * (9.0 * REPS[II] * ypro1 - 1.0 * REPS[II2] * ypro2 - 8. * epsurf);
  double rkii = idir * (9.000 * RK[II] * ypro1 - 1.000 * RK[II2] * ypro2 - 8. * rksurf);
  rkii = idir * MAXD(idir * rkii, 0.0);
  double f6v = surfrk * rkii * MAXD(1.0, 1.0);
  double f7v = surfep * evii * MAXD(1.0, 1.0);
  F[0] = 0.;
  F[1] = A[IF1] * (ax * pb + f2v);
  F[2] = A[IF1] * (ay * pb + f3v);
  F[3] = A[IF1] * (az * pb + f4v);
  F[4] = A[IF1] * (0. * pb1 + f5v + f6v);
  F[5] = A[IF1] * f6v;
  F[6] = A[IF1] * f7v;
}

/* FLXCYC res3c.f:6424 for one direction on level 1 (FULLNS): face fluxes of
 * the five flow equations and k, omega into F1R..F1E, F1RK, F1EPS. */
void orc_flux_dir_sst(orc_block *b, const ff_params *p, int dir) {
  dims_t d = dims_of(b);
  int S = dir == 1 ? 1 : (dir == 2 ? d.is : d.il);
  int nmax = dir == 1 ? d.imax : (dir == 2 ? d.jmax : d.kmax);
  int intem = dir == 1 ? p->interi : (dir == 2 ? p->interj : p->interk);
  int intet = (intem > -5 && intem < 5) ? 1 : intem;          /* res3c.f:3641-3647 */
  double *F[7] = {b->a[FF_F1R], b->a[FF_F1RM], b->a[FF_F1RN], b->a[FF_F1RW], b->a[FF_F1E],
                  b->a[FF_F1RK], b->a[FF_F1EPS]};
  for (int v = 0; v < 7; v++) memset(F[v], 0, sizeof(double) * d.ntot);
  const double *A = b->a[FF_A1 + 4 * (dir - 1)], *NX = b->a[FF_A1XA + 4 * (dir - 1)];
  const double *NY = b->a[FF_A1YA + 4 * (dir - 1)], *NZ = b->a[FF_A1ZA + 4 * (dir - 1)];
  const double *RO = b->a[FF_RO], *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W];
  const double *P = b->a[FF_P], *C = b->a[FF_C], *DRDP = b->a[FF_DRDP], *DRDH = b->a[FF_DRDH];
  const double *RK = b->a[FF_RK], *REPS = b->a[FF_REPS];
  int t1max = dir == 1 ? d.jmax : d.imax, t2max = dir == 3 ? d.jmax : d.kmax;
  int idi = dir == 1 ? p->idi1 : (dir == 2 ? p->idi2 : p->idi3);
  for (int t2 = 1; t2 <= t2max; t2++)
    for (int t1 = 1; t1 <= t1max; t1++)
      for (int m = 1; m <= nmax + 1; m++) {
        size_t L = dir == 1 ? IX(d, m, t1, t2) : (dir == 2 ? IX(d, t1, m, t2) : IX(d, t1, t2, m));
        double f[7] = {0, 0, 0, 0, 0, 0, 0};
        if (m <= MIND(idi, nmax + 1)) {
          double frk, feps, fv[5];
          flkebl_face(b, L, S, dir, &frk, &feps);
          f[5] = frk; f[6] = feps;
          f[4] = frk;                                   /* FE = FRK, SETV12 */
          fluxbl_face(b, p, L, S, dir, fv);
          f[0] = 0.; f[1] = fv[1]; f[2] = fv[2]; f[3] = fv[3];
          f[4] = f[4] + fv[4];                          /* FE = FE - F5VIB */
        }
        double q[7][4];
        const double *arr[7] = {RO, U, V, W, P, RK, REPS};
        for (int v = 0; v < 7; v++) {
          q[v][0] = arr[v][L - 2 * S]; q[v][1] = arr[v][L - S];
          q[v][2] = arr[v][L]; q[v][3] = arr[v][L + S];
        }
        double nrm[3] = {NX[L], NY[L], NZ[L]};
        double cr[5] = {C[L], DRDP[L], DRDH[L], RO[L], P[L]};
        size_t L2 = dir == 3 ? L : L - S;
        double cl[5] = {C[L2], DRDP[L2], DRDH[L2], RO[L2], P[L2]};
        if (p->flux != FF_FLUX_ROE) alt_face(b, p, dir, L, S, intem, intet, 7, f);   /* IFLUX 7, 8 */
        else {
          double dd[4];
          roe_face_ke(q, nrm, A[L], intem, intet, p, C[L], C[L - S], cr, cl, stencil_d(b, p, dir, L, S, dd), f);
          if (p->rjk2 > 0. || p->rjk4 > 0.) jst_face(b, p, L, S, f);   /* res3c.f:6955 */
        }
        for (int v = 0; v < 7; v++) F[v][L] = f[v];
      }
  for (int ip = 0; ip < b->npatch; ip++) {
    const ff_patch *pa = &b->patch[ip];
    if (pa->ityp < 8 || pa->ityp > 10) continue;
    face_t f = face_geom(&d, pa->iface);
    if (f.dir != dir) continue;
    for (int bb = pa->r2a; bb <= pa->r2b; bb++)
      for (int a = pa->r1a; a <= pa->r1b; a++) {
        size_t II = face_cell(&d, &f, a, bb);
        double fw[7];
        botske_face_ke(b, p, II, S, f.idir, dir, pa->iheat, intem, fw);
        size_t IF1 = f.idir == 1 ? II : II + S;
        for (int v = 0; v < 7; v++) F[v][IF1] = fw[v];
      }
  }
}

/* SWEEPK res3c.f:1342: like SWEEP for the seven equations. */
static void sweepk(orc_block *b, int dir, int ido) {
  dims_t d = dims_of(b);
  int S = dir == 1 ? 1 : (dir == 2 ? d.is : d.il);
  double *D[7] = {b->a[FF_DRO], b->a[FF_DM], b->a[FF_DN], b->a[FF_DW], b->a[FF_DE], b->a[FF_DRK], b->a[FF_DEPS]};
  double *F[7] = {b->a[FF_F1R], b->a[FF_F1RM], b->a[FF_F1RN], b->a[FF_F1RW], b->a[FF_F1E],
                  b->a[FF_F1RK], b->a[FF_F1EPS]};
  const double *VOL = b->a[FF_VOL];
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t n = IX(d, I, J, K);
        if (ido == 0) {
          for (int v = 0; v < 7; v++) D[v][n] = D[v][n] - (F[v][n + S] - F[v][n]);
        } else {
          double dt1 = 1. / VOL[n];
          for (int v = 0; v < 7; v++) D[v][n] = (D[v][n] - (F[v][n + S] - F[v][n])) * dt1;
        }
      }
}

/* SOURKO turb3.f:7624 (KOVER=0, RANS, no rotation correction, TRANSL and
 * TUR_FRS_SOURCE false) into SRK, SEPS; SEPS holds the cross diffusion on
 * entry.  Then ADDSKE res3c.f:1473. */
static void sourko_addske(orc_block *b) {
  dims_t d = dims_of(b);
  const double *PTUR = b->a[FF_PTUR], *EPS2 = b->a[FF_EPS2], *VIS = b->a[FF_VIS], *RO = b->a[FF_RO];
  const double *RK = b->a[FF_RK], *ROM = b->a[FF_REPS], *FUN1 = b->a[FF_FUN1];
  double *SRK = b->a[FF_SRK], *SOM = b->a[FF_SEPS], *DRK = b->a[FF_DRK], *DEPS = b->a[FF_DEPS];
  const double pbstar = 1.0 / SST_BSTAR, persbs = 1.0 / sqrt(SST_BSTAR), eps = 1.0E-10;
  const double rotco = 0.0;
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t L = IX(d, I, J, K);
        double onemf1 = MAXD(0.0, (1.0 - FUN1[L]));
        double beta = FUN1[L] * SST_BETA1 + onemf1 * SST_BETA2;
        double sigom = FUN1[L] * SST_SIGOM1 + onemf1 * SST_SIGOM2;
        double gamkom = beta * pbstar - sigom * (SST_CKAPPA * SST_CKAPPA) * persbs;
        double rmutrb = MAXD(eps, EPS2[L] - 1.0) * VIS[L];
        double fco = MAXD(0.0, (1.0 - rotco)) + MAXD(0.0, rotco / (1.0 + 3.6 * 0.0));
        double trueomega = ROM[L];
        double prol = 1.0 / RO[L];
        SOM[L] = onemf1 * SOM[L];
        SRK[L] = PTUR[L] - SST_BSTAR * RK[L] * trueomega * prol;
        double omepro = gamkom * RO[L] * PTUR[L] / (rmutrb * ROM[L]);
        double omedis = fco * beta * prol * trueomega;
        SOM[L] = SOM[L] + ROM[L] * (omepro - omedis);
      }
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t n = IX(d, I, J, K);
        DRK[n] = DRK[n] + SRK[n];
        DEPS[n] = DEPS[n] + SOM[n];
      }
}

/* FLUDKE base3c.f:5547: thin-layer k and omega diffusion of one face
 * (coarse levels, or FULLNS off). */
static void fludke_face(const orc_block *b, size_t I, int S, int dir, double *frk, double *feps) {
  const double *A = b->a[FF_A1 + 4 * (dir - 1)], *VOL = b->a[FF_VOL], *FUN1 = b->a[FF_FUN1];
  const double *VIS = b->a[FF_VIS], *EPS2 = b->a[FF_EPS2], *RO = b->a[FF_RO];
  const double *RK = b->a[FF_RK], *REPS = b->a[FF_REPS];
  size_t M = I - S;
  double onemf1 = MAXD(0.0, (1.0 - FUN1[I]));
  double psigk = FUN1[I] * SST_SIGRK1 + onemf1 * SST_SIGRK2;
  double psige = FUN1[I] * SST_SIGOM1 + onemf1 * SST_SIGOM2;
  double ypd2 = A[I] / (VOL[I] + VOL[M]);
  double surg = -A[I] * ypd2;
  double rmut2 = (EPS2[I] - 1.) * VIS[I] + (EPS2[M] - 1.) * VIS[M];
  double surfk = surg * (VIS[I] + VIS[M] + rmut2 * psigk);
  double surfep = surg * (VIS[I] + VIS[M] + rmut2 * psige);
  double ypro1 = 1. / RO[I], ypro2 = 1. / RO[M];
  *frk = surfk * (RK[I] * ypro1 - RK[M] * ypro2);
  *feps = surfep * (REPS[I] * ypro1 - REPS[M] * ypro2);
}

/* FLXCYC on a coarse level (M > 1): FLUDKE + FLUXDO, first-order Roe
 * (INTERI/J/K = INTET = 55), BOTSKE walls; no inlet/outlet update. */
static void flux_dir_sst_coarse(orc_block *b, const ff_params *p, int dir) {
  dims_t d = dims_of(b);
  int S = dir == 1 ? 1 : (dir == 2 ? d.is : d.il);
  int nmax = dir == 1 ? d.imax : (dir == 2 ? d.jmax : d.kmax);
  int intem = p->coarse_inter, intet = (intem > -5 && intem < 5) ? 1 : intem;
  double *F[7] = {b->a[FF_F1R], b->a[FF_F1RM], b->a[FF_F1RN], b->a[FF_F1RW], b->a[FF_F1E],
                  b->a[FF_F1RK], b->a[FF_F1EPS]};
  for (int v = 0; v < 7; v++) memset(F[v], 0, sizeof(double) * d.ntot);
  const double *A = b->a[FF_A1 + 4 * (dir - 1)], *NX = b->a[FF_A1XA + 4 * (dir - 1)];
  const double *NY = b->a[FF_A1YA + 4 * (dir - 1)], *NZ = b->a[FF_A1ZA + 4 * (dir - 1)];
  const double *RO = b->a[FF_RO], *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W];
  const double *P = b->a[FF_P], *C = b->a[FF_C], *DRDP = b->a[FF_DRDP], *DRDH = b->a[FF_DRDH];
  const double *RK = b->a[FF_RK], *REPS = b->a[FF_REPS];
  int t1max = dir == 1 ? d.jmax : d.imax, t2max = dir == 3 ? d.jmax : d.kmax;
  int idi = dir == 1 ? p->idi1 : (dir == 2 ? p->idi2 : p->idi3);
  for (int t2 = 1; t2 <= t2max; t2++)
    for (int t1 = 1; t1 <= t1max; t1++)
      for (int m = 1; m <= nmax + 1; m++) {
        size_t L = dir == 1 ? IX(d, m, t1, t2) : (dir == 2 ? IX(d, t1, m, t2) : IX(d, t1, t2, m));
        double f[7] = {0, 0, 0, 0, 0, 0, 0};
        if (m <= MIND(idi, nmax + 1)) {
          double frk, feps, fv[5];
          fludke_face(b, L, S, dir, &frk, &feps);
          f[5] = frk; f[6] = feps;
          fluxdo_face_fe(b, p, L, S, dir, frk, fv);
          f[0] = 0.; f[1] = fv[1]; f[2] = fv[2]; f[3] = fv[3]; f[4] = fv[4];
        }
        double q[7][4];
        const double *arr[7] = {RO, U, V, W, P, RK, REPS};
        for (int v = 0; v < 7; v++) {
          q[v][0] = arr[v][L - 2 * S]; q[v][1] = arr[v][L - S];
          q[v][2] = arr[v][L]; q[v][3] = arr[v][L + S];
        }
        double nrm[3] = {NX[L], NY[L], NZ[L]};
        double cr[5] = {C[L], DRDP[L], DRDH[L], RO[L], P[L]};
        size_t L2 = dir == 3 ? L : L - S;
        double cl[5] = {C[L2], DRDP[L2], DRDH[L2], RO[L2], P[L2]};
        if (p->flux != FF_FLUX_ROE) alt_face(b, p, dir, L, S, intem, intet, 7, f);   /* IFLUX 7, 8 */
        else {
          double dd[4];
          roe_face_ke(q, nrm, A[L], intem, intet, p, C[L], C[L - S], cr, cl, stencil_d(b, p, dir, L, S, dd), f);
        }
        for (int v = 0; v < 7; v++) F[v][L] = f[v];
      }
  for (int ip = 0; ip < b->npatch; ip++) {
    const ff_patch *pa = &b->patch[ip];
    if (pa->ityp < 8 || pa->ityp > 10) continue;
    face_t f = face_geom(&d, pa->iface);
    if (f.dir != dir) continue;
    for (int bb = pa->r2a; bb <= pa->r2b; bb++)
      for (int a = pa->r1a; a <= pa->r1b; a++) {
        size_t II = face_cell(&d, &f, a, bb);
        double fw[7];
        botske_face_ke(b, p, II, S, f.idir, dir, pa->iheat, intem, fw);
        size_t IF1 = f.idir == 1 ? II : II + S;
        for (int v = 0; v < 7; v++) F[v][IF1] = fw[v];
      }
  }
}

/* RESIKE res3c.f:3423 for SST on level lev (1 = finest) with CYCLES at
 * multigrid depth m2: zero the increments and sources; for m2 >= 2 zero and
 * recompute the velocity gradients (DERFUN at this level); CROSKO + FUN1KO;
 * REFCEN on level 1; MAKE_EPS + PRODKE; TEMDER of T, k, omega; the k, i, j
 * direction cycles with SWEEPK; SOURKO + ADDSKE.  For m2 = 1 the velocity
 * gradients are the ones TURBEQ computed this cycle. */
void orc_residu_sst_lev(orc_block *b, const ff_params *p, int lev, int m2, int icycle) {
  dims_t d = dims_of(b);
  for (int s = FF_DRO; s <= FF_DEPS; s++) memset(b->a[s], 0, sizeof(double) * d.ntot);
  memset(b->a[FF_SRK], 0, sizeof(double) * d.ntot);
  memset(b->a[FF_FUN1], 0, sizeof(double) * d.ntot);
  if (lev == 1 && (p->rjk2 > 0. || p->rjk4 > 0.)) orc_scalard(b);   /* res3c.f:3599 */
  if (m2 >= 2) {
    static const int z[] = {FF_OHMI, FF_W12, FF_W13, FF_W23, FF_DTDX, FF_DTDY, FF_DTDZ, FF_DKDX, FF_DKDY,
                            FF_DKDZ, FF_DEDX, FF_DEDY, FF_DEDZ, FF_S11, FF_S12, FF_S13, FF_S22, FF_S23, FF_S33};
    for (size_t q = 0; q < sizeof(z) / sizeof(z[0]); q++) memset(b->a[z[q]], 0, sizeof(double) * d.ntot);
    orc_gradients(b, lev);
  }
  crosko(b);
  fun1ko(b, p);
  if (lev == 1) orc_refcen(b, p);
  double *tmp = calloc((size_t)d.ntot, sizeof(double));
  prodke(b, tmp);
  if (p->fullns) {
    temder_field(b, lev, b->a[FF_TEMP], b->a[FF_DTDX], b->a[FF_DTDY], b->a[FF_DTDZ]);
    for (int L = 0; L < d.ntot; L++) tmp[L] = b->a[FF_RK][L] / b->a[FF_RO][L];     /* DIVV12 */
    temder_field(b, lev, tmp, b->a[FF_DKDX], b->a[FF_DKDY], b->a[FF_DKDZ]);
    for (int L = 0; L < d.ntot; L++) tmp[L] = b->a[FF_REPS][L] / b->a[FF_RO][L];
    temder_field(b, lev, tmp, b->a[FF_DEDX], b->a[FF_DEDY], b->a[FF_DEDZ]);
  }
  free(tmp);
  const int order[3] = {3, 1, 2};
  for (int o = 0; o < 3; o++) {
    int dir = order[o];
    if (lev == 1) {
      orc_inlet_outlet(b, p, dir, icycle);
      orc_flux_dir_sst(b, p, dir);
    } else {
      flux_dir_sst_coarse(b, p, dir);
    }
    sweepk(b, dir, dir == 2);
  }
  sourko_addske(b);
  if (p->timel && lev == 1) orc_timder(b, p, 7);   /* TIMDER + TIMDKE, res3c.f:5097 */
}

void orc_residu_sst(orc_block *b, const ff_params *p, int icycle) {
  orc_residu_sst_lev(b, p, 1, 1, icycle);
}

/* LOCDTK imps3.f:807 (DTURB=1), IMSOKO imps3.f:972 and COPRKE imps3.f:1113
 * on the interior cells. */
static void locdtk_imsoko_coprke(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  double *DRO = b->a[FF_DRO], *DM = b->a[FF_DM], *DN = b->a[FF_DN], *DW = b->a[FF_DW], *DE = b->a[FF_DE];
  double *DRK = b->a[FF_DRK], *DEPS = b->a[FF_DEPS];
  const double *DTL = b->a[FF_DTL], *RO = b->a[FF_RO], *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W];
  const double *E = b->a[FF_E], *P = b->a[FF_P], *C = b->a[FF_C], *DRDP = b->a[FF_DRDP], *DRDH = b->a[FF_DRDH];
  const double *RK = b->a[FF_RK], *ROM = b->a[FF_REPS], *PTUR = b->a[FF_PTUR], *EPS2 = b->a[FF_EPS2];
  const double *VIS = b->a[FF_VIS];
  const double gamkom = SST_BETA1 / SST_BSTAR - SST_SIGOM1 * (SST_CKAPPA * SST_CKAPPA) / (sqrt(SST_BSTAR));
  const double ckmax = 1.0 / (2.0 * p->csimps), comax = 1.0 / (2.0 * p->csimps), eps = 1.0E-10;
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t i = IX(d, I, J, K);
        double dt1 = DTL[i];
        DRO[i] = dt1 * DRO[i]; DM[i] = dt1 * DM[i]; DN[i] = dt1 * DN[i];
        DW[i] = dt1 * DW[i]; DE[i] = dt1 * DE[i];
        DRK[i] = 1. * dt1 * DRK[i]; DEPS[i] = 1. * dt1 * DEPS[i];
      }
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t L = IX(d, I, J, K);
        double emeanf = E[L] - RK[L];
        double drkmax = MAXD(ckmax * MIND(RK[L], fabs(0.1 * emeanf - 0.9 * RK[L])), eps);
        double dommax = comax * ROM[L];
        double prol = 1. / RO[L];
        double atprod = fabs(PTUR[L]);
        double rnutrb = MAXD((EPS2[L] - 1.0), eps) * VIS[L] * prol;
        double drkden = 1.0 + DTL[L] * (atprod / drkmax + prol * SST_BSTAR * ROM[L]);
        double domden = 1.0 + DTL[L] * (gamkom * atprod / (rnutrb * dommax) + 2. * SST_BETA1 * ROM[L]);
        DRK[L] = DRK[L] / drkden;
        DEPS[L] = DEPS[L] / domden;
      }
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t i = IX(d, I, J, K);
        double vel2 = (U[i] * U[i] + V[i] * V[i] + W[i] * W[i]);
        double drodh = DRDH[i], drodp = DRDP[i];
        double ypro = 1. / RO[i], rki = RK[i] * ypro;
        double dri = DRO[i], dmi = DM[i], dni = DN[i], dwi = DW[i], dre = DE[i], dki = DRK[i];
        double dkin = U[i] * dmi + V[i] * dni + W[i] * dwi + dki;
        DM[i] = ypro * (-U[i] * DRO[i] + dmi);
        DN[i] = ypro * (-V[i] * DRO[i] + dni);
        DW[i] = ypro * (-W[i] * DRO[i] + dwi);
        DRK[i] = ypro * (-rki * DRO[i] + dki);
        DEPS[i] = ypro * (-ROM[i] * ypro * DRO[i] + DEPS[i]);
        double hi = ypro * (E[i] + P[i]);
        double dei = dre - (hi - vel2 - rki) * dri - dkin;
        double dpi = C[i] * C[i] * (dri - drodh * ypro * dei);
        double dhi = (dri - drodp * dpi) / drodh;
        DRO[i] = dhi;
        DE[i] = dpi;
        DE[i] = dpi + .667 * dki;
      }
}

/* SYIKE / SYM1KE imps4.f:982/1034 and the characteristic product of PRKEGS /
 * COKEGS (diag(l1,l2,l1,l1,l5,l1,l1)). */
static void jac_product_ke(double *out, const double *x, double rk, double c, double ro, double drdp,
                           double drdh, double nx, double ny, double nz, double l1, double l2, double l5) {
  double a21, a22, a23, a31, a32, a33;
  surfvects(nx, ny, nz, &a21, &a22, &a23, &a31, &a32, &a33);
  double z1 = x[0], z5 = x[4], z6 = x[5], z7 = x[6];
  double z2 = nx * x[1] + ny * x[2] + nz * x[3];
  double z3 = a21 * x[1] + a22 * x[2] + a23 * x[3];
  double z4 = a31 * x[1] + a32 * x[2] + a33 * x[3];
  double roc = ro * c, pc2 = 1. / ro, dpres = z5;
  double w1 = z1 - pc2 * dpres, w2 = roc * z2 + dpres, w3 = z3, w4 = z4, w6 = z6, w7 = z7;
  double w5 = -roc * z2 + dpres;
  w1 = l1 * w1; w2 = l2 * w2; w3 = l1 * w3; w4 = l1 * w4; w5 = l5 * w5; w6 = l1 * w6; w7 = l1 * w7;
  double ypro = 1. / ro, pc2b = .5 * ypro, proc = pc2b / c;
  double drh = .667 * rk * (ypro * ypro) * drdh;
  double ydrp = 1. / (1. + .667 * rk * ypro * drdp);
  double dh = w1 + pc2b * (w2 + w5);
  out[0] = dh;
  double x2i = proc * (w2 - w5), x3i = w3, x4i = w4;
  double x5 = .5 * (w2 + w5);
  out[4] = ydrp * (x5 - drh * ro * dh - .667 * ro * w6);
  out[5] = w6;
  out[6] = w7;
  out[1] = nx * x2i + a21 * x3i + a31 * x4i;
  out[2] = ny * x2i + a22 * x3i + a32 * x4i;
  out[3] = nz * x2i + a23 * x3i + a33 * x4i;
}

/* PRKEGS imps4.f:1462 (lower sweep, 7 equations).  Unlike PREDGS its row
 * buffer shift starts at MAX(IALKU-1,1) (imps4.f:1763), so the last j row
 * keeps its i+1 coupling. */
static void prkegs(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  const int IS = d.is, IL = d.il, IMAX = d.imax, JMAX = d.jmax, KMAX = d.kmax;
  double *D[7] = {b->a[FF_DRO], b->a[FF_DM], b->a[FF_DN], b->a[FF_DW], b->a[FF_DE], b->a[FF_DRK], b->a[FF_DEPS]};
  const double *VOL = b->a[FF_VOL], *DTL = b->a[FF_DTL];
  const double *A1 = b->a[FF_A1], *A2 = b->a[FF_A2], *A3 = b->a[FF_A3];
  const double *A1X = b->a[FF_A1XA], *A1Y = b->a[FF_A1YA], *A1Z = b->a[FF_A1ZA];
  const double *A2X = b->a[FF_A2XA], *A2Y = b->a[FF_A2YA], *A2Z = b->a[FF_A2ZA];
  const double *A3X = b->a[FF_A3XA], *A3Y = b->a[FF_A3YA], *A3Z = b->a[FF_A3ZA];
  const double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *C = b->a[FF_C], *RO = b->a[FF_RO];
  const double *VIS = b->a[FF_VIS], *VIST = b->a[FF_VIST], *RK = b->a[FF_RK];
  const double *DRDP = b->a[FF_DRDP], *DRDH = b->a[FF_DRDH];
  const int maw = JMAX * IS + 8;
  double *cd = calloc((size_t)7 * maw, sizeof(double));
  double *xi = calloc((size_t)3 * maw, sizeof(double)), *xj = calloc((size_t)3 * maw, sizeof(double));
  double *xk = calloc((size_t)3 * maw, sizeof(double)), *dt = calloc((size_t)maw, sizeof(double));
  double *scinv = calloc((size_t)maw, sizeof(double)), *scinp = calloc((size_t)maw, sizeof(double));
  double *yd = calloc((size_t)7 * (IMAX + 2), sizeof(double)), *bd = calloc((size_t)7 * (IMAX + 2), sizeof(double));
  const double cdiff = 2.;
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
        for (int v = 0; v < 7; v++) cd[7 * L + v] = -dt1 * A3[N + IL] * cd[7 * L + v] + VOL[N] * D[v][N];
        scinv[L] = 1. / (VOL[N] + dt1 * (xia * A1[N] + xja * A2[N] + xka * A3[N]) + VOL[N] * 0.);
        scinp[L] = 1. / (VOL[N] + dt1 * (rimax * A1[N] + rjmax * A2[N] + rkmax * A3[N]) + VOL[N] * 0.);
      }
    }
    for (int l = 0; l < 7 * (IMAX + 2); l++) { yd[l] = 0.; bd[l] = 0.; }
    for (int M = IMAX + JMAX; M >= 2; M--) {
      int ialku = MAXD(1, M - JMAX), iloppu = MIND(IMAX, M - 1);
      for (int I = ialku; I <= iloppu; I++) {
        int J = M - I;
        size_t N = kk + (size_t)(J + 1) * IS + (I + 1);
        int L = (J - 1) * IS + 2 + I;
        double dt1 = dt[L];
        for (int v = 0; v < 7; v++)
          cd[7 * L + v] = cd[7 * L + v] - dt1 * (A1[N + 1] * yd[7 * I + v] + A2[N + IS] * bd[7 * I + v]);
        for (int v = 0; v < 4; v++) cd[7 * L + v] = cd[7 * L + v] * scinv[L];
        cd[7 * L + 4] = cd[7 * L + 4] * scinp[L];
        cd[7 * L + 5] = cd[7 * L + 5] * scinv[L];
        cd[7 * L + 6] = cd[7 * L + 6] * scinv[L];
        double dw[7], out[7];
        for (int v = 0; v < 7; v++) { D[v][N] = cd[7 * L + v]; dw[v] = cd[7 * L + v]; }
        jac_product_ke(out, dw, RK[N], C[N], RO[N], DRDP[N], DRDH[N], A1X[N], A1Y[N], A1Z[N],
                       xi[3 * L], xi[3 * L + 1], xi[3 * L + 2]);
        for (int v = 0; v < 7; v++) yd[7 * I + v] = out[v];
        jac_product_ke(out, dw, RK[N], C[N], RO[N], DRDP[N], DRDH[N], A2X[N], A2Y[N], A2Z[N],
                       xj[3 * L], xj[3 * L + 1], xj[3 * L + 2]);
        for (int v = 0; v < 7; v++) bd[7 * I + v] = out[v];
      }
      for (int I = MAXD(ialku - 1, 1); I <= iloppu - 1; I++)
        for (int v = 0; v < 7; v++) yd[7 * I + v] = yd[7 * (I + 1) + v];
      for (int v = 0; v < 7; v++) yd[7 * iloppu + v] = 0.;
    }
    for (int l = 1; l <= JMAX * IS; l++) {
      size_t N = kk + l + 2 * IS - 1;
      double dw[7], out[7];
      for (int v = 0; v < 7; v++) dw[v] = D[v][N];
      jac_product_ke(out, dw, RK[N], C[N], RO[N], DRDP[N], DRDH[N], A3X[N], A3Y[N], A3Z[N],
                     xk[3 * l], xk[3 * l + 1], xk[3 * l + 2]);
      for (int v = 0; v < 7; v++) cd[7 * l + v] = out[v];
    }
  }
  free(cd); free(xi); free(xj); free(xk); free(dt); free(scinv); free(scinp); free(yd); free(bd);
}

/* DIKEGS imps4.f:1841 on the interior cells (7 equations). */
static void dikegs(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  const int IS = d.is, IL = d.il;
  double *D[7] = {b->a[FF_DRO], b->a[FF_DM], b->a[FF_DN], b->a[FF_DW], b->a[FF_DE], b->a[FF_DRK], b->a[FF_DEPS]};
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
        for (int v = 0; v < 7; v++) D[v][N] = D[v][N] * (1. + dt1 * scinv + 0.);
      }
}

/* COKEGS imps4.f:1078 (upper sweep, 7 equations), the CORRGS order. */
static void cokegs(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  const int IS = d.is, IL = d.il, IMAX = d.imax, JMAX = d.jmax, KMAX = d.kmax;
  double *D[7] = {b->a[FF_DRO], b->a[FF_DM], b->a[FF_DN], b->a[FF_DW], b->a[FF_DE], b->a[FF_DRK], b->a[FF_DEPS]};
  const double *VOL = b->a[FF_VOL], *DTL = b->a[FF_DTL];
  const double *A1 = b->a[FF_A1], *A2 = b->a[FF_A2], *A3 = b->a[FF_A3];
  const double *A1X = b->a[FF_A1XA], *A1Y = b->a[FF_A1YA], *A1Z = b->a[FF_A1ZA];
  const double *A2X = b->a[FF_A2XA], *A2Y = b->a[FF_A2YA], *A2Z = b->a[FF_A2ZA];
  const double *A3X = b->a[FF_A3XA], *A3Y = b->a[FF_A3YA], *A3Z = b->a[FF_A3ZA];
  const double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *C = b->a[FF_C], *RO = b->a[FF_RO];
  const double *VIS = b->a[FF_VIS], *VIST = b->a[FF_VIST], *RK = b->a[FF_RK];
  const double *DRDP = b->a[FF_DRDP], *DRDH = b->a[FF_DRDH];
  const int maw = JMAX * IS + 8;
  double *cd = calloc((size_t)7 * maw, sizeof(double));
  double *xi = calloc((size_t)3 * maw, sizeof(double)), *xj = calloc((size_t)3 * maw, sizeof(double));
  double *xk = calloc((size_t)3 * maw, sizeof(double)), *dt = calloc((size_t)maw, sizeof(double));
  double *scinv = calloc((size_t)maw, sizeof(double)), *scinp = calloc((size_t)maw, sizeof(double));
  double *yd = calloc((size_t)7 * (IMAX + 3), sizeof(double)), *bd = calloc((size_t)7 * (IMAX + 3), sizeof(double));
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
        for (int v = 0; v < 7; v++) cd[7 * L + v] = dt1 * A3[N] * cd[7 * L + v] + VOL[N] * D[v][N];
        scinv[L] = 1. / (VOL[N] + dt1 * (xia * A1[N + 1] + xja * A2[N + IS] + xka * A3[N + IL]) + VOL[N] * 0.);
        scinp[L] = 1. / (VOL[N] + dt1 * (rimax * A1[N] + rjmax * A2[N] + rkmax * A3[N]) + VOL[N] * 0.);
      }
    }
    for (int l = 0; l < 7 * (IMAX + 3); l++) { yd[l] = 0.; bd[l] = 0.; }
    for (int M = 2; M <= IMAX + JMAX; M++) {
      int ialku = MAXD(1, M - JMAX), iloppu = MIND(IMAX, M - 1);
      for (int I = ialku; I <= iloppu; I++) {
        int J = M - I;
        size_t N = kk + (size_t)(J + 1) * IS + (I + 1);
        int L = (J - 1) * IS + 2 + I;
        double dt1 = dt[L];
        for (int v = 0; v < 7; v++)
          cd[7 * L + v] = cd[7 * L + v] + dt1 * (A1[N] * yd[7 * I + v] + A2[N] * bd[7 * I + v]);
        for (int v = 0; v < 4; v++) cd[7 * L + v] = cd[7 * L + v] * scinv[L];
        cd[7 * L + 4] = cd[7 * L + 4] * scinp[L];
        cd[7 * L + 5] = cd[7 * L + 5] * scinv[L];
        cd[7 * L + 6] = cd[7 * L + 6] * scinv[L];
        double dw[7], out[7];
        for (int v = 0; v < 7; v++) { D[v][N] = cd[7 * L + v]; dw[v] = cd[7 * L + v]; }
        jac_product_ke(out, dw, RK[N], C[N], RO[N], DRDP[N], DRDH[N], A1X[N + 1], A1Y[N + 1], A1Z[N + 1],
                       xi[3 * L], xi[3 * L + 1], xi[3 * L + 2]);
        for (int v = 0; v < 7; v++) yd[7 * I + v] = out[v];
        jac_product_ke(out, dw, RK[N], C[N], RO[N], DRDP[N], DRDH[N], A2X[N + IS], A2Y[N + IS], A2Z[N + IS],
                       xj[3 * L], xj[3 * L + 1], xj[3 * L + 2]);
        for (int v = 0; v < 7; v++) bd[7 * I + v] = out[v];
      }
      for (int I = iloppu + 1; I >= MAXD(ialku + 1, 2); I--)
        for (int v = 0; v < 7; v++) yd[7 * I + v] = yd[7 * (I - 1) + v];
      for (int v = 0; v < 7; v++) yd[7 * ialku + v] = 0.;
    }
    for (int l = 1; l <= JMAX * IS; l++) {
      size_t N = kk + l + 2 * IS - 1;
      double dw[7], out[7];
      for (int v = 0; v < 7; v++) dw[v] = D[v][N];
      jac_product_ke(out, dw, RK[N], C[N], RO[N], DRDP[N], DRDH[N], A3X[N + IL], A3Y[N + IL], A3Z[N + IL],
                     xk[3 * l], xk[3 * l + 1], xk[3 * l + 2]);
      for (int v = 0; v < 7; v++) cd[7 * l + v] = out[v];
    }
  }
  free(cd); free(xi); free(xj); free(xk); free(dt); free(scinv); free(scinp); free(yd); free(bd);
}

/* IMPS imps3.f:6 for SST (JRIMP=0): TIME3, LOCDTK, IMSOKO, COPRKE, then
 * PRKEGS, DIKEGS, COKEGS (LUSGS=1) or the DDADI line sweeps (LUSGS=0), then
 * DRO/CP, DRK and DEPS times RO. */
void orc_imps_sst_lev(orc_block *b, const ff_params *p, int lev) {
  dims_t d = dims_of(b);
  orc_time3(b, p, lev == 1 ? p->cfl : p->cfll);
  locdtk_imsoko_coprke(b, p);
  if (p->ddadi) {   /* LUSGS=0: PREDKE, DIAGKE, CORRKE per direction */
    ddadi_sweeps(b, p, 7);
  } else {
    prkegs(b, p);
    dikegs(b, p);
    cokegs(b, p);
  }
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t n = IX(d, I, J, K);
        b->a[FF_DRO][n] = b->a[FF_DRO][n] / b->a[FF_CP][n];
        b->a[FF_DRK][n] = b->a[FF_DRK][n] * b->a[FF_RO][n];
        b->a[FF_DEPS][n] = b->a[FF_DEPS][n] * b->a[FF_RO][n];
      }
}

void orc_imps_sst(orc_block *b, const ff_params *p) { orc_imps_sst_lev(b, p, 1); }

/* FIN res3c.f:1077-1208 (ITURB>=3, single phase) and the CYCLES limits
 * (ns3c.f:1553-1596, LOLIM(REPS,EPSLIM) included). */
static void fin_sst_core(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  double *RK = b->a[FF_RK], *REPS = b->a[FF_REPS];
  for (int K = 1; K <= d.kmax; K++)
    for (int J = 1; J <= d.jmax; J++)
      for (int I = 1; I <= d.imax; I++) {
        size_t n = IX(d, I, J, K);
        b->a[FF_TEMP][n] = b->a[FF_TOLD][n] + b->a[FF_DRO][n];
        b->a[FF_U][n] = b->a[FF_UOLD][n] + b->a[FF_DM][n];
        b->a[FF_V][n] = b->a[FF_VOLD][n] + b->a[FF_DN][n];
        b->a[FF_W][n] = b->a[FF_WOLD][n] + b->a[FF_DW][n];
        b->a[FF_PDIFF][n] = b->a[FF_POLD][n] + b->a[FF_DE][n];
        double rkoldn = .45 * b->a[FF_RKOLD][n];
        double epoldn = .90 * b->a[FF_EPSOLD][n];
        double absdrk = fabs(b->a[FF_DRK][n]), absdep = fabs(b->a[FF_DEPS][n]);
        RK[n] = b->a[FF_RKOLD][n] + b->a[FF_DRK][n] / (1. + absdrk / rkoldn);
        REPS[n] = b->a[FF_EPSOLD][n] + b->a[FF_DEPS][n] / (1. + absdep / epoldn);
      }
  for (int n = 0; n < d.ntot; n++) RK[n] = MAXD(RK[n], p->rklim);
  for (int n = 0; n < d.ntot; n++) REPS[n] = MAXD(REPS[n], p->epslim);
}

void orc_fin_limits_sst(orc_block *b, const ff_params *p) {
  dims_t d = dims_of(b);
  double *REPS = b->a[FF_REPS];
  fin_sst_core(b, p);
  double *T = b->a[FF_TEMP], *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *PD = b->a[FF_PDIFF];
  double *P = b->a[FF_P];
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
  for (int n = 0; n < d.ntot; n++) P[n] = PD[n] + p->frspre;
  for (int n = 0; n < d.ntot; n++) REPS[n] = MAXD(REPS[n], p->epslim);
  for (int n = 0; n < d.ntot; n++) {
    double prelim = MIND(0., P[n] - 0.01 * p->frspre);
    P[n] = P[n] - prelim;
    PD[n] = PD[n] - prelim;
  }
}

/* SUBIN ns3c.f:9742 for SST: cap k (RKMAX = FRSDEN*REFVEL^2), the max |dp|
 * monitor and the *OLD copies including RKOLD, EPSOLD. */
void orc_subin_sst(orc_block *b, const ff_params *p, double *dromax) {
  dims_t d = dims_of(b);
  double rkmax = .5 * p->frsden * p->frsvel * p->frsvel * 2.;
  for (int L = 0; L < d.ntot; L++) {
    double *RK = b->a[FF_RK];
    RK[L] = MIND(RK[L], MAXD(0.1 * b->a[FF_E][L], rkmax));
    RK[L] = MIND(RK[L], rkmax);
  }
  orc_subin(b, dromax);
  memcpy(b->a[FF_RKOLD], b->a[FF_RK], sizeof(double) * d.ntot);
  memcpy(b->a[FF_EPSOLD], b->a[FF_REPS], sizeof(double) * d.ntot);
}

/* One single-grid SST cycle: STATIM, TURBEQ, RESIKE (+RESL2), IMPS, FIN +
 * limits, BOUNDI, SUBIN. */
void orc_cycle_sst(orc_block *b, const ff_params *p, int icycle, double *resi5, double *dromax) {
  orc_statim(b, p);
  orc_turbeq_sst(b, p);
  orc_residu_sst(b, p, icycle);
  orc_resl2(b, resi5);
  orc_imps_sst(b, p);
  orc_fin_limits_sst(b, p);
  orc_boundi(b, p);
  orc_subin_sst(b, p, dromax);
}

/* ---- multigrid with k and omega (CYCLES ns3c.f:1607-2120) -------------- */

/* TRANKE multi.f:434: restriction of RK, REPS (into RO2/RM2), EPS2, VIST and
 * of DRK, DEPS into the forcing RKP2H/EPP2H over coarse cells 0..MAX+1, the
 * interior RKOLD/EPSOLD copies and the ghost rings (same order as TRANSF). */
void orc_tranke(orc_block *f, orc_block *c) {
  dims_t df = dims_of(f), dc = dims_of(c);
  static const int vs[4] = {FF_RK, FF_REPS, FF_EPS2, FF_VIST};
  static const int rs[2] = {FF_DRK, FF_DEPS};
  static const int ps[2] = {FF_RKP2H, FF_EPP2H};
  const double *VOL = f->a[FF_VOL], *VOL2 = c->a[FF_VOL];
  int kind = df.kmax == 1 ? 1 : 2;
  for (int K = 0; K <= dc.kmax + 1; K++)
    for (int J = 0; J <= dc.jmax + 1; J++)
      for (int I = 0; I <= dc.imax + 1; I++) {
        size_t N = IX(dc, I, J, K);
        size_t ijk = IX(df, 2 * I - 1, 2 * J - 1, kind * K - kind + 1);
        size_t imjm2 = df.kmax == 1 ? 0 : df.il;
        size_t ipjk = ijk + 1, ijpk = ijk + df.is, ipjpk = ijk + df.is + 1;
        size_t ijkp = ijk + imjm2, ipjpkp = ipjpk + imjm2, ijpkp = ijpk + imjm2, ipjkp = ipjk + imjm2;
        double pvol = 1. / VOL2[N];
#define R8(X) ((VOL[ipjpk] * X[ipjpk] + VOL[ijk] * X[ijk] + VOL[ipjk] * X[ipjk] + VOL[ijpk] * X[ijpk] + \
                VOL[ipjpkp] * X[ipjpkp] + VOL[ijkp] * X[ijkp] + VOL[ipjkp] * X[ipjkp] + VOL[ijpkp] * X[ijpkp]) * pvol)
        for (int v = 0; v < 4; v++) c->a[vs[v]][N] = R8(f->a[vs[v]]);
        for (int v = 0; v < 2; v++) c->a[ps[v]][N] = R8(f->a[rs[v]]);
#undef R8
      }
  for (int K = 1; K <= dc.kmax; K++)
    for (int J = 1; J <= dc.jmax; J++)
      for (int I = 1; I <= dc.imax; I++) {
        size_t N = IX(dc, I, J, K);
        c->a[FF_RKOLD][N] = c->a[FF_RK][N];
        c->a[FF_EPSOLD][N] = c->a[FF_REPS][N];
      }
#define RING(N0, OFF)                                                            \
  do {                                                                           \
    size_t n0 = (N0);                                                            \
    for (int v = 0; v < 2; v++) { c->a[ps[v]][n0] = 0.; c->a[ps[v]][n0 + (OFF)] = 0.; } \
    for (int v = 0; v < 4; v++) c->a[vs[v]][n0 + (OFF)] = c->a[vs[v]][n0];       \
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

/* FORCFU / ADDRES multi.f:1609/1686 for k and omega (ITURB>=3 branch). */
void orc_forcfu_ke(orc_block *c) {
  dims_t d = dims_of(c);
  orc_forcfu(c);
  for (int n = 0; n < d.ntot; n++) c->a[FF_RKP2H][n] = c->a[FF_RKP2H][n] - c->a[FF_DRK][n];
  for (int n = 0; n < d.ntot; n++) c->a[FF_EPP2H][n] = c->a[FF_EPP2H][n] - c->a[FF_DEPS][n];
}

void orc_addres_ke(orc_block *c) {
  dims_t d = dims_of(c);
  orc_addres(c);
  for (int n = 0; n < d.ntot; n++) c->a[FF_DRK][n] = c->a[FF_RKP2H][n] + c->a[FF_DRK][n];
  for (int n = 0; n < d.ntot; n++) c->a[FF_DEPS][n] = c->a[FF_EPP2H][n] + c->a[FF_DEPS][n];
}

/* INTERT multi.f:2051 -> INTERO 2007: damped injection of the coarse k and
 * omega corrections, RO += CC1*RO*DROK/(CC2*RO + |DROK|). */
void orc_intert(orc_block *c, orc_block *f, const ff_params *pf) {
  dims_t dc = dims_of(c), df = dims_of(f);
  const int ss[2] = {FF_RK, FF_REPS}, so[2] = {FF_RKOLD, FF_EPSOLD};
  const double cc[2] = {pf->cmgk, pf->cmgeps};
  for (int q = 0; q < 2; q++) {
    const double cc1 = cc[q], cc2 = cc1 + 1.E-7;
    for (int K = 1; K <= df.kmax; K++)
      for (int J = 1; J <= df.jmax; J++)
        for (int I = 1; I <= df.imax; I++) {
          size_t N = IX(dc, (I + 1) / 2, (J + 1) / 2, (K + 1) / 2), F = IX(df, I, J, K);
          double drok = c->a[ss[q]][N] - c->a[so[q]][N];
          double alpo = fabs(drok);
          double *R = f->a[ss[q]];
          R[F] = R[F] + cc1 * R[F] * drok / (cc2 * R[F] + alpo);
        }
  }
}

/* Coarse-level FIN (ns3c.f:1935-1990): FIN with k and omega, then UPLIM /
 * LOLIM of T and LOLIMP (no PDTOP, as there). */
void orc_fin_coarse_sst(orc_block *b, const ff_params *p) {
  fin_sst_core(b, p);
  temp_p_limits(b, p);
}

/* One multigrid SST cycle of CYCLES (same order as orc_mg_cycle). */
/* The per-block part of the k-omega multigrid cycle (see orc_mg_body). */
void orc_mg_body_sst(orc_block **lv, int nlev, const ff_params *prm, int icycle, double *resi5) {
  orc_block *b = lv[0];
  orc_statim(b, &prm[0]);
  orc_turbeq_sst(b, &prm[0]);
  orc_residu_sst_lev(b, &prm[0], 1, 1, icycle);
  orc_resl2(b, resi5);
  orc_imps_sst_lev(b, &prm[0], 1);
  orc_fin_limits_sst(b, &prm[0]);
  for (int m = 1; m < nlev; m++) {
    orc_block *f = lv[m - 1], *c = lv[m];
    orc_statim(f, &prm[m - 1]);
    orc_residu_sst_lev(f, &prm[m - 1], m, m + 1, icycle);
    if (m == 1) orc_resl2(f, resi5);
    if (m > 1) orc_addres_ke(f);
    orc_transf(f, c);
    orc_tranke(f, c);
    orc_statim(c, &prm[m]);
    orc_residu_sst_lev(c, &prm[m], m + 1, m + 1, icycle);
    orc_forcfu_ke(c);
    orc_addres_ke(c);
    orc_imps_sst_lev(c, &prm[m], m + 1);
    orc_fin_coarse_sst(c, &prm[m]);
  }
  for (int m = nlev - 1; m >= 1; m--) orc_interp_limits(lv[m], lv[m - 1], &prm[m - 1]);
  reflec(b, &prm[0]);
}

void orc_mg_cycle_sst(orc_block **lv, int nlev, const ff_params *prm, int icycle, double *resi5, double *dromax) {
  orc_mg_body_sst(lv, nlev, prm, icycle, resi5);
  orc_boundi(lv[0], &prm[0]);
  orc_subin_sst(lv[0], &prm[0], dromax);
}
