/*
 * CPU oracle (test infrastructure): the inviscid face fluxes that IFLUX
 * selects besides Roe's (FLUXKE) and van Leer's (FLUXVL, vl_face), one face
 * at a time, restated from the reference in its own order of operations:
 *
 *   FLUXWP  base3c.f:1967-2195  IFLUX = 2  wave/particle splitting (laminar)
 *   FLUXAU  base3c.f:2201-2466  IFLUX = 3  AUSM form of WPS (laminar)
 *   FLUXKT  base3c.f:4403-4747  IFLUX = 7  Kurganov-Tadmor central upwind
 *   FLUCUSP base3c.f:5133-5540  IFLUX = 8  H-CUSP
 *
 * FLUCYC (res3c.f:7890-7990) calls all four for a laminar block with k and
 * omega zero (RKLIM = EPSLIM = 0, res3c.f:7680); RESIKE (res3c.f:7017-7036)
 * calls FLUXKT and FLUCUSP with the k-omega variables.  nv = 5 is the
 * laminar form (the k and omega entries of q are not read), nv = 7 the
 * two-equation one.  Perfect gas (ISTATE = 1), no grid rotation (UROT = 0),
 * XXTRAP, or XXTRAA for KT and H-CUSP when XXTRAL is set (FLUXVL, FLUXWP
 * and FLUXAU have no XXTRAL branch), no transition model.
 *
 * Included by finflo_oracle.c (uses its xxtrap and surfvects).
 */

/* The MUSCL pair of one variable: q[0..3] = cells I-2S, I-S, I, I+S. */
static void xx4(const double *q, int intem, double *ip, double *im) {
  xxtrap(q[0], q[1], q[2], q[3], intem, ip, im);
}

/* XXTRAL: the extents D1/D2/D3 (the face direction's) of cells L-2S..L+S
 * into dd, returned for XXTRAA; NULL (XXTRAP) when XXTRAL is off. */
static const double *stencil_d(const orc_block *b, const ff_params *p, int dir, size_t L, int S, double *dd) {
  if (!p->xxtral) return NULL;
  const double *D = b->a[FF_D1 + dir - 1];
  for (int m = 0; m < 4; m++) dd[m] = D[L + (m - 2) * S];
  return dd;
}

/* FLUXAU base3c.f:2201-2466 (IFLUX = 3) at one face.  q[v][m]: v = RO, U,
 * V, W, P, PDIFF.  c_r = C(I), c_l = C(I-IL).  Adds 5 components to f. */
static void ausm_face(const double q[6][4], const double *nrm, double area, int intem, const ff_params *p,
                      double c_r, double c_l, double *f) {
  double roip, roim, uip, uim, vip, vim, wip, wim, ppi, pmi, pdpi, pdmi;
  xx4(q[0], intem, &roip, &roim);
  xx4(q[1], intem, &uip, &uim);
  xx4(q[2], intem, &vip, &vim);
  xx4(q[3], intem, &wip, &wim);
  xx4(q[4], intem, &ppi, &pmi);
  xx4(q[5], intem, &pdpi, &pdmi);
  roip = MAXD(0.001 * p->frsden, roip);
  ppi = MAXD(0.001 * p->frspre, ppi);
  roim = MAXD(0.001 * p->frsden, roim);
  pmi = MAXD(0.001 * p->frspre, pmi);
  pdpi = MAXD(-0.999 * p->frspre, pdpi);
  pdmi = MAXD(-0.999 * p->frspre, pdmi);
  const double gm1 = p->gamma - 1.;
  double eip = (ppi + 0.) / (gm1 * roip) - p->e0ref;   /* EFPRO state.f:620, FRSPRE = 0 */
  double eim = (pmi + 0.) / (gm1 * roim) - p->e0ref;
  double a11 = nrm[0], a12 = nrm[1], a13 = nrm[2], a21, a22, a23, a31, a32, a33;
  surfvects(a11, a12, a13, &a21, &a22, &a23, &a31, &a32, &a33);
  double ur = a11 * uip + a12 * vip + a13 * wip;
  double vr = a21 * uip + a22 * vip + a23 * wip;
  double wr = a31 * uip + a32 * vip + a33 * wip;
  double ul = a11 * uim + a12 * vim + a13 * wim;
  double vl = a21 * uim + a22 * vim + a23 * wim;
  double wl = a31 * uim + a32 * vim + a33 * wim;
  const double uc = 0.;
  double eir = eip + .5 * (ur * ur + vr * vr + wr * wr);
  double eil = eim + .5 * (ul * ul + vl * vl + wl * wl);
  double pdr = pdpi, cr = c_r, rmaip = (ur - uc) / cr, rmar;
  if (fabs(rmaip) <= 1.) {
    double h = .5 * (rmaip - 1.);
    rmar = -(h * h);
    pdr = pdr * .50 * ((rmaip - 1.) * (rmaip - 1.)) * (2. + rmaip);
  } else {
    rmar = .5 * (rmaip - fabs(rmaip));
    pdr = pdr * (rmaip - fabs(rmaip)) / rmaip;
  }
  double pdl = pdmi, cl = c_l, rmaim = (ul - uc) / cl, rmal;
  if (fabs(rmaim) <= 1.) {
    double h = .5 * (rmaim + 1.);
    rmal = h * h;
    pdl = pdl * .50 * ((rmaim + 1.) * (rmaim + 1.)) * (2. - rmaim);
  } else {
    rmal = .5 * (rmaim + fabs(rmaim));
    pdl = pdl * (rmaim + fabs(rmaim)) / rmaim;
  }
  double rma = rmar + rmal, absrma = fabs(rma);
  double roucr = roip * cr, roucl = roim * cl;
  double rouur = roucr * ur, rouul = roucl * ul, rouvr = roucr * vr, rouvl = roucl * vl;
  double rouwr = roucr * wr, rouwl = roucl * wl, rouer = roucr * eir, rouel = roucl * eil;
  double f1 = .5 * area * (rma * (roucr + roucl) - absrma * (roucr - roucl));
  double f2 = .5 * area * (rma * (rouur + rouul) - absrma * (rouur - rouul) + pdr + pdl);
  double f3 = .5 * area * (rma * (rouvr + rouvl) - absrma * (rouvr - rouvl));
  double f4 = .5 * area * (rma * (rouwr + rouwl) - absrma * (rouwr - rouwl));
  double f5 = .5 * area * (rma * (rouer + rouel) - absrma * (rouer - rouel) + pdpi * ur + pdmi * ul);
  double f2pm = a11 * f2 + a21 * f3 + a31 * f4;
  double f3pm = a12 * f2 + a22 * f3 + a32 * f4;
  double f4pm = a13 * f2 + a23 * f3 + a33 * f4;
  f[0] = f1 + f[0];
  f[1] = f2pm + f[1];
  f[2] = f3pm + f[2];
  f[3] = f4pm + f[3];
  f[4] = f5 + f[4];
}

/* The Roe-averaged state and sound speed that FLUXKE, FLUXKT and FLUCUSP
 * share (base3c.f:4620-4660, 5290-5330): DERIV base3c.f:707 from the
 * cells (cr / cl2 = {C, DRDP, DRDH, RO, P} of I and of its DERIV partner)
 * and the extrapolated pairs, the hat averages, PHAT and CHAT. */
typedef struct {
  double rohat, uhat, vhat, what, hhat, rkhat, epshat, chat, dedph;
} hat_t;

static hat_t hat_state(double roip, double roim, double ppi, double pmi, double eip, double eim, double elr,
                       double erl, double ur, double vr, double wr, double ul, double vl, double wl, double rkr,
                       double rkl, double epsr, double epsl, double hr, double hl, double c_r, double c_l,
                       const double *cr, const double *cl2) {
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
  hat_t h;
  double pr = ppi, pl = pmi, er = eip, el = eim;
  h.rohat = sqrt(roip * roim);
  double yproh = 1. / h.rohat;
  double sqrl = 1. / (roim + h.rohat), cql = roim * sqrl, cqr = 1. - cql;
  h.uhat = cqr * ur + cql * ul;
  h.vhat = cqr * vr + cql * vl;
  h.what = cqr * wr + cql * wl;
  h.hhat = cqr * hr + cql * hl;
  double ehat = cqr * er + cql * el;
  h.rkhat = cqr * rkr + cql * rkl;
  h.epshat = cqr * epsr + cql * epsl;
  double phat = h.rohat * (h.hhat - ehat - .5 * (h.uhat * h.uhat + h.vhat * h.vhat + h.what * h.what) - h.rkhat);
  double pmin = MIND(pr, pl), pmax = MAXD(pr, pl);
  phat = MIND(pmax, phat);
  phat = MAXD(pmin, phat);
  double drdhh = 1. / (dedrh - phat * (yproh * yproh));
  double drdph = -drdhh * (dedph + yproh);
  double xturb = 1. + .6667 * h.rkhat * yproh * drdph;
  double chat2 = xturb / (drdhh * yproh + drdph);
  double cmin = MIND(c_r, c_l), cmax = MAXD(c_r, c_l);
  chat2 = MIND(cmax * cmax, chat2);
  chat2 = MAXD(cmin * cmin, chat2);
  h.chat = sqrt(chat2);
  h.dedph = dedph;
  return h;
}

/* FLUCUSP base3c.f:5133-5540 (IFLUX = 8) at one face.  q[v][m]: v = RO, U,
 * V, W, P (, RK, REPS for nv = 7).  The characteristic multipliers and the
 * entropy-fixed eigenvalues of the reference feed only HAT1..HAT4 (scalar
 * transport), not the fluxes, and are left out. */
static void hcusp_face(const double q[7][4], int nv, const double *nrm, double area, int intem, int intet,
                       const ff_params *p, double c_r, double c_l, const double *cr, const double *cl2,
                       const double *dd, double *f) {
  double roip, roim, uip, uim, vip, vim, wip, wim, ppi, pmi, rkip = 0., rkim = 0., reip = 0., reim = 0.;
  xxm(q[0], dd, intem, &roip, &roim);
  xxm(q[1], dd, intem, &uip, &uim);
  xxm(q[2], dd, intem, &vip, &vim);
  xxm(q[3], dd, intem, &wip, &wim);
  xxm(q[4], dd, intem, &ppi, &pmi);
  if (nv == 7) {   /* XXTRAA takes INTEM for k and omega too (base3c.f:5244-5245) */
    xxm(q[5], dd, dd ? intem : intet, &rkip, &rkim);
    xxm(q[6], dd, dd ? intem : intet, &reip, &reim);
  }
  const double rklim = nv == 7 ? p->rklim : 0., epslim = nv == 7 ? p->epslim : 0.;
  roip = MAXD(0.001 * p->frsden, roip);
  ppi = MAXD(0.001 * p->frspre, ppi);
  roim = MAXD(0.001 * p->frsden, roim);
  pmi = MAXD(0.001 * p->frspre, pmi);
  const double gm1 = p->gamma - 1.;
  double eip = (ppi + 0.) / (gm1 * roip) - p->e0ref;
  double eim = (pmi + 0.) / (gm1 * roim) - p->e0ref;
  double elr = (ppi + 0.) / (gm1 * roim) - p->e0ref;
  double erl = (pmi + 0.) / (gm1 * roip) - p->e0ref;
  double a11 = nrm[0], a12 = nrm[1], a13 = nrm[2], a21, a22, a23, a31, a32, a33;
  surfvects(a11, a12, a13, &a21, &a22, &a23, &a31, &a32, &a33);
  double ur = a11 * uip + a12 * vip + a13 * wip;
  double vr = a21 * uip + a22 * vip + a23 * wip;
  double wr = a31 * uip + a32 * vip + a33 * wip;
  double ul = a11 * uim + a12 * vim + a13 * wim;
  double vl = a21 * uim + a22 * vim + a23 * wim;
  double wl = a31 * uim + a32 * vim + a33 * wim;
  double rkipi = MAXD(0.001 * rklim, rkip), reipi = MAXD(0.001 * epslim, reip);
  double rkimi = MAXD(0.001 * rklim, rkim), reimi = MAXD(0.001 * epslim, reim);
  double ypror = 1. / roip, rkr = rkipi * ypror;
  double yprol = 1. / roim, rkl = rkimi * yprol;
  double eir = eip + .5 * (ur * ur + vr * vr + wr * wr) + rkr;
  double eil = eim + .5 * (ul * ul + vl * vl + wl * wl) + rkl;
  double pr = ppi, pkr = .6667 * rkipi, epsr = reipi * ypror, hr = eir + pr * ypror;
  double pl = pmi, pkl = .6667 * rkimi, epsl = reimi * yprol, hl = eil + yprol * pl;
  hat_t h = hat_state(roip, roim, ppi, pmi, eip, eim, elr, erl, ur, vr, wr, ul, vl, wl, rkr, rkl, epsr, epsl,
                      hr, hl, c_r, c_l, cr, cl2);
  double chat = h.chat, uhat = h.uhat, rma = uhat / chat;
  const double uc = 0.;
  double roucr = roip * (ur - uc), roucl = roim * (ul - uc);
  double alfa, beta;
  if (fabs(rma) > .2) alfa = fabs(rma);
  else alfa = (rma * rma + .04) / .4;
  if (rma >= 0. && rma <= 1.) beta = MAXD(0., 2. * rma - 1.);
  else if (rma > -1. && rma < 0.) beta = MIND(0., 2 * rma + 1.);
  else beta = rma >= 0. ? 1. : -1.;                            /* SIGN(1.,RMA) */
  double ac = alfa * chat - beta * uhat;
  double damp, f1, f2, f3, f4, f5, f6, f7;
  damp = ac * (roip - roim) + beta * (roucr - roucl);
  f1 = .5 * area * (roucr + roucl - damp);
  damp = ac * (roip * ur - roim * ul) + beta * (roucr * ur + pr + pkr - roucl * ul - pl - pkl);
  f2 = .5 * area * (roucr * ur + pr + pkr + roucl * ul + pl + pkl - damp);
  damp = ac * (roip * vr - roim * vl) + beta * (roucr * vr - roucl * vl);
  f3 = .5 * area * (roucr * vr + roucl * vl - damp);
  damp = ac * (roip * wr - roim * wl) + beta * (roucr * wr - roucl * wl);
  f4 = .5 * area * (roucr * wr + roucl * wl - damp);
  double hkr = hr + pkr * ypror, hkl = hl + pkl * yprol;
  damp = ac * (roip * hkr - roim * hkl) + beta * (roucr * hkr - roucl * hkl);
  f5 = .5 * area * (roucr * hkr + roucl * hkl + uc * (pr + pkr + pl + pkl) - damp);
  damp = ac * (roip * rkr - roim * rkl) + beta * (roucr * rkr - roucl * rkl);
  f6 = .5 * area * (roucr * rkr + roucl * rkl - damp);
  damp = ac * (roip * epsr - roim * epsl) + beta * (roucr * epsr - roucl * epsl);
  f7 = .5 * area * (roucr * epsr + roucl * epsl - damp);
  double f2pm = a11 * f2 + a21 * f3 + a31 * f4;
  double f3pm = a12 * f2 + a22 * f3 + a32 * f4;
  double f4pm = a13 * f2 + a23 * f3 + a33 * f4;
  f[0] = f1 + f[0];
  f[1] = f2pm + f[1];
  f[2] = f3pm + f[2];
  f[3] = f4pm + f[3];
  f[4] = f5 + f[4];
  if (nv == 7) {
    f[5] = f6 + f[5];
    f[6] = f7 + f[6];
  }
}

/* FLUXKT base3c.f:4403-4747 (IFLUX = 7) at one face.  q[v][m]: v = TEMP, U,
 * V, W, P, PDIFF (, RK, REPS for nv = 7).  Density and internal energy of
 * the extrapolated pairs from pressure and temperature (ROFPT state.f:667
 * with IUPPTL = 0, EFPT state.f:876).  FLUXKT hands DERIV the arrays ELR and
 * ERL without filling them (base3c.f:4562-4572: no EFPRO calls), so the
 * reference reads whatever its work space holds there; they are taken
 * here as FLUXKE and FLUCUSP fill them, e(P of one side, RO of the other)
 * (EFPRO, base3c.f:5213-5216).  CHAT enters only the mass flux's pressure
 * damping; the eigenvalues and their entropy fix feed HAT4 alone and are
 * left out. */
static void kt_face(const double q[8][4], int nv, const double *nrm, double area, int intem, int intet,
                    const ff_params *p, double c_r, double c_l, const double *cr, const double *cl2,
                    const double *dd, double *f) {
  double teip, teim, uip, uim, vip, vim, wip, wim, ppi, pmi, pdpi, pdmi;
  double rkip = 0., rkim = 0., reip = 0., reim = 0.;
  xxm(q[0], dd, intem, &teip, &teim);
  xxm(q[1], dd, intem, &uip, &uim);
  xxm(q[2], dd, intem, &vip, &vim);
  xxm(q[3], dd, intem, &wip, &wim);
  xxm(q[4], dd, intem, &ppi, &pmi);
  xxm(q[5], dd, intem, &pdpi, &pdmi);
  if (nv == 7) {   /* XXTRAA takes INTEM for k and omega too (base3c.f:4507-4508) */
    xxm(q[6], dd, dd ? intem : intet, &rkip, &rkim);
    xxm(q[7], dd, dd ? intem : intet, &reip, &reim);
  }
  const double rklim = nv == 7 ? p->rklim : 0., epslim = nv == 7 ? p->epslim : 0.;
  ppi = MAXD(0.001 * p->frspre, ppi);
  pmi = MAXD(0.001 * p->frspre, pmi);
  pdpi = MAXD(-0.999 * p->frspre, pdpi);
  pdmi = MAXD(-0.999 * p->frspre, pdmi);
  rkip = MAXD(0., rkip);
  rkim = MAXD(0., rkim);
  reip = MAXD(0., reip);
  reim = MAXD(0., reim);
  const double gm1 = p->gamma - 1.;
  double roip = ppi / (p->rgas * teip), roim = pmi / (p->rgas * teim);     /* ROFPT */
  double eip = p->rgas / gm1 * teip, eim = p->rgas / gm1 * teim;           /* EFPT  */
  double elr = (ppi + 0.) / (gm1 * roim) - p->e0ref;
  double erl = (pmi + 0.) / (gm1 * roip) - p->e0ref;
  double a11 = nrm[0], a12 = nrm[1], a13 = nrm[2], a21, a22, a23, a31, a32, a33;
  surfvects(a11, a12, a13, &a21, &a22, &a23, &a31, &a32, &a33);
  double rkipi = MAXD(0.001 * rklim, rkip), reipi = MAXD(0.001 * epslim, reip);
  double rkimi = MAXD(0.001 * rklim, rkim), reimi = MAXD(0.001 * epslim, reim);
  double ur = a11 * uip + a12 * vip + a13 * wip;
  double vr = a21 * uip + a22 * vip + a23 * wip;
  double wr = a31 * uip + a32 * vip + a33 * wip;
  double ul = a11 * uim + a12 * vim + a13 * wim;
  double vl = a21 * uim + a22 * vim + a23 * wim;
  double wl = a31 * uim + a32 * vim + a33 * wim;
  double ypror = 1. / roip, rkr = rkipi * ypror;
  double yprol = 1. / roim, rkl = rkimi * yprol;
  double eir = eip + .5 * (ur * ur + vr * vr + wr * wr) + rkr;
  double eil = eim + .5 * (ul * ul + vl * vl + wl * wl) + rkl;
  double pdr = pdpi, pr = ppi, pkr = .6667 * rkipi, epsr = reipi * ypror, hr = eir + pr * ypror;
  double pdl = pdmi, pl = pmi, pkl = .6667 * rkimi, epsl = reimi * yprol, hl = eil + yprol * pl;
  hat_t h = hat_state(roip, roim, ppi, pmi, eip, eim, elr, erl, ur, vr, wr, ul, vl, wl, rkr, rkl, epsr, epsl,
                      hr, hl, c_r, c_l, cr, cl2);
  double chat = h.chat;
  double sr = MAXD(fabs(ur) + c_r, fabs(ul) + c_l);
  const double uc = 0.;
  double roucr = roip * (ur - uc), roucl = roim * (ul - uc);
  double uhat = .5 * (ur + ul);
  double damp = sr * (pdr - pdl) / (chat * chat);
  double f1 = .5 * area * (roucr + roucl - damp);
  double f2 = .5 * area * (roucr * ur + pdr + pkr + roucl * ul + pdl + pkl - sr * (roip * ur - roim * ul));
  double f3 = .5 * area * (roucr * vr + roucl * vl - sr * (roip * vr - roim * vl));
  double f4 = .5 * area * (roucr * wr + roucl * wl - sr * (roip * wr - roim * wl));
  double f5 = .5 * area * (roucr * (hr + pkr * ypror) + roucl * (hl + pkl * yprol) + uc * (pr + pkr + pl + pkl)
                           - sr * (roip * eir - roim * eil));
  double f6 = .5 * area * (roucr * rkr + roucl * rkl - fabs(uhat) * (roip * rkr - roim * rkl));
  double f7 = .5 * area * (roucr * epsr + roucl * epsl - fabs(uhat) * (roip * epsr - roim * epsl));
  double f2pm = a11 * f2 + a21 * f3 + a31 * f4;
  double f3pm = a12 * f2 + a22 * f3 + a32 * f4;
  double f4pm = a13 * f2 + a23 * f3 + a33 * f4;
  f[0] = f1 + f[0];
  f[1] = f2pm + f[1];
  f[2] = f3pm + f[2];
  f[3] = f4pm + f[3];
  f[4] = f5 + f[4];
  if (nv == 7) {
    f[5] = f6 + f[5];
    f[6] = f7 + f[6];
  }
}

/* The inviscid flux of face L (cells L-S | L) for ff_params.flux other than
 * Roe, added to f (nv = 5 laminar, 7 with k and omega): the stencil each
 * scheme extrapolates, then its face function.  L2 = DERIV's partner of L. */
static void alt_face(const orc_block *b, const ff_params *p, int dir, size_t L, int S, int intem, int intet,
                     int nv, double *f) {
  size_t L2 = dir == 3 ? L : L - S;
  const double nrm[3] = {b->a[FF_A1XA + 4 * (dir - 1)][L], b->a[FF_A1YA + 4 * (dir - 1)][L],
                         b->a[FF_A1ZA + 4 * (dir - 1)][L]};
  const double area = b->a[FF_A1 + 4 * (dir - 1)][L];
  const double *C = b->a[FF_C];
  double cr[5] = {C[L], b->a[FF_DRDP][L], b->a[FF_DRDH][L], b->a[FF_RO][L], b->a[FF_P][L]};
  double cl[5] = {C[L2], b->a[FF_DRDP][L2], b->a[FF_DRDH][L2], b->a[FF_RO][L2], b->a[FF_P][L2]};
  switch (p->flux) {
    case FF_FLUX_VANLEER:
    case FF_FLUX_WPS: {
      const int s[5] = {FF_RO, FF_RM, FF_RN, FF_RW, FF_E};
      double qc[5][4];
      for (int v = 0; v < 5; v++)
        for (int m = 0; m < 4; m++) qc[v][m] = b->a[s[v]][L + (m - 2) * S];
      vl_face(qc, nrm, area, intem, p, p->flux == FF_FLUX_WPS, f);
      return;
    }
    case FF_FLUX_AUSM: {
      const int s[6] = {FF_RO, FF_U, FF_V, FF_W, FF_P, FF_PDIFF};
      double q[6][4];
      for (int v = 0; v < 6; v++)
        for (int m = 0; m < 4; m++) q[v][m] = b->a[s[v]][L + (m - 2) * S];
      ausm_face(q, nrm, area, intem, p, C[L], C[L - S], f);
      return;
    }
    case FF_FLUX_KT: {
      const int s[8] = {FF_TEMP, FF_U, FF_V, FF_W, FF_P, FF_PDIFF, FF_RK, FF_REPS};
      double q[8][4];
      const int n = nv == 7 ? 8 : 6;
      for (int v = 0; v < n; v++)
        for (int m = 0; m < 4; m++) q[v][m] = b->a[s[v]][L + (m - 2) * S];
      double dd[4];
      kt_face(q, nv, nrm, area, intem, intet, p, C[L], C[L - S], cr, cl, stencil_d(b, p, dir, L, S, dd), f);
      return;
    }
    case FF_FLUX_HCUSP: {
      const int s[7] = {FF_RO, FF_U, FF_V, FF_W, FF_P, FF_RK, FF_REPS};
      double q[7][4];
      for (int v = 0; v < nv; v++)
        for (int m = 0; m < 4; m++) q[v][m] = b->a[s[v]][L + (m - 2) * S];
      double dd[4];
      hcusp_face(q, nv, nrm, area, intem, intet, p, C[L], C[L - S], cr, cl, stencil_d(b, p, dir, L, S, dd), f);
      return;
    }
    default:
      return;
  }
}

/* SCALARD base3c.f:6-78 (IPRESC = 0, UROT = VROT = WROT = 0): SCALEJ of the
 * cells 0..MAX+1 in each direction, |contravariant velocity| summed over the
 * cell's mean face vectors plus C times the mean face areas. */
void orc_scalard(orc_block *b) {
  dims_t d = dims_of(b);
  double *SJ = b->a[FF_SCALEJ];
  memset(SJ, 0, sizeof(double) * d.ntot);
  const double *A1 = b->a[FF_A1], *A2 = b->a[FF_A2], *A3 = b->a[FF_A3];
  const double *A1X = b->a[FF_A1XA], *A1Y = b->a[FF_A1YA], *A1Z = b->a[FF_A1ZA];
  const double *A2X = b->a[FF_A2XA], *A2Y = b->a[FF_A2YA], *A2Z = b->a[FF_A2ZA];
  const double *A3X = b->a[FF_A3XA], *A3Y = b->a[FF_A3YA], *A3Z = b->a[FF_A3ZA];
  const double *U = b->a[FF_U], *V = b->a[FF_V], *W = b->a[FF_W], *C = b->a[FF_C];
  const int is = d.is, il = d.il;
  for (int K = 0; K <= d.kmax + 1; K++)
    for (int J = 0; J <= d.jmax + 1; J++)
      for (int I = 0; I <= d.imax + 1; I++) {
        size_t kk = IX(d, I, J, K);
        double chat = C[kk];
        double a1k = .5 * (A1[kk] + A1[kk + 1]);
        double a2k = .5 * (A2[kk] + A2[kk + is]);
        double a3k = .5 * (A3[kk] + A3[kk + il]);
        double a1xk = .5 * (A1X[kk] * A1[kk] + A1X[kk + 1] * A1[kk + 1]);
        double a1yk = .5 * (A1Y[kk] * A1[kk] + A1Y[kk + 1] * A1[kk + 1]);
        double a1zk = .5 * (A1Z[kk] * A1[kk] + A1Z[kk + 1] * A1[kk + 1]);
        double a2xk = .5 * (A2X[kk] * A2[kk] + A2X[kk + is] * A2[kk + is]);
        double a2yk = .5 * (A2Y[kk] * A2[kk] + A2Y[kk + is] * A2[kk + is]);
        double a2zk = .5 * (A2Z[kk] * A2[kk] + A2Z[kk + is] * A2[kk + is]);
        double a3xk = .5 * (A3X[kk] * A3[kk] + A3X[kk + il] * A3[kk + il]);
        double a3yk = .5 * (A3Y[kk] * A3[kk] + A3Y[kk + il] * A3[kk + il]);
        double a3zk = .5 * (A3Z[kk] * A3[kk] + A3Z[kk + il] * A3[kk + il]);
        double ucii = a1xk * U[kk] + a1yk * V[kk] + a1zk * W[kk] - 0.;
        double vcii = a2xk * U[kk] + a2yk * V[kk] + a2zk * W[kk] - 0.;
        double wcii = a3xk * U[kk] + a3yk * V[kk] + a3zk * W[kk] - 0.;
        double ccii = (a1k + a2k + a3k) * chat;
        SJ[kk] = sqrt(ucii * ucii + vcii * vcii + wcii * wcii) + ccii;
      }
}

/* JAMESON base3c.f:2827-3019 (IPRESC = 0) at face L (cells L-S | L): the
 * pressure sensors of the two cells (PDIFF second differences), EPS2 =
 * RJK2 * max, EPS4 = max(0, RJK4 - EPS2), SCALEJ averaged to the face; the
 * second- and fourth-difference dissipation of RO, RM, RN, RW, E subtracted
 * from f.  FLUCYC and RESIKE add it to Roe's flux on the finest level
 * (res3c.f:7899-7906, 6955-6962); k and omega keep theirs. */
static void jst_face(const orc_block *b, const ff_params *p, size_t L, int S, double *f) {
  const double *PD = b->a[FF_PDIFF], *SJ = b->a[FF_SCALEJ];
  const double fp4 = 4. * p->frspre;
  double pres1 = fabs(PD[L] - 2. * PD[L - S] + PD[L - 2 * S]) / (PD[L] + 2. * PD[L - S] + PD[L - 2 * S] + fp4);
  double pres2 = fabs(PD[L + S] - 2. * PD[L] + PD[L - S]) / (PD[L + S] + 2. * PD[L] + PD[L - S] + fp4);
  double eps2i = p->rjk2 * MAXD(pres1, pres2);
  double eps4i = MAXD(0., (p->rjk4 - eps2i));
  double rlami = .5 * (SJ[L] + SJ[L - S]);
  const int sl[5] = {FF_RO, FF_RM, FF_RN, FF_RW, FF_E};
  for (int v = 0; v < 5; v++) {
    const double *Q = b->a[sl[v]];
    double fj = rlami * (eps2i * (Q[L] - Q[L - S]) - eps4i * (Q[L + S] - 3. * Q[L] + 3. * Q[L - S] - Q[L - 2 * S]));
    f[v] = -fj + f[v];
  }
}
