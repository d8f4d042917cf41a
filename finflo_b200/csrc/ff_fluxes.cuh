// The inviscid face fluxes that IFLUX selects besides Roe's (ff_params.flux,
// enum ff_flux): wave/particle splitting (FLUXWP, in vl_flux), its AUSM form
// (FLUXAU), Kurganov-Tadmor (FLUXKT) and H-CUSP (FLUCUSP), one face per
// thread, FP64, UROT = 0, perfect gas, MUSCL by XXTRAP (XXTRAA for KT and
// H-CUSP when XXTRAL is set; FLUXVL, FLUXWP and FLUXAU have no XXTRAL
// branch).  NV = 5: the laminar form that FLUCYC calls (k and omega zero,
// RKLIM = EPSLIM = 0, res3c.f:7680); NV = 7: RESIKE's, with the k-omega
// variables (res3c.f:7017-7036).  Included by ff_kernels.cuh after vl_flux.
#pragma once

// The MUSCL pair of one variable (q = cells I-2S..I+S): XXTRAA over the
// extents d when XXTRAL gives them, else XXTRAP.
FF_DI void muscl_d(const double q[4], const double* d, int intem, double& ip, double& im) {
  if (d) xxtraa(q[0], q[1], q[2], q[3], d, intem, ip, im);
  else xxtrap(q[0], q[1], q[2], q[3], intem, ip, im);
}

// FLUXAU base3c.f:2201-2466 (IFLUX = 3).  q[v][m]: v = RO, U, V, W, P, PDIFF,
// m = cells I-2S..I+S; c_r = C(I), c_l = C(I-S).  Adds to f[0..4].
FF_DI void ausm_flux(const double q[6][4], double nx, double ny, double nz, double area, int intem,
                     const ff_params& p, double c_r, double c_l, double f[5]) {
  double roip, roim, uip, uim, vip, vim, wip, wim, ppi, pmi, pdpi, pdmi;
  xxtrap(q[0][0], q[0][1], q[0][2], q[0][3], intem, roip, roim);
  xxtrap(q[1][0], q[1][1], q[1][2], q[1][3], intem, uip, uim);
  xxtrap(q[2][0], q[2][1], q[2][2], q[2][3], intem, vip, vim);
  xxtrap(q[3][0], q[3][1], q[3][2], q[3][3], intem, wip, wim);
  xxtrap(q[4][0], q[4][1], q[4][2], q[4][3], intem, ppi, pmi);
  xxtrap(q[5][0], q[5][1], q[5][2], q[5][3], intem, pdpi, pdmi);
  roip = dmax(0.001 * p.frsden, roip);
  ppi = dmax(0.001 * p.frspre, ppi);
  roim = dmax(0.001 * p.frsden, roim);
  pmi = dmax(0.001 * p.frspre, pmi);
  pdpi = dmax(-0.999 * p.frspre, pdpi);
  pdmi = dmax(-0.999 * p.frspre, pdmi);
  const double gm1 = p.gamma - 1.;
  const double eip = ppi / (gm1 * roip) - p.e0ref, eim = pmi / (gm1 * roim) - p.e0ref;   // EFPRO
  double a21, a22, a23, a31, a32, a33;
  surfvects(nx, ny, nz, a21, a22, a23, a31, a32, a33);
  const double ur = nx * uip + ny * vip + nz * wip, vr = a21 * uip + a22 * vip + a23 * wip,
               wr = a31 * uip + a32 * vip + a33 * wip;
  const double ul = nx * uim + ny * vim + nz * wim, vl = a21 * uim + a22 * vim + a23 * wim,
               wl = a31 * uim + a32 * vim + a33 * wim;
  const double eir = eip + .5 * (ur * ur + vr * vr + wr * wr);
  const double eil = eim + .5 * (ul * ul + vl * vl + wl * wl);
  // split Mach numbers and pressure differences of the two sides
  double pdr = pdpi, rmar;
  const double rmaip = ur / c_r;
  if (fabs(rmaip) <= 1.) {
    const double h = .5 * (rmaip - 1.);
    rmar = -(h * h);
    pdr = pdr * .50 * ((rmaip - 1.) * (rmaip - 1.)) * (2. + rmaip);
  } else {
    rmar = .5 * (rmaip - fabs(rmaip));
    pdr = pdr * (rmaip - fabs(rmaip)) / rmaip;
  }
  double pdl = pdmi, rmal;
  const double rmaim = ul / c_l;
  if (fabs(rmaim) <= 1.) {
    const double h = .5 * (rmaim + 1.);
    rmal = h * h;
    pdl = pdl * .50 * ((rmaim + 1.) * (rmaim + 1.)) * (2. - rmaim);
  } else {
    rmal = .5 * (rmaim + fabs(rmaim));
    pdl = pdl * (rmaim + fabs(rmaim)) / rmaim;
  }
  const double rma = rmar + rmal, absrma = fabs(rma);
  const double roucr = roip * c_r, roucl = roim * c_l;
  // RMA*(a_R + a_L) - |RMA|*(a_R - a_L) of each convected quantity a
  auto up = [&](double ar, double al) { return rma * (ar + al) - absrma * (ar - al); };
  const double ha = .5 * area;
  const double f1 = ha * up(roucr, roucl);
  const double f2 = ha * (up(roucr * ur, roucl * ul) + pdr + pdl);
  const double f3 = ha * up(roucr * vr, roucl * vl);
  const double f4 = ha * up(roucr * wr, roucl * wl);
  const double f5 = ha * (up(roucr * eir, roucl * eil) + pdpi * ur + pdmi * ul);
  f[0] += f1;
  f[1] += nx * f2 + a21 * f3 + a31 * f4;
  f[2] += ny * f2 + a22 * f3 + a32 * f4;
  f[3] += nz * f2 + a23 * f3 + a33 * f4;
  f[4] += f5;
}

// The Roe-averaged state and sound speed shared by FLUXKE, FLUXKT and FLUCUSP:
// DERIV base3c.f:707 (cr / cl2 = {DRDP, DRDH, RO, P} of cell I and of its
// DERIV partner; the jump forms from e(P, RO) of the pairs), the hat
// averages, PHAT clipped to the side pressures, CHAT clipped to the cells'
// sound speeds.
struct HatState {
  double rohat, uhat, chat;
};

FF_DI HatState hat_state(double roip, double roim, double ppi, double pmi, double eip, double eim, double elr,
                         double erl, double ur, double vr, double wr, double ul, double vl, double wl, double rkr,
                         double rkl, double hr, double hl, double c_r, double c_l, const double cr[4],
                         const double cl2[4]) {
  const double ypro1 = rcp(cr[2]), ypro2 = rcp(cl2[2]);
  const double rdh1 = rcp(cr[1]), rdh2 = rcp(cl2[1]);
  double dedph = 0.5 * ((-cr[0] * rdh1 - ypro1) + (-cl2[0] * rdh2 - ypro2));
  double dedrh = 0.5 * ((rdh1 + cr[3] * (ypro1 * ypro1)) + (rdh2 + cl2[3] * (ypro2 * ypro2)));
  {
    const double dpp = 2. * (ppi - pmi), drr = 2. * (roip - roim);
    if (fabs(dpp) >= 1.e-2 * (ppi + pmi)) dedph = (eip + elr - eim - erl) / dpp;
    if (fabs(drr) >= 1.e-2 * (roip + roim)) dedrh = (eip + erl - eim - elr) / drr;
  }
  HatState h;
  h.rohat = sqrt(roip * roim);
  const double yproh = rcp(h.rohat);
  const double sqrl = rcp(roim + h.rohat), cql = roim * sqrl, cqr = 1. - cql;
  h.uhat = cqr * ur + cql * ul;
  const double vhat = cqr * vr + cql * vl, what = cqr * wr + cql * wl;
  const double hhat = cqr * hr + cql * hl, ehat = cqr * eip + cql * eim, rkhat = cqr * rkr + cql * rkl;
  double phat = h.rohat * (hhat - ehat - .5 * (h.uhat * h.uhat + vhat * vhat + what * what) - rkhat);
  phat = dmin(dmax(ppi, pmi), phat);
  phat = dmax(dmin(ppi, pmi), phat);
  const double drdhh = rcp(dedrh - phat * (yproh * yproh));
  const double drdph = -drdhh * (dedph + yproh);
  const double xturb = 1. + .6667 * rkhat * yproh * drdph;
  double chat2 = xturb / (drdhh * yproh + drdph);
  const double cmin = dmin(c_r, c_l), cmax = dmax(c_r, c_l);
  chat2 = dmin(cmax * cmax, chat2);
  chat2 = dmax(cmin * cmin, chat2);
  h.chat = sqrt(chat2);
  return h;
}

// FLUCUSP base3c.f:5133-5540 (IFLUX = 8).  q[v][m]: v = RO, U, V, W, P (, RK,
// REPS).  Adds to f[0..NV-1].  The characteristic multipliers and the
// (entropy-fixed) eigenvalues of the reference reach only HAT1..HAT4, the
// scalar-transport hand-over, and are not formed.
template <int NV>
FF_DI void hcusp_flux(const double q[NV][4], double nx, double ny, double nz, double area, int intem, int intet,
                      const ff_params& p, double c_r, double c_l, const double cr[4], const double cl2[4],
                      const double* dd, double f[NV]) {
  double roip, roim, uip, uim, vip, vim, wip, wim, ppi, pmi, rkip = 0., rkim = 0., reip = 0., reim = 0.;
  muscl_d(q[0], dd, intem, roip, roim);
  muscl_d(q[1], dd, intem, uip, uim);
  muscl_d(q[2], dd, intem, vip, vim);
  muscl_d(q[3], dd, intem, wip, wim);
  muscl_d(q[4], dd, intem, ppi, pmi);
  if constexpr (NV == 7) {   // XXTRAA takes INTEM for k and omega (base3c.f:5244-5245)
    muscl_d(q[5], dd, dd ? intem : intet, rkip, rkim);
    muscl_d(q[6], dd, dd ? intem : intet, reip, reim);
  }
  const double rklim = NV == 7 ? p.rklim : 0., epslim = NV == 7 ? p.epslim : 0.;
  roip = dmax(0.001 * p.frsden, roip);
  ppi = dmax(0.001 * p.frspre, ppi);
  roim = dmax(0.001 * p.frsden, roim);
  pmi = dmax(0.001 * p.frspre, pmi);
  const double gm1 = p.gamma - 1.;
  const double eip = ppi / (gm1 * roip) - p.e0ref, eim = pmi / (gm1 * roim) - p.e0ref;
  const double elr = ppi / (gm1 * roim) - p.e0ref, erl = pmi / (gm1 * roip) - p.e0ref;
  double a21, a22, a23, a31, a32, a33;
  surfvects(nx, ny, nz, a21, a22, a23, a31, a32, a33);
  const double ur = nx * uip + ny * vip + nz * wip, vr = a21 * uip + a22 * vip + a23 * wip,
               wr = a31 * uip + a32 * vip + a33 * wip;
  const double ul = nx * uim + ny * vim + nz * wim, vl = a21 * uim + a22 * vim + a23 * wim,
               wl = a31 * uim + a32 * vim + a33 * wim;
  const double rkipi = dmax(0.001 * rklim, rkip), reipi = dmax(0.001 * epslim, reip);
  const double rkimi = dmax(0.001 * rklim, rkim), reimi = dmax(0.001 * epslim, reim);
  const double ypror = rcp(roip), yprol = rcp(roim);
  const double rkr = rkipi * ypror, rkl = rkimi * yprol;
  const double eir = eip + .5 * (ur * ur + vr * vr + wr * wr) + rkr;
  const double eil = eim + .5 * (ul * ul + vl * vl + wl * wl) + rkl;
  const double pr = ppi, pl = pmi, pkr = .6667 * rkipi, pkl = .6667 * rkimi;
  const double epsr = reipi * ypror, epsl = reimi * yprol;
  const double hr = eir + pr * ypror, hl = eil + yprol * pl;
  const HatState h = hat_state(roip, roim, ppi, pmi, eip, eim, elr, erl, ur, vr, wr, ul, vl, wl, rkr, rkl, hr, hl,
                               c_r, c_l, cr, cl2);
  const double rma = h.uhat / h.chat;
  const double roucr = roip * ur, roucl = roim * ul;
  const double alfa = fabs(rma) > .2 ? fabs(rma) : (rma * rma + .04) / .4;
  double beta;
  if (rma >= 0. && rma <= 1.) beta = dmax(0., 2. * rma - 1.);
  else if (rma > -1. && rma < 0.) beta = dmin(0., 2. * rma + 1.);
  else beta = rma >= 0. ? 1. : -1.;
  const double ac = alfa * h.chat - beta * h.uhat;
  // (a_R ro_R - a_L ro_L) scaled by ALFA*CHAT - BETA*UHAT, plus BETA times
  // the jump of the convective flux
  auto damp = [&](double ar, double al, double fr, double fl) { return ac * (roip * ar - roim * al) + beta * (fr - fl); };
  const double ha = .5 * area;
  const double f1 = ha * (roucr + roucl - (ac * (roip - roim) + beta * (roucr - roucl)));
  const double f2 = ha * (roucr * ur + pr + pkr + roucl * ul + pl + pkl -
                          (ac * (roip * ur - roim * ul) + beta * (roucr * ur + pr + pkr - roucl * ul - pl - pkl)));
  const double f3 = ha * (roucr * vr + roucl * vl - damp(vr, vl, roucr * vr, roucl * vl));
  const double f4 = ha * (roucr * wr + roucl * wl - damp(wr, wl, roucr * wr, roucl * wl));
  const double hkr = hr + pkr * ypror, hkl = hl + pkl * yprol;
  const double f5 = ha * (roucr * hkr + roucl * hkl - damp(hkr, hkl, roucr * hkr, roucl * hkl));
  f[0] += f1;
  f[1] += nx * f2 + a21 * f3 + a31 * f4;
  f[2] += ny * f2 + a22 * f3 + a32 * f4;
  f[3] += nz * f2 + a23 * f3 + a33 * f4;
  f[4] += f5;
  if constexpr (NV == 7) {
    f[5] += ha * (roucr * rkr + roucl * rkl - damp(rkr, rkl, roucr * rkr, roucl * rkl));
    f[6] += ha * (roucr * epsr + roucl * epsl - damp(epsr, epsl, roucr * epsr, roucl * epsl));
  }
}

// FLUXKT base3c.f:4403-4747 (IFLUX = 7).  q[v][m]: v = TEMP, U, V, W, P, PDIFF
// (, RK, REPS).  Density and internal energy of the pairs from P and T
// (ROFPT state.f:667 with IUPPTL = 0, EFPT state.f:876).  DERIV's ELR / ERL,
// which FLUXKT passes unset, are e(P of one side, RO of the other) as in
// FLUXKE.  Adds to f[0..NV-1].
template <int NV>
FF_DI void kt_flux(const double q[NV + 1][4], double nx, double ny, double nz, double area, int intem, int intet,
                   const ff_params& p, double c_r, double c_l, const double cr[4], const double cl2[4],
                   const double* dd, double f[NV]) {
  double teip, teim, uip, uim, vip, vim, wip, wim, ppi, pmi, pdpi, pdmi, rkip = 0., rkim = 0., reip = 0., reim = 0.;
  muscl_d(q[0], dd, intem, teip, teim);
  muscl_d(q[1], dd, intem, uip, uim);
  muscl_d(q[2], dd, intem, vip, vim);
  muscl_d(q[3], dd, intem, wip, wim);
  muscl_d(q[4], dd, intem, ppi, pmi);
  muscl_d(q[5], dd, intem, pdpi, pdmi);
  if constexpr (NV == 7) {   // XXTRAA takes INTEM for k and omega (base3c.f:4507-4508)
    muscl_d(q[6], dd, dd ? intem : intet, rkip, rkim);
    muscl_d(q[7], dd, dd ? intem : intet, reip, reim);
  }
  const double rklim = NV == 7 ? p.rklim : 0., epslim = NV == 7 ? p.epslim : 0.;
  ppi = dmax(0.001 * p.frspre, ppi);
  pmi = dmax(0.001 * p.frspre, pmi);
  pdpi = dmax(-0.999 * p.frspre, pdpi);
  pdmi = dmax(-0.999 * p.frspre, pdmi);
  rkip = dmax(0., rkip); rkim = dmax(0., rkim); reip = dmax(0., reip); reim = dmax(0., reim);
  const double gm1 = p.gamma - 1.;
  const double roip = ppi / (p.rgas * teip), roim = pmi / (p.rgas * teim);
  const double eip = p.rgas / gm1 * teip, eim = p.rgas / gm1 * teim;
  const double elr = ppi / (gm1 * roim) - p.e0ref, erl = pmi / (gm1 * roip) - p.e0ref;
  double a21, a22, a23, a31, a32, a33;
  surfvects(nx, ny, nz, a21, a22, a23, a31, a32, a33);
  const double rkipi = dmax(0.001 * rklim, rkip), reipi = dmax(0.001 * epslim, reip);
  const double rkimi = dmax(0.001 * rklim, rkim), reimi = dmax(0.001 * epslim, reim);
  const double ur = nx * uip + ny * vip + nz * wip, vr = a21 * uip + a22 * vip + a23 * wip,
               wr = a31 * uip + a32 * vip + a33 * wip;
  const double ul = nx * uim + ny * vim + nz * wim, vl = a21 * uim + a22 * vim + a23 * wim,
               wl = a31 * uim + a32 * vim + a33 * wim;
  const double ypror = rcp(roip), yprol = rcp(roim);
  const double rkr = rkipi * ypror, rkl = rkimi * yprol;
  const double eir = eip + .5 * (ur * ur + vr * vr + wr * wr) + rkr;
  const double eil = eim + .5 * (ul * ul + vl * vl + wl * wl) + rkl;
  const double pkr = .6667 * rkipi, pkl = .6667 * rkimi;
  const double epsr = reipi * ypror, epsl = reimi * yprol;
  const double hr = eir + ppi * ypror, hl = eil + yprol * pmi;
  const HatState h = hat_state(roip, roim, ppi, pmi, eip, eim, elr, erl, ur, vr, wr, ul, vl, wl, rkr, rkl, hr, hl,
                               c_r, c_l, cr, cl2);
  const double sr = dmax(fabs(ur) + c_r, fabs(ul) + c_l);
  const double roucr = roip * ur, roucl = roim * ul;
  const double ha = .5 * area;
  const double f1 = ha * (roucr + roucl - sr * (pdpi - pdmi) / (h.chat * h.chat));
  const double f2 = ha * (roucr * ur + pdpi + pkr + roucl * ul + pdmi + pkl - sr * (roip * ur - roim * ul));
  const double f3 = ha * (roucr * vr + roucl * vl - sr * (roip * vr - roim * vl));
  const double f4 = ha * (roucr * wr + roucl * wl - sr * (roip * wr - roim * wl));
  const double f5 = ha * (roucr * (hr + pkr * ypror) + roucl * (hl + pkl * yprol) - sr * (roip * eir - roim * eil));
  f[0] += f1;
  f[1] += nx * f2 + a21 * f3 + a31 * f4;
  f[2] += ny * f2 + a22 * f3 + a32 * f4;
  f[3] += nz * f2 + a23 * f3 + a33 * f4;
  f[4] += f5;
  if constexpr (NV == 7) {
    const double au = fabs(.5 * (ur + ul));
    f[5] += ha * (roucr * rkr + roucl * rkl - au * (roip * rkr - roim * rkl));
    f[6] += ha * (roucr * epsr + roucl * epsl - au * (roip * epsr - roim * epsl));
  }
}

// The inviscid flux of face L (cells L-S | L) for a scheme other than Roe,
// added to f: each scheme's MUSCL stencil from the block arrays (cells
// L-2S..L+S), then its face function.  Van Leer and WPS read the
// conservative variables, AUSM the primitive ones with PDIFF, KT T, the
// velocities, P and PDIFF, H-CUSP those of FLUXKE.
template <int NV>
FF_DI void alt_flux(const DevBlock& b, const ff_params& p, int dir, size_t L, int S, int intem, int intet,
                    double f[NV]) {
  const int ao = 4 * (dir - 1);
  const double nx = __ldg(b.a[FF_A1XA + ao] + L), ny = __ldg(b.a[FF_A1YA + ao] + L),
               nz = __ldg(b.a[FF_A1ZA + ao] + L), area = __ldg(b.a[FF_A1 + ao] + L);
  auto ld4 = [&](int slot, double* out) {
    const double* a = b.a[slot];
    out[0] = __ldg(a + L - 2 * S); out[1] = __ldg(a + L - S); out[2] = __ldg(a + L); out[3] = __ldg(a + L + S);
  };
  const double c_r = __ldg(b.a[FF_C] + L), c_l = __ldg(b.a[FF_C] + L - S);
  if (p.flux == FF_FLUX_VANLEER || p.flux == FF_FLUX_WPS) {
    double qc[5][4];
    const int sc[5] = {FF_RO, FF_RM, FF_RN, FF_RW, FF_E};
#pragma unroll
    for (int v = 0; v < 5; v++) ld4(sc[v], qc[v]);
    vl_flux(qc, nx, ny, nz, area, intem, p, p.flux == FF_FLUX_WPS, f);
    return;
  }
  if (p.flux == FF_FLUX_AUSM) {
    double q[6][4];
    const int sl[6] = {FF_RO, FF_U, FF_V, FF_W, FF_P, FF_PDIFF};
#pragma unroll
    for (int v = 0; v < 6; v++) ld4(sl[v], q[v]);
    ausm_flux(q, nx, ny, nz, area, intem, p, c_r, c_l, f);
    return;
  }
  const size_t L2 = dir == 3 ? L : L - S;
  double ddv[4];
  const double* dd = nullptr;
  if (p.xxtral) {   // XXTRAA over the cells' extents along the normal
    ld4(FF_D1 + dir - 1, ddv);
    dd = ddv;
  }
  const double cr[4] = {__ldg(b.a[FF_DRDP] + L), __ldg(b.a[FF_DRDH] + L), __ldg(b.a[FF_RO] + L),
                        __ldg(b.a[FF_P] + L)};
  const double cl[4] = {__ldg(b.a[FF_DRDP] + L2), __ldg(b.a[FF_DRDH] + L2), __ldg(b.a[FF_RO] + L2),
                        __ldg(b.a[FF_P] + L2)};
  if (p.flux == FF_FLUX_KT) {
    double q[NV + 1][4];
    const int sl[8] = {FF_TEMP, FF_U, FF_V, FF_W, FF_P, FF_PDIFF, FF_RK, FF_REPS};
#pragma unroll
    for (int v = 0; v < NV + 1; v++) ld4(sl[v], q[v]);
    kt_flux<NV>(q, nx, ny, nz, area, intem, intet, p, c_r, c_l, cr, cl, dd, f);
    return;
  }
  // FF_FLUX_HCUSP (the host admits no other value)
  double q[NV][4];
  const int sl[7] = {FF_RO, FF_U, FF_V, FF_W, FF_P, FF_RK, FF_REPS};
#pragma unroll
  for (int v = 0; v < NV; v++) ld4(sl[v], q[v]);
  hcusp_flux<NV>(q, nx, ny, nz, area, intem, intet, p, c_r, c_l, cr, cl, dd, f);
}
