// k-omega SST (ITURB=6, KOVER=0, IDIS=2) on the device, level 1.
//
// The per-cycle steps of the reference's two-equation path: TURBEQ
// (res3c.f:5845: DERFUN + EPS2KO turb3.f:7454), RESIKE (res3c.f:3423:
// CROSKO turb3.f:7790, FUN1KO 7385, MAKE_EPS 7905, PRODKE 4687, TEMDER of k
// and omega, FLXCYC res3c.f:6424 faces with FLKEBL base3c.f:5727, FLUXBL,
// FLUXKE base3c.f:4753 and BOTSKE base3c.f:6147, SWEEPK 1342, SOURKO
// turb3.f:7624, ADDSKE res3c.f:1473), the point-implicit and conversion
// steps of IMPS (LOCDTK imps3.f:807, IMSOKO 972, COPRKE 1113) and the k cap
// of SUBIN (ns3c.f:9742).  Included by ff_kernels.cuh inside namespace ff.

// COEFKO turb3.f:8068 (ITURB=6, KOVER<5)
constexpr double SST_A1KLEB = 0.31, SST_BSTAR = 0.09, SST_CKAPPA = 0.41, SST_BETA1 = 0.075;
constexpr double SST_SIGRK1 = 0.85, SST_SIGOM1 = 0.5, SST_BETA2 = 0.0828, SST_SIGRK2 = 1.0,
                 SST_SIGOM2 = 0.856;

// ---- TURBEQ: EPS2KO with STRAIN (res3c.f:6338), interior cells ----------
__global__ void k_eps2ko(DevBlock b, ff_params p) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.imax * b.jmax * b.kmax) return;
  int I = t % b.imax + 1, J = (t / b.imax) % b.jmax + 1, K = t / (b.imax * b.jmax) + 1;
  size_t L = ix(b, I, J, K);
  const double eps = 1.e-20, frsmut = 1.e-3 * p.frsvis;
  double ro = b.a[FF_RO][L], rk = b.a[FF_RK][L], rom = b.a[FF_REPS][L], dw = b.a[FF_DISTW][L];
  double vis = b.a[FF_VIS][L], st = b.a[FF_STRAIN][L];
  double prol = 1. / ro;
  double rkl = dmax(rk * prol, 0.0);
  double oml = rom * prol;
  double dis2 = dw * dw;
  double arg21 = 2. * sqrt(rkl) / dmax(eps, SST_BSTAR * oml * dw);
  double auxvi = vis / dmax(eps, rom * dis2);
  double arg2 = dmax(arg21, 500. * auxvi);
  double arg4 = 150. * auxvi;
  double fun2 = tanh(arg2 * arg2);
  double fun3 = 1. - tanh(arg4 * arg4 * arg4 * arg4);
  double rmubas = rk / oml;
  double rmumen = SST_A1KLEB * rk / dmax(eps, st * fun2 * fun3);
  double rmutrb = dmin(rmubas, rmumen);
  rmutrb = dmax(rmutrb, frsmut);
  rmutrb = dmin(rmutrb, p.turlim * vis);
  b.a[FF_VIST][L] = rmutrb;
  b.a[FF_EPS2][L] = 1.0 + rmutrb / vis;
}

// ---- CROSKO: cross diffusion into SEPS (interior).  k and omega of every
// stencil cell are RK/RO and REPS/RO as the reference's in-place division
// leaves them; k_rk_roundtrip then applies its RK = (RK/RO)*RO round trip.
__global__ void k_crosko(DevBlock b) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.imax * b.jmax * b.kmax) return;
  int I = t % b.imax + 1, J = (t / b.imax) % b.jmax + 1, K = t / (b.imax * b.jmax) + 1;
  const int IS = b.is, IL = b.il;
  size_t L = ix(b, I, J, K);
  const double *RK = b.a[FF_RK], *RE = b.a[FF_REPS], *RO = b.a[FF_RO];
#define KV(n) (RK[n] * (1. / RO[n]))
#define OV(n) (RE[n] * (1. / RO[n]))
#define LD(s, n) __ldg(b.a[s] + (n))
  double k0 = KV(L), o0 = OV(L);
  double rk1m = LD(FF_A1, L) * (k0 + KV(L - 1)), rk1p = LD(FF_A1, L + 1) * (k0 + KV(L + 1));
  double om1m = LD(FF_A1, L) * (o0 + OV(L - 1)), om1p = LD(FF_A1, L + 1) * (o0 + OV(L + 1));
  double rk2m = LD(FF_A2, L) * (k0 + KV(L - IS)), rk2p = LD(FF_A2, L + IS) * (k0 + KV(L + IS));
  double om2m = LD(FF_A2, L) * (o0 + OV(L - IS)), om2p = LD(FF_A2, L + IS) * (o0 + OV(L + IS));
  double rk3m = LD(FF_A3, L) * (k0 + KV(L - IL)), rk3p = LD(FF_A3, L + IL) * (k0 + KV(L + IL));
  double om3m = LD(FF_A3, L) * (o0 + OV(L - IL)), om3p = LD(FF_A3, L + IL) * (o0 + OV(L + IL));
  double pvol = 0.5 / LD(FF_VOL, L);
#define CSUM(c, p3, m3, p2, m2, p1, m1)                                                                   \
  (pvol * (LD(FF_A3##c, L + IL) * p3 - LD(FF_A3##c, L) * m3 + LD(FF_A2##c, L + IS) * p2 -               \
           LD(FF_A2##c, L) * m2 + LD(FF_A1##c, L + 1) * p1 - LD(FF_A1##c, L) * m1))
  double dkdx = CSUM(XA, rk3p, rk3m, rk2p, rk2m, rk1p, rk1m);
  double dkdy = CSUM(YA, rk3p, rk3m, rk2p, rk2m, rk1p, rk1m);
  double dkdz = CSUM(ZA, rk3p, rk3m, rk2p, rk2m, rk1p, rk1m);
  double dodx = CSUM(XA, om3p, om3m, om2p, om2m, om1p, om1m);
  double dody = CSUM(YA, om3p, om3m, om2p, om2m, om1p, om1m);
  double dodz = CSUM(ZA, om3p, om3m, om2p, om2m, om1p, om1m);
#undef CSUM
#undef LD
#undef KV
#undef OV
  double divdot = dkdx * dodx + dkdy * dody + dkdz * dodz;
  b.a[FF_SEPS][L] = 2.0 * SST_SIGOM2 * RO[L] * divdot / o0;
}

__global__ void k_rk_roundtrip(DevBlock b) {
  size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (size_t)b.ntot) return;
  double ro = b.a[FF_RO][n], prol = 1. / ro;
  b.a[FF_RK][n] = (b.a[FF_RK][n] * prol) * ro;
  b.a[FF_REPS][n] = (b.a[FF_REPS][n] * prol) * ro;
}

// CDMAX of FUN1KO: max(0, CROSSD) over the storage range from cell (1,1,1)
// to (IMAX,JMAX,KMAX); non-negative doubles order like their bit patterns.
__global__ void k_cdmax(DevBlock b, unsigned long long* out) {
  size_t lbeg = ix(b, 1, 1, 1), lend = ix(b, b.imax, b.jmax, b.kmax);
  double m = 0.;
  for (size_t n = lbeg + (size_t)blockIdx.x * blockDim.x + threadIdx.x; n <= lend;
       n += (size_t)gridDim.x * blockDim.x)
    m = dmax(b.a[FF_SEPS][n], m);
  for (int o = 16; o > 0; o >>= 1) m = dmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

__global__ void k_fun1ko(DevBlock b, ff_params p, const unsigned long long* cdmax_bits) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.imax * b.jmax * b.kmax) return;
  int I = t % b.imax + 1, J = (t / b.imax) % b.jmax + 1, K = t / (b.imax * b.jmax) + 1;
  size_t L = ix(b, I, J, K);
  const double eps = 1.e-20;
  double cdmin = 1e-8 * __longlong_as_double((long long)*cdmax_bits);
  double ro = b.a[FF_RO][L], rk = b.a[FF_RK][L], rom = b.a[FF_REPS][L], dw = b.a[FF_DISTW][L];
  double prol = 1. / ro;
  double rkl = dmax(rk * prol, 0.0);
  double oml = rom * prol;
  double dis2 = dw * dw;
  double cdkom = dmax(b.a[FF_SEPS][L], cdmin);
  double arg11 = sqrt(rkl) / dmax(eps, SST_BSTAR * oml * dw);
  double arg12 = 500. * b.a[FF_VIS][L] / dmax(eps, rom * dis2);
  double arg13 = dmax(arg11, arg12);
  double arg14 = 4. * SST_SIGOM2 * rk / dmax(eps, cdkom * dis2);
  double arg1 = dmin(arg13, arg14);
  double f1 = tanh(arg1 * arg1 * arg1 * arg1);
  if (dw < .40559E-7 * sqrt(p.re)) f1 = 1.;
  b.a[FF_FUN1][L] = f1;
}

// MAKE_EPS + PRODKE (Kato-Launder): rows J = 1..JMAX of the interior
// k-planes, i ghosts included, as the reference loops.
__global__ void k_prodke(DevBlock b) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int per = b.jmax * b.is;
  if (t >= per * b.kmax) return;
  int K = t / per + 1, jj = t % per;
  size_t L = (size_t)(K + 1) * b.il + 2 * b.is + jj;
#define A(s) b.a[s][L]
  double s11 = A(FF_S11), s12 = A(FF_S12), s13 = A(FF_S13), s22 = A(FF_S22), s23 = A(FF_S23), s33 = A(FF_S33);
  double strain = s11 * s11 + s12 * s12 + s13 * s13 + s12 * s12 + s22 * s22 + s23 * s23 + s13 * s13 + s23 * s23 +
                  s33 * s33;
  strain = sqrt(2. * strain);
  double trueps = 0.09 * A(FF_REPS) * A(FF_RK) / A(FF_RO);
  double pt = (A(FF_EPS2) - 1.) * A(FF_VIS) * strain * A(FF_OHMI);
  b.a[FF_PTUR][L] = dmin(pt, 20. * trueps);
#undef A
}

// TEMDER of k = RK/RO and omega = REPS/RO (DIVV12 + TEMDER, res3c.f:3994-4006)
// over the TEMDER range of level 1.
__global__ void k_temder_ke(DevBlock b, int level) {
  const int lo = level == 1 ? 0 : 1, g = level == 1 ? 2 : 0;
  int ni = b.imax + g, nj = b.jmax + g;
  int klo = (level == 1 && b.kmax > 1) ? 0 : 1, nk = (level == 1 && b.kmax > 1) ? b.kmax + 2 : b.kmax;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ni * nj * nk) return;
  int I = t % ni + lo, J = (t / ni) % nj + lo, K = t / (ni * nj) + klo;
  const int IS = b.is, IL = b.il;
  size_t L = ix(b, I, J, K);
  const double *RO = b.a[FF_RO];
#define LD(s, n) __ldg(b.a[s] + (n))
  const size_t nb[6] = {L - 1, L + 1, L - (size_t)IS, L + IS, L - (size_t)IL, L + IL};
  const int dslot[6] = {FF_D1, FF_D1, FF_D2, FF_D2, FF_D3, FF_D3};
  double w1[6], w2[6];
#pragma unroll
  for (int q = 0; q < 6; q++) {
    double dl = LD(dslot[q], L);
    w1[q] = 2.0 * (dl / (dl + LD(dslot[q], nb[q])));
    w2[q] = 2.0 - w1[q];
  }
  double pvol = .5 / LD(FF_VOL, L);
#pragma unroll
  for (int f = 0; f < 2; f++) {
    const double* PH = b.a[f == 0 ? FF_RK : FF_REPS];
    double ph0 = PH[L] / RO[L];
    double t_[6];
#pragma unroll
    for (int q = 0; q < 6; q++) t_[q] = w2[q] * ph0 + w1[q] * (PH[nb[q]] / RO[nb[q]]);
    // t_: 1m, 1p, 2m, 2p, 3m, 3p
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const int x1 = FF_A1XA + c, x2 = FF_A2XA + c, x3 = FF_A3XA + c;
      double g = pvol * (LD(FF_A3, L + IL) * LD(x3, L + IL) * t_[5] - LD(FF_A3, L) * LD(x3, L) * t_[4] +
                         LD(FF_A2, L + IS) * LD(x2, L + IS) * t_[3] - LD(FF_A2, L) * LD(x2, L) * t_[2] +
                         LD(FF_A1, L + 1) * LD(x1, L + 1) * t_[1] - LD(FF_A1, L) * LD(x1, L) * t_[0]);
      b.a[(f == 0 ? FF_DKDX : FF_DEDX) + c][L] = g;
    }
  }
#undef LD
}

// ---- face fluxes of the seven equations ---------------------------------

// FLUXKE base3c.f:4753-5120 with k and omega (UROT = 0); q[v][m], v = ro, u,
// v, w, p, rk, reps; m = cells I-2S..I+S.  Adds to f[7].  T = float for a
// coarse face pass in FP32.
// DD: XXTRAA over the extents dd (XXTRAL), with INTEM for k and omega too
// (base3c.f:4861-4862).
template <typename T, bool DD = false>
FF_DI void roe_flux_ke(const T q[7][4], T nx, T ny, T nz, T area, int intem, int intet, const ff_params& p,
                       T c_r, T c_l, const T cr[4], const T cl2[4], T f[7], const T* dd = nullptr) {
  T roip, roim, rmip, rmim, rnip, rnim, rwip, rwim, ppi, pmi, rkip, rkim, reip, reim;
  muscl<DD>(q[0], dd, intem, roip, roim);
  muscl<DD>(q[1], dd, intem, rmip, rmim);
  muscl<DD>(q[2], dd, intem, rnip, rnim);
  muscl<DD>(q[3], dd, intem, rwip, rwim);
  muscl<DD>(q[4], dd, intem, ppi, pmi);
  muscl<DD>(q[5], dd, DD ? intem : intet, rkip, rkim);
  muscl<DD>(q[6], dd, DD ? intem : intet, reip, reim);
  roip = dmax(T(0.001) * T(p.frsden), roip);
  ppi = dmax(T(0.001) * T(p.frspre), ppi);
  roim = dmax(T(0.001) * T(p.frsden), roim);
  pmi = dmax(T(0.001) * T(p.frspre), pmi);
  const T rgm1 = rcp(T(p.gamma) - T(1.)), e0 = T(p.e0ref);
  const T ypror = rcp(roip), yprol = rcp(roim);
  T eip = ppi * rgm1 * ypror - e0;
  T eim = pmi * rgm1 * yprol - e0;
  T elr = ppi * rgm1 * yprol - e0;
  T erl = pmi * rgm1 * ypror - e0;
  T ypro1 = rcp(cr[2]), ypro2 = rcp(cl2[2]);
  T rdh1 = rcp(cr[1]), rdh2 = rcp(cl2[1]);
  T dedph = T(0.5) * ((-cr[0] * rdh1 - ypro1) + (-cl2[0] * rdh2 - ypro2));
  T dedrh = T(0.5) * ((rdh1 + cr[3] * (ypro1 * ypro1)) + (rdh2 + cl2[3] * (ypro2 * ypro2)));
  {
    T dpp = T(2.) * (ppi - pmi), drr = T(2.) * (roip - roim);
    if (fabs(dpp) >= T(1.e-2) * (ppi + pmi)) dedph = (eip + elr - eim - erl) / dpp;
    if (fabs(drr) >= T(1.e-2) * (roip + roim)) dedrh = (eip + erl - eim - elr) / drr;
  }
  // normal velocities; the tangential parts as Cartesian vectors (the
  // SURFVECTS tangents t1, t2 only ever appear as t1 t1' + t2 t2' = I - n n')
  T ur = nx * rmip + ny * rnip + nz * rwip;
  T ul = nx * rmim + ny * rnim + nz * rwim;
  const T txr = rmip - ur * nx, tyr = rnip - ur * ny, tzr = rwip - ur * nz;
  const T txl = rmim - ul * nx, tyl = rnim - ul * ny, tzl = rwim - ul * nz;
  T rkipi = dmax(T(0.001) * T(p.rklim), rkip), reipi = dmax(T(0.001) * T(p.epslim), reip);
  T rkimi = dmax(T(0.001) * T(p.rklim), rkim), reimi = dmax(T(0.001) * T(p.epslim), reim);
  T rkr = rkipi * ypror, rkl = rkimi * yprol;
  T eir = eip + T(.5) * (rmip * rmip + rnip * rnip + rwip * rwip) + rkr;
  T eil = eim + T(.5) * (rmim * rmim + rnim * rnim + rwim * rwim) + rkl;
  T pr = ppi, pl = pmi, pkr = T(.6667) * rkipi, pkl = T(.6667) * rkimi;
  T epsr = reipi * ypror, epsl = reimi * yprol;
  T hr = eir + pr * ypror, hl = eil + yprol * pl;
  T rohat = sqrt(roip * roim), yproh = rcp(rohat);
  T sqrl = rcp(roim + rohat), cql = roim * sqrl, cqr = T(1.) - cql;
  T uhat = cqr * ur + cql * ul;
  const T thx = cqr * txr + cql * txl, thy = cqr * tyr + cql * tyl, thz = cqr * tzr + cql * tzl;
  T hhat = cqr * hr + cql * hl, ehat = cqr * eip + cql * eim;
  T rkhat = cqr * rkr + cql * rkl, epshat = cqr * epsr + cql * epsl;
  T phat = rohat * (hhat - ehat - T(.5) * (uhat * uhat + thx * thx + thy * thy + thz * thz) - rkhat);
  phat = dmin(dmax(pr, pl), phat);
  phat = dmax(dmin(pr, pl), phat);
  T drdhh = rcp(dedrh - phat * (yproh * yproh));
  T drdph = -drdhh * (dedph + yproh);
  T xturb = T(1.) + T(.6667) * rkhat * yproh * drdph;
  T chat2 = xturb / (drdhh * yproh + drdph);
  T cmin = dmin(c_r, c_l), cmax = dmax(c_r, c_l);
  chat2 = dmin(cmax * cmax, chat2);
  chat2 = dmax(cmin * cmin, chat2);
  T chat = sqrt(chat2);
  T pdpde = dedph;
  T dro = roip - roim, du = ur - ul, dk = rkr - rkl;
  T dp = pr - pl + T(.6667) * (rkhat * dro + rohat * dk);
  T pchat2 = rcp(chat * chat);
  T alfa1 = T(.5) * (dp + rohat * chat * du) * pchat2;
  T alfa2 = T(.5) * (dp - rohat * chat * du) * pchat2;
  T alfa3 = dro - dp * pchat2;
  T alfa6 = rohat * dk, alfa7 = rohat * (epsr - epsl);
  T rl1h = uhat + chat, rl2h = uhat - chat, rl3h = uhat;
  T rl1 = fabs(rl1h), rl2 = fabs(rl2h), rl3 = fabs(rl3h);
  if (p.entropy_fix) {
    T e22;
    e22 = T(4.) * dmax(dmax(T(1.e-10), rl1h - (ul + c_l)), (ur + c_r) - rl1h);
    if (rl1 <= e22) rl1 = T(.5) * (rl1h * rl1h + e22 * e22) / e22;
    e22 = T(4.) * dmax(dmax(T(1.e-10), rl2h - (ul - c_l)), (ur - c_r) - rl2h);
    if (rl2 <= e22) rl2 = T(.5) * (rl2h * rl2h + e22 * e22) / e22;
    e22 = T(4.) * dmax(dmax(T(1.e-10), rl3h - ul), ur - rl3h);
    if (rl3 <= e22) rl3 = T(.5) * (rl3h * rl3h + e22 * e22) / e22;
  }
  T roucr = roip * ur, roucl = roim * ul;
  T damp = rl1 * alfa1 + rl2 * alfa2 + rl3 * alfa3;
  T ha = T(.5) * area;
  T f1 = ha * (roucr + roucl - damp);
  T f2 = ha * (roucr * ur + pr + pkr + roucl * ul + pl + pkl - (damp * uhat + (rl1 * alfa1 - rl2 * alfa2) * chat));
  // the tangential momentum flux as a vector (f3, f4 of the reference's
  // rotated frame) and its jump term of the energy flux
  const T rr = rl3 * rohat;
  const T ftx = ha * (roucr * txr + roucl * txl - damp * thx - rr * (txr - txl));
  const T fty = ha * (roucr * tyr + roucl * tyl - damp * thy - rr * (tyr - tyl));
  const T ftz = ha * (roucr * tzr + roucl * tzl - damp * thz - rr * (tzr - tzl));
  const T tj = rr * ((txr - txl) * thx + (tyr - tyl) * thy + (tzr - tzl) * thz);
  T f5 = ha * (roucr * (hr + pkr * ypror) + roucl * (hl + pkl * yprol) - damp * hhat -
               ((rl1 * alfa1 - rl2 * alfa2) * uhat * chat - rl3 * alfa3 * rohat * (chat * chat) * pdpde + tj) +
               rl3 * alfa6 * (T(1.) - T(.6667) * rohat * pdpde));
  T f6 = ha * (roucr * rkr + roucl * rkl - damp * rkhat - rl3 * alfa6);
  T f7 = ha * (roucr * epsr + roucl * epsl - damp * epshat - rl3 * alfa7);
  f[0] += f1;
  f[1] += nx * f2 + ftx;
  f[2] += ny * f2 + fty;
  f[3] += nz * f2 + ftz;
  f[4] += f5;
  f[5] += f6;
  f[6] += f7;
}

// FLKEBL: k and omega diffusion of one face (I = high-side cell).
FF_DI void flkebl_face(const DevBlock& b, size_t I, int S, int dir, const FaceGeom& g, double& frk, double& feps) {
#define LD(s, n) __ldg(b.a[s] + (n))
  size_t M = I - S;
  double f1 = LD(FF_FUN1, I), onemf1 = dmax(0.0, 1.0 - f1);
  double psigk = f1 * SST_SIGRK1 + onemf1 * SST_SIGRK2;
  double psige = f1 * SST_SIGOM1 + onemf1 * SST_SIGOM2;
  const double w1 = g.w1, w2 = g.w2;
  double dkdxi = 0.5 * (w2 * LD(FF_DKDX, I) + w1 * LD(FF_DKDX, M));
  double dkdyi = 0.5 * (w2 * LD(FF_DKDY, I) + w1 * LD(FF_DKDY, M));
  double dkdzi = 0.5 * (w2 * LD(FF_DKDZ, I) + w1 * LD(FF_DKDZ, M));
  double dedxi = 0.5 * (w2 * LD(FF_DEDX, I) + w1 * LD(FF_DEDX, M));
  double dedyi = 0.5 * (w2 * LD(FF_DEDY, I) + w1 * LD(FF_DEDY, M));
  double dedzi = 0.5 * (w2 * LD(FF_DEDZ, I) + w1 * LD(FF_DEDZ, M));
  const double sxi = g.sx, syi = g.sy, szi = g.sz, rslen = g.rslen;
  const double nx = g.nx, ny = g.ny, nz = g.nz;
  double alfa = dmax(sxi * nx + syi * ny + szi * nz, 0.);
  double rmut2 = LD(FF_VIST, I) + LD(FF_VIST, M);
  double vv = LD(FF_VIS, I) + LD(FF_VIS, M), area = g.area;
  double surfk = 0.5 * area * (vv + rmut2 * psigk);
  double surfep = 0.5 * area * (vv + rmut2 * psige);
  double ypro1 = rcp(LD(FF_RO, I)), ypro2 = rcp(LD(FF_RO, M));
  frk = -surfk * (alfa * (LD(FF_RK, I) * ypro1 - LD(FF_RK, M) * ypro2) * rslen + dkdxi * (nx - alfa * sxi) +
                  dkdyi * (ny - alfa * syi) + dkdzi * (nz - alfa * szi));
  feps = -surfep * (alfa * (LD(FF_REPS, I) * ypro1 - LD(FF_REPS, M) * ypro2) * rslen + dedxi * (nx - alfa * sxi) +
                    dedyi * (ny - alfa * syi) + dedzi * (nz - alfa * szi));
#undef LD
}

// FLUDKE base3c.f:5547: thin-layer k and omega diffusion (coarse levels).
template <typename T>
FF_DI void fludke_face(const DevBlock& b, size_t I, int S, int dir, T& frk, T& feps) {
#define LD(s, n) T(__ldg(b.a[s] + (n)))
  size_t M = I - S;
  T f1 = LD(FF_FUN1, I), onemf1 = dmax(T(0.0), T(1.0) - f1);
  T psigk = f1 * T(SST_SIGRK1) + onemf1 * T(SST_SIGRK2);
  T psige = f1 * T(SST_SIGOM1) + onemf1 * T(SST_SIGOM2);
  T area = LD(FF_A1 + 4 * (dir - 1), I);
  T ypd2 = area / (LD(FF_VOL, I) + LD(FF_VOL, M));
  T surg = -area * ypd2;
  T rmut2 = (LD(FF_EPS2, I) - T(1.)) * LD(FF_VIS, I) + (LD(FF_EPS2, M) - T(1.)) * LD(FF_VIS, M);
  T vv = LD(FF_VIS, I) + LD(FF_VIS, M);
  T ypro1 = rcp(LD(FF_RO, I)), ypro2 = rcp(LD(FF_RO, M));
  frk = surg * (vv + rmut2 * psigk) * (LD(FF_RK, I) * ypro1 - LD(FF_RK, M) * ypro2);
  feps = surg * (vv + rmut2 * psige) * (LD(FF_REPS, I) * ypro1 - LD(FF_REPS, M) * ypro2);
#undef LD
}

// BOTSKE with k and omega (smooth wall, IDIS=2): seven wall fluxes (T =
// float for a coarse face pass in FP32).
template <typename T>
FF_DI void wall_flux_ke(const DevBlock& b, const ff_params& p, size_t II, int S, int idir, int dir, int iheat,
                        int intem, T f[7]) {
#define LD(s, n) T(__ldg(b.a[s] + (n)))
  T rc1 = intem == 6 ? T(1.) : T(1.5), rc2 = rc1 - T(1.);
  const T prs = T(p.pr) / T(p.prt), ymr = T(.166666667), eps = T(1.e-3);
  int lstrid = S * idir;
  size_t II2 = II + lstrid, IF1 = idir == 1 ? II : II + S;
  int ihfl = (iheat == 2 || iheat >= 12) ? 1 : 0;
  int iht = (iheat == 0 || iheat == 15) ? 0 : 1;
  const int ao = 4 * (dir - 1);
  T a_f = LD(FF_A1 + ao, IF1);
  T dist = (a_f + LD(FF_A1 + ao, IF1 + lstrid)) / LD(FF_VOL, II);
  T surg = -dist * ymr;
  T visb = dmax(T(0.01) * T(p.frsvis), rc1 * LD(FF_VIS, II) - rc2 * LD(FF_VIS, II2));
  T chsb = dmax(eps, rc1 * LD(FF_CH, II) - rc2 * LD(FF_CH, II2));
  T straib = dmax(eps, rc1 * LD(FF_STRAIN, II) - rc2 * LD(FF_STRAIN, II2));
  // PB = YP1*PB1 + YP4*PB4 (base3c.f:6304-6315, 6487): the extrapolated
  // pressure, or its difference from FRSPRE for KT (IFLUX=7)
  T pb1 = p.flux == FF_FLUX_KT
              ? dmax(T(-.99) * T(p.frspre), rc1 * LD(FF_PDIFF, II) - rc2 * LD(FF_PDIFF, II2))
              : dmax(T(0.01) * T(p.frspre), rc1 * LD(FF_P, II) - rc2 * LD(FF_P, II2));
  T rob = dmax(T(0.001) * T(p.frsden), rc1 * LD(FF_RO, II) - rc2 * LD(FF_RO, II2));
  T surf = surg * visb;
  T surfe = surg * (prs * T(0.) / visb + T(1.)) * chsb;
  T rapub = T(1.0E-20);
  T surfrk = surg * (T(1.0) + T(SST_SIGRK1) * rapub) * visb;
  T surfep = surg * (T(1.0) + T(SST_SIGOM1) * rapub) * visb;
  T ypro1 = rcp(LD(FF_RO, II)), ypro2 = rcp(LD(FF_RO, II2));
  T rnub = visb / rob;
  T plusfc = sqrt(rnub * straib) / rnub;
  T yplus1 = T(2.0) * plusfc / dist;
  T skpmin = dmax(dmin(T(2.4) * pow(yplus1, T(0.85)), T(8.0)), T(1.e-3));
  T skplus = dmax(T(0.0) * plusfc, skpmin);
  T pskp = T(1.0) / skplus;
  T omsurf = straib * dmax(T(2500.0) * pskp * pskp, T(100.0) * pskp);
  T tempb = dmax(T(0.01) * T(p.frstem), rc1 * LD(FF_TEMP, II) - rc2 * LD(FF_TEMP, II2));
  T tsurf = iheat == 3 ? tempb : T(p.frstem);
  T cvii = T(iht * idir) * (T(9.000) * LD(FF_TEMP, II) - T(1.000) * LD(FF_TEMP, II2) - T(8.) * tsurf);
  T uvii = T(idir) * (T(9.000) * LD(FF_U, II) - T(1.000) * LD(FF_U, II2));
  T vvii = T(idir) * (T(9.000) * LD(FF_V, II) - T(1.000) * LD(FF_V, II2));
  T wvii = T(idir) * (T(9.000) * LD(FF_W, II) - T(1.000) * LD(FF_W, II2));
  T ax = LD(FF_A1XA + ao, IF1), ay = LD(FF_A1YA + ao, IF1), az = LD(FF_A1ZA + ao, IF1);
  T duc = T(.33333) * (ay * vvii + az * wvii + ax * uvii);
  T f2v = surf * (uvii + ax * duc);
  T f3v = surf * (vvii + ay * duc);
  T f4v = surf * (wvii + az * duc);
  T f5v = T(1 - ihfl) * surfe * cvii;
  T evii = T(idir) * (T(9.0) * LD(FF_REPS, II) * ypro1 - T(1.0) * LD(FF_REPS, II2) * ypro2 - T(8.) * omsurf);
  T rkii = T(idir) * (T(9.000) * LD(FF_RK, II) * ypro1 - T(1.000) * LD(FF_RK, II2) * ypro2);
  rkii = T(idir) * dmax(T(idir) * rkii, T(0.0));
  T f6v = surfrk * rkii;
  T f7v = surfep * evii;
  f[0] = T(0.);
  f[1] = a_f * (ax * pb1 + f2v);
  f[2] = a_f * (ay * pb1 + f3v);
  f[3] = a_f * (az * pb1 + f4v);
  f[4] = a_f * (f5v + f6v);
  f[5] = a_f * f6v;
  f[6] = a_f * f7v;
#undef LD
}

// Flux of one face with k and omega (FLXCYC order: FLKEBL, SETV12, FLUXBL,
// FLUXKE; BOTSKE on walls).
// sq (optional): the seven MUSCL variables of cell L in a staged stencil,
// variable v at sq[v * vs], the cells along the face normal es apart.
template <typename T, bool ALT = true>
FF_DI void face_flux_ke(const DevBlock& b, const ff_params& p, int dir, size_t L, int m, int t1, int t2,
                        int level, T f[7], const double* sq = nullptr, int es = 0, int vs = 0) {
  const int S = dir == 1 ? 1 : (dir == 2 ? b.is : b.il);
  const int nmax = dir == 1 ? b.imax : (dir == 2 ? b.jmax : b.kmax);
  int intem = dir == 1 ? p.interi : (dir == 2 ? p.interj : p.interk);
  if (level > 1) intem = p.coarse_inter;
  int intet = (intem > -5 && intem < 5) ? 1 : intem;
  if (m == 1 || m == nmax + 1) {
    int iface = m == 1 ? dir : dir + 3;
    for (int ip = 0; ip < b.npatch; ip++) {
      const ff_patch& pa = b.patch[ip];
      if (pa.iface != iface || pa.ityp < 8 || pa.ityp > 10) continue;
      if (t1 < pa.r1a || t1 > pa.r1b || t2 < pa.r2a || t2 > pa.r2b) continue;
      int idir = m == 1 ? 1 : -1;
      size_t II = m == 1 ? L : L - S;
      wall_flux_ke(b, p, II, S, idir, dir, pa.iheat, intem, f);
      return;
    }
  }
  const int idi = dir == 1 ? p.idi1 : (dir == 2 ? p.idi2 : p.idi3);
  // The inviscid flux first, into f from zero; the viscous flux after it,
  // when the MUSCL stencil is no longer live.  The reference adds the
  // inviscid flux to the viscous one (F = Fv + Fi per component), and one
  // addition is the same either way round.
#pragma unroll
  for (int v = 0; v < 7; v++) f[v] = T(0.);
  bool alt = false;
  if constexpr (ALT && sizeof(T) == sizeof(double)) {
    if (p.flux != FF_FLUX_ROE) {   // KT or H-CUSP (RESIKE res3c.f:7017-7036)
      alt_flux<7>(b, p, dir, L, S, intem, intet, f);
      alt = true;
    }
  }
  if (!alt) {
    T q[7][4];
    const int sl[7] = {FF_RO, FF_U, FF_V, FF_W, FF_P, FF_RK, FF_REPS};
    if (sq) {
#pragma unroll
      for (int v = 0; v < 7; v++) {
        const double* a = sq + v * vs;
        q[v][0] = T(a[-2 * es]); q[v][1] = T(a[-es]); q[v][2] = T(a[0]); q[v][3] = T(a[es]);
      }
    } else {
#pragma unroll
      for (int v = 0; v < 7; v++) {
        const double* a = b.a[sl[v]];
        q[v][0] = T(__ldg(a + L - 2 * S)); q[v][1] = T(__ldg(a + L - S)); q[v][2] = T(__ldg(a + L));
        q[v][3] = T(__ldg(a + L + S));
      }
    }
    size_t L2 = dir == 3 ? L : L - S;
    T cr[4] = {T(__ldg(b.a[FF_DRDP] + L)), T(__ldg(b.a[FF_DRDH] + L)), q[0][2], q[4][2]};
    // RO and P of cell L2 (L itself for k faces) are in the stencil
    T cl[4] = {T(__ldg(b.a[FF_DRDP] + L2)), T(__ldg(b.a[FF_DRDH] + L2)), dir == 3 ? q[0][2] : q[0][1],
               dir == 3 ? q[4][2] : q[4][1]};
    const int ao = 4 * (dir - 1);
    bool done = false;
    if constexpr (ALT && sizeof(T) == sizeof(double)) {
      if (p.xxtral) {   // XXTRAA over the cells' extents along the normal
        const double* D = b.a[FF_D1 + dir - 1];
        const double dd[4] = {__ldg(D + L - 2 * S), __ldg(D + L - S), __ldg(D + L), __ldg(D + L + S)};
        roe_flux_ke<double, true>(q, __ldg(b.a[FF_A1XA + ao] + L), __ldg(b.a[FF_A1YA + ao] + L),
                                  __ldg(b.a[FF_A1ZA + ao] + L), __ldg(b.a[FF_A1 + ao] + L), intem, intet, p,
                                  __ldg(b.a[FF_C] + L), __ldg(b.a[FF_C] + L - S), cr, cl, f, dd);
        done = true;
      }
    }
    if (!done)
      roe_flux_ke(q, T(__ldg(b.a[FF_A1XA + ao] + L)), T(__ldg(b.a[FF_A1YA + ao] + L)),
                  T(__ldg(b.a[FF_A1ZA + ao] + L)), T(__ldg(b.a[FF_A1 + ao] + L)), intem, intet, p,
                  T(__ldg(b.a[FF_C] + L)), T(__ldg(b.a[FF_C] + L - S)), cr, cl, f);
  }
  if (m <= min(idi, nmax + 1)) {
    T frk, feps, fv[5], f4;
    bool full = false;
    if constexpr (sizeof(T) == sizeof(double)) {
      if (level == 1 && p.fullns) {   // FLKEBL, SETV12, FLUXBL
        const FaceGeom g = face_geom(b, L, S, dir);
        flkebl_face(b, L, S, dir, g, frk, feps);
        visc_flux(b, p, L, S, dir, g, fv);
        f4 = frk + fv[4];
        full = true;
      }
    }
    if (!full) {                      // FLUDKE, FLUXDO
      fludke_face(b, L, S, dir, frk, feps);
      visc_flux_thin(b, p, L, S, dir, fv, frk);
      f4 = fv[4];
    }
    f[1] = fv[1] + f[1]; f[2] = fv[2] + f[2]; f[3] = fv[3] + f[3];
    f[4] = f4 + f[4]; f[5] = frk + f[5]; f[6] = feps + f[6];
  }
  if constexpr (ALT && sizeof(T) == sizeof(double)) {   // JAMESON after the viscous and Roe fluxes
    if (!alt && level == 1 && (p.rjk2 > 0. || p.rjk4 > 0.)) jst_flux(b, p, L, S, f);
  }
}

// RESIKE face cycles + SWEEPK for a 32x4x4 tile (k, i, j, then 1/VOL).
// NT threads per CTA (128, 256 or 512): each thread sums the faces of
// CPT = 512 / NT cells of the 32x4x4 tile (a k column of CPT cells); the
// register budget gives RES_MIN_CTAS * 128 threads per SM at every NT.
template <int NT>
__global__ void __launch_bounds__(NT, RES_MIN_CTAS * 128 / NT) k_residual_sst(DevBlock b, ff_params p, int level) {
  constexpr int CPT = TI * TJ * TK / NT;
  constexpr int NF = TI * (TJ + 1) * TK, NC = TI * TJ * TK;
  // one direction's faces (at most 640) x 7, then the cells' running sums
  // (in shared memory, not registers: the face flux needs the registers)
  extern __shared__ double res_smem[];
  double(*sF)[NF] = reinterpret_cast<double(*)[NF]>(res_smem);
  double(*sAcc)[NC] = reinterpret_cast<double(*)[NC]>(res_smem + 7 * NF);
  const int tid = threadIdx.x;
  const int i0 = blockIdx.x * TI, j0 = blockIdx.y * TJ, k0 = blockIdx.z * TK;
  const int ci = tid % TI, cj = (tid / TI) % TJ, ck0 = (tid / (TI * TJ)) * CPT;
#pragma unroll
  for (int c = 0; c < CPT; c++)
#pragma unroll
    for (int v = 0; v < 7; v++) sAcc[v][ci + TI * (cj + TJ * (ck0 + c))] = 0.;
  // the directions in SWEEP order (k, i, j; RESIKE res3c.f:3423); one call site of the
  // face flux keeps a single copy of its code in the instruction stream
#pragma unroll 1
  for (int pass = 0; pass < 3; pass++) {
    const int dir = pass == 0 ? 3 : pass;   // k, i, j
    const int ni = TI + (dir == 1), nj = TJ + (dir == 2), nk = TK + (dir == 3);
    for (int f = tid; f < ni * nj * nk; f += blockDim.x) {
      const int fi = f % ni, fj = (f / ni) % nj, fk = f / (ni * nj);
      const int I = i0 + fi + 1, J = j0 + fj + 1, K = k0 + fk + 1;
      if (I > b.imax + (dir == 1) || J > b.jmax + (dir == 2) || K > b.kmax + (dir == 3)) continue;
      const int m = dir == 1 ? I : (dir == 2 ? J : K);
      const int t1 = dir == 1 ? J : I, t2 = dir == 3 ? J : K;
      double fl[7];
      face_flux_ke(b, p, dir, ix(b, I, J, K), m, t1, t2, level, fl);
#pragma unroll
      for (int v = 0; v < 7; v++) sF[v][f] = fl[v];
    }
    __syncthreads();
    const int fs = dir == 1 ? 1 : (dir == 2 ? ni : ni * nj);   // low face -> high face of a cell
#pragma unroll
    for (int c = 0; c < CPT; c++) {
      const int f0 = ci + ni * (cj + nj * (ck0 + c));
      const int I = i0 + ci + 1, J = j0 + cj + 1, K = k0 + ck0 + c + 1;
      if (I > b.imax || J > b.jmax || K > b.kmax) continue;
      const int ca = ci + TI * (cj + TJ * (ck0 + c));
      if (pass < 2) {
#pragma unroll
        for (int v = 0; v < 7; v++) sAcc[v][ca] = sAcc[v][ca] - (sF[v][f0 + fs] - sF[v][f0]);
      } else {   // last direction, then 1/VOL (SWEEP IDO = 1)
        const size_t n = ix(b, I, J, K);
        const double rv = 1. / __ldg(b.a[FF_VOL] + n);
#pragma unroll
        for (int v = 0; v < 7; v++) b.a[FF_DRO + v][n] = (sAcc[v][ca] - (sF[v][f0 + fs] - sF[v][f0])) * rv;
      }
    }
    __syncthreads();
  }
}

// RESIDU/RESIKE for a 32x4x4 tile with all three directions' faces in one
// work list: the k, i and j faces (640 + 528 + 640) are computed by NT
// threads into one shared-memory face buffer with a single barrier, then
// each cell sums its six faces in the reference order (k, i, j, then
// 1/VOL, SWEEP res3c.f:992 / SWEEPK res3c.f:1342).  Against one barrier per
// direction this balances the face work over the threads (8 rounds for the
// 1808 faces at 256 threads, against 3 + 3 + 3) and drops two barriers.
//
// The tile shape (TI_ x TJ_ x TK_ cells, 512 of them) is a template
// parameter: 32x4x4, 16x8x4 and 8x8x8 trade i-direction coalescing against
// the faces computed per cell (3.53, 3.44, 3.38); the autotuner picks one
// per block shape.
//
// STAGE: the MUSCL variables (RO, U, V, W, P(, RK, REPS)) of the tile's
// cells and of the two cells beyond each of its six faces are first copied
// into shared memory (a box of (TI+4)(TJ+4)(TK+4) cells of which the
// tile's three cross arms are filled), and every face reads its four-cell
// stencil from there instead of global memory.
//
// FT = float: the face fluxes of a coarse level in FP32 (the cells' sums
// of their faces and the result stay FP64).
template <int NV, int NT, int TI_, int TJ_, int TK_, bool STAGE = false, typename FT = double, bool ALT = false>
FF_DI void residual_tile(const DevBlock& b, const ff_params& p, int level, int i0, int j0, int k0,
                         double* res_smem) {
  constexpr int TI = TI_, TJ = TJ_, TK = TK_;
  constexpr int NFK = TI * TJ * (TK + 1), NFI = (TI + 1) * TJ * TK, NFJ = TI * (TJ + 1) * TK;
  constexpr int NFT = NFK + NFI + NFJ, NC = TI * TJ * TK;
  constexpr int BI = TI + 4, BJ = TJ + 4, BOX = BI * BJ * (TK + 4);
  double(*sF)[NFT] = reinterpret_cast<double(*)[NFT]>(res_smem);
  double* sQ = res_smem + NV * NFT;
  const int tid = threadIdx.x;
  if constexpr (STAGE) {
    const int sl[7] = {FF_RO, FF_U, FF_V, FF_W, FF_P, FF_RK, FF_REPS};
    for (int e = tid; e < BOX; e += NT) {
      const int ci = e % BI - 2, cj = (e / BI) % BJ - 2, ck = e / (BI * BJ) - 2;
      const int out = (ci < 0 || ci >= TI) + (cj < 0 || cj >= TJ) + (ck < 0 || ck >= TK);
      const int I = i0 + ci + 1, J = j0 + cj + 1, K = k0 + ck + 1;
      if (out > 1 || I < -1 || I > b.imax + 2 || J < -1 || J > b.jmax + 2 || K < -1 || K > b.kmax + 2) continue;
      const size_t n = ix(b, I, J, K);
#pragma unroll
      for (int v = 0; v < NV; v++) sQ[v * BOX + e] = __ldg(b.a[sl[v]] + n);
    }
    __syncthreads();
  }
  for (int f = tid; f < NFT; f += NT) {
    int dir, l, ni, nj;
    if (f < NFK) { dir = 3; l = f; ni = TI; nj = TJ; }
    else if (f < NFK + NFI) { dir = 1; l = f - NFK; ni = TI + 1; nj = TJ; }
    else { dir = 2; l = f - NFK - NFI; ni = TI; nj = TJ + 1; }
    const int fi = l % ni, fj = (l / ni) % nj, fk = l / (ni * nj);
    const int I = i0 + fi + 1, J = j0 + fj + 1, K = k0 + fk + 1;
    if (I > b.imax + (dir == 1) || J > b.jmax + (dir == 2) || K > b.kmax + (dir == 3)) continue;
    const int m = dir == 1 ? I : (dir == 2 ? J : K);
    const int t1 = dir == 1 ? J : I, t2 = dir == 3 ? J : K;
    FT fl[NV];
    const double* sq = nullptr;
    int es = 0;
    if constexpr (STAGE) {   // the face's high cell in the staged box
      sq = sQ + ((fk + 2) * BJ + (fj + 2)) * BI + (fi + 2);
      es = dir == 1 ? 1 : (dir == 2 ? BI : BI * BJ);
    }
    if constexpr (NV == 7) face_flux_ke<FT, ALT>(b, p, dir, ix(b, I, J, K), m, t1, t2, level, fl, sq, es, BOX);
    else face_flux<FT, ALT>(b, p, dir, ix(b, I, J, K), m, t1, t2, level, fl, sq, es, BOX);
#pragma unroll
    for (int v = 0; v < NV; v++) sF[v][f] = double(fl[v]);
  }
  __syncthreads();
  for (int c = tid; c < NC; c += NT) {
    const int ci = c % TI, cj = (c / TI) % TJ, ck = c / (TI * TJ);
    const int I = i0 + ci + 1, J = j0 + cj + 1, K = k0 + ck + 1;
    if (I > b.imax || J > b.jmax || K > b.kmax) continue;
    const int fk0 = ci + TI * (cj + TJ * ck);                       // face K-1/2; K+1/2 at + TI*TJ
    const int fi0 = NFK + ci + (TI + 1) * (cj + TJ * ck);          // face I-1/2; I+1/2 at + 1
    const int fj0 = NFK + NFI + ci + TI * (cj + (TJ + 1) * ck);    // face J-1/2; J+1/2 at + TI
    const size_t n = ix(b, I, J, K);
    const double rv = 1. / __ldg(b.a[FF_VOL] + n);
#pragma unroll
    for (int v = 0; v < NV; v++) {
      double acc = 0. - (sF[v][fk0 + TI * TJ] - sF[v][fk0]);
      acc = acc - (sF[v][fi0 + 1] - sF[v][fi0]);
      b.a[FF_DRO + v][n] = (acc - (sF[v][fj0 + TI] - sF[v][fj0])) * rv;
    }
  }
}

// ALT: the selectable variants compiled in (the other IFLUX schemes, XXTRAA,
// JAMESON); the plain Roe/XXTRAP forms leave them out.
template <int NV, int NT, int TI_ = TI, int TJ_ = TJ, int TK_ = TK, bool STAGE = false, typename FT = double,
          bool ALT = false>
__global__ void __launch_bounds__(NT, RES_MIN_CTAS * 128 / NT) k_residual_fused(DevBlock b, ff_params p, int level) {
  extern __shared__ double res_smem[];
  residual_tile<NV, NT, TI_, TJ_, TK_, STAGE, FT, ALT>(b, p, level, blockIdx.x * TI_, blockIdx.y * TJ_,
                                                       blockIdx.z * TK_, res_smem);
}

// Whether a block's residual on `level` needs the selectable variants.
inline bool residual_alt(const ff_params& p, int level) {
  return p.flux != FF_FLUX_ROE || p.xxtral || (level == 1 && (p.rjk2 > 0. || p.rjk4 > 0.));
}

// The same residual for several blocks in one launch: a block work-list of
// tiles (north-star batching: one launch per stage over all blocks of
// uneven size).  CTA t takes tile t of the concatenated lists; blocks and
// their parameters travel in the kernel's parameter space.
constexpr int RB_MAX = 16;
struct ResBatch {
  int nblk;
  int tile0[RB_MAX + 1];   // first tile of each block, and the total
  int ntx[RB_MAX], nty[RB_MAX];
  DevBlock b[RB_MAX];
  ff_params p[RB_MAX];
};

template <int NV, int NT, int TI_, int TJ_, int TK_, bool STAGE = false>
__global__ void __launch_bounds__(NT, RES_MIN_CTAS * 128 / NT)
    k_residual_batch(const __grid_constant__ ResBatch rb, int level) {
  extern __shared__ double res_smem[];
  const int t = blockIdx.x;
  int bi = 0;
  while (bi + 1 < rb.nblk && t >= rb.tile0[bi + 1]) bi++;
  const int l = t - rb.tile0[bi], nx = rb.ntx[bi], ny = rb.nty[bi];
  const int ti = l % nx, tj = (l / nx) % ny, tk = l / (nx * ny);
  residual_tile<NV, NT, TI_, TJ_, TK_, STAGE>(rb.b[bi], rb.p[bi], level, ti * TI_, tj * TJ_, tk * TK_, res_smem);
}

inline size_t residual_fused_smem(int nv, int ti = TI, int tj = TJ, int tk = TK, bool stage = false) {
  const size_t faces = (size_t)nv * (ti * tj * (tk + 1) + (ti + 1) * tj * tk + ti * (tj + 1) * tk);
  const size_t box = stage ? (size_t)nv * (ti + 4) * (tj + 4) * (tk + 4) : 0;
  return (faces + box) * sizeof(double);
}

// The residual forms the autotuner chooses from: tile shape (cells in i,
// j, k) and staged stencil or not (form s: shape s % 3, staged for s >= 3).
constexpr int RES_NSHAPE = 3, RES_NFORM = 6;
constexpr int RES_SHAPES[RES_NSHAPE][3] = {{32, 4, 4}, {16, 8, 4}, {8, 8, 8}};

// SOURKO (KOVER=0, RANS, no rotation correction) + ADDSKE, interior cells.
__global__ void k_sourko_addske(DevBlock b) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.imax * b.jmax * b.kmax) return;
  int I = t % b.imax + 1, J = (t / b.imax) % b.jmax + 1, K = t / (b.imax * b.jmax) + 1;
  size_t L = ix(b, I, J, K);
  const double pbstar = 1.0 / SST_BSTAR, persbs = 1.0 / sqrt(SST_BSTAR), eps = 1.0E-10;
  double f1 = b.a[FF_FUN1][L], onemf1 = dmax(0.0, 1.0 - f1);
  double beta = f1 * SST_BETA1 + onemf1 * SST_BETA2;
  double sigom = f1 * SST_SIGOM1 + onemf1 * SST_SIGOM2;
  double gamkom = beta * pbstar - sigom * (SST_CKAPPA * SST_CKAPPA) * persbs;
  double rmutrb = dmax(eps, b.a[FF_EPS2][L] - 1.0) * b.a[FF_VIS][L];
  double ro = b.a[FF_RO][L], rom = b.a[FF_REPS][L], pt = b.a[FF_PTUR][L];
  double prol = 1.0 / ro;
  double som = onemf1 * b.a[FF_SEPS][L];
  double srk = pt - SST_BSTAR * b.a[FF_RK][L] * rom * prol;
  double omepro = gamkom * ro * pt / (rmutrb * rom);
  double omedis = 1.0 * beta * prol * rom;
  som = som + rom * (omepro - omedis);
  b.a[FF_SRK][L] = srk;
  b.a[FF_SEPS][L] = som;
  b.a[FF_DRK][L] = b.a[FF_DRK][L] + srk;
  b.a[FF_DEPS][L] = b.a[FF_DEPS][L] + som;
}

// LOCDTK (DTURB=1) + IMSOKO + COPRKE, after TIME3 wrote DTL (interior).
__global__ void k_locdtk_imsoko_coprke(DevBlock b, ff_params p) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.imax * b.jmax * b.kmax) return;
  int I = t % b.imax + 1, J = (t / b.imax) % b.jmax + 1, K = t / (b.imax * b.jmax) + 1;
  size_t i = ix(b, I, J, K);
  double dtl = b.a[FF_DTL][i];
  double dri = dtl * b.a[FF_DRO][i], dmi = dtl * b.a[FF_DM][i], dni = dtl * b.a[FF_DN][i];
  double dwi = dtl * b.a[FF_DW][i], dre = dtl * b.a[FF_DE][i];
  double drk = 1. * dtl * b.a[FF_DRK][i], deps = 1. * dtl * b.a[FF_DEPS][i];
  // IMSOKO imps3.f:972
  const double gamkom = SST_BETA1 / SST_BSTAR - SST_SIGOM1 * (SST_CKAPPA * SST_CKAPPA) / sqrt(SST_BSTAR);
  const double ckmax = 1.0 / (2.0 * p.csimps), eps = 1.0E-10;
  double E = b.a[FF_E][i], rk = b.a[FF_RK][i], rom = b.a[FF_REPS][i], ro = b.a[FF_RO][i];
  double emeanf = E - rk;
  double drkmax = dmax(ckmax * dmin(rk, fabs(0.1 * emeanf - 0.9 * rk)), eps);
  double dommax = ckmax * rom;
  double prol = 1. / ro;
  double atprod = fabs(b.a[FF_PTUR][i]);
  double rnutrb = dmax(b.a[FF_EPS2][i] - 1.0, eps) * b.a[FF_VIS][i] * prol;
  double drkden = 1.0 + dtl * (atprod / drkmax + prol * SST_BSTAR * rom);
  double domden = 1.0 + dtl * (gamkom * atprod / (rnutrb * dommax) + 2. * SST_BETA1 * rom);
  drk = drk / drkden;
  deps = deps / domden;
  // COPRKE imps3.f:1113
  double u = b.a[FF_U][i], v = b.a[FF_V][i], w = b.a[FF_W][i];
  double vel2 = u * u + v * v + w * w;
  double drodh = b.a[FF_DRDH][i], drodp = b.a[FF_DRDP][i];
  double ypro = 1. / ro, rki = rk * ypro;
  double dkin = u * dmi + v * dni + w * dwi + drk;
  b.a[FF_DM][i] = ypro * (-u * dri + dmi);
  b.a[FF_DN][i] = ypro * (-v * dri + dni);
  b.a[FF_DW][i] = ypro * (-w * dri + dwi);
  b.a[FF_DRK][i] = ypro * (-rki * dri + drk);
  b.a[FF_DEPS][i] = ypro * (-rom * ypro * dri + deps);
  double hi = ypro * (E + b.a[FF_P][i]);
  double dei = dre - (hi - vel2 - rki) * dri - dkin;
  double c = b.a[FF_C][i];
  double dpi = c * c * (dri - drodh * ypro * dei);
  b.a[FF_DRO][i] = (dri - drodp * dpi) / drodh;
  b.a[FF_DE][i] = dpi + .667 * drk;
}

// SUBIN for SST: the k cap (RKMAX = FRSDEN*FRSVEL^2) and RKOLD/EPSOLD over
// all cells.
__global__ void k_subin_sst(DevBlock b, ff_params p) {
  size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (size_t)b.ntot) return;
  double rkmax = .5 * p.frsden * p.frsvel * p.frsvel * 2.;
  double rk = b.a[FF_RK][n];
  rk = dmin(rk, dmax(0.1 * b.a[FF_E][n], rkmax));
  rk = dmin(rk, rkmax);
  b.a[FF_RK][n] = rk;
  b.a[FF_RKOLD][n] = rk;
  b.a[FF_EPSOLD][n] = b.a[FF_REPS][n];
}
