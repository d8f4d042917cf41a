// sm_100a kernels of the FINFLO per-iteration hot path (FP64).
//
// Launch shapes:
//   k_state / k_fin / k_time3_copr ...  element-wise, one thread per cell
//   k_patch_*                         one grid row per boundary patch
//   k_grad                            one thread per cell incl. ghost layer 1
//   k_residual                        32x4x4-cell tiles, all three face
//                                     directions fused, face fluxes staged
//                                     in shared memory, residual written once
//   k_sweep_coef + k_lusgs_sweep      coefficient pass into the skewed sweep
//                                     layout, then a cooperative persistent
//                                     kernel marching the i+j+k hyperplanes
//                                     with a bounded grid barrier
//   k_lusgs_lines                     the same sweep as a line wavefront in
//                                     one thread-block cluster (DSMEM)
#pragma once
#include "ff_device.cuh"
#include <cooperative_groups.h>

namespace ff {

constexpr int TI = 32, TJ = 4, TK = 4;   // residual tile
#ifndef RES_MIN_CTAS
#define RES_MIN_CTAS 4                    // residual threads per SM the register budget aims at, / 128
#endif
constexpr int NCOEF = 13;                 // LU-SGS coefficients per cell

// ---------------------------------------------------------------------------
// STATIM: PDTOP state.f:1690, PERFGA state.f:159, CONSVA base3c.f:489, and the
// laminar TURBDI (ADJUIN res3c.f:9447: EPS2 = 1, VIST = 0 on interior cells).
FF_DI void state_cell(const DevBlock& b, const ff_params& p, size_t n) {
  double* a_P = b.a[FF_P];
  double pd = b.a[FF_PDIFF][n], T = b.a[FF_TEMP][n];
  double P = pd + p.frspre;
  const double gm1 = p.gamma - 1., cp2 = p.gamma / gm1 * p.rgas;
  double trgs = T * p.rgas;
  double drdp = 1. / trgs;
  double ro = P * drdp;
  double vis = p.visu0 * T * sqrt(T) / (T + p.tsu0);
  double e = trgs / gm1;
  double drdh = -ro / e / p.gamma;
  double u = b.a[FF_U][n], v = b.a[FF_V][n], w = b.a[FF_W][n];
  double rkin = (u * u + v * v + w * w) * .5;
  double c, rk = 0.;
  if (p.iturb < 3) {
    c = sqrt(dmax(1. / (drdh / ro + drdp), 1.0));
  } else {   // CONSVA two-equation branch: k in the sound speed and E
    rk = b.a[FF_RK][n];
    double ypro = 1. / ro;
    double xturb = 1. + (2. / 3.) * rk * ypro * drdp;
    c = sqrt(dmax(xturb / (drdh * ypro + drdp), 1.0));
  }
  a_P[n] = P;
  b.a[FF_DRDP][n] = drdp;
  b.a[FF_RO][n] = ro;
  b.a[FF_VIS][n] = vis;
  b.a[FF_DRDH][n] = drdh;
  b.a[FF_CP][n] = cp2;
  b.a[FF_CH][n] = vis * cp2 / p.pr;
  b.a[FF_C][n] = c;
  b.a[FF_E][n] = p.iturb < 3 ? (e + rkin) * ro : (e + rkin) * ro + rk;
  b.a[FF_RM][n] = ro * u;
  b.a[FF_RN][n] = ro * v;
  b.a[FF_RW][n] = ro * w;
}

__global__ void k_state(DevBlock b, ff_params p) {
  size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (size_t)b.ntot) return;
  state_cell(b, p, n);
  if (p.iturb >= 3) return;   // TURBEQ, not ADJUIN, sets EPS2 and VIST
  int i = (int)(n % b.is), j = (int)((n / b.is) % (b.jmax + 4)), k = (int)(n / b.il);
  if (i >= 2 && i < b.imax + 2 && j >= 2 && j < b.jmax + 2 && k >= 2 && k < b.kmax + 2) {
    b.a[FF_EPS2][n] = 1.0;
    b.a[FF_VIST][n] = 0.0;
  }
}

// Face description of a patch: direction, sign, normal stride, interior layer.
struct FaceG { int dir, idir, s, layer; };
FF_DI FaceG face_g(const DevBlock& b, int iface) {
  FaceG f;
  f.dir = (iface - 1) % 3 + 1;
  f.idir = iface <= 3 ? 1 : -1;
  f.s = f.dir == 1 ? 1 : (f.dir == 2 ? b.is : b.il);
  int mx = f.dir == 1 ? b.imax : (f.dir == 2 ? b.jmax : b.kmax);
  f.layer = iface <= 3 ? 1 : mx;
  return f;
}
FF_DI size_t face_cell(const DevBlock& b, const FaceG& f, int a, int c) {
  if (f.dir == 1) return ix(b, f.layer, a, c);
  if (f.dir == 2) return ix(b, a, f.layer, c);
  return ix(b, a, c, f.layer);
}

// Patch-cell iteration: blockIdx.y = patch, x covers r1 x r2.
#define FF_PATCH_LOOP(b)                                                       \
  const ff_patch& pa = (b).patch[blockIdx.y];                                  \
  int n1 = pa.r1b - pa.r1a + 1, n2 = pa.r2b - pa.r2a + 1;                      \
  int t = blockIdx.x * blockDim.x + threadIdx.x;                               \
  if (t >= n1 * n2) return;                                                    \
  int pa1 = pa.r1a + t % n1, pa2 = pa.r2a + t / n1;                            \
  FaceG fg = face_g((b), pa.iface);                                            \
  int ls = fg.idir * fg.s;                                                     \
  (void)ls;                                                                    \
  size_t L = face_cell((b), fg, pa1, pa2);

// REFLEC turb3.f:5294: solid walls (viscous, wall at rest) and the inlet
// pressure extrapolation.  mode 0: REFLEC; mode 1: re-evaluate the equation of
// state in the two ghost cells first (the second STATIM pass).
__global__ void k_reflec(DevBlock b, ff_params p, int mode) {
  FF_PATCH_LOOP(b)
  size_t LB = L - ls, LT = L + ls, LC = L - 2 * ls;
  bool wall = pa.ityp >= 7 && pa.ityp <= 10;
  if (!wall && pa.ityp != FF_BC_INL) return;
  if (mode == 1) { state_cell(b, p, LB); state_cell(b, p, LC); }
  double* P = b.a[FF_P]; double* PD = b.a[FF_PDIFF];
  if (pa.ityp == FF_BC_INL) {
    P[LB] = P[L]; PD[LB] = PD[L]; P[LC] = P[L]; PD[LC] = PD[L];
    return;
  }
  double *T = b.a[FF_TEMP], *RO = b.a[FF_RO];
  int ihfl = pa.iheat == 1 ? 1 : 0;
  double tsurf = pa.iheat == 1 ? pa.bount : 0.0;
  double tb = (1 - ihfl) * T[L] + ihfl * (2. * tsurf - T[L]);
  tb = dmax(dmin(tb, p.tuplim), p.tlolim);
  T[LB] = tb; T[LC] = tb;
  b.a[FF_VIS][LB] = b.a[FF_VIS][L]; b.a[FF_CH][LB] = b.a[FF_CH][L]; b.a[FF_C][LB] = b.a[FF_C][L];
  b.a[FF_DRDP][LB] = b.a[FF_DRDP][L]; b.a[FF_DRDH][LB] = b.a[FF_DRDH][L];
  double u = -b.a[FF_U][L], v = -b.a[FF_V][L], w = -b.a[FF_W][L];
  b.a[FF_U][LB] = u; b.a[FF_V][LB] = v; b.a[FF_W][LB] = w;
  b.a[FF_U][LC] = u; b.a[FF_V][LC] = v; b.a[FF_W][LC] = w;
  double ro = dmax(0.001 * p.frsden, RO[L]);
  double pb = dmax(0.001 * p.frspre, 2. * P[L] - P[LT]);
  double pdb = dmax(-0.999 * p.frspre, 2. * PD[L] - PD[LT]);
  RO[LB] = ro; RO[LC] = ro; P[LB] = pb; P[LC] = pb; PD[LB] = pdb; PD[LC] = pdb;
  b.a[FF_EPS2][LB] = 1.; b.a[FF_VIST][LB] = 0.; b.a[FF_EPS2][LC] = 1.; b.a[FF_VIST][LC] = 0.;
  b.a[FF_RM][LB] = ro * u; b.a[FF_RN][LB] = ro * v; b.a[FF_RW][LB] = ro * w;
  b.a[FF_RM][LC] = ro * u; b.a[FF_RN][LC] = ro * v; b.a[FF_RW][LC] = ro * w;
  b.a[FF_E][LB] = b.a[FF_E][L]; b.a[FF_E][LC] = b.a[FF_E][L];
  if (p.iturb >= 3) {   // turb3.f:5646-5658 (ITURB = 6)
    b.a[FF_RK][LB] = -b.a[FF_RK][L];
    b.a[FF_REPS][LB] = dmax(0., 2. * b.a[FF_REPS][L] - b.a[FF_REPS][LT]);
  }
}

// REFCEN turb3.f:5881: linear extrapolation into the first wall ghost.
__global__ void k_refcen(DevBlock b, ff_params p) {
  FF_PATCH_LOOP(b)
  if (pa.ityp < 7 || pa.ityp > 10) return;
  size_t LB = L - ls, LT = L + ls;
  double* RO = b.a[FF_RO]; double* P = b.a[FF_P]; double* PD = b.a[FF_PDIFF];
  RO[LB] = dmax(0.001 * p.frsden, 2. * RO[L] - RO[LT]);
  P[LB] = dmax(0.001 * p.frspre, 2. * P[L] - P[LT]);
  PD[LB] = dmax(-0.999 * p.frspre, 2. * PD[L] - PD[LT]);
  const int sl[7] = {FF_E, FF_U, FF_V, FF_W, FF_RM, FF_RN, FF_RW};
#pragma unroll
  for (int s = 0; s < 7; s++) { double* q = b.a[sl[s]]; q[LB] = 2. * q[L] - q[LT]; }
  if (p.iturb >= 3) {   // turb3.f:6013-6027
    double *RK = b.a[FF_RK], *RE = b.a[FF_REPS];
    RK[LB] = dmax(p.rklim, 2. * RK[L] - 1. * RK[LT]);
    RE[LB] = dmax(p.epslim, 2. * RE[L] - 1. * RE[LT]);
  }
}

// INLET base3c.f:9223 (INLOUT 4) and OUTLET base3c.f:9595 (INLOUT 2, 3): the
// level-1 ghost update FLUCYC does before the fluxes (res3c.f:7730-7834).
__global__ void k_inlet_outlet(DevBlock b, ff_params p, int icycle) {
  FF_PATCH_LOOP(b)
  bool inl = pa.ityp == FF_BC_INL && pa.ibtype == 4;
  bool out = pa.ityp == FF_BC_OUT && (pa.ibtype == 2 || pa.ibtype == 3);
  if (!inl && !out) return;
  size_t II = L, IM1 = L - ls, IM2 = IM1 - ls;
  size_t IF1 = fg.idir == 1 ? II : II + fg.s;
  double *U = b.a[FF_U], *V = b.a[FF_V], *W = b.a[FF_W], *T = b.a[FF_TEMP], *RO = b.a[FF_RO];
  double *P = b.a[FF_P], *PD = b.a[FF_PDIFF], *E = b.a[FF_E], *RM = b.a[FF_RM], *RN = b.a[FF_RN];
  double *RW = b.a[FF_RW], *EPS2 = b.a[FF_EPS2], *VIST = b.a[FF_VIST], *VIS = b.a[FF_VIS];
  if (inl) {
    double dpkoe = P[II], dpdif = PD[II];
    EPS2[IM1] = EPS2[II]; EPS2[IM2] = EPS2[II];
    VIST[IM1] = VIST[II]; VIST[IM2] = VIST[II];
    double rm = pa.bounu * pa.bounr, rn = pa.bounv * pa.bounr, rw = pa.bounw * pa.bounr;
    RM[IM1] = rm; RN[IM1] = rn; RW[IM1] = rw; RM[IM2] = rm; RN[IM2] = rn; RW[IM2] = rw;
    if (icycle == 1) RO[IM1] = pa.bounr;
    T[IM1] = pa.bount; T[IM2] = pa.bount;
    P[IM1] = dpkoe; P[IM2] = dpkoe; PD[IM1] = dpdif; PD[IM2] = dpdif;
    double e = p.rgas / (p.gamma - 1.) * pa.bount;
    double r1 = RO[IM1], r2 = RO[IM2];
    double u1 = rm / r1, v1 = rn / r1, w1 = rw / r1, u2 = rm / r2, v2 = rn / r2, w2 = rw / r2;
    U[IM1] = u1; V[IM1] = v1; W[IM1] = w1; U[IM2] = u2; V[IM2] = v2; W[IM2] = w2;
    E[IM1] = r1 * (e + .5 * (u1 * u1 + v1 * v1 + w1 * w1));
    E[IM2] = r2 * (e + .5 * (u2 * u2 + v2 * v2 + w2 * w2));
    if (p.iturb >= 3) {   // base3c.f:9534-9541
      b.a[FF_RK][IM1] = pa.bounrk; b.a[FF_RK][IM2] = pa.bounrk;
      b.a[FF_REPS][IM1] = pa.bounep; b.a[FF_REPS][IM2] = pa.bounep;
      E[IM1] = E[IM1] + pa.bounrk;
      E[IM2] = E[IM2] + pa.bounrk;
    }
    return;
  }
  // FLUCYC's local TURLIM (res3c.f:7750); FLXCYC passes the real one
  const double turlim = p.iturb >= 3 ? p.turlim : 1.e-6;
  double rk3 = pa.ibtype == 2 ? 0.7 : 1.0, rk4 = pa.ibtype == 2 ? 0.3 : 0.0;
  const double* NX = b.a[FF_A1XA + 4 * (fg.dir - 1)];
  const double* NY = b.a[FF_A1YA + 4 * (fg.dir - 1)];
  const double* NZ = b.a[FF_A1ZA + 4 * (fg.dir - 1)];
  double a11 = NX[IF1], a12 = NY[IF1], a13 = NZ[IF1], a21, a22, a23, a31, a32, a33;
  surfvects(a11, a12, a13, a21, a22, a23, a31, a32, a33);
  double veloc = .5 * (a11 * (U[II] + pa.bounu) + a12 * (V[II] + pa.bounv) + a13 * (W[II] + pa.bounw));
  P[IM1] = pa.bounp; P[IM2] = pa.bounp; PD[IM1] = pa.bounpd; PD[IM2] = pa.bounpd;
  double eps2 = dmin(EPS2[II], turlim), vist = dmin(VIST[II], turlim * VIS[IM2]);
  EPS2[IM1] = eps2; EPS2[IM2] = eps2; VIST[IM1] = vist; VIST[IM2] = vist;
  if (-veloc * fg.idir > 0.) {
    double u = RO[II] * U[II] / RO[IM1], v = V[II], w = W[II];
    U[IM1] = u; U[IM2] = u; V[IM1] = v; V[IM2] = v; W[IM1] = w; W[IM2] = w;
    T[IM1] = T[II]; T[IM2] = T[II];
    RM[IM1] = RO[IM1] * u; RM[IM2] = RO[IM2] * u;
    RN[IM1] = RO[IM1] * v; RN[IM2] = RO[IM2] * v;
    RW[IM1] = RO[IM1] * w; RW[IM2] = RO[IM2] * w;
  } else {
    double velc1 = a11 * U[II] + a12 * V[II] + a13 * W[II];
    double velc2 = a21 * pa.bounu + a22 * pa.bounv + a23 * pa.bounw;
    double velc3 = a31 * pa.bounu + a32 * pa.bounv + a33 * pa.bounw;
    double uu = a11 * velc1 + a21 * velc2 + a31 * velc3;
    double vv = a12 * velc1 + a22 * velc2 + a32 * velc3;
    double ww = a13 * velc1 + a23 * velc2 + a33 * velc3;
    double u = rk3 * U[IM1] + rk4 * uu, v = rk3 * V[IM1] + rk4 * vv, w = rk3 * W[IM1] + rk4 * ww;
    U[IM1] = u; U[IM2] = u; V[IM1] = v; V[IM2] = v; W[IM1] = w; W[IM2] = w;
    T[IM1] = pa.bount; T[IM2] = pa.bount;
    RO[IM1] = pa.bounr; RO[IM2] = pa.bounr;
  }
  if (p.iturb >= 3 && -veloc * fg.idir > 0.) {   // base3c.f:10134-10146
    double rk = b.a[FF_RK][II], re = b.a[FF_REPS][II];
    b.a[FF_RK][IM1] = rk; b.a[FF_RK][IM2] = rk;
    b.a[FF_REPS][IM1] = re; b.a[FF_REPS][IM2] = re;
    E[IM1] = E[IM1] + rk;
    E[IM2] = E[IM2] + rk;
  }
}

// MIR ns3c.f:9003 -> MIRROR gluebm.f:3911 for symmetry patches.
__global__ void k_mir(DevBlock b) {
  FF_PATCH_LOOP(b)
  if (pa.ityp != FF_BC_MIR) return;
  (void)ls;
  int kdir = fg.idir == 1 ? -1 : 1, koff = fg.idir == 1 ? 0 : 1;
  size_t IC1 = L, IT = IC1 + (size_t)koff * fg.s;
  size_t IT1 = IC1 + kdir * fg.s, IT2 = IC1 + 2 * kdir * fg.s, IC2 = IC1 - kdir * fg.s;
  double nx = b.a[FF_A1XA + 4 * (fg.dir - 1)][IT];
  double ny = b.a[FF_A1YA + 4 * (fg.dir - 1)][IT];
  double nz = b.a[FF_A1ZA + 4 * (fg.dir - 1)][IT];
  double a11 = -2. * nx * nx + 1.0, a12 = -2. * nx * ny, a13 = -2. * nx * nz;
  double a22 = -2. * ny * ny + 1.0, a23 = -2. * ny * nz, a33 = -2. * nz * nz + 1.0;
  double *U = b.a[FF_U], *V = b.a[FF_V], *W = b.a[FF_W];
  double u1 = U[IC1], v1 = V[IC1], w1 = W[IC1], u2 = U[IC2], v2 = V[IC2], w2 = W[IC2];
  U[IT1] = a11 * u1 + a12 * v1 + a13 * w1;
  V[IT1] = a12 * u1 + a22 * v1 + a23 * w1;
  W[IT1] = a13 * u1 + a23 * v1 + a33 * w1;
  U[IT2] = a11 * u2 + a12 * v2 + a13 * w2;
  V[IT2] = a12 * u2 + a22 * v2 + a23 * w2;
  W[IT2] = a13 * u2 + a23 * v2 + a33 * w2;
  const int sc[8] = {FF_TEMP, FF_E, FF_P, FF_PDIFF, FF_EPS2, FF_VIST, FF_RK, FF_REPS};
#pragma unroll
  for (int s = 0; s < 8; s++) { double* q = b.a[sc[s]]; q[IT1] = q[IC1]; q[IT2] = q[IC2]; }
}

// REFCOR turb3.f:6040: ghost cells with two or three ghost indices copy the
// interior edge/corner cell next to them.
__global__ void k_refcor(DevBlock b) {
  size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (size_t)b.ntot) return;
  int i = (int)(n % b.is) - 1, j = (int)((n / b.is) % (b.jmax + 4)) - 1, k = (int)(n / b.il) - 1;
  int gi = i < 1 || i > b.imax, gj = j < 1 || j > b.jmax, gk = k < 1 || k > b.kmax;
  if (gi + gj + gk < 2) return;
  int ic = i < 1 ? 1 : (i > b.imax ? b.imax : i);
  int jc = j < 1 ? 1 : (j > b.jmax ? b.jmax : j);
  int kc = k < 1 ? 1 : (k > b.kmax ? b.kmax : k);
  size_t src = ix(b, ic, jc, kc);
  const int sl[20] = {FF_RO, FF_RM, FF_RN, FF_RW, FF_E, FF_U, FF_V, FF_W, FF_P, FF_PDIFF,
                      FF_EPS2, FF_VIST, FF_TEMP, FF_VIS, FF_CH, FF_C, FF_DRDP, FF_DRDH, FF_RK, FF_REPS};
#pragma unroll
  for (int s = 0; s < 20; s++) b.a[sl[s]][n] = b.a[sl[s]][src];
}

// DERFUN turb3.f:2476 + TEMDER turb3.f:3456 (IDERI = 1), interior + first
// ghost layer on level 1.
__global__ void k_grad(DevBlock b, int level) {
  int lo = level == 1 ? 0 : 1, hi = level == 1 ? 1 : 0;
  int ni = b.imax + hi - lo + 1, nj = b.jmax + hi - lo + 1, nk = b.kmax + hi - lo + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ni * nj * nk) return;
  int I = lo + t % ni, J = lo + (t / ni) % nj, K = lo + t / (ni * nj);
  const int IS = b.is, IL = b.il;
  size_t L = ix(b, I, J, K);
  const double *U = b.a[FF_U], *V = b.a[FF_V], *W = b.a[FF_W], *T = b.a[FF_TEMP];
  const double *A1 = b.a[FF_A1], *A2 = b.a[FF_A2], *A3 = b.a[FF_A3];
  const double *D1 = b.a[FF_D1], *D2 = b.a[FF_D2], *D3 = b.a[FF_D3];
  double q[4][6];   // face-weighted values of u,v,w,T on the 6 faces (m/p per dir)
  double aa[6];     // areas: 1m,1p,2m,2p,3m,3p
  const double* Dd[3] = {D1, D2, D3};
  const double* Ad[3] = {A1, A2, A3};
  const int st[3] = {1, IS, IL};
  const double* F[4] = {U, V, W, T};
#pragma unroll
  for (int d = 0; d < 3; d++) {
#pragma unroll
    for (int side = 0; side < 2; side++) {
      size_t nb = side == 0 ? L - st[d] : L + st[d];
      double w1 = 2.0 * (Dd[d][L] / (Dd[d][L] + Dd[d][nb])), w2 = 2.0 - w1;
      aa[2 * d + side] = side == 0 ? Ad[d][L] : Ad[d][L + st[d]];
#pragma unroll
      for (int v = 0; v < 4; v++) q[v][2 * d + side] = w2 * F[v][L] + w1 * F[v][nb];
    }
  }
  double pvol = .5 / b.a[FF_VOL][L];
  double g[3][3];   // g[v][x] = d(u_v)/dx_x
#pragma unroll
  for (int x = 0; x < 3; x++) {
    const double* N1 = b.a[FF_A1XA + x];
    const double* N2 = b.a[FF_A2XA + x];
    const double* N3 = b.a[FF_A3XA + x];
    double n3p = N3[L + IL], n3m = N3[L], n2p = N2[L + IS], n2m = N2[L], n1p = N1[L + 1], n1m = N1[L];
#pragma unroll
    for (int v = 0; v < 3; v++)
      g[v][x] = pvol * (n3p * (aa[5] * q[v][5]) - n3m * (aa[4] * q[v][4]) + n2p * (aa[3] * q[v][3])
                        - n2m * (aa[2] * q[v][2]) + n1p * (aa[1] * q[v][1]) - n1m * (aa[0] * q[v][0]));
    bool tk = !(level == 1 && (K == 0 || K == b.kmax + 1) && b.kmax <= 1);
    if (tk)
      b.a[FF_DTDX + x][L] = pvol * (aa[5] * n3p * q[3][5] - aa[4] * n3m * q[3][4] + aa[3] * n2p * q[3][3]
                                    - aa[2] * n2m * q[3][2] + aa[1] * n1p * q[3][1] - aa[0] * n1m * q[3][0]);
  }
  double w12 = .5 * (g[0][1] - g[1][0]), w13 = .5 * (g[0][2] - g[2][0]), w23 = .5 * (g[1][2] - g[2][1]);
  b.a[FF_W12][L] = w12; b.a[FF_W13][L] = w13; b.a[FF_W23][L] = w23;
  b.a[FF_OHMI][L] = 2. * sqrt(w12 * w12 + w13 * w13 + w23 * w23);
  double s11 = g[0][0], s22 = g[1][1], s33 = g[2][2];
  double s12 = .5 * (g[0][1] + g[1][0]), s13 = .5 * (g[0][2] + g[2][0]), s23 = .5 * (g[1][2] + g[2][1]);
  b.a[FF_S11][L] = s11; b.a[FF_S12][L] = s12; b.a[FF_S13][L] = s13;
  b.a[FF_S22][L] = s22; b.a[FF_S23][L] = s23; b.a[FF_S33][L] = s33;
  double stn = s11 * s11 + 2. * s12 * s12 + 2. * s13 * s13 + s22 * s22 + 2. * s23 * s23 + s33 * s33;
  b.a[FF_STRAIN][L] = sqrt(2. * stn);
}

// FLUXBL base3c.f:4085 (IDIFF = 1) for the face between M = L-S and L; the
// result is the viscous part of the face flux (FRO untouched).
// Face geometry both viscous face fluxes (FLUXBL, FLKEBL) read: the
// interpolation weights from the cell thicknesses D1..D3, the unit vector s
// between the two cell centres with its length and reciprocal, and the face's
// unit normal and area.  Computed once per face.
struct FaceGeom {
  double w1, w2, sx, sy, sz, slen, rslen, nx, ny, nz, area;
};

FF_DI FaceGeom face_geom(const DevBlock& b, size_t L, int S, int dir) {
#define LD(s, n) __ldg(b.a[s] + (n))
  FaceGeom g;
  const size_t M = L - S;
  const double* D = b.a[FF_D1 + dir - 1];
  g.w1 = 2.0 * (__ldg(D + L) / (__ldg(D + L) + __ldg(D + M)));
  g.w2 = 2.0 - g.w1;
  double sx = LD(FF_XC, L) - LD(FF_XC, M), sy = LD(FF_YC, L) - LD(FF_YC, M), sz = LD(FF_ZC, L) - LD(FF_ZC, M);
  g.slen = sqrt(sx * sx + sy * sy + sz * sz) + 1.e-21;
  g.rslen = rcp(g.slen);
  g.sx = sx * g.rslen; g.sy = sy * g.rslen; g.sz = sz * g.rslen;
  const int ao = 4 * (dir - 1);
  g.nx = LD(FF_A1XA + ao, L); g.ny = LD(FF_A1YA + ao, L); g.nz = LD(FF_A1ZA + ao, L);
  g.area = LD(FF_A1 + ao, L);
#undef LD
  return g;
}

FF_DI void visc_flux(const DevBlock& b, const ff_params& p, size_t L, int S, int dir, const FaceGeom& g,
                     double f[5]) {
  size_t M = L - S;
  const double w1 = g.w1, w2 = g.w2;
  double w1p = .5 * w1, w2p = .5 * w2;
#define LD(s, n) __ldg(b.a[s] + (n))
  double s11l = LD(FF_S11, L), s11m = LD(FF_S11, M), s22l = LD(FF_S22, L), s22m = LD(FF_S22, M);
  double s33l = LD(FF_S33, L), s33m = LD(FF_S33, M), s12l = LD(FF_S12, L), s12m = LD(FF_S12, M);
  double s13l = LD(FF_S13, L), s13m = LD(FF_S13, M), s23l = LD(FF_S23, L), s23m = LD(FF_S23, M);
  double w12l = LD(FF_W12, L), w12m = LD(FF_W12, M), w13l = LD(FF_W13, L), w13m = LD(FF_W13, M);
  double w23l = LD(FF_W23, L), w23m = LD(FF_W23, M);
  double dudx = w2p * s11l + w1p * s11m, dvdy = w2p * s22l + w1p * s22m, dwdz = w2p * s33l + w1p * s33m;
  double dudy = w2p * (s12l + w12l) + w1p * (s12m + w12m);
  double dudz = w2p * (s13l + w13l) + w1p * (s13m + w13m);
  double dvdx = w2p * (s12l - w12l) + w1p * (s12m - w12m);
  double dvdz = w2p * (s23l + w23l) + w1p * (s23m + w23m);
  double dwdx = w2p * (s13l - w13l) + w1p * (s13m - w13m);
  double dwdy = w2p * (s23l - w23l) + w1p * (s23m - w23m);
  double s11i = w2 * s11l + w1 * s11m, s12i = w2 * s12l + w1 * s12m, s13i = w2 * s13l + w1 * s13m;
  double s22i = w2 * s22l + w1 * s22m, s23i = w2 * s23l + w1 * s23m, s33i = w2 * s33l + w1 * s33m;
  double dtdxi = w2p * LD(FF_DTDX, L) + w1p * LD(FF_DTDX, M);
  double dtdyi = w2p * LD(FF_DTDY, L) + w1p * LD(FF_DTDY, M);
  double dtdzi = w2p * LD(FF_DTDZ, L) + w1p * LD(FF_DTDZ, M);
  const double sxi = g.sx, syi = g.sy, szi = g.sz, rslen = g.rslen;
  const double nx = g.nx, ny = g.ny, nz = g.nz, area = g.area;
  double alfa = sxi * nx + syi * ny + szi * nz;
  double surf = 0.5 * area * (LD(FF_EPS2, L) * LD(FF_VIS, L) + LD(FF_EPS2, M) * LD(FF_VIS, M));
  const double rprt = rcp(p.prt);
  double surfe = 0.5 * area * (LD(FF_CP, L) * LD(FF_VIST, L) * rprt + LD(FF_CH, L)
                               + LD(FF_CP, M) * LD(FF_VIST, M) * rprt + LD(FF_CH, M));
  double ul = LD(FF_U, L), um = LD(FF_U, M), vl = LD(FF_V, L), vm = LD(FF_V, M), wl = LD(FF_W, L), wm = LD(FF_W, M);
  double duvwsj = nx * (dudx * sxi + dudy * syi + dudz * szi) + ny * (dvdx * sxi + dvdy * syi + dvdz * szi)
                + nz * (dwdx * sxi + dwdy * syi + dwdz * szi);
  double f2 = nx * s11i + ny * s12i + nz * s13i;
  double f3 = nx * s12i + ny * s22i + nz * s23i;
  double f4 = nx * s13i + ny * s23i + nz * s33i;
  if (alfa > 0.) {
    double adotu = nx * (ul - um) + ny * (vl - vm) + nz * (wl - wm);
    double cc = adotu * rslen - duvwsj;
    f2 = alfa * ((ul - um) * rslen - (sxi * dudx + syi * dudy + szi * dudz)) + sxi * cc + f2;
    f3 = alfa * ((vl - vm) * rslen - (sxi * dvdx + syi * dvdy + szi * dvdz)) + syi * cc + f3;
    f4 = alfa * ((wl - wm) * rslen - (sxi * dwdx + syi * dwdy + szi * dwdz)) + szi * cc + f4;
  }
  const double R23 = .6666667;
  double dv = dudx + dvdy + dwdz;
  f2 = surf * (f2 - R23 * nx * dv);
  f3 = surf * (f3 - R23 * ny * dv);
  f4 = surf * (f4 - R23 * nz * dv);
  double f5 = .5 * ((ul + um) * f2 + (vl + vm) * f3 + (wl + wm) * f4) + surfe * (dtdxi * nx + dtdyi * ny + dtdzi * nz);
  if (alfa > 0.)
    f5 = surfe * alfa * ((LD(FF_TEMP, L) - LD(FF_TEMP, M)) * rslen - sxi * dtdxi - syi * dtdyi - szi * dtdzi) + f5;
#undef LD
  f[0] = 0.; f[1] = -f2; f[2] = -f3; f[3] = -f4; f[4] = -f5;
}

FF_DI void visc_flux(const DevBlock& b, const ff_params& p, size_t L, int S, int dir, double f[5]) {
  visc_flux(b, p, L, S, dir, face_geom(b, L, S, dir), f);
}

// FLUXDO base3c.f:3677 (thin layer, IDIFF = 1): the viscous flux on coarse
// levels and whenever FULLNS is off (T = float for a coarse face pass in
// FP32).
template <typename T>
FF_DI void visc_flux_thin(const DevBlock& b, const ff_params& p, size_t L, int S, int dir, T f[5], T fe0 = T(0.)) {
#define LD(s, n) T(__ldg(b.a[s] + (n)))
  size_t M = L - S;
  const int ao = 4 * (dir - 1);
  T area = LD(FF_A1 + ao, L);
  T nx = LD(FF_A1XA + ao, L), ny = LD(FF_A1YA + ao, L), nz = LD(FF_A1ZA + ao, L);
  T surg = -area * (area / (LD(FF_VOL, L) + LD(FF_VOL, M)));
  T surf = surg * (LD(FF_EPS2, L) * LD(FF_VIS, L) + LD(FF_EPS2, M) * LD(FF_VIS, M));
  const T prt = T(p.prt);
  T surfe = surg * (LD(FF_CP, L) * LD(FF_VIST, L) / prt + LD(FF_CH, L)
                    + LD(FF_CP, M) * LD(FF_VIST, M) / prt + LD(FF_CH, M));
  T ul = LD(FF_U, L), um = LD(FF_U, M), vl = LD(FF_V, L), vm = LD(FF_V, M), wl = LD(FF_W, L), wm = LD(FF_W, M);
  T duc = T(.333333) * (nx * (ul - um) + ny * (vl - vm) + nz * (wl - wm));
  T f2 = surf * (ul - um + nx * duc);
  T f3 = surf * (vl - vm + ny * duc);
  T f4 = surf * (wl - wm + nz * duc);
  T f5 = T(.5) * ((ul + um) * f2 + (vl + vm) * f3 + (wl + wm) * f4);
  f[0] = T(0.); f[1] = f2; f[2] = f3; f[3] = f4;
  f[4] = fe0 + f5 + surfe * (LD(FF_TEMP, L) - LD(FF_TEMP, M));
#undef LD
}

// BOTSKE base3c.f:6147 wall-face flux (laminar, TURCOR false as FLUCYC passes
// it, wall at rest).  II = interior cell at the wall.
template <typename T>
FF_DI void wall_flux(const DevBlock& b, const ff_params& p, size_t II, int S, int idir, int dir,
                     int iheat, int intem, T f[5]) {
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
  // PB = YP1*PB1 + YP4*PB4 (base3c.f:6304-6315, 6487): the extrapolated
  // pressure, or its difference from FRSPRE for KT (IFLUX=7)
  T pb1 = p.flux == FF_FLUX_KT
              ? dmax(T(-.99) * T(p.frspre), rc1 * LD(FF_PDIFF, II) - rc2 * LD(FF_PDIFF, II2))
              : dmax(T(0.01) * T(p.frspre), rc1 * LD(FF_P, II) - rc2 * LD(FF_P, II2));
  T surf = surg * visb;
  T surfe = surg * (prs * T(0.) / visb + T(1.)) * chsb;
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
  f[0] = T(0.);
  f[1] = a_f * (ax * pb1 + f2v);
  f[2] = a_f * (ay * pb1 + f3v);
  f[3] = a_f * (az * pb1 + f4v);
  f[4] = a_f * f5v;
#undef LD
}

// Flux of one face (dir, cell L on the high side, normal index m).
// FLUXVL base3c.f:1733-1961 (IFLUX=0) at one face: van Leer flux-vector
// splitting of the MUSCL-extrapolated conservative variables qc[v][m]
// (v = RO, RM, RN, RW, E; cells I-2S..I+S), perfect gas, added to f.
// wps: FLUXWP base3c.f:1967-2195 (IFLUX=2), the wave/particle split of the
// subsonic momentum and energy fluxes (base3c.f:2118-2125, 2156-2163).
FF_DI void vl_flux(const double qc[5][4], double nx, double ny, double nz, double area, int intem,
                   const ff_params& p, bool wps, double f[5]) {
  const double gamma = p.gamma, gm1 = gamma - 1., ygm = 1. / gamma;
  double ip[5], im[5];
#pragma unroll
  for (int v = 0; v < 5; v++) xxtrap(qc[v][0], qc[v][1], qc[v][2], qc[v][3], intem, ip[v], im[v]);
  double ppi = (gamma - 1.) * (ip[4] - .5 / ip[0] * (ip[1] * ip[1] + ip[2] * ip[2] + ip[3] * ip[3]));
  double pmi = (gamma - 1.) * (im[4] - .5 / im[0] * (im[1] * im[1] + im[2] * im[2] + im[3] * im[3]));
  ip[0] = dmax(0.001 * p.frsden, ip[0]);
  ppi = dmax(0.001 * p.frspre, ppi);
  im[0] = dmax(0.001 * p.frsden, im[0]);
  pmi = dmax(0.001 * p.frspre, pmi);
  double a21, a22, a23, a31, a32, a33;
  surfvects(nx, ny, nz, a21, a22, a23, a31, a32, a33);
  const double rip0 = nx * ip[1] + ny * ip[2] + nz * ip[3], rip1 = a21 * ip[1] + a22 * ip[2] + a23 * ip[3],
               rip2 = a31 * ip[1] + a32 * ip[2] + a33 * ip[3];
  const double rim0 = nx * im[1] + ny * im[2] + nz * im[3], rim1 = a21 * im[1] + a22 * im[2] + a23 * im[3],
               rim2 = a31 * im[1] + a32 * im[2] + a33 * im[3];
  double fm[5], fp[5];
  {  // F- from the right state
    const double ypro = 1. / ip[0], u = ypro * rip0, v = ypro * rip1, w = ypro * rip2;
    const double pp = dmax(0.01, ppi), c = sqrt(gamma * pp * ypro), rma = u / c;
    if (rma < -1.) {
      fm[0] = area * rip0; fm[1] = area * (rip0 * u + pp); fm[2] = area * rip0 * v;
      fm[3] = area * rip0 * w; fm[4] = area * u * (ip[4] + pp);
    } else if (rma < 1.) {
      const double h = .5 * (rma - 1.), f1 = -area * ip[0] * c * (h * h);
      fm[0] = f1; fm[2] = f1 * v; fm[3] = f1 * w;
      if (wps) {
        const double rma2 = .25 * ((rma - 1.) * (rma - 1.)) * (2. + rma);
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
  {  // F+ from the left state
    const double ypro = 1. / im[0], u = ypro * rim0, v = ypro * rim1, w = ypro * rim2;
    const double pm = dmax(0.01, pmi), c = sqrt(gamma * pm * ypro), rma = u / c;
    if (rma > 1.) {
      fp[0] = area * rim0; fp[1] = area * (rim0 * u + pm); fp[2] = area * rim0 * v;
      fp[3] = area * rim0 * w; fp[4] = area * u * (im[4] + pm);
    } else if (rma > -1.) {
      const double h = .5 * (rma + 1.), f1 = +area * im[0] * c * (h * h);
      fp[0] = f1; fp[2] = f1 * v; fp[3] = f1 * w;
      if (wps) {
        const double rma2 = .25 * ((rma + 1.) * (rma + 1.)) * (2. - rma);
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
  const double f2 = fp[1] + fm[1], f3 = fp[2] + fm[2], f4 = fp[3] + fm[3];
  f[0] = fm[0] + fp[0] + f[0];
  f[1] = nx * f2 + a21 * f3 + a31 * f4 + f[1];
  f[2] = ny * f2 + a22 * f3 + a32 * f4 + f[2];
  f[3] = nz * f2 + a23 * f3 + a33 * f4 + f[3];
  f[4] = fm[4] + fp[4] + f[4];
}

#include "ff_fluxes.cuh"

// JAMESON base3c.f:2827-3019 (IPRESC = 0) at face L (cells L-S | L): the
// pressure sensors of the two cells (second differences of PDIFF), EPS2 =
// RJK2 * their max, EPS4 = max(0, RJK4 - EPS2), SCALEJ averaged to the face;
// the second- and fourth-difference dissipation of RO, RM, RN, RW, E taken
// off f.  Added to Roe's flux on the finest level when RJK2 or RJK4 > 0
// (FLUCYC res3c.f:7899-7906, RESIKE 6955-6962); k and omega keep theirs.
FF_DI void jst_flux(const DevBlock& b, const ff_params& p, size_t L, int S, double* f) {
  const double* PD = b.a[FF_PDIFF];
  const double pd0 = __ldg(PD + L - 2 * S), pd1 = __ldg(PD + L - S), pd2 = __ldg(PD + L), pd3 = __ldg(PD + L + S);
  const double fp4 = 4. * p.frspre;
  const double pres1 = fabs(pd2 - 2. * pd1 + pd0) / (pd2 + 2. * pd1 + pd0 + fp4);
  const double pres2 = fabs(pd3 - 2. * pd2 + pd1) / (pd3 + 2. * pd2 + pd1 + fp4);
  const double eps2 = p.rjk2 * dmax(pres1, pres2), eps4 = dmax(0., p.rjk4 - eps2);
  const double rlami = .5 * (__ldg(b.a[FF_SCALEJ] + L) + __ldg(b.a[FF_SCALEJ] + L - S));
  const int sl[5] = {FF_RO, FF_RM, FF_RN, FF_RW, FF_E};
#pragma unroll
  for (int v = 0; v < 5; v++) {
    const double* q = b.a[sl[v]];
    const double q0 = __ldg(q + L - 2 * S), q1 = __ldg(q + L - S), q2 = __ldg(q + L), q3 = __ldg(q + L + S);
    f[v] = -(rlami * (eps2 * (q2 - q1) - eps4 * (q3 - 3. * q2 + 3. * q1 - q0))) + f[v];
  }
}

// SCALARD base3c.f:6-78 (IPRESC = 0, no grid rotation): SCALEJ of cells
// 0..MAX+1 in each direction, |(U,V,W) . mean face vectors| + C * the mean
// face areas; the JAMESON dissipation scale.
__global__ void k_scalard(DevBlock b) {
  const int ni = b.imax + 2, nj = b.jmax + 2;
  const long n = (long)ni * nj * (b.kmax + 2);
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int I = t % ni, J = (t / ni) % nj, K = t / ((long)ni * nj);
  const size_t kk = ix(b, I, J, K), is = b.is, il = b.il;
#define LD(s, n) __ldg(b.a[s] + (n))
  const double a1 = LD(FF_A1, kk), a1p = LD(FF_A1, kk + 1), a2 = LD(FF_A2, kk), a2p = LD(FF_A2, kk + is);
  const double a3 = LD(FF_A3, kk), a3p = LD(FF_A3, kk + il);
  const double a1k = .5 * (a1 + a1p), a2k = .5 * (a2 + a2p), a3k = .5 * (a3 + a3p);
  const double a1xk = .5 * (LD(FF_A1XA, kk) * a1 + LD(FF_A1XA, kk + 1) * a1p);
  const double a1yk = .5 * (LD(FF_A1YA, kk) * a1 + LD(FF_A1YA, kk + 1) * a1p);
  const double a1zk = .5 * (LD(FF_A1ZA, kk) * a1 + LD(FF_A1ZA, kk + 1) * a1p);
  const double a2xk = .5 * (LD(FF_A2XA, kk) * a2 + LD(FF_A2XA, kk + is) * a2p);
  const double a2yk = .5 * (LD(FF_A2YA, kk) * a2 + LD(FF_A2YA, kk + is) * a2p);
  const double a2zk = .5 * (LD(FF_A2ZA, kk) * a2 + LD(FF_A2ZA, kk + is) * a2p);
  const double a3xk = .5 * (LD(FF_A3XA, kk) * a3 + LD(FF_A3XA, kk + il) * a3p);
  const double a3yk = .5 * (LD(FF_A3YA, kk) * a3 + LD(FF_A3YA, kk + il) * a3p);
  const double a3zk = .5 * (LD(FF_A3ZA, kk) * a3 + LD(FF_A3ZA, kk + il) * a3p);
  const double u = LD(FF_U, kk), v = LD(FF_V, kk), w = LD(FF_W, kk);
  const double ucii = a1xk * u + a1yk * v + a1zk * w, vcii = a2xk * u + a2yk * v + a2zk * w;
  const double wcii = a3xk * u + a3yk * v + a3zk * w;
  b.a[FF_SCALEJ][kk] = sqrt(ucii * ucii + vcii * vcii + wcii * wcii) + (a1k + a2k + a3k) * LD(FF_C, kk);
#undef LD
}

// sq (optional): RO, U, V, W, P of cell L in a staged stencil, variable v
// at sq[v * vs], the cells along the face normal es apart.  T = float: a
// coarse level's face in FP32 (loads converted, fluxes in FP32).
// ALT = false compiles out the selectable variants (the other IFLUX schemes,
// XXTRAA, JAMESON) for the residual kernels of the plain Roe/XXTRAP case:
// their code would raise the register count of every face.
template <typename T, bool ALT = true>
FF_DI void face_flux(const DevBlock& b, const ff_params& p, int dir, size_t L, int m, int t1, int t2,
                     int level, T f[5], const double* sq = nullptr, int es = 0, int vs = 0) {
  const int S = dir == 1 ? 1 : (dir == 2 ? b.is : b.il);
  const int nmax = dir == 1 ? b.imax : (dir == 2 ? b.jmax : b.kmax);
  int intem = dir == 1 ? p.interi : (dir == 2 ? p.interj : p.interk);
  if (level > 1) intem = p.coarse_inter;
  // wall face?  (BOTSKE overwrites, res3c.f:8092)
  if (m == 1 || m == nmax + 1) {
    int iface = m == 1 ? dir : dir + 3;
    for (int ip = 0; ip < b.npatch; ip++) {
      const ff_patch& pa = b.patch[ip];
      if (pa.iface != iface || pa.ityp < 8 || pa.ityp > 10) continue;
      if (t1 < pa.r1a || t1 > pa.r1b || t2 < pa.r2a || t2 > pa.r2b) continue;
      int idir = m == 1 ? 1 : -1;
      size_t II = m == 1 ? L : L - S;
      wall_flux(b, p, II, S, idir, dir, pa.iheat, intem, f);
      return;
    }
  }
  const int idi = dir == 1 ? p.idi1 : (dir == 2 ? p.idi2 : p.idi3);
  if (m <= min(idi, nmax + 1)) {   // SINVIS base3c.f:3876: viscous faces
    bool full = false;
    if constexpr (sizeof(T) == sizeof(double)) {
      if (level == 1 && p.fullns) { visc_flux(b, p, L, S, dir, f); full = true; }
    }
    if (!full) visc_flux_thin(b, p, L, S, dir, f);
  } else {
    f[0] = f[1] = f[2] = f[3] = f[4] = T(0.);
  }
  const int ao = 4 * (dir - 1);
  if constexpr (ALT && sizeof(T) == sizeof(double)) {
    if (p.flux != FF_FLUX_ROE) {   // the other IFLUX schemes (FLUCYC res3c.f:7890-7990)
      alt_flux<5>(b, p, dir, L, S, intem, 1, f);
      return;
    }
  }
  T q[5][4];
  const int sl[5] = {FF_RO, FF_U, FF_V, FF_W, FF_P};
  if (sq) {
#pragma unroll
    for (int v = 0; v < 5; v++) {
      const double* a = sq + v * vs;
      q[v][0] = T(a[-2 * es]); q[v][1] = T(a[-es]); q[v][2] = T(a[0]); q[v][3] = T(a[es]);
    }
  } else {
#pragma unroll
    for (int v = 0; v < 5; v++) {
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
  if constexpr (ALT && sizeof(T) == sizeof(double)) {
    if (p.xxtral) {   // XXTRAA over the cells' extents along the normal
      const double* D = b.a[FF_D1 + dir - 1];
      const double dd[4] = {__ldg(D + L - 2 * S), __ldg(D + L - S), __ldg(D + L), __ldg(D + L + S)};
      roe_flux<double, true>(q, __ldg(b.a[FF_A1XA + ao] + L), __ldg(b.a[FF_A1YA + ao] + L),
                             __ldg(b.a[FF_A1ZA + ao] + L), __ldg(b.a[FF_A1 + ao] + L), intem, p, __ldg(b.a[FF_C] + L),
                             __ldg(b.a[FF_C] + L - S), cr, cl, f, dd);
    } else {
      roe_flux(q, __ldg(b.a[FF_A1XA + ao] + L), __ldg(b.a[FF_A1YA + ao] + L), __ldg(b.a[FF_A1ZA + ao] + L),
               __ldg(b.a[FF_A1 + ao] + L), intem, p, __ldg(b.a[FF_C] + L), __ldg(b.a[FF_C] + L - S), cr, cl, f);
    }
    if (level == 1 && (p.rjk2 > 0. || p.rjk4 > 0.)) jst_flux(b, p, L, S, f);
    return;
  }
  roe_flux(q, T(__ldg(b.a[FF_A1XA + ao] + L)), T(__ldg(b.a[FF_A1YA + ao] + L)), T(__ldg(b.a[FF_A1ZA + ao] + L)),
           T(__ldg(b.a[FF_A1 + ao] + L)), intem, p, T(__ldg(b.a[FF_C] + L)), T(__ldg(b.a[FF_C] + L - S)), cr, cl, f);
}

// RESIDU: fused k, i, j face fluxes and SWEEP res3c.f:992 for a 32x4x4 tile.
// NT threads per CTA (128, 256 or 512): each thread sums the faces of
// CPT = 512 / NT cells of the 32x4x4 tile (a k column of CPT cells); the
// register budget gives RES_MIN_CTAS * 128 threads per SM at every NT.
template <int NT>
__global__ void __launch_bounds__(NT, RES_MIN_CTAS * 128 / NT) k_residual(DevBlock b, ff_params p, int level) {
  constexpr int CPT = TI * TJ * TK / NT;
  constexpr int NF = TI * (TJ + 1) * TK, NC = TI * TJ * TK;
  // one direction's faces (at most 640) x 5, then the cells' running sums
  // (in shared memory, not registers: the face flux needs the registers)
  extern __shared__ double res_smem[];
  double(*sF)[NF] = reinterpret_cast<double(*)[NF]>(res_smem);
  double(*sAcc)[NC] = reinterpret_cast<double(*)[NC]>(res_smem + 5 * NF);
  const int tid = threadIdx.x;
  const int i0 = blockIdx.x * TI, j0 = blockIdx.y * TJ, k0 = blockIdx.z * TK;
  const int ci = tid % TI, cj = (tid / TI) % TJ, ck0 = (tid / (TI * TJ)) * CPT;
#pragma unroll
  for (int c = 0; c < CPT; c++)
#pragma unroll
    for (int v = 0; v < 5; v++) sAcc[v][ci + TI * (cj + TJ * (ck0 + c))] = 0.;
  // the directions in SWEEP order (k, i, j; res3c.f:355); one call site of the
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
      double fl[5];
      face_flux(b, p, dir, ix(b, I, J, K), m, t1, t2, level, fl);
#pragma unroll
      for (int v = 0; v < 5; v++) sF[v][f] = fl[v];
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
        for (int v = 0; v < 5; v++) sAcc[v][ca] = sAcc[v][ca] - (sF[v][f0 + fs] - sF[v][f0]);
      } else {   // last direction, then 1/VOL (SWEEP IDO = 1)
        const size_t n = ix(b, I, J, K);
        const double rv = 1. / __ldg(b.a[FF_VOL] + n);
#pragma unroll
        for (int v = 0; v < 5; v++) b.a[FF_DRO + v][n] = (sAcc[v][ca] - (sF[v][f0 + fs] - sF[v][f0])) * rv;
      }
    }
    __syncthreads();
  }
}

// Sum of squares (RESL2 res3c.f:8920) of the five residuals into out[0..4].
__global__ void k_resl2(DevBlock b, double* out) {
  __shared__ double red[5][8];
  double s[5] = {0, 0, 0, 0, 0};
  int n_int = b.imax * b.jmax * b.kmax;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n_int; t += gridDim.x * blockDim.x) {
    int I = t % b.imax + 1, J = (t / b.imax) % b.jmax + 1, K = t / (b.imax * b.jmax) + 1;
    size_t n = ix(b, I, J, K);
#pragma unroll
    for (int v = 0; v < 5; v++) { double d = b.a[FF_DRO + v][n]; s[v] += d * d; }
  }
#pragma unroll
  for (int v = 0; v < 5; v++) {
    double x = s[v];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[v][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    double x = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) x += red[threadIdx.x][w];
    atomicAdd(out + threadIdx.x, x);
  }
}

// TIME3 base3c.f:79 + LOCDT imps3.f:784 + COPR imps3.f:891 (interior cells).
// mode 1: TIME3 only (the two-equation path converts in k_locdtk_imsoko_coprke).
__global__ void k_time3_copr(DevBlock b, ff_params p, double cfl, int mode = 0) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.imax * b.jmax * b.kmax) return;
  int I = t % b.imax + 1, J = (t / b.imax) % b.jmax + 1, K = t / (b.imax * b.jmax) + 1;
  const int IS = b.is, IL = b.il;
  size_t kk = ix(b, I, J, K);
#define LD(s, n) __ldg(b.a[s] + (n))
  double a1 = LD(FF_A1, kk), a1p = LD(FF_A1, kk + 1), a2 = LD(FF_A2, kk), a2p = LD(FF_A2, kk + IS);
  double a3 = LD(FF_A3, kk), a3p = LD(FF_A3, kk + IL);
  double zz = 0.;
  if (p.idi1 != 0 && I <= min(p.idi1, b.imax)) zz = .5 * (a1 + a1p);
  if (p.idi2 != 0 && J <= min(p.idi2, b.jmax)) zz = dmax(.5 * (a2 + a2p), zz);
  if (p.idi3 != 0 && K <= min(p.idi3, b.kmax)) zz = dmax(.5 * (a3 + a3p), zz);
  double ro = b.a[FF_RO][kk], u = b.a[FF_U][kk], v = b.a[FF_V][kk], w = b.a[FF_W][kk];
  double c = b.a[FF_C][kk], P = b.a[FF_P][kk];
  double pvol = 1. / LD(FF_VOL, kk), ypro = 1. / (ro + 1.e-10);
  double a1k = .5 * (a1 + a1p), a2k = .5 * (a2 + a2p), a3k = .5 * (a3 + a3p);
  double ucii = .5 * (LD(FF_A1XA, kk) * a1 + LD(FF_A1XA, kk + 1) * a1p) * u
              + .5 * (LD(FF_A1YA, kk) * a1 + LD(FF_A1YA, kk + 1) * a1p) * v
              + .5 * (LD(FF_A1ZA, kk) * a1 + LD(FF_A1ZA, kk + 1) * a1p) * w;
  double vcii = .5 * (LD(FF_A2XA, kk) * a2 + LD(FF_A2XA, kk + IS) * a2p) * u
              + .5 * (LD(FF_A2YA, kk) * a2 + LD(FF_A2YA, kk + IS) * a2p) * v
              + .5 * (LD(FF_A2ZA, kk) * a2 + LD(FF_A2ZA, kk + IS) * a2p) * w;
  double wcii = .5 * (LD(FF_A3XA, kk) * a3 + LD(FF_A3XA, kk + IL) * a3p) * u
              + .5 * (LD(FF_A3YA, kk) * a3 + LD(FF_A3YA, kk + IL) * a3p) * v
              + .5 * (LD(FF_A3ZA, kk) * a3 + LD(FF_A3ZA, kk + IL) * a3p) * w;
#undef LD
  double b1 = pvol * (fabs(ucii) + fabs(vcii) + fabs(wcii) + c * sqrt(a1k * a1k + a2k * a2k + a3k * a3k)) / cfl;
  double rnum = zz * zz * (pvol * pvol) * ypro;
  double tt = rnum * (b.a[FF_VIS][kk] + p.pr / p.prt * b.a[FF_VIST][kk]) / p.cdiff;
  double b11 = dmax(b1, 2. * tt * p.pvisc);
  double denlow = 1. + dmax(0., (p.frspre - 2. * P) / P);
  double denmax = 1. + dmax(0., (ro - 2. * p.frsden) * ypro) * 5.;
  double dtl = 1. / (b11 * dmax(denlow, denmax));
  if (p.timel) dtl = dtl * p.dt / (1.5 * dtl + p.dt);   // TIMEL dual time step, base3c.f:206-215
  b.a[FF_DTL][kk] = dtl;
  if (mode == 1) return;
  // LOCDT + COPR
  double dri = dtl * b.a[FF_DRO][kk], dmi = dtl * b.a[FF_DM][kk], dni = dtl * b.a[FF_DN][kk];
  double dwi = dtl * b.a[FF_DW][kk], dre = dtl * b.a[FF_DE][kk];
  double yp = 1. / ro, drodh = b.a[FF_DRDH][kk], drodp = b.a[FF_DRDP][kk];
  double beta = .5 * (u * u + v * v + w * w);
  double dkin = u * dmi + v * dni + w * dwi;
  b.a[FF_DM][kk] = yp * (-u * dri + dmi);
  b.a[FF_DN][kk] = yp * (-v * dri + dni);
  b.a[FF_DW][kk] = yp * (-w * dri + dwi);
  double hi = yp * (b.a[FF_E][kk] + P);
  double dei = dre - (hi - 2 * beta) * dri - dkin;
  double dpi = c * c * (dri - drodh * yp * dei);
  b.a[FF_DRO][kk] = (dri - drodp * dpi) / drodh;
  b.a[FF_DE][kk] = dpi;
}

// LU-SGS coefficients of one interior cell (PREDGS imps4.f:388-470 for
// upper=1, CORRGS imps4.f:120-200 + DIAGGS imps4.f:604 for upper=0): the
// split eigenvalue coefficients x[d][0..2] of the face the cell's product in
// direction d crosses, DT1 = THETA*DTL, the scalings SCINV / SCINP and the
// diagonal factor of the lower sweep.
struct CellCoef {
  double x[3][3], dt1, scinv, scinp, fdiag;
};

FF_DI void lusgs_cell_coef(const DevBlock& b, const ff_params& p, int I, int J, int K, int upper, CellCoef& cc) {
  const int IS = b.is, IL = b.il;
  size_t N = ix(b, I, J, K);
#define LD(s, n) __ldg(b.a[s] + (n))
  double u = LD(FF_U, N), v = LD(FF_V, N), w = LD(FF_W, N), c = LD(FF_C, N), ro = LD(FF_RO, N);
  double vol = LD(FF_VOL, N), mu = LD(FF_VIST, N) + LD(FF_VIS, N);
  const int st[3] = {1, IS, IL};
  const int idi[3] = {p.idi1, p.idi2, p.idi3};
  const int idx[3] = {I, J, K};
  double xa[3], rmax_lo[3];
  for (int d = 0; d < 3; d++) {
    const int ao = 4 * d;
    size_t fN = upper ? N : N + st[d];          // face normal used for the eigenvalue
    size_t nb = upper ? N - st[d] : N + st[d];  // cell across that face
    double ff = 2.;
    if (upper && idx[d] == 1) ff = 4.;
    if (idx[d] > idi[d]) ff = 0.;
    double rl1 = LD(FF_A1XA + ao, fN) * u + LD(FF_A1YA + ao, fN) * v + LD(FF_A1ZA + ao, fN) * w;
    double rnum = (vol + LD(FF_VOL, nb)) * (ro + LD(FF_RO, nb));
    double tt = (ff * 2.) * LD(FF_A1 + ao, N) / rnum * (mu + LD(FF_VIST, nb) + LD(FF_VIS, nb));
    double rmax = fabs(rl1) + c;
    double sg = upper ? -1. : 1.;
    cc.x[d][0] = (rl1 + sg * rmax) * .5 + sg * tt;
    cc.x[d][1] = (rl1 + c + sg * rmax) * .5 + sg * tt;
    cc.x[d][2] = (rl1 - c + sg * rmax) * .5 + sg * tt;
    xa[d] = rmax + tt;
    // SCINP uses the spectral radius of the eigenvalue face in both sweeps
    rmax_lo[d] = fabs(rl1) + c;
  }
  double dt1 = p.theta * LD(FF_DTL, N);
  double a1 = LD(FF_A1, N), a2 = LD(FF_A2, N), a3 = LD(FF_A3, N);
  double a1p = LD(FF_A1, N + 1), a2p = LD(FF_A2, N + IS), a3p = LD(FF_A3, N + IL);
  cc.dt1 = dt1;
  cc.scinv = upper ? 1. / (vol + dt1 * (xa[0] * a1 + xa[1] * a2 + xa[2] * a3))
                   : 1. / (vol + dt1 * (xa[0] * a1p + xa[1] * a2p + xa[2] * a3p));
  cc.scinp = 1. / (vol + dt1 * (rmax_lo[0] * a1 + rmax_lo[1] * a2 + rmax_lo[2] * a3));
  cc.fdiag = 1.;
  if (!upper) {   // DIAGGS imps4.f:614-660
    double r[6];
    for (int d = 0; d < 3; d++) {
      const int ao = 4 * d;
      size_t fp = N + st[d];
      r[2 * d] = fabs(LD(FF_A1XA + ao, N) * u + LD(FF_A1YA + ao, N) * v + LD(FF_A1ZA + ao, N) * w) + c;
      r[2 * d + 1] = fabs(LD(FF_A1XA + ao, fp) * u + LD(FF_A1YA + ao, fp) * v + LD(FF_A1ZA + ao, fp) * w) + c;
    }
    double sc = .5 * (a1 * r[0] + a1p * r[1] + a2 * r[2] + a2p * r[3] + a3 * r[4] + a3p * r[5]);
    cc.fdiag = 1. + p.theta * LD(FF_DTL, N) / vol * sc;
  }
#undef LD
}

// Coefficients in the storage layout, coef[c*ntot + n], c = xi(3) xj(3)
// xk(3) dt1 scinv scinp fdiag (the allocation-free stage's sweep).
template <typename CT>
__global__ void k_lusgs_coef(DevBlock b, ff_params p, CT* coef, int upper) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.imax * b.jmax * b.kmax) return;
  int I = t % b.imax + 1, J = (t / b.imax) % b.jmax + 1, K = t / (b.imax * b.jmax) + 1;
  CellCoef cc;
  lusgs_cell_coef(b, p, I, J, K, upper, cc);
  size_t nt = b.ntot, N = ix(b, I, J, K);
  for (int d = 0; d < 3; d++)
    for (int e = 0; e < 3; e++) coef[(3 * d + e) * nt + N] = (CT)cc.x[d][e];
  coef[9 * nt + N] = (CT)cc.dt1;
  coef[10 * nt + N] = (CT)cc.scinv;
  coef[11 * nt + N] = (CT)cc.scinp;
  coef[12 * nt + N] = (CT)cc.fdiag;
}

// The static part of one sweep's layout (see sw_index): the unit normals
// of the three products' faces, the areas and the volume -- the metrics
// only, written once per block.
template <typename CT>
__global__ void k_sweep_static(DevBlock b, CT* sw, int upper) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t row = (size_t)(b.imax + b.jmax - 1) * b.jmax;
  if (t >= row * b.kmax) return;
  const int K = (int)(t / row) + 1;
  const int r = (int)(t % row), J = r % b.jmax + 1, I = r / b.jmax + 2 - J;
  if (I < 1 || I > b.imax) return;
  const size_t ns = sw_size(b.imax, b.jmax, b.kmax), S = sw_index(b, I, J, K);
  const size_t N = ix(b, I, J, K);
  const int IS = b.is, IL = b.il;
  const int st[3] = {1, IS, IL};
  sw[SW_VOL * ns + S] = (CT)__ldg(b.a[FF_VOL] + N);
  sw[SW_A1 * ns + S] = (CT)__ldg(b.a[FF_A1] + (upper ? N + 1 : N));
  sw[SW_A2 * ns + S] = (CT)__ldg(b.a[FF_A2] + (upper ? N + IS : N));
  sw[SW_A3 * ns + S] = (CT)__ldg(b.a[FF_A3] + (upper ? N + IL : N));
  for (int d = 0; d < 3; d++) {
    const int ao = 4 * d;
    size_t fN = upper ? N : N + st[d];   // the face the product in direction d crosses
    sw[(SW_F + 3 * d + 0) * ns + S] = (CT)__ldg(b.a[FF_A1XA + ao] + fN);
    sw[(SW_F + 3 * d + 1) * ns + S] = (CT)__ldg(b.a[FF_A1YA + ao] + fN);
    sw[(SW_F + 3 * d + 2) * ns + S] = (CT)__ldg(b.a[FF_A1ZA + ao] + fN);
  }
}

// The state-dependent part of one sweep's layout (see sw_index; the static
// part is k_sweep_static's), and for the first sweep (upper = 1) the
// right-hand side DRO..DE(,DRK,DEPS) copied into dwp in the same layout and
// type.
template <typename CT>
__global__ void k_sweep_coef(DevBlock b, ff_params p, CT* sw, CT* dwp, int upper) {
  // one thread per slot of the sweep layout, in slot order, so that the
  // ~50 stores of a warp are contiguous; slots outside the block (I < 1 or
  // I > IMAX on a diagonal) have no cell
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t row = (size_t)(b.imax + b.jmax - 1) * b.jmax;
  if (t >= row * b.kmax) return;
  const int K = (int)(t / row) + 1;
  const int r = (int)(t % row), J = r % b.jmax + 1, I = r / b.jmax + 2 - J;
  if (I < 1 || I > b.imax) return;
  CellCoef cc;
  lusgs_cell_coef(b, p, I, J, K, upper, cc);
  const size_t ns = sw_size(b.imax, b.jmax, b.kmax), S = sw_index(b, I, J, K);
  const size_t N = ix(b, I, J, K);
  sw[SW_DT1 * ns + S] = (CT)cc.dt1;
  sw[SW_SCINV * ns + S] = (CT)cc.scinv;
  sw[SW_SCINP * ns + S] = (CT)cc.scinp;
  sw[SW_FD * ns + S] = (CT)cc.fdiag;
  CT ro = (CT)__ldg(b.a[FF_RO] + N), c = (CT)__ldg(b.a[FF_C] + N);
  sw[SW_RO * ns + S] = ro;
  CT ypro = CT(1) / ro;
  sw[(SW_SC + 0) * ns + S] = ypro;
  sw[(SW_SC + 1) * ns + S] = ro * c;
  sw[(SW_SC + 2) * ns + S] = (CT(.5) * ypro) / c;
  if (p.iturb >= 3) {
    CT rk = (CT)__ldg(b.a[FF_RK] + N), drdp = (CT)__ldg(b.a[FF_DRDP] + N), drdh = (CT)__ldg(b.a[FF_DRDH] + N);
    sw[(SW_SC + 3) * ns + S] = CT(.667) * rk * (ypro * ypro) * drdh;
    sw[(SW_SC + 4) * ns + S] = CT(1) / (CT(1) + CT(.667) * rk * ypro * drdp);
  }
  for (int d = 0; d < 3; d++)
    for (int e = 0; e < 3; e++) sw[(SW_L + 3 * d + e) * ns + S] = (CT)cc.x[d][e];
  if (upper) {
    const int nv = p.iturb >= 3 ? 7 : 5;
    for (int v = 0; v < nv; v++) dwp[v * ns + S] = (CT)b.a[FF_DRO + v][N];
  }
}

// The increments back from the sweep layout into DRO..DE(,DRK,DEPS).
template <typename CT>
__global__ void k_sweep_out(DevBlock b, const CT* __restrict__ dwp, int nv) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.imax * b.jmax * b.kmax) return;
  int I = t % b.imax + 1, J = (t / b.imax) % b.jmax + 1, K = t / (b.imax * b.jmax) + 1;
  const size_t ns = sw_size(b.imax, b.jmax, b.kmax), S = sw_index(b, I, J, K);
  const size_t N = ix(b, I, J, K);
  for (int v = 0; v < nv; v++) b.a[FF_DRO + v][N] = (double)dwp[v * ns + S];
}

// One LU-SGS sweep as i+j+k hyperplanes (cooperative, persistent).  The
// triangular system is the reference's (PREDGS: neighbours i+1, j+1, k+1 with
// the reference's dropped i+1 coupling in row J = JMAX, imps4.f:547-559;
// CORRGS: i-1, j-1, k-1), so the result equals its slab-by-slab order.
// dw: increment arrays (5 x ntot) of type CT; read through L2 (__ldcg)
// because other blocks write them during the sweep.
template <typename CT, int NV>
__global__ void k_lusgs_sweep_basic(DevBlock b, const CT* __restrict__ coef, CT* dw, int upper,
                                    unsigned* bar, int* err) {
  const int IMAX = b.imax, JMAX = b.jmax, KMAX = b.kmax, IS = b.is, IL = b.il;
  const size_t nt = b.ntot;
  const int nthreads = gridDim.x * blockDim.x;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nplanes = IMAX + JMAX + KMAX - 2;
  for (int s = 0; s < nplanes; s++) {
    int m = upper ? IMAX + JMAX + KMAX - s : 3 + s;
    int klo = max(1, m - IMAX - JMAX), khi = min(KMAX, m - 2);
    int npairs = (khi - klo + 1) * JMAX;
    for (int q = tid; q < npairs; q += nthreads) {
      int K = klo + q / JMAX, J = q % JMAX + 1, I = m - J - K;
      if (I < 1 || I > IMAX) continue;
      size_t N = ix(b, I, J, K);
      CT dt1 = coef[9 * nt + N];
      CT vol = (CT)__ldg(b.a[FF_VOL] + N);
      CT cd[NV];
      CT fd = upper ? CT(1) : coef[12 * nt + N];
#pragma unroll
      for (int v = 0; v < NV; v++) cd[v] = __ldcg(dw + v * nt + N) * fd;
      // the three neighbours: k first (reference order), then i and j
      CT ck[NV], yd[NV], bd[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) { ck[v] = 0; yd[v] = 0; bd[v] = 0; }
      const int st[3] = {1, IS, IL};
      // PREDGS drops the i+1 coupling of row J = JMAX unless bit 2 of upper
      // (predgs_full) asks for it; PRKEGS does not drop it
      const bool has[3] = {upper ? (I < IMAX && (NV == 7 || J < JMAX || (upper & 2))) : (I > 1), upper ? (J < JMAX) : (J > 1),
                           upper ? (K < KMAX) : (K > 1)};
#pragma unroll
      for (int d = 2; d >= 0; d--) {
        if (!has[d]) continue;
        size_t nb = upper ? N + st[d] : N - st[d];
        size_t fN = upper ? nb : N;              // shared face
        const int ao = 4 * d;
        CT x[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) x[v] = __ldcg(dw + v * nt + nb);
        CT out[NV];
        nb_product<CT, NV>(out, x, b, nb, (CT)__ldg(b.a[FF_C] + nb), (CT)__ldg(b.a[FF_RO] + nb),
                           (CT)__ldg(b.a[FF_A1XA + ao] + fN), (CT)__ldg(b.a[FF_A1YA + ao] + fN),
                           (CT)__ldg(b.a[FF_A1ZA + ao] + fN), coef[(3 * d) * nt + nb],
                           coef[(3 * d + 1) * nt + nb], coef[(3 * d + 2) * nt + nb]);
        CT* dst = d == 2 ? ck : (d == 0 ? yd : bd);
#pragma unroll
        for (int v = 0; v < NV; v++) dst[v] = out[v];
      }
      CT a3 = (CT)__ldg(b.a[FF_A3] + (upper ? N + IL : N));
      CT a1 = (CT)__ldg(b.a[FF_A1] + (upper ? N + 1 : N));
      CT a2 = (CT)__ldg(b.a[FF_A2] + (upper ? N + IS : N));
      CT scinv = coef[10 * nt + N], scinp = coef[11 * nt + N];
      CT res[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) {
        CT x = upper ? (-dt1 * a3 * ck[v] + vol * cd[v]) : (dt1 * a3 * ck[v] + vol * cd[v]);
        x = upper ? x - dt1 * (a1 * yd[v] + a2 * bd[v]) : x + dt1 * (a1 * yd[v] + a2 * bd[v]);
        res[v] = x * (v == 4 ? scinp : scinv);
      }
#pragma unroll
      for (int v = 0; v < NV; v++) __stcg(dw + v * nt + N, res[v]);
    }
    if (!grid_barrier(bar, bar + 1, gridDim.x, err)) return;
  }
}

// The hyperplane sweep on the sweep layout (k_sweep_coef): the cells of a
// plane with one K and consecutive J are consecutive in sw and dwp, so each
// warp's loads are coalesced.  Each cell pulls the products of its three
// upstream neighbours from their increments and their precomputed frames,
// scalars and eigenvalue coefficients.
template <typename CT, int NV>
__global__ void k_lusgs_sweep(DevBlock b, const CT* __restrict__ sw, CT* dwp, int upper, unsigned* bar, int* err) {
  const int IMAX = b.imax, JMAX = b.jmax, KMAX = b.kmax;
  const int W = IMAX + JMAX - 1;
  const size_t ns = sw_size(IMAX, JMAX, KMAX);
  const int nthreads = gridDim.x * blockDim.x;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nplanes = IMAX + JMAX + KMAX - 2;
  const long off[3] = {JMAX, JMAX + 1, (long)W * JMAX};
  for (int s = 0; s < nplanes; s++) {
    const int m = upper ? IMAX + JMAX + KMAX - s : 3 + s;
    const int klo = max(1, m - IMAX - JMAX), khi = min(KMAX, m - 2);
    const int npairs = (khi - klo + 1) * JMAX;
    for (int q = tid; q < npairs; q += nthreads) {
      const int K = klo + q / JMAX, J = q % JMAX + 1, I = m - J - K;
      if (I < 1 || I > IMAX) continue;
      const size_t S = ((size_t)(K - 1) * W + (m - K - 2)) * JMAX + (J - 1);
      // PREDGS drops the i+1 coupling of row J = JMAX unless bit 2 of upper
      // (predgs_full) asks for it; PRKEGS does not drop it
      const bool has[3] = {upper ? (I < IMAX && (NV == 7 || J < JMAX || (upper & 2))) : (I > 1), upper ? (J < JMAX) : (J > 1),
                           upper ? (K < KMAX) : (K > 1)};
      CT ck[NV], yd[NV], bd[NV];
#pragma unroll
      for (int d = 2; d >= 0; d--) {   // k first (reference order), then i and j
        CT* dst = d == 2 ? ck : (d == 0 ? yd : bd);
        if (!has[d]) {
#pragma unroll
          for (int v = 0; v < NV; v++) dst[v] = CT(0);
          continue;
        }
        const size_t nb = upper ? S + off[d] : S - off[d];
        CT x[NV], f[3], sc[5], l[3];
#pragma unroll
        for (int v = 0; v < NV; v++) x[v] = __ldcg(dwp + v * ns + nb);
#pragma unroll
        for (int c = 0; c < 3; c++) f[c] = __ldg(sw + (SW_F + 3 * d + c) * ns + nb);
#pragma unroll
        for (int c = 0; c < (NV == 7 ? 5 : 3); c++) sc[c] = __ldg(sw + (SW_SC + c) * ns + nb);
#pragma unroll
        for (int e = 0; e < 3; e++) l[e] = __ldg(sw + (SW_L + 3 * d + e) * ns + nb);
        nb_product_pre<CT, NV>(dst, x, f, sc, NV == 7 ? __ldg(sw + SW_RO * ns + nb) : CT(0), l[0], l[1], l[2]);
      }
      const CT dt1 = __ldg(sw + SW_DT1 * ns + S), vol = __ldg(sw + SW_VOL * ns + S);
      const CT fd = upper ? CT(1) : __ldg(sw + SW_FD * ns + S);
      const CT a1 = __ldg(sw + SW_A1 * ns + S), a2 = __ldg(sw + SW_A2 * ns + S), a3 = __ldg(sw + SW_A3 * ns + S);
      const CT scinv = __ldg(sw + SW_SCINV * ns + S), scinp = __ldg(sw + SW_SCINP * ns + S);
#pragma unroll
      for (int v = 0; v < NV; v++) {
        CT cd = __ldcg(dwp + v * ns + S) * fd;
        CT x = upper ? (-dt1 * a3 * ck[v] + vol * cd) : (dt1 * a3 * ck[v] + vol * cd);
        x = upper ? x - dt1 * (a1 * yd[v] + a2 * bd[v]) : x + dt1 * (a1 * yd[v] + a2 * bd[v]);
        __stcg(dwp + v * ns + S, x * (v == 4 ? scinp : scinv));
      }
    }
    if (!grid_barrier(bar, bar + 1, gridDim.x, err)) return;
  }
}

// DRO/CP (imps3.f:483), FIN res3c.f:1077, the limits of CYCLES
// (ns3c.f:1553-1596: UPLIM/LOLIM res3c.f:3314-3401, PDTOP, LOLIMP), the
// interior *OLD copies of SUBIN and the max|dp| monitor (DROMXX, IDRXX=6).
__global__ void k_fin(DevBlock b, ff_params p, unsigned long long* dromax_bits, int divide_cp) {
  size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double amax = 0.;
  if (n < (size_t)b.ntot) {
    int i = (int)(n % b.is), j = (int)((n / b.is) % (b.jmax + 4)), k = (int)(n / b.il);
    bool kin = k >= 2 && k < b.kmax + 2, jin = j >= 2 && j < b.jmax + 2;
    bool interior = kin && jin && i >= 2 && i < b.imax + 2;
    double T = b.a[FF_TEMP][n], U = b.a[FF_U][n], V = b.a[FF_V][n], W = b.a[FF_W][n], PD = b.a[FF_PDIFF][n];
    const bool sst = p.iturb >= 3;
    if (interior) {
      double dt = b.a[FF_DRO][n];
      if (divide_cp) { dt = dt / b.a[FF_CP][n]; b.a[FF_DRO][n] = dt; }
      if (sst) {   // imps3.f:488-492, then FIN res3c.f:1190-1198
        double ro = b.a[FF_RO][n], drk = b.a[FF_DRK][n], deps = b.a[FF_DEPS][n];
        if (divide_cp) { drk = drk * ro; deps = deps * ro; b.a[FF_DRK][n] = drk; b.a[FF_DEPS][n] = deps; }
        double rkold = b.a[FF_RKOLD][n], epold = b.a[FF_EPSOLD][n];
        double rk = rkold + drk / (1. + fabs(drk) / (.45 * rkold));
        double re = epold + deps / (1. + fabs(deps) / (.90 * epold));
        b.a[FF_RK][n] = rk;
        b.a[FF_REPS][n] = re;
      }
      T = b.a[FF_TOLD][n] + dt;
      U = b.a[FF_UOLD][n] + b.a[FF_DM][n];
      V = b.a[FF_VOLD][n] + b.a[FF_DN][n];
      W = b.a[FF_WOLD][n] + b.a[FF_DW][n];
      PD = b.a[FF_POLD][n] + b.a[FF_DE][n];
      amax = fabs(b.a[FF_DE][n]);
    }
    if (kin && jin) {   // UPLIM range: interior k-planes, interior rows
      T = dmin(T, p.tuplim); U = dmin(U, 5000.); V = dmin(V, 5000.); W = dmin(W, 5000.);
    }
    T = dmax(T, p.tlolim); U = dmax(U, -5000.); V = dmax(V, -5000.); W = dmax(W, -5000.);
    double P = PD + p.frspre;
    double prelim = dmin(0., P - 0.01 * p.frspre);
    P = P - prelim; PD = PD - prelim;
    b.a[FF_TEMP][n] = T; b.a[FF_U][n] = U; b.a[FF_V][n] = V; b.a[FF_W][n] = W;
    b.a[FF_PDIFF][n] = PD; b.a[FF_P][n] = P;
    if (sst) {   // LOLIM of RK and REPS over every cell (FIN, then CYCLES)
      b.a[FF_RK][n] = dmax(b.a[FF_RK][n], p.rklim);
      b.a[FF_REPS][n] = dmax(b.a[FF_REPS][n], p.epslim);
    }
    if (interior) {
      b.a[FF_TOLD][n] = T; b.a[FF_UOLD][n] = U; b.a[FF_VOLD][n] = V; b.a[FF_WOLD][n] = W;
      b.a[FF_POLD][n] = PD;
    }
  }
  for (int o = 16; o > 0; o >>= 1) amax = dmax(amax, __shfl_down_sync(0xffffffffu, amax, o));
  if ((threadIdx.x & 31) == 0 && amax > 0.) atomicMax(dromax_bits, (unsigned long long)__double_as_longlong(amax));
}

// Standalone DRO/CP that ends IMPS (imps3.f:483) when it is called as a stage.
__global__ void k_fin_divide(DevBlock b, int sst) {
  size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (size_t)b.ntot) return;
  int i = (int)(n % b.is), j = (int)((n / b.is) % (b.jmax + 4)), k = (int)(n / b.il);
  if (i >= 2 && i < b.imax + 2 && j >= 2 && j < b.jmax + 2 && k >= 2 && k < b.kmax + 2) {
    b.a[FF_DRO][n] = b.a[FF_DRO][n] / b.a[FF_CP][n];
    if (sst) {   // imps3.f:488-492
      b.a[FF_DRK][n] = b.a[FF_DRK][n] * b.a[FF_RO][n];
      b.a[FF_DEPS][n] = b.a[FF_DEPS][n] * b.a[FF_RO][n];
    }
  }
}

// ---------------------------------------------------------------------------
// Multigrid transfers (FAS V-cycle of CYCLES ns3c.f:1607-2170)
// ---------------------------------------------------------------------------

// TRANSF multi.f:156: volume-weighted restriction of TEMP,U,V,W,PDIFF,EPS2,
// VIST and of the residuals (into P2H) for coarse cells 0..MAX+1, and the
// interior *OLD copies.
__global__ void k_transf(DevBlock f, DevBlock c, int sst) {
  int ni = c.imax + 2, nj = c.jmax + 2, nk = c.kmax + 2;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ni * nj * nk) return;
  int I = t % ni, J = (t / ni) % nj, K = t / (ni * nj);
  size_t N = ix(c, I, J, K);
  size_t ijk = ix(f, 2 * I - 1, 2 * J - 1, 2 * K - 1);
  size_t o[8] = {ijk + f.is + 1, ijk, ijk + 1, ijk + f.is,
                 ijk + f.is + 1 + f.il, ijk + f.il, ijk + 1 + f.il, ijk + f.is + f.il};
  const double* VOL = f.a[FF_VOL];
  double vv[8];
#pragma unroll
  for (int q = 0; q < 8; q++) vv[q] = VOL[o[q]];
  double pvol = 1. / c.a[FF_VOL][N];
  const int vs[12] = {FF_TEMP, FF_U, FF_V, FF_W, FF_PDIFF, FF_EPS2, FF_VIST, FF_DRO, FF_DM, FF_DN, FF_DW, FF_DE};
  const int ds[12] = {FF_TEMP, FF_U, FF_V, FF_W, FF_PDIFF, FF_EPS2, FF_VIST, FF_ROP2H, FF_RMP2H, FF_RNP2H, FF_RWP2H, FF_EP2H};
#pragma unroll
  for (int v = 0; v < 12; v++) {
    const double* X = f.a[vs[v]];
    double s = 0.;
#pragma unroll
    for (int q = 0; q < 8; q++) s += vv[q] * X[o[q]];
    c.a[ds[v]][N] = s * pvol;
  }
  if (sst) {   // TRANKE multi.f:434: RK, REPS and DRK, DEPS into RKP2H, EPP2H
    const int vk[4] = {FF_RK, FF_REPS, FF_DRK, FF_DEPS}, dk[4] = {FF_RK, FF_REPS, FF_RKP2H, FF_EPP2H};
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const double* X = f.a[vk[v]];
      double s = 0.;
#pragma unroll
      for (int q = 0; q < 8; q++) s += vv[q] * X[o[q]];
      c.a[dk[v]][N] = s * pvol;
    }
  }
  if (I >= 1 && I <= c.imax && J >= 1 && J <= c.jmax && K >= 1 && K <= c.kmax) {
    c.a[FF_TOLD][N] = c.a[FF_TEMP][N];
    c.a[FF_UOLD][N] = c.a[FF_U][N];
    c.a[FF_VOLD][N] = c.a[FF_V][N];
    c.a[FF_WOLD][N] = c.a[FF_W][N];
    c.a[FF_POLD][N] = c.a[FF_PDIFF][N];
    if (sst) { c.a[FF_RKOLD][N] = c.a[FF_RK][N]; c.a[FF_EPSOLD][N] = c.a[FF_REPS][N]; }
  }
}

// Coarse ghost rings of TRANSF (multi.f:250-432): P2H = 0 in both ghost
// layers; the second ghost layer of each face copies the first one.
__global__ void k_transf_ring(DevBlock c, int sst) {
  size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (size_t)c.ntot) return;
  int i = (int)(n % c.is) - 1, j = (int)((n / c.is) % (c.jmax + 4)) - 1, k = (int)(n / c.il) - 1;
  bool gi = i < 1 || i > c.imax, gj = j < 1 || j > c.jmax, gk = k < 1 || k > c.kmax;
  if (!(gi || gj || gk)) return;
#pragma unroll
  for (int v = 0; v < 5; v++) c.a[FF_ROP2H + v][n] = 0.;
  if (sst) { c.a[FF_RKP2H][n] = 0.; c.a[FF_EPP2H][n] = 0.; }
  // second-layer face ghosts copy the first layer along the face normal
  // (cells in the second layer of two directions are not used on coarse
  // levels and are left alone)
  int second = (i == -1 || i == c.imax + 2) + (j == -1 || j == c.jmax + 2) + (k == -1 || k == c.kmax + 2);
  if (second != 1) return;
  int src_off = 0;
  if (i == -1) src_off = 1; else if (i == c.imax + 2) src_off = -1;
  else if (j == -1) src_off = c.is; else if (j == c.jmax + 2) src_off = -c.is;
  else if (k == -1) src_off = c.il; else if (k == c.kmax + 2) src_off = -c.il;
  if (src_off == 0) return;
  const int vs[9] = {FF_TEMP, FF_U, FF_V, FF_W, FF_PDIFF, FF_EPS2, FF_VIST, FF_RK, FF_REPS};
  const int nv = sst ? 9 : 7;
  for (int v = 0; v < nv; v++) c.a[vs[v]][n] = c.a[vs[v]][n + src_off];
}

// FORCFU multi.f:1609 (mode 0: P2H -= R) and ADDRES multi.f:1686 (mode 1:
// R = P2H + R), every cell of the level.
__global__ void k_forcing(DevBlock b, int mode, int sst) {
  size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (size_t)b.ntot) return;
  const int ps[7] = {FF_ROP2H, FF_RMP2H, FF_RNP2H, FF_RWP2H, FF_EP2H, FF_RKP2H, FF_EPP2H};
  const int nv = sst ? 7 : 5;
  for (int v = 0; v < nv; v++) {
    double* P2 = b.a[ps[v]];
    double* R = b.a[FF_DRO + v];
    if (mode == 0) P2[n] = P2[n] - R[n];
    else R[n] = P2[n] + R[n];
  }
}

// INTERT multi.f:2051 -> INTERO 2007: damped injection of the coarse k and
// omega corrections (CMGK, CMGEPS) into the fine interior.
__global__ void k_intert(DevBlock c, DevBlock f, ff_params p) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= f.imax * f.jmax * f.kmax) return;
  int I = t % f.imax + 1, J = (t / f.imax) % f.jmax + 1, K = t / (f.imax * f.jmax) + 1;
  size_t N = ix(c, (I + 1) / 2, (J + 1) / 2, (K + 1) / 2), F = ix(f, I, J, K);
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const double cc1 = q == 0 ? p.cmgk : p.cmgeps, cc2 = cc1 + 1.E-7;
    double drok = c.a[q == 0 ? FF_RK : FF_REPS][N] - c.a[q == 0 ? FF_RKOLD : FF_EPSOLD][N];
    double* R = f.a[q == 0 ? FF_RK : FF_REPS];
    double r = R[F];
    R[F] = r + cc1 * r * drok / (cc2 * r + fabs(drok));
  }
}

// INTERP multi.f:1763: inject the coarse correction into the 8 children.
__global__ void k_interp(DevBlock c, DevBlock f) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= f.imax * f.jmax * f.kmax) return;
  int I = t % f.imax + 1, J = (t / f.imax) % f.jmax + 1, K = t / (f.imax * f.jmax) + 1;
  size_t N = ix(c, (I + 1) / 2, (J + 1) / 2, (K + 1) / 2), F = ix(f, I, J, K);
  double dp = c.a[FF_PDIFF][N] - c.a[FF_POLD][N];
  f.a[FF_TEMP][F] = f.a[FF_TEMP][F] + (c.a[FF_TEMP][N] - c.a[FF_TOLD][N]);
  f.a[FF_U][F] = f.a[FF_U][F] + (c.a[FF_U][N] - c.a[FF_UOLD][N]);
  f.a[FF_V][F] = f.a[FF_V][F] + (c.a[FF_V][N] - c.a[FF_VOLD][N]);
  f.a[FF_W][F] = f.a[FF_W][F] + (c.a[FF_W][N] - c.a[FF_WOLD][N]);
  f.a[FF_P][F] = f.a[FF_P][F] + dp;
  f.a[FF_PDIFF][F] = f.a[FF_PDIFF][F] + dp;
}

// FIN on a coarse level (update = 1: UPLIM/LOLIM TEMP, LOLIMP, no PDTOP,
// ns3c.f:1935-1990) and the limits after INTERP (update = 0, ns3c.f:2059-2125:
// LOLIMP; the two-equation branch also limits TEMP, RK and REPS).
__global__ void k_fin_coarse(DevBlock b, ff_params p, int update) {
  size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (size_t)b.ntot) return;
  int i = (int)(n % b.is), j = (int)((n / b.is) % (b.jmax + 4)), k = (int)(n / b.il);
  bool kin = k >= 2 && k < b.kmax + 2, jin = j >= 2 && j < b.jmax + 2;
  bool interior = kin && jin && i >= 2 && i < b.imax + 2;
  const bool sst = p.iturb >= 3;
  double T = b.a[FF_TEMP][n];
  if (update && interior) {
    T = b.a[FF_TOLD][n] + b.a[FF_DRO][n];
    b.a[FF_U][n] = b.a[FF_UOLD][n] + b.a[FF_DM][n];
    b.a[FF_V][n] = b.a[FF_VOLD][n] + b.a[FF_DN][n];
    b.a[FF_W][n] = b.a[FF_WOLD][n] + b.a[FF_DW][n];
    b.a[FF_PDIFF][n] = b.a[FF_POLD][n] + b.a[FF_DE][n];
    if (sst) {   // FIN res3c.f:1190-1198
      double drk = b.a[FF_DRK][n], deps = b.a[FF_DEPS][n];
      double rkold = b.a[FF_RKOLD][n], epold = b.a[FF_EPSOLD][n];
      b.a[FF_RK][n] = rkold + drk / (1. + fabs(drk) / (.45 * rkold));
      b.a[FF_REPS][n] = epold + deps / (1. + fabs(deps) / (.90 * epold));
    }
  }
  if (sst) {   // LOLIM of RK, REPS over every cell (FIN; after INTERP, CYCLES)
    b.a[FF_RK][n] = dmax(b.a[FF_RK][n], p.rklim);
    b.a[FF_REPS][n] = dmax(b.a[FF_REPS][n], p.epslim);
  }
  // TEMP limits after a coarse FIN, and after INTERP on the two-equation branch
  if (update || sst) {
    if (kin && jin) T = dmin(T, p.tuplim);
    T = dmax(T, p.tlolim);
    b.a[FF_TEMP][n] = T;
  }
  double P = b.a[FF_P][n];
  double prelim = dmin(0., P - 0.01 * p.frspre);
  b.a[FF_P][n] = P - prelim;
  b.a[FF_PDIFF][n] = b.a[FF_PDIFF][n] - prelim;
}

// CONNEC ns3c.f:8605 (EXPTOT/IMPVO2 gluebm.f:6819/6964) for aligned 1:1
// patches of all blocks in one launch: blockIdx.y = connection item; the two
// interior layers of the source block fill the two ghost layers of the
// destination patch (TEMP,U,V,W,E,EPS2,VIST,CH,P,PDIFF,RK,REPS, as BOUNDI passes).
struct ConnItem { int dst, src; ff_patch pa; };

// The donor face cell (ad, cd) of receiver patch point (a, c) of a 1:1
// connection in orientation ICON(14) = pa.iori: the donor's export order
// (second in-face index fastest on odd faces, first on even faces; EXPVOL
// gluebm.f:6115-6136), the receiver's import order (first index fastest on
// odd faces, second on even; IMPVO2 7040-7080) and PERMUT's turn of the
// receiver sequence (gluebm.f:4868).
FF_DI void conn_donor(const ff_patch& pa, int a, int c, int& ad, int& cd) {
  const int n1 = pa.r1b - pa.r1a + 1, n2 = pa.r2b - pa.r2a + 1;
  const bool rodd = pa.iface & 1, dodd = pa.nface & 1;
  const int P = rodd ? n1 : n2, Q = rodd ? n2 : n1;
  const int x = rodd ? a - pa.r1a + 1 : c - pa.r2a + 1;
  const int y = rodd ? c - pa.r2a + 1 : a - pa.r1a + 1;
  int u, v;
  switch (pa.iori & 3) {
    case 1: u = Q + 1 - y; v = x; break;
    case 2: u = P + 1 - x; v = Q + 1 - y; break;
    case 3: u = y; v = P + 1 - x; break;
    default: u = x; v = y;
  }
  if (dodd) { cd = pa.n2a + u - 1; ad = pa.n1a + v - 1; }
  else { ad = pa.n1a + u - 1; cd = pa.n2a + v - 1; }
}

__global__ void k_connec(const DevBlock* __restrict__ blocks, const ConnItem* __restrict__ items) {
  const ConnItem& it = items[blockIdx.y];
  const ff_patch& pa = it.pa;
  int n1 = pa.r1b - pa.r1a + 1, n2 = pa.r2b - pa.r2a + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n1 * n2) return;
  int a = pa.r1a + t % n1, c = pa.r2a + t / n1;
  const DevBlock& d = blocks[it.dst];
  const DevBlock& s = blocks[it.src];
  FaceG fd = face_g(d, pa.iface), fs = face_g(s, pa.nface);
  int ad, cd;
  conn_donor(pa, a, c, ad, cd);
  size_t L = face_cell(d, fd, a, c);
  size_t S = face_cell(s, fs, ad, cd);
  const int vs[12] = {FF_TEMP, FF_U, FF_V, FF_W, FF_E, FF_EPS2, FF_VIST, FF_CH, FF_P, FF_PDIFF, FF_RK, FF_REPS};
  int lsd = fd.idir * fd.s, lss = fs.idir * fs.s;
#pragma unroll
  for (int g = 1; g <= 2; g++) {
    size_t G = L - g * lsd, Q = S + (g - 1) * lss;
#pragma unroll
    for (int v = 0; v < 12; v++) d.a[vs[v]][G] = s.a[vs[v]][Q];
  }
}

// Halo pack (mode 0, from the source block) / unpack (mode 1, into the
// destination's ghost layers) of remote 1:1 patches; blockIdx.y = item.
struct HaloItem { int blk, mode; long long offset; ff_patch pa; };

__global__ void k_halo(const DevBlock* __restrict__ blocks, const HaloItem* __restrict__ items,
                       int mode, double* __restrict__ sbuf, const double* __restrict__ rbuf) {
  const HaloItem& it = items[blockIdx.y];
  if (it.mode != mode) return;
  const ff_patch& pa = it.pa;
  int n1 = pa.r1b - pa.r1a + 1, n2 = pa.r2b - pa.r2a + 1, n = n1 * n2;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int a = t % n1, c = t / n1;
  const DevBlock& b = blocks[it.blk];
  const int vs[12] = {FF_TEMP, FF_U, FF_V, FF_W, FF_E, FF_EPS2, FF_VIST, FF_CH, FF_P, FF_PDIFF, FF_RK, FF_REPS};
  if (mode == 0) {
    FaceG fs = face_g(b, pa.nface);
    int ad, cd;
    conn_donor(pa, a + pa.r1a, c + pa.r2a, ad, cd);
    size_t S = face_cell(b, fs, ad, cd);
    int lss = fs.idir * fs.s;
    double* o = sbuf + it.offset;
#pragma unroll
    for (int g = 0; g < 2; g++)
#pragma unroll
      for (int v = 0; v < 12; v++) o[(size_t)(g * 12 + v) * n + t] = b.a[vs[v]][S + g * lss];
  } else {
    FaceG fd = face_g(b, pa.iface);
    size_t L = face_cell(b, fd, a + pa.r1a, c + pa.r2a);
    int lsd = fd.idir * fd.s;
    const double* o = rbuf + it.offset;
#pragma unroll
    for (int g = 0; g < 2; g++)
#pragma unroll
      for (int v = 0; v < 12; v++) b.a[vs[v]][L - (g + 1) * lsd] = o[(size_t)(g * 12 + v) * n + t];
  }
}

// SUBIN ns3c.f:9742: the *OLD copies of the interior cells.
__global__ void k_subin_copy(DevBlock b) {
  size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (size_t)b.ntot) return;
  int i = (int)(n % b.is), j = (int)((n / b.is) % (b.jmax + 4)), k = (int)(n / b.il);
  if (!(i >= 2 && i < b.imax + 2 && j >= 2 && j < b.jmax + 2 && k >= 2 && k < b.kmax + 2)) return;
  b.a[FF_TOLD][n] = b.a[FF_TEMP][n];
  b.a[FF_UOLD][n] = b.a[FF_U][n];
  b.a[FF_VOLD][n] = b.a[FF_V][n];
  b.a[FF_WOLD][n] = b.a[FF_W][n];
  b.a[FF_POLD][n] = b.a[FF_PDIFF][n];
}

// max |DE| over the interior (DROMXX, IDRXX = 6) into dm_bits.
__global__ void k_maxabs_de(DevBlock b, unsigned long long* dm_bits) {
  double amax = 0.;
  int ncell = b.imax * b.jmax * b.kmax;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += gridDim.x * blockDim.x) {
    int I = t % b.imax + 1, J = (t / b.imax) % b.jmax + 1, K = t / (b.imax * b.jmax) + 1;
    amax = dmax(amax, fabs(b.a[FF_DE][ix(b, I, J, K)]));
  }
  for (int o = 16; o > 0; o >>= 1) amax = dmax(amax, __shfl_down_sync(0xffffffffu, amax, o));
  if ((threadIdx.x & 31) == 0 && amax > 0.) atomicMax(dm_bits, (unsigned long long)__double_as_longlong(amax));
}

// TIMDER res3c.f:3014 / TIMDKE res3c.f:3062 on the interior cells: the
// second-order physical-time derivative of TIMEL added to the residual,
// PDT * (-1.5 VOL (Q - Q2) + 0.5 VOL (Q2 - Q3)) with PDT = 1 / (VOL DT).
template <int NV>
__global__ void k_timder(DevBlock b, ff_params p) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.imax * b.jmax * b.kmax) return;
  int I = t % b.imax + 1, J = (t / b.imax) % b.jmax + 1, K = t / (b.imax * b.jmax) + 1;
  const size_t n = ix(b, I, J, K);
  const int sq[7] = {FF_RO, FF_RM, FF_RN, FF_RW, FF_E, FF_RK, FF_REPS};
  const double vol = b.a[FF_VOL][n], pdt = 1. / (vol * p.dt);
#pragma unroll
  for (int v = 0; v < NV; v++) {
    const double q = b.a[sq[v]][n], q2 = b.a[FF_ROLE2 + v][n], q3 = b.a[FF_ROLE3 + v][n];
    b.a[FF_DRO + v][n] = b.a[FF_DRO + v][n] + pdt * (-1.5 * vol * (q - q2) + 0.5 * vol * (q2 - q3));
  }
}

// STARTI res3c.f:3175 (mode 0: both old time levels = the state, every
// cell) and NEWTIM ns3c.f:9420 with R1 = 1 (mode 1: level n-1 <- level n,
// level n <- the state, interior cells).
__global__ void k_time_levels(DevBlock b, int nv, int mode) {
  const int sq[7] = {FF_RO, FF_RM, FF_RN, FF_RW, FF_E, FF_RK, FF_REPS};
  if (mode == 0) {
    size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= (size_t)b.ntot) return;
    for (int v = 0; v < nv; v++) {
      const double q = b.a[sq[v]][n];
      b.a[FF_ROLE3 + v][n] = q;
      b.a[FF_ROLE2 + v][n] = q;
    }
    return;
  }
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.imax * b.jmax * b.kmax) return;
  int I = t % b.imax + 1, J = (t / b.imax) % b.jmax + 1, K = t / (b.imax * b.jmax) + 1;
  const size_t n = ix(b, I, J, K);
  for (int v = 0; v < nv; v++) {
    b.a[FF_ROLE3 + v][n] = b.a[FF_ROLE2 + v][n];
    b.a[FF_ROLE2 + v][n] = b.a[sq[v]][n];
  }
}

#include "ff_sst.cuh"

}  // namespace ff

// ---------------------------------------------------------------------------
// LU-SGS sweep as a line wavefront inside one thread-block cluster.
//
// Thread (lj, lk) of tile t owns the i-line (J, K); at hyperplane m it
// handles the cell I = m - J - K of its line.  Like the reference (PREDGS
// imps4.f:345 / CORRGS imps4.f:76) each cell, once solved, produces the
// split-Jacobian products for its three downstream neighbours: the i
// neighbour is on the same line (kept in shared memory), the j and k
// neighbours are the lines (J -/+ 1, K) and (J, K -/+ 1), read at the next
// plane from shared memory -- from another CTA's shared memory (DSMEM) when
// the line belongs to another tile.  The triangular system is the
// reference's (incl. the dropped i+1 coupling in row J = JMAX of PREDGS), so
// the result equals the hyperplane and slab orders up to rounding.
//
// A CTA of the cluster holds tpc tiles, ng = min(tpc, 4) of them side by
// side (ng x 128 threads; a thread group takes every ng-th tile).  One split
// cluster barrier per plane: a thread arrives once its products are
// published and waits only before the next plane.  With STAGE (one tile per
// thread group) the thread starts, between arrive and wait, the
// asynchronous copy (cp.async) of its next cell's sweep data (the SW_N
// values of the sweep layout and the right-hand side) into its own
// shared-memory slots, so the memory latency of the next plane overlaps the
// barrier.  Without STAGE the cell data is read from global memory where it
// is used: the variant for many blocks' sweeps running side by side, where
// the other blocks' warps hide the latency and the smaller shared-memory
// footprint keeps more CTAs resident.  The published values are
// double-buffered, so a plane reads only the previous plane's outputs.
// ---------------------------------------------------------------------------
// 16x4-line tiles (two warps, each 16 consecutive J of two K rows, so a
// warp's sweep-layout loads are two 128-byte runs): a 16-CTA cluster then
// holds up to 160 tiles in one pass (10 per CTA, 640 threads), enough for
// the ~9,000 i-lines of a 2.4M-cell block.
constexpr int LTJ = 16, LTK = 4, LTHREADS = LTJ * LTK;
constexpr int LMAX_TPC = 10;         // tile groups per CTA (threads per CTA <= 640)
constexpr int LMAX_TPC_STAGE = 4;    // staged: <= 256 threads, so up to 255 registers a thread
constexpr int LSTAGE = SW_N + 7;     // staged values per thread: sweep data + right-hand side

struct LineGeom {
  int ntj, ntk, ntiles, cs, tpc;   // tiles in j/k, cluster size, tiles per CTA
  int ng;                          // thread groups of 128 per CTA (tiles in parallel)
};

// Shared memory of k_lusgs_lines: pub [2][tpc][2*NV][128] (j and k
// products), ydb [tpc][NV][128] (i products), with STAGE (one tile per
// thread group, ng == tpc) stage [LSTAGE][tpc*128].
__host__ __device__ inline size_t lines_smem_bytes(int nv, int tpc, size_t elem, bool stage) {
  return ((size_t)5 * nv + (stage ? LSTAGE : 0)) * tpc * LTHREADS * elem;
}

FF_DI void cp_async_ca(void* smem, const double* g) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(g) : "memory");
}
FF_DI void cp_async_ca(void* smem, const float* g) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(g) : "memory");
}
FF_DI void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
FF_DI void cluster_arrive_release() { asm volatile("barrier.cluster.arrive.release;\n" ::: "memory"); }
FF_DI void cluster_wait_acquire() { asm volatile("barrier.cluster.wait.acquire;\n" ::: "memory"); }

// Start the copy of one cell's sweep data into the thread's stage slots
// (stride = threads per CTA).
template <typename CT, int NV>
FF_DI void lines_stage(CT* stg, int stride, const CT* __restrict__ sw, const CT* dwp, size_t ns, size_t S,
                       int upper) {
#pragma unroll
  for (int c = 0; c < SW_N; c++) {
    if (c == SW_FD && upper) continue;
    if (NV == 5 && (c == SW_RO || c == SW_SC + 3 || c == SW_SC + 4)) continue;
    cp_async_ca(stg + c * stride, sw + c * ns + S);
  }
#pragma unroll
  for (int v = 0; v < NV; v++) cp_async_ca(stg + (SW_N + v) * stride, dwp + v * ns + S);
}

FF_DI void prefetch_l2(const void* g) { asm volatile("prefetch.global.L2 [%0];\n" ::"l"(g)); }

// The sweep data and right-hand side of one cell into L2 (the values
// lines_stage copies, without a destination).
template <typename CT, int NV>
FF_DI void lines_prefetch_l2(const CT* __restrict__ sw, const CT* dwp, size_t ns, size_t S, int upper) {
#pragma unroll
  for (int c = 0; c < SW_N; c++) {
    if (c == SW_FD && upper) continue;
    if (NV == 5 && (c == SW_RO || c == SW_SC + 3 || c == SW_SC + 4)) continue;
    prefetch_l2(sw + c * ns + S);
  }
#pragma unroll
  for (int v = 0; v < NV; v++) prefetch_l2(dwp + v * ns + S);
}

// A lane's line in one tile slot of its CTA, with the DSMEM sources of its
// j and k neighbours' products (offsets within one pub buffer).
template <typename CT>
struct LineDesc {
  bool ok, hj, hk;
  int J, K;
  const CT* srcj;
  const CT* srck;
};

template <typename CT, int NV>
FF_DI LineDesc<CT> line_desc(const cooperative_groups::cluster_group& cluster, CT* pub, const LineGeom& lg,
                             int JMAX, int KMAX, int upper, int rank, int q, int lj, int lk) {
  LineDesc<CT> d;
  d.ok = false;
  d.hj = d.hk = false;
  d.J = d.K = 0;
  d.srcj = d.srck = pub;
  const int t = q * lg.cs + rank;
  if (t >= lg.ntiles) return d;
  const int tj = t % lg.ntj, tk = t / lg.ntj;
  d.J = tj * LTJ + lj + 1;
  d.K = tk * LTK + lk + 1;
  d.ok = d.J <= JMAX && d.K <= KMAX;
  d.hj = upper ? (d.J < JMAX) : (d.J > 1);
  d.hk = upper ? (d.K < KMAX) : (d.K > 1);
  if (d.ok && d.hj) {   // line (J -/+ 1, K)
    const int Jn = upper ? d.J + 1 : d.J - 1;
    const int tn = tk * lg.ntj + (Jn - 1) / LTJ, ln = lk * LTJ + (Jn - 1) % LTJ;
    d.srcj = cluster.map_shared_rank(pub, tn % lg.cs) + (tn / lg.cs) * 2 * NV * LTHREADS + ln;
  }
  if (d.ok && d.hk) {   // line (J, K -/+ 1)
    const int Kn = upper ? d.K + 1 : d.K - 1;
    const int tn = ((Kn - 1) / LTK) * lg.ntj + tj, ln = ((Kn - 1) % LTK) * LTJ + lj;
    d.srck = cluster.map_shared_rank(pub, tn % lg.cs) + ((tn / lg.cs) * 2 * NV + NV) * LTHREADS + ln;
  }
  return d;
}

// The sweep of one block by one cluster.  The CTA may hold more thread
// groups than lg.ng (a batched launch sized for its largest block): the
// extra groups own no tile and only take part in the cluster barriers.
template <typename CT, int NV, bool STAGE>
FF_DI void lines_body(const DevBlock& b, const CT* __restrict__ sw, CT* dwp, int upper, const LineGeom& lg) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tpc = lg.tpc, ng = lg.ng, nthr = ng * LTHREADS;
  CT* pub = reinterpret_cast<CT*>(smem_raw);        // [2][tpc][2*NV][LTHREADS]: bd(NV), ck(NV)
  CT* ydb = pub + 2 * tpc * 2 * NV * LTHREADS;      // [tpc][NV][LTHREADS]
  CT* my = ydb + tpc * NV * LTHREADS + threadIdx.x; // stage [LSTAGE][nthr] (STAGE: ng == tpc)
  const int IMAX = b.imax, JMAX = b.jmax, KMAX = b.kmax;
  const int W = IMAX + JMAX - 1;
  const size_t ns = sw_size(IMAX, JMAX, KMAX);
  const int rank = (int)cluster.block_rank();
  const int g0 = threadIdx.x / LTHREADS, lane = threadIdx.x % LTHREADS, lj = lane % LTJ, lk = lane / LTJ;
  const int nplanes = IMAX + JMAX + KMAX - 2;
  const int pstride = tpc * 2 * NV * LTHREADS;   // one buffer of pub
  auto plane_cell = [&](int s, int J, int K, int& I, size_t& S) {
    const int m = upper ? IMAX + JMAX + KMAX - s : 3 + s;
    I = m - J - K;
    S = ((size_t)(K - 1) * W + (m - K - 2)) * JMAX + (J - 1);
    return I >= 1 && I <= IMAX;
  };
  for (int q = g0; q < tpc; q += ng)
#pragma unroll
    for (int v = 0; v < NV; v++) ydb[(q * NV + v) * LTHREADS + lane] = CT(0);
  // the thread group's first tile (its only one with STAGE), computed once
  const LineDesc<CT> d0 = line_desc<CT, NV>(cluster, pub, lg, JMAX, KMAX, upper, rank, g0, lj, lk);
  if (STAGE) {
    int I;
    size_t S;
    if (d0.ok && plane_cell(0, d0.J, d0.K, I, S)) lines_stage<CT, NV>(my, nthr, sw, dwp, ns, S, upper);
  }
  cluster.sync();
  for (int s = 0; s < nplanes; s++) {
    const int bin = s & 1, bout = bin ^ 1;
    for (int q = g0; q < (STAGE ? g0 + 1 : tpc); q += ng) {
      const LineDesc<CT> ld =
          STAGE || q == g0 ? d0 : line_desc<CT, NV>(cluster, pub, lg, JMAX, KMAX, upper, rank, q, lj, lk);
      const int J = ld.J;
      int I;
      size_t S;
      if (!ld.ok || !plane_cell(s, J, ld.K, I, S)) continue;
      if (STAGE) cp_async_wait_all();
      // value c of the cell's sweep data (c >= SW_N: right-hand side)
      auto cd_ = [&](int c) -> CT {
        if (STAGE) return my[c * nthr];
        return c < SW_N ? __ldg(sw + c * ns + S) : dwp[(c - SW_N) * ns + S];
      };
      // PREDGS drops the i+1 coupling of row J = JMAX unless bit 2 of upper
      // (predgs_full) asks for it; PRKEGS does not drop it
      const bool hy = upper ? (I < IMAX && (NV == 7 || J < JMAX || (upper & 2))) : (I > 1);
      // ---- consume: neighbour contributions of the previous plane ----
      CT yd[NV], bd[NV], ck[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) {
        yd[v] = hy ? ydb[(q * NV + v) * LTHREADS + lane] : CT(0);
        bd[v] = ld.hj ? ld.srcj[bin * pstride + v * LTHREADS] : CT(0);
        ck[v] = ld.hk ? ld.srck[bin * pstride + v * LTHREADS] : CT(0);
      }
      // ---- solve the cell ----
      const CT dt1 = cd_(SW_DT1), vol = cd_(SW_VOL), fd = upper ? CT(1) : cd_(SW_FD);
      const CT a1 = cd_(SW_A1), a2 = cd_(SW_A2), a3 = cd_(SW_A3);
      const CT scinv = cd_(SW_SCINV), scinp = cd_(SW_SCINP);
      CT res[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) {
        CT cd = cd_(SW_N + v) * fd;
        CT x = upper ? (-dt1 * a3 * ck[v] + vol * cd) : (dt1 * a3 * ck[v] + vol * cd);
        x = upper ? x - dt1 * (a1 * yd[v] + a2 * bd[v]) : x + dt1 * (a1 * yd[v] + a2 * bd[v]);
        res[v] = x * (v == 4 ? scinp : scinv);
        dwp[v * ns + S] = res[v];
      }
      // ---- produce: contributions to the three downstream neighbours ----
      CT sc[5];
#pragma unroll
      for (int c = 0; c < (NV == 7 ? 5 : 3); c++) sc[c] = cd_(SW_SC + c);
      const CT ro = NV == 7 ? cd_(SW_RO) : CT(0);
#pragma unroll
      for (int d = 0; d < 3; d++) {
        CT f[3], l[3];
#pragma unroll
        for (int c = 0; c < 3; c++) f[c] = cd_(SW_F + 3 * d + c);
#pragma unroll
        for (int e = 0; e < 3; e++) l[e] = cd_(SW_L + 3 * d + e);
        CT out[NV];
        nb_product_pre<CT, NV>(out, res, f, sc, ro, l[0], l[1], l[2]);
        if (d == 0) {
#pragma unroll
          for (int v = 0; v < NV; v++) ydb[(q * NV + v) * LTHREADS + lane] = out[v];
        } else {
#pragma unroll
          for (int v = 0; v < NV; v++)
            pub[bout * pstride + (q * 2 * NV + (d == 1 ? 0 : NV) + v) * LTHREADS + lane] = out[v];
        }
      }
    }
    cluster_arrive_release();
    // the next plane's sweep data, in flight while the other CTAs finish
    if (STAGE && s + 1 < nplanes && d0.ok) {
      int I;
      size_t S;
      if (plane_cell(s + 1, d0.J, d0.K, I, S)) lines_stage<CT, NV>(my, nthr, sw, dwp, ns, S, upper);
    }
    if (!STAGE && s + 1 < nplanes) {
      // unstaged: pull the next plane's cells of every tile of the thread
      // group into L2 (a hint: no registers or shared memory held)
      for (int q = g0; q < tpc; q += ng) {
        const int t = q * lg.cs + rank;
        if (t >= lg.ntiles) break;
        const int J = (t % lg.ntj) * LTJ + lj + 1, K = (t / lg.ntj) * LTK + lk + 1;
        int I;
        size_t S;
        if (J > JMAX || K > KMAX || !plane_cell(s + 1, J, K, I, S)) continue;
        lines_prefetch_l2<CT, NV>(sw, dwp, ns, S, upper);
      }
    }
    cluster_wait_acquire();
  }
}

template <typename CT, int NV, bool STAGE>
__global__ void __launch_bounds__(LTHREADS * (STAGE ? LMAX_TPC_STAGE : LMAX_TPC))
    k_lusgs_lines(DevBlock b, const CT* __restrict__ sw, CT* dwp, int upper, LineGeom lg) {
  lines_body<CT, NV, STAGE>(b, sw, dwp, upper, lg);
}

// Several blocks' sweeps in one launch (a block work-list): cluster e of
// the grid sweeps entry e.  All entries share the cluster size; each has its
// own tile geometry and sweep flags.
constexpr int LB_MAX = 16;
struct LinesBatch {
  int n;
  int upper[LB_MAX];
  LineGeom lg[LB_MAX];
  const void* sw[LB_MAX];
  void* dwp[LB_MAX];
  DevBlock b[LB_MAX];
};

template <typename CT, int NV>
__global__ void __launch_bounds__(LTHREADS * LMAX_TPC)
    k_lusgs_lines_batch(const __grid_constant__ LinesBatch lb) {
  const int e = blockIdx.x / lb.lg[0].cs;
  if (e >= lb.n) return;   // whole clusters only: the launch has n * cs CTAs
  lines_body<CT, NV, false>(lb.b[e], static_cast<const CT*>(lb.sw[e]), static_cast<CT*>(lb.dwp[e]), lb.upper[e],
                            lb.lg[e]);
}

#include "ff_pipe.cuh"
#include "ff_ddadi.cuh"
