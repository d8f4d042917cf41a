// Device-side numerics of the FINFLO hot path (sm_100a, FP64).
//
// Each function is the per-face or per-cell body of a reference routine; the
// kernels in ff_kernels.cu decide the launch shape and data movement.
// Reference citations are to the Fortran sources of mattipalin/finflo.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/finflo_types.h"

#define FF_DI __device__ __forceinline__

// Storage geometry of one block on one grid level.  a[] holds device
// pointers to the FF_NSLOTS per-cell arrays (enum ff_slot).
struct DevBlock {
  int imax, jmax, kmax;
  int is, il, ntot;
  int npatch, pad;
  const ff_patch* patch;   // device copy of the patch table
  double* a[FF_NSLOTS];
};

FF_DI size_t ix(const DevBlock& b, int I, int J, int K) {
  return (size_t)(K + 1) * b.il + (size_t)(J + 1) * b.is + (size_t)(I + 1);
}

template <typename T> FF_DI T dmax(T a, T b) { return a > b ? a : b; }
// 1/x correctly rounded (the same value as 1. / x), through the reciprocal
// intrinsic rather than the general division
FF_DI double rcp(double x) { return __drcp_rn(x); }
FF_DI float rcp(float x) { return __frcp_rn(x); }
template <typename T> FF_DI T dmin(T a, T b) { return a < b ? a : b; }

// SURFVECTS base3c.f:12245: two tangent unit vectors completing the normal.
template <typename T>
FF_DI void surfvects(T a11, T a12, T a13, T& a21, T& a22, T& a23, T& a31, T& a32, T& a33) {
  T am = fabs(a11);
  int idir = 1;
  if (fabs(a12) < am) { am = fabs(a12); idir = 2; }
  if (fabs(a13) < am) idir = 3;
  T b1, b2, b3;
  if (idir == 1) { b1 = T(0); b2 = -a13; b3 = a12; }
  else if (idir == 2) { b1 = a13; b2 = T(0); b3 = -a11; }
  else { b1 = -a12; b2 = a11; b3 = T(0); }
  T palpo = T(1) / sqrt(b1 * b1 + b2 * b2 + b3 * b3);
  a21 = b1 * palpo; a22 = b2 * palpo; a23 = b3 * palpo;
  a31 = a12 * a23 - a13 * a22;
  a32 = a13 * a21 - a11 * a23;
  a33 = a11 * a22 - a12 * a21;
}

// XXTRAP base3c.f:750 (kappa scheme, van Albada limiter); r0..r3 are the
// cells I-2S, I-S, I, I+S of the face between I-S and I.  T = double, or
// float for a coarse level's face pass in FP32.
template <typename T>
FF_DI void xxtrap(T r0, T r1, T r2, T r3, int intem, T& rip, T& rim) {
  int inter = intem < 0 ? -intem : intem;
  int inte2 = inter < 1 ? 1 : (inter > 5 ? 5 : inter);
  T rk1 = inte2 == 1 ? T(0.) : (inte2 == 2 ? T(1.) : (inte2 == 3 ? T(1.3333333) : (inte2 == 4 ? T(2.) : T(1.5))));
  T rk2 = T(2.) - rk1;
  T R1 = T(.25) * rk1, R2 = T(.25) * rk2;
  T diff0 = r1 - r0, diff1 = r2 - r1, diff2 = r3 - r2;
  if (intem <= 0 && intem >= -5) {
    rip = r2 - (diff1 * R1 + diff2 * R2);
    rim = r1 + (diff1 * R1 + diff0 * R2);
  } else if (inter <= 4) {
    // the two van Albada ratios through one reciprocal of the product of
    // their denominators (each at least 1e-10, far from over- or underflow)
    T diff12 = diff1 * diff1 + T(1.e-10);
    T db = diff12 + diff0 * diff0, df = diff12 + diff2 * diff2;
    T r = rcp(db * df);
    T phibi = (diff12 + diff1 * diff0) * (df * r);
    T phifi = (diff12 + diff1 * diff2) * (db * r);
    rip = r2 - phifi * (diff1 * R1 + diff2 * R2);
    rim = r1 + phibi * (diff1 * R1 + diff0 * R2);
  } else {
    rip = r2;
    rim = r1;
  }
}

// XXTRAA base3c.f:1444-1570: XXTRAP with the cells' extents d[0..3] along
// the face normal (D1/D2/D3 of cells I-2S..I+S): differences become slopes
// over the centre distances, the half extents scale the extrapolation.
// FLUXKE, FLUXKT and FLUCUSP use it in place of XXTRAP when XXTRAL is set.
template <typename T>
FF_DI void xxtraa(T r0, T r1, T r2, T r3, const T d[4], int intem, T& rip, T& rim) {
  int inter = intem < 0 ? -intem : intem;
  int inte2 = inter < 1 ? 1 : (inter > 5 ? 5 : inter);
  T rk1 = inte2 == 1 ? T(0.) : (inte2 == 2 ? T(1.) : (inte2 == 3 ? T(1.3333333) : (inte2 == 4 ? T(2.) : T(1.5))));
  T rk2 = T(2.) - rk1;
  if (inter > 4 && !(intem <= 0 && intem >= -5)) {
    rip = r2;
    rim = r1;
    return;
  }
  const T eps = T(1.e-10);
  const T dxl = T(.5) * d[1], dxr = T(.5) * d[2];
  const T dx0 = T(1.) / (d[0] + d[1] + eps), dx1 = T(1.) / (d[1] + d[2] + eps), dx2 = T(1.) / (d[2] + d[3] + eps);
  if (intem <= 0 && intem >= -5) {
    rip = r2 - dxr * (dx1 * (r2 - r1) * rk1 + dx2 * (r3 - r2) * rk2);
    rim = r1 + dxl * (dx1 * (r2 - r1) * rk1 + dx0 * (r1 - r0) * rk2);
  } else {
    const T diff0 = dx0 * (r1 - r0), diff1 = dx1 * (r2 - r1), diff2 = dx2 * (r3 - r2);
    const T diff12 = diff1 * diff1 + eps;
    const T phibi = (diff12 + diff1 * diff0) / (diff12 + diff0 * diff0);
    const T phifi = (diff12 + diff1 * diff2) / (diff12 + diff2 * diff2);
    rip = r2 - dxr * phifi * (diff1 * rk1 + diff2 * rk2);
    rim = r1 + dxl * phibi * (diff1 * rk1 + diff0 * rk2);
  }
}

// The MUSCL pair of one variable (q = cells I-2S..I+S): XXTRAP, or XXTRAA
// over the extents d (DD, XXTRAL set).
template <bool DD, typename T>
FF_DI void muscl(const T q[4], const T* d, int intem, T& ip, T& im) {
  if constexpr (DD) xxtraa(q[0], q[1], q[2], q[3], d, intem, ip, im);
  else xxtrap(q[0], q[1], q[2], q[3], intem, ip, im);
}

// Roe flux-difference splitting for a general EOS (FLUXKE base3c.f:4753-5120)
// at one face; laminar (k = omega = 0), UROT = 0.  q[v][m]: v = ro,u,v,w,p,
// m = cells I-2S, I-S, I, I+S.  cr / cl2 = {DRDP, DRDH, RO, P} of cell I and of
// the cell DERIV pairs it with (I-S, or I itself for the k direction,
// base3c.f:4892 with IL > NTOT).  DD: XXTRAA over the extents dd (XXTRAL).
// Adds the 5 flux components to f.
template <typename T, bool DD = false>
FF_DI void roe_flux(const T q[5][4], T nx, T ny, T nz, T area, int intem, const ff_params& p, T c_r, T c_l,
                    const T cr[4], const T cl2[4], T f[5], const T* dd = nullptr) {
  T roip, roim, rmip, rmim, rnip, rnim, rwip, rwim, ppi, pmi;
  muscl<DD>(q[0], dd, intem, roip, roim);
  muscl<DD>(q[1], dd, intem, rmip, rmim);
  muscl<DD>(q[2], dd, intem, rnip, rnim);
  muscl<DD>(q[3], dd, intem, rwip, rwim);
  muscl<DD>(q[4], dd, intem, ppi, pmi);
  roip = dmax(T(0.001) * T(p.frsden), roip);
  ppi = dmax(T(0.001) * T(p.frspre), ppi);
  roim = dmax(T(0.001) * T(p.frsden), roim);
  pmi = dmax(T(0.001) * T(p.frspre), pmi);
  const T rgm1 = rcp(T(p.gamma) - T(1.)), e0 = T(p.e0ref);
  const T ypror = rcp(roip), yprol = rcp(roim);
  // EFPRO state.f:620 (perfect gas): p / ((gamma - 1) rho)
  T eip = ppi * rgm1 * ypror - e0;
  T eim = pmi * rgm1 * yprol - e0;
  T elr = ppi * rgm1 * yprol - e0;
  T erl = pmi * rgm1 * ypror - e0;
  // DERIV base3c.f:707 (Glaister hat derivatives)
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
  T eir = eip + T(.5) * (rmip * rmip + rnip * rnip + rwip * rwip);
  T eil = eim + T(.5) * (rmim * rmim + rnim * rnim + rwim * rwim);
  T pr = ppi, pl = pmi;
  T hr = eir + pr * ypror, hl = eil + yprol * pl;
  T rohat = sqrt(roip * roim), yproh = rcp(rohat);
  T sqrl = rcp(roim + rohat), cql = roim * sqrl, cqr = T(1.) - cql;
  T uhat = cqr * ur + cql * ul;
  const T thx = cqr * txr + cql * txl, thy = cqr * tyr + cql * tyl, thz = cqr * tzr + cql * tzl;
  T hhat = cqr * hr + cql * hl, ehat = cqr * eip + cql * eim;
  T phat = rohat * (hhat - ehat - T(.5) * (uhat * uhat + thx * thx + thy * thy + thz * thz));
  phat = dmin(dmax(pr, pl), phat);
  phat = dmax(dmin(pr, pl), phat);
  T drdhh = rcp(dedrh - phat * (yproh * yproh));
  T drdph = -drdhh * (dedph + yproh);
  T chat2 = rcp(drdhh * yproh + drdph);
  T cmin = dmin(c_r, c_l), cmax = dmax(c_r, c_l);
  chat2 = dmin(cmax * cmax, chat2);
  chat2 = dmax(cmin * cmin, chat2);
  T chat = sqrt(chat2);
  T pdpde = dedph;
  T dro = roip - roim, du = ur - ul;
  T dp = pr - pl;
  T pchat2 = rcp(chat * chat);
  T alfa1 = T(.5) * (dp + rohat * chat * du) * pchat2;
  T alfa2 = T(.5) * (dp - rohat * chat * du) * pchat2;
  T alfa3 = dro - dp * pchat2;
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
  T f2 = ha * (roucr * ur + pr + roucl * ul + pl - (damp * uhat + (rl1 * alfa1 - rl2 * alfa2) * chat));
  // the tangential momentum flux as a vector (f3, f4 of the reference's
  // rotated frame) and its jump term of the energy flux
  const T rr = rl3 * rohat;
  const T ftx = ha * (roucr * txr + roucl * txl - damp * thx - rr * (txr - txl));
  const T fty = ha * (roucr * tyr + roucl * tyl - damp * thy - rr * (tyr - tyl));
  const T ftz = ha * (roucr * tzr + roucl * tzl - damp * thz - rr * (tzr - tzl));
  const T tj = rr * ((txr - txl) * thx + (tyr - tyl) * thy + (tzr - tzl) * thz);
  T f5 = ha * (roucr * hr + roucl * hl - damp * hhat
               - ((rl1 * alfa1 - rl2 * alfa2) * uhat * chat - rl3 * alfa3 * rohat * (chat * chat) * pdpde + tj));
  f[0] += f1;
  f[1] += nx * f2 + ftx;
  f[2] += ny * f2 + fty;
  f[3] += nz * f2 + ftz;
  f[4] += f5;
}

// SYI / SYM1I imps4.f:10/46 and the split-eigenvalue product of one
// neighbour: SYM1I(diag(l1,l2,l1,l1,l5) * SYI(dw)).
template <typename T>
FF_DI void jac_product(T out[5], const T dw[5], T c, T ro, T nx, T ny, T nz, T l1, T l2, T l5) {
  T a21, a22, a23, a31, a32, a33;
  surfvects(nx, ny, nz, a21, a22, a23, a31, a32, a33);
  T z2 = nx * dw[1] + ny * dw[2] + nz * dw[3];
  T z3 = a21 * dw[1] + a22 * dw[2] + a23 * dw[3];
  T z4 = a31 * dw[1] + a32 * dw[2] + a33 * dw[3];
  T roc = ro * c;
  T w1 = l1 * (dw[0] - dw[4] / ro);
  T w2 = l2 * (roc * z2 + dw[4]);
  T w3 = l1 * z3;
  T w4 = l1 * z4;
  T w5 = l5 * (-roc * z2 + dw[4]);
  T ypro = T(1) / ro, pc2 = T(.5) * ypro, proc = pc2 / c;
  out[0] = w1 + pc2 * (w2 + w5);
  T x2i = proc * (w2 - w5);
  out[4] = T(.5) * (w2 + w5);
  out[1] = nx * x2i + a21 * w3 + a31 * w4;
  out[2] = ny * x2i + a22 * w3 + a32 * w4;
  out[3] = nz * x2i + a23 * w3 + a33 * w4;
}

// SYIKE / SYM1KE imps4.f:982/1034: the seven-equation product of PRKEGS /
// COKEGS, SYM1KE(diag(l1,l2,l1,l1,l5,l1,l1) * SYIKE(dw)).
template <typename T>
FF_DI void jac_product_ke(T out[7], const T dw[7], T rk, T c, T ro, T drdp, T drdh, T nx, T ny, T nz, T l1,
                          T l2, T l5) {
  T a21, a22, a23, a31, a32, a33;
  surfvects(nx, ny, nz, a21, a22, a23, a31, a32, a33);
  T z2 = nx * dw[1] + ny * dw[2] + nz * dw[3];
  T z3 = a21 * dw[1] + a22 * dw[2] + a23 * dw[3];
  T z4 = a31 * dw[1] + a32 * dw[2] + a33 * dw[3];
  T roc = ro * c, pc2 = T(1) / ro, dpres = dw[4];
  T w1 = l1 * (dw[0] - pc2 * dpres);
  T w2 = l2 * (roc * z2 + dpres);
  T w3 = l1 * z3, w4 = l1 * z4;
  T w5 = l5 * (-roc * z2 + dpres);
  T w6 = l1 * dw[5], w7 = l1 * dw[6];
  T ypro = T(1) / ro, pc2b = T(.5) * ypro, proc = pc2b / c;
  T drh = T(.667) * rk * (ypro * ypro) * drdh;
  T ydrp = T(1) / (T(1) + T(.667) * rk * ypro * drdp);
  T dh = w1 + pc2b * (w2 + w5);
  out[0] = dh;
  T x2i = proc * (w2 - w5);
  out[4] = ydrp * (T(.5) * (w2 + w5) - drh * ro * dh - T(.667) * ro * w6);
  out[5] = w6;
  out[6] = w7;
  out[1] = nx * x2i + a21 * w3 + a31 * w4;
  out[2] = ny * x2i + a22 * w3 + a32 * w4;
  out[3] = nz * x2i + a23 * w3 + a33 * w4;
}

// Sweep layout.  The LU-SGS sweeps visit the cells plane by plane (i+j+k =
// m); in the storage order (i fastest) the cells of one plane lie a j-stride
// apart, so every load of a warp touches 32 cache lines.  The sweeps
// therefore work on a skewed copy of their data, index
//   S(I,J,K) = ((K-1) * (IMAX+JMAX-1) + (I+J-2)) * JMAX + (J-1),
// in which the cells of one plane with the same K and consecutive J are
// consecutive, and the upstream/downstream neighbours of a cell are at
// S -/+ JMAX (i), S -/+ (JMAX+1) (j) and S -/+ (IMAX+JMAX-1)*JMAX (k).
// Per cell (sw[c * ns + S]): its own solve data, then the data of the
// products that it sends to its three downstream neighbours (the face frame
// of each direction, the split eigenvalue coefficients, and the cell's
// scalars 1/RO, RO*C, (.5/RO)/C and, for k-omega, DRH and
// 1/(1+.667*RK*DRDP/RO) of SYM1KE).
enum : int {
  SW_DT1 = 0, SW_SCINV, SW_SCINP, SW_FD, SW_VOL, SW_A1, SW_A2, SW_A3, SW_RO,
  SW_SC = 9,     // 5 scalars
  SW_F = 14,     // 3 directions x the face's unit normal
  SW_L = 23,     // 3 directions x 3 eigenvalue coefficients
  SW_N = 32
};

__host__ __device__ inline size_t sw_size(int imax, int jmax, int kmax) {
  return (size_t)kmax * (imax + jmax - 1) * jmax;
}

FF_DI size_t sw_index(const DevBlock& b, int I, int J, int K) {
  return ((size_t)(K - 1) * (b.imax + b.jmax - 1) + (I + J - 2)) * b.jmax + (J - 1);
}

// The product of one cell with its precomputed frame f[9] and scalars
// sc = {ypro, roc, proc, drh, ydrp}: SYM1I/SYM1KE(diag(l) * SYI/SYIKE(dw)).
template <typename T, int NV>
FF_DI void nb_product_pre(T* out, const T* dw, const T f[3], const T sc[5], T ro, T l1, T l2, T l5) {
  // The tangential part of SYM1I(diag * SYI(dw)): with {n, t1, t2}
  // orthonormal (the normal and its SURFVECTS tangents), t1 (t1 . dw) +
  // t2 (t2 . dw) = dw - n (n . dw), so only the normal is needed:
  // out_m = n (x2i - l1 z2) + l1 dw_m, the same operator in fewer steps.
  const T nx = f[0], ny = f[1], nz = f[2];
  const T ypro = sc[0], roc = sc[1], proc = sc[2];
  T z2 = nx * dw[1] + ny * dw[2] + nz * dw[3];
  T w1 = l1 * (dw[0] - ypro * dw[4]);
  T w2 = l2 * (roc * z2 + dw[4]);
  T w5 = l5 * (-roc * z2 + dw[4]);
  T pc2 = T(.5) * ypro;
  T dh = w1 + pc2 * (w2 + w5);
  out[0] = dh;
  T x2i = proc * (w2 - w5);
  if constexpr (NV == 5) {
    out[4] = T(.5) * (w2 + w5);
  } else {
    T w6 = l1 * dw[5];
    out[4] = sc[4] * (T(.5) * (w2 + w5) - sc[3] * ro * dh - T(.667) * ro * w6);
    out[5] = w6;
    out[6] = l1 * dw[6];
  }
  const T g = x2i - l1 * z2;
  out[1] = nx * g + l1 * dw[1];
  out[2] = ny * g + l1 * dw[2];
  out[3] = nz * g + l1 * dw[3];
}

// One neighbour's product for NV = 5 (laminar) or 7 (k-omega) equations.
template <typename T, int NV>
FF_DI void nb_product(T* out, const T* dw, const DevBlock& b, size_t n, T c, T ro, T nx, T ny, T nz, T l1, T l2,
                      T l5) {
  if constexpr (NV == 5) {
    jac_product<T>(out, dw, c, ro, nx, ny, nz, l1, l2, l5);
  } else {
    jac_product_ke<T>(out, dw, (T)__ldg(b.a[FF_RK] + n), c, ro, (T)__ldg(b.a[FF_DRDP] + n),
                      (T)__ldg(b.a[FF_DRDH] + n), nx, ny, nz, l1, l2, l5);
  }
}

// Bounded grid-wide barrier for a co-resident (cooperative) grid.  Every
// spin has an iteration limit; on time-out the error word is set and all
// blocks leave the kernel at their next barrier.
FF_DI bool grid_barrier(unsigned* count, unsigned* gen, unsigned nblocks, int* err) {
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
    volatile unsigned* vg = gen;
    unsigned g = *vg;
    __threadfence();
    unsigned arrived = atomicAdd(count, 1u);
    if (arrived == nblocks - 1) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      long it = 0;
      while (*vg == g) {
        if (++it > (1L << 24)) { atomicExch(err, 1); break; }
        if ((it & 1023) == 0 && *((volatile int*)err)) break;
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *((volatile int*)err) == 0;
}
