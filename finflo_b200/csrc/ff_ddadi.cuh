// DDADI implicit stage (LUSGS=0, the reference's default): per direction
// (k, then i, then j, imps3.f:320-356) a backward sweep PRED + point factor
// DIAG and a forward sweep CORR along every grid line (IMPSWE
// imps3.f:578-778; PRED/DIAG/CORR imps4.f:788/911/671, the k-omega forms
// PREDKE/DIAGKE/CORRKE imps4.f:2084/2235/1939).
//
// Lines are independent, so one thread owns one line and walks it in the
// FINFLO storage (stride 1, IS or IL); neighbouring threads own neighbouring
// lines, so for the j and k directions every load of a warp is one
// contiguous 256-byte run.  The recurrence carries only the five (seven)
// components of BD from cell to cell; everything else a step needs is
// independent of it.  Each thread therefore prefetches the data of the next
// PD-1 steps with cp.async into its own column of a shared-memory ring and
// computes step s while steps s+1..s+PD-1 are in flight.  The values of the
// neighbour cell and of the shared face that step s loaded are the cell and
// face values of step s+1, and are carried in registers.
//
// PRED+DIAG and CORR are separate launches: CORR reads the increments that
// PRED wrote, and the kernel boundary orders those stores before its
// cp.async reads.
#pragma once

// SYI / SYM1I imps4.f:10/46 (NV = 5) and SYIKE / SYM1KE imps4.f:982/1034
// (NV = 7): primitive increments <-> characteristic variables in the frame
// of the face normal n (tangents t from SURFVECTS).
template <typename T>
struct DdFrame {
  T nx, ny, nz, t21, t22, t23, t31, t32, t33;
};

template <typename T>
FF_DI DdFrame<T> dd_frame(T nx, T ny, T nz) {
  DdFrame<T> f;
  f.nx = nx; f.ny = ny; f.nz = nz;
  surfvects(nx, ny, nz, f.t21, f.t22, f.t23, f.t31, f.t32, f.t33);
  return f;
}

// The cell scalars the transforms use (RK, DRDP, DRDH for NV = 7 only).
template <typename T>
struct DdCell {
  T c, ro, rk, drdp, drdh;
};

template <typename T, int NV>
FF_DI void dd_syi(T w[NV], const T x[NV], const DdFrame<T>& f, const DdCell<T>& q) {
  T z2 = f.nx * x[1] + f.ny * x[2] + f.nz * x[3];
  T z3 = f.t21 * x[1] + f.t22 * x[2] + f.t23 * x[3];
  T z4 = f.t31 * x[1] + f.t32 * x[2] + f.t33 * x[3];
  T roc = q.ro * q.c;
  if constexpr (NV == 5) {
    w[0] = x[0] - x[4] / q.ro;
  } else {
    w[0] = x[0] - (T(1) / q.ro) * x[4];
    w[5] = x[5];
    w[6] = x[6];
  }
  w[1] = roc * z2 + x[4];
  w[2] = z3;
  w[3] = z4;
  w[4] = -roc * z2 + x[4];
}

template <typename T, int NV>
FF_DI void dd_sym1i(T x[NV], const T w[NV], const DdFrame<T>& f, const DdCell<T>& q) {
  T ypro = T(1) / q.ro, pc2 = T(.5) * ypro, proc = pc2 / q.c;
  T dh = w[0] + pc2 * (w[1] + w[4]);
  T x2i = proc * (w[1] - w[4]);
  T x5 = T(.5) * (w[1] + w[4]);
  x[0] = dh;
  if constexpr (NV == 5) {
    x[4] = x5;
  } else {
    T drh = T(.667) * q.rk * (ypro * ypro) * q.drdh;
    T ydrp = T(1) / (T(1) + T(.667) * q.rk * ypro * q.drdp);
    x[4] = ydrp * (x5 - drh * q.ro * dh - T(.667) * q.ro * w[5]);
    x[5] = w[5];
    x[6] = w[6];
  }
  x[1] = f.nx * x2i + f.t21 * w[2] + f.t31 * w[3];
  x[2] = f.ny * x2i + f.t22 * w[2] + f.t32 * w[3];
  x[3] = f.nz * x2i + f.t23 * w[2] + f.t33 * w[3];
}

// One line of one direction: the first cell, stride, length and the face
// arrays of the direction (entry N = face between N - stride and N).
struct DdLine {
  size_t n0, st;
  int n, idi;
  const double *A, *AX, *AY, *AZ;
};

FF_DI bool dd_line(const DevBlock& b, const ff_params& p, int dir, int t, DdLine& L) {
  int na, nb;
  if (dir == 1) { na = b.jmax; nb = b.kmax; } else if (dir == 2) { na = b.imax; nb = b.kmax; }
  else { na = b.imax; nb = b.jmax; }
  if (t >= na * nb) return false;
  const int aa = t % na + 1, bb = t / na + 1;
  if (dir == 1) {
    L.n0 = ix(b, 1, aa, bb); L.st = 1; L.n = b.imax; L.idi = p.idi1;
    L.A = b.a[FF_A1]; L.AX = b.a[FF_A1XA]; L.AY = b.a[FF_A1YA]; L.AZ = b.a[FF_A1ZA];
  } else if (dir == 2) {
    L.n0 = ix(b, aa, 1, bb); L.st = (size_t)b.is; L.n = b.jmax; L.idi = p.idi2;
    L.A = b.a[FF_A2]; L.AX = b.a[FF_A2XA]; L.AY = b.a[FF_A2YA]; L.AZ = b.a[FF_A2ZA];
  } else {
    L.n0 = ix(b, aa, bb, 1); L.st = (size_t)b.il; L.n = b.kmax; L.idi = p.idi3;
    L.A = b.a[FF_A3]; L.AX = b.a[FF_A3XA]; L.AY = b.a[FF_A3YA]; L.AZ = b.a[FF_A3ZA];
  }
  return true;
}

// Values loaded per step: the increments and DTL, U, V, W, C (and RK, DRDP,
// DRDH) of the cell, RO, VOL, VIS, VIST of the neighbour on the side the
// sweep goes next, and A, AX, AY, AZ of the face between them.
template <int NV>
struct DdSlots {
  static constexpr int D = 0, DTL = NV, U = NV + 1, V = NV + 2, W = NV + 3, C = NV + 4;
  static constexpr int RK = NV + 5, DRDP = NV + 6, DRDH = NV + 7;   // NV = 7 only
  static constexpr int Q = NV == 7 ? NV + 8 : NV + 5;                // neighbour RO, VOL, VIS, VIST
  static constexpr int F = Q + 4;                                    // face A, AX, AY, AZ
  static constexpr int N = F + 4;
};

FF_DI void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int K>
FF_DI void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(K) : "memory"); }

template <int NV, int TPB>
FF_DI void dd_issue(double* slot, const DevBlock& b, const DdLine& L, size_t N, size_t Q, size_t F) {
  using S = DdSlots<NV>;
#pragma unroll
  for (int v = 0; v < NV; v++) cp_async_ca(slot + (S::D + v) * TPB, b.a[FF_DRO + v] + N);
  cp_async_ca(slot + S::DTL * TPB, b.a[FF_DTL] + N);
  cp_async_ca(slot + S::U * TPB, b.a[FF_U] + N);
  cp_async_ca(slot + S::V * TPB, b.a[FF_V] + N);
  cp_async_ca(slot + S::W * TPB, b.a[FF_W] + N);
  cp_async_ca(slot + S::C * TPB, b.a[FF_C] + N);
  if constexpr (NV == 7) {
    cp_async_ca(slot + S::RK * TPB, b.a[FF_RK] + N);
    cp_async_ca(slot + S::DRDP * TPB, b.a[FF_DRDP] + N);
    cp_async_ca(slot + S::DRDH * TPB, b.a[FF_DRDH] + N);
  }
  cp_async_ca(slot + (S::Q + 0) * TPB, b.a[FF_RO] + Q);
  cp_async_ca(slot + (S::Q + 1) * TPB, b.a[FF_VOL] + Q);
  cp_async_ca(slot + (S::Q + 2) * TPB, b.a[FF_VIS] + Q);
  cp_async_ca(slot + (S::Q + 3) * TPB, b.a[FF_VIST] + Q);
  cp_async_ca(slot + (S::F + 0) * TPB, L.A + F);
  cp_async_ca(slot + (S::F + 1) * TPB, L.AX + F);
  cp_async_ca(slot + (S::F + 2) * TPB, L.AY + F);
  cp_async_ca(slot + (S::F + 3) * TPB, L.AZ + F);
}

template <typename CT, int NV>
FF_DI DdCell<CT> dd_cell(const double* slot, int tpb, CT ro) {
  using S = DdSlots<NV>;
  DdCell<CT> q;
  q.c = (CT)slot[S::C * tpb];
  q.ro = ro;
  if constexpr (NV == 7) {
    q.rk = (CT)slot[S::RK * tpb];
    q.drdp = (CT)slot[S::DRDP * tpb];
    q.drdh = (CT)slot[S::DRDH * tpb];
  } else {
    q.rk = q.drdp = q.drdh = CT(0);
  }
  return q;
}

// y[v] / (VOL (+ VREL) + DT * XA_v * A) of PRED/CORR; the k-omega forms add
// VREL = 1e-21 and group the k and omega terms as DT * (XA * A + 0).
template <typename CT, int NV>
FF_DI void dd_scale(CT y[NV], CT vol, CT dt1, CT a, CT x1a, CT x2a, CT x5a) {
  if constexpr (NV == 5) {
    y[0] = y[0] / (vol + dt1 * x1a * a);
    y[1] = y[1] / (vol + dt1 * x2a * a);
    y[2] = y[2] / (vol + dt1 * x1a * a);
    y[3] = y[3] / (vol + dt1 * x1a * a);
    y[4] = y[4] / (vol + dt1 * x5a * a);
  } else {
    const CT vr = vol + CT(1.e-21);
    y[0] = y[0] / (vr + dt1 * x1a * a);
    y[1] = y[1] / (vr + dt1 * x2a * a);
    y[2] = y[2] / (vr + dt1 * x1a * a);
    y[3] = y[3] / (vr + dt1 * x1a * a);
    y[4] = y[4] / (vr + dt1 * x5a * a);
    y[5] = y[5] / (vr + dt1 * (x1a * a));
    y[6] = y[6] / (vr + dt1 * (x1a * a));
  }
}

template <typename CT, int NV>
FF_DI void dd_xmul(CT y[NV], CT x1, CT x2, CT x5) {
  y[0] = x1 * y[0]; y[1] = x2 * y[1]; y[2] = x1 * y[2]; y[3] = x1 * y[3]; y[4] = x5 * y[4];
  if constexpr (NV == 7) { y[5] = x1 * y[5]; y[6] = x1 * y[6]; }
}

// PRED (K = n .. 1, BD from cell K+1 through face K+1/2, frame and split
// eigenvalues of face K-1/2) followed on each cell by DIAG (frame of face
// K+1/2, positive eigenvalues of face K-1/2 and negative of face K+1/2).
template <typename CT, int NV, int PD, int TPB>
__global__ void __launch_bounds__(TPB) k_ddadi_pred(DevBlock b, ff_params p, int dir) {
  using S = DdSlots<NV>;
  extern __shared__ double dd_smem[];
  DdLine L;
  if (!dd_line(b, p, dir, blockIdx.x * TPB + threadIdx.x, L)) return;
  double* ring = dd_smem + threadIdx.x;   // slot s at ring + s * S::N * TPB
  const size_t st = L.st;
  auto cell = [&](int K) { return L.n0 + (size_t)(K - 1) * st; };
  // step s visits K = n - s: cell N, neighbour N - st, face N
#pragma unroll
  for (int s = 0; s < PD - 1; s++) {
    if (s < L.n) dd_issue<NV, TPB>(ring + s * S::N * TPB, b, L, cell(L.n - s), cell(L.n - s) - st, cell(L.n - s));
    cp_async_commit();
  }
  // the cell values of K = n and face n+1/2
  const size_t Nn = cell(L.n);
  CT ro = (CT)b.a[FF_RO][Nn], vol = (CT)b.a[FF_VOL][Nn];
  CT vis = (CT)b.a[FF_VIS][Nn], vist = (CT)b.a[FF_VIST][Nn];
  CT au = (CT)L.A[Nn + st], nxu = (CT)L.AX[Nn + st], nyu = (CT)L.AY[Nn + st], nzu = (CT)L.AZ[Nn + st];
  const CT theta = (CT)p.theta;
  CT bd[NV];
#pragma unroll
  for (int v = 0; v < NV; v++) bd[v] = CT(0);
  for (int s = 0; s < L.n; s++) {
    const int K = L.n - s;
    const int sp = s + PD - 1;
    if (sp < L.n) {
      const size_t Np = cell(L.n - sp);
      dd_issue<NV, TPB>(ring + (sp % PD) * S::N * TPB, b, L, Np, Np - st, Np);
    }
    cp_async_commit();
    cp_async_wait_group<PD - 1>();
    const double* sl = ring + (s % PD) * S::N * TPB;
    const size_t N = cell(K);
    const CT dt1 = theta * (CT)sl[S::DTL * TPB];
    const CT u = (CT)sl[S::U * TPB], vv = (CT)sl[S::V * TPB], w = (CT)sl[S::W * TPB];
    const CT ro_b = (CT)sl[(S::Q + 0) * TPB], vol_b = (CT)sl[(S::Q + 1) * TPB];
    const CT vis_b = (CT)sl[(S::Q + 2) * TPB], vist_b = (CT)sl[(S::Q + 3) * TPB];
    const CT al = (CT)sl[(S::F + 0) * TPB];
    const DdFrame<CT> fl = dd_frame<CT>((CT)sl[(S::F + 1) * TPB], (CT)sl[(S::F + 2) * TPB], (CT)sl[(S::F + 3) * TPB]);
    const DdCell<CT> q = dd_cell<CT, NV>(sl, TPB, ro);
    CT bdx[NV], y[NV], out[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) bdx[v] = dt1 * au * bd[v] + vol * (CT)sl[(S::D + v) * TPB];
    dd_syi<CT, NV>(y, bdx, fl, q);
    const CT rl1 = fl.nx * u + fl.ny * vv + fl.nz * w;
    const CT rl2 = rl1 + q.c, rl5 = rl1 - q.c;
    const CT ff = K == 1 ? CT(.25) : CT(.5);
    const CT cdiff = K <= L.idi ? CT(2) : CT(0);
    const CT rnum = ff * (vol + vol_b) * (ro + ro_b);
    const CT T = cdiff * al / rnum * (vist + vis + vist_b + vis_b);
    const CT x1 = dmax(-rl1, CT(0)) + T, x2 = dmax(-rl2, CT(0)) + T, x5 = dmax(-rl5, CT(0)) + T;
    dd_scale<CT, NV>(y, vol, dt1, al, fabs(rl1) + T, fabs(rl2) + T, fabs(rl5) + T);
    dd_sym1i<CT, NV>(out, y, fl, q);
    dd_xmul<CT, NV>(y, x1, x2, x5);
    dd_sym1i<CT, NV>(bd, y, fl, q);
    // DIAG on cell K
    {
      const DdFrame<CT> fu = dd_frame<CT>(nxu, nyu, nzu);
      CT z[NV];
      dd_syi<CT, NV>(z, out, fu, q);
      CT ucon = fu.nx * u + fu.ny * vv + fu.nz * w;
      const CT rl2n = dmax(-(ucon + q.c), CT(0)), rl5n = dmax(-(ucon - q.c), CT(0)), rl1n = dmax(-ucon, CT(0));
      const CT rl2p = dmax(rl2, CT(0)), rl5p = dmax(rl5, CT(0)), rl1p = dmax(rl1, CT(0));
      const CT dtv = NV == 5 ? dt1 / vol : dt1 / (vol + CT(1.e-21));
      const CT f1 = CT(1) + dtv * (al * rl1p + au * rl1n);
      z[0] = z[0] * f1;
      z[1] = z[1] * (CT(1) + dtv * (al * rl2p + au * rl2n));
      z[2] = z[2] * f1;
      z[3] = z[3] * f1;
      z[4] = z[4] * (CT(1) + dtv * (al * rl5p + au * rl5n));
      if constexpr (NV == 7) { z[5] = z[5] * f1; z[6] = z[6] * f1; }
      dd_sym1i<CT, NV>(out, z, fu, q);
    }
#pragma unroll
    for (int v = 0; v < NV; v++) b.a[FF_DRO + v][N] = (double)out[v];
    // the neighbour and the lower face become the next step's cell and upper face
    ro = ro_b; vol = vol_b; vis = vis_b; vist = vist_b;
    au = al; nxu = fl.nx; nyu = fl.ny; nzu = fl.nz;
  }
  cp_async_wait_group<0>();
}

// CORR (K = 1 .. n, BD from cell K-1 through face K-1/2, frame and split
// eigenvalues of face K+1/2).
template <typename CT, int NV, int PD, int TPB>
__global__ void __launch_bounds__(TPB) k_ddadi_corr(DevBlock b, ff_params p, int dir) {
  using S = DdSlots<NV>;
  extern __shared__ double dd_smem[];
  DdLine L;
  if (!dd_line(b, p, dir, blockIdx.x * TPB + threadIdx.x, L)) return;
  double* ring = dd_smem + threadIdx.x;
  const size_t st = L.st;
  auto cell = [&](int K) { return L.n0 + (size_t)(K - 1) * st; };
  // step s visits K = s + 1: cell N, neighbour N + st, face N + st
#pragma unroll
  for (int s = 0; s < PD - 1; s++) {
    if (s < L.n) dd_issue<NV, TPB>(ring + s * S::N * TPB, b, L, cell(s + 1), cell(s + 1) + st, cell(s + 1) + st);
    cp_async_commit();
  }
  const size_t N1 = L.n0;
  CT ro = (CT)b.a[FF_RO][N1], vol = (CT)b.a[FF_VOL][N1];
  CT vis = (CT)b.a[FF_VIS][N1], vist = (CT)b.a[FF_VIST][N1];
  CT alo = (CT)L.A[N1];
  const CT theta = (CT)p.theta;
  CT bd[NV];
#pragma unroll
  for (int v = 0; v < NV; v++) bd[v] = CT(0);
  for (int s = 0; s < L.n; s++) {
    const int K = s + 1;
    const int sp = s + PD - 1;
    if (sp < L.n) {
      const size_t Np = cell(sp + 1);
      dd_issue<NV, TPB>(ring + (sp % PD) * S::N * TPB, b, L, Np, Np + st, Np + st);
    }
    cp_async_commit();
    cp_async_wait_group<PD - 1>();
    const double* sl = ring + (s % PD) * S::N * TPB;
    const size_t N = cell(K);
    const CT dt1 = theta * (CT)sl[S::DTL * TPB];
    const CT u = (CT)sl[S::U * TPB], vv = (CT)sl[S::V * TPB], w = (CT)sl[S::W * TPB];
    const CT ro_a = (CT)sl[(S::Q + 0) * TPB], vol_a = (CT)sl[(S::Q + 1) * TPB];
    const CT vis_a = (CT)sl[(S::Q + 2) * TPB], vist_a = (CT)sl[(S::Q + 3) * TPB];
    const CT au = (CT)sl[(S::F + 0) * TPB];
    const DdFrame<CT> fu = dd_frame<CT>((CT)sl[(S::F + 1) * TPB], (CT)sl[(S::F + 2) * TPB], (CT)sl[(S::F + 3) * TPB]);
    const DdCell<CT> q = dd_cell<CT, NV>(sl, TPB, ro);
    CT bdx[NV], y[NV], out[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) bdx[v] = dt1 * alo * bd[v] + vol * (CT)sl[(S::D + v) * TPB];
    dd_syi<CT, NV>(y, bdx, fu, q);
    const CT rl1 = fu.nx * u + fu.ny * vv + fu.nz * w;
    const CT rl2 = rl1 + q.c, rl5 = rl1 - q.c;
    const CT cdiff = K <= L.idi ? CT(2) : CT(0);
    const CT rnum = CT(.5) * (vol + vol_a) * (ro + ro_a);
    const CT T = cdiff * au / rnum * (vist + vis + vist_a + vis_a);
    const CT x1 = dmax(rl1, CT(0)) + T, x2 = dmax(rl2, CT(0)) + T, x5 = dmax(rl5, CT(0)) + T;
    dd_scale<CT, NV>(y, vol, dt1, au, fabs(rl1) + T, fabs(rl2) + T, fabs(rl5) + T);
    dd_sym1i<CT, NV>(out, y, fu, q);
#pragma unroll
    for (int v = 0; v < NV; v++) b.a[FF_DRO + v][N] = (double)out[v];
    dd_xmul<CT, NV>(y, x1, x2, x5);
    dd_sym1i<CT, NV>(bd, y, fu, q);
    ro = ro_a; vol = vol_a; vis = vis_a; vist = vist_a;
    alo = au;
  }
  cp_async_wait_group<0>();
}

// Shared memory of one CTA: PD slots of S::N doubles per thread.
inline size_t ddadi_smem_bytes(int nv, int pd, int tpb) {
  const int n = nv == 7 ? 7 + 8 + 8 : 5 + 5 + 8;
  return (size_t)pd * n * tpb * sizeof(double);
}
