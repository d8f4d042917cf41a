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

// ---------------------------------------------------------------------------
// Producer/consumer form.  With one thread per line a 128 x 64 x 64 block
// has only 4096-8192 threads in flight, one or two warps per SM, and each
// step's ~600 instructions (two frames with a square root and a division,
// four divisions, the DIAG transforms) run back to back on that lone warp.
// Only a few of them are on the recurrence.  So a CTA owns 32 lines and
// splits the work: CH producer warps compute, for the next CH cells of all
// 32 lines (one cell per thread), everything that does not depend on BD --
// the face frames, the cell scalars of SYI/SYM1I, the reciprocal
// denominators, the split eigenvalues X and the DIAG factors -- into a
// shared-memory chunk, while warp 0 (one lane per line) runs the recurrence
// over the previous chunk: ~100 multiply-adds per step.  Two chunk buffers
// and one __syncthreads per chunk keep the two sides in step.  The
// reciprocals are taken once per cell, so y / den becomes y * (1 / den).

// PRED chunk slots per cell: right-hand side VOL*D, BD multiplier
// THETA*DTL*A(K+1/2), frames of faces K-1/2 and K+1/2, RO*C, 1/RO, .5/RO,
// (.5/RO)/C, the reciprocal denominators of waves 1, 2, 5 (and k, omega),
// X1, X2, X5, the DIAG factors of waves 1, 2, 5 and RO, DRH, YDRP (NV = 7).
template <int NV>
struct DdPredSlots {
  static constexpr int RHS = 0, A = NV, FL = NV + 1, FU = NV + 10, ROC = NV + 19, YPRO = NV + 20, PC2 = NV + 21,
                       PROC = NV + 22, R1 = NV + 23, R2 = NV + 24, R5 = NV + 25, X1 = NV + 26, X2 = NV + 27,
                       X5 = NV + 28, F1 = NV + 29, F2 = NV + 30, F5 = NV + 31, RO = NV + 32, DRH = NV + 33,
                       YDRP = NV + 34, R6 = NV + 35;
  static constexpr int N = NV == 7 ? NV + 36 : NV + 32;
};

// CORR chunk slots per cell: VOL*D, THETA*DTL*A(K-1/2), frame of face
// K+1/2, the cell scalars, reciprocal denominators, X, and RO, DRH, YDRP.
template <int NV>
struct DdCorrSlots {
  static constexpr int RHS = 0, A = NV, FU = NV + 1, ROC = NV + 10, YPRO = NV + 11, PC2 = NV + 12, PROC = NV + 13,
                       R1 = NV + 14, R2 = NV + 15, R5 = NV + 16, X1 = NV + 17, X2 = NV + 18, X5 = NV + 19,
                       RO = NV + 20, DRH = NV + 21, YDRP = NV + 22, R6 = NV + 23;
  static constexpr int N = NV == 7 ? NV + 24 : NV + 20;
};

template <typename CT>
FF_DI void dd_put_frame(CT* s, int stride, const DdFrame<CT>& f) {
  s[0] = f.nx; s[stride] = f.ny; s[2 * stride] = f.nz;
  s[3 * stride] = f.t21; s[4 * stride] = f.t22; s[5 * stride] = f.t23;
  s[6 * stride] = f.t31; s[7 * stride] = f.t32; s[8 * stride] = f.t33;
}

template <typename CT>
FF_DI DdFrame<CT> dd_get_frame(const CT* s, int stride) {
  DdFrame<CT> f;
  f.nx = s[0]; f.ny = s[stride]; f.nz = s[2 * stride];
  f.t21 = s[3 * stride]; f.t22 = s[4 * stride]; f.t23 = s[5 * stride];
  f.t31 = s[6 * stride]; f.t32 = s[7 * stride]; f.t33 = s[8 * stride];
  return f;
}

// The SYI/SYM1I cell scalars of one cell (RO*C, 1/RO, .5/RO, (.5/RO)/C and
// for NV = 7 RO, .667*RK/RO^2*DRDH, 1/(1+.667*RK/RO*DRDP)).
template <typename CT>
struct DdScal {
  CT roc, ypro, pc2, proc, ro, drh, ydrp;
};

template <typename CT, int NV>
FF_DI DdScal<CT> dd_scal(CT ro, CT c, CT rk, CT drdp, CT drdh) {
  DdScal<CT> q;
  q.roc = ro * c;
  q.ypro = CT(1) / ro;
  q.pc2 = CT(.5) * q.ypro;
  q.proc = q.pc2 / c;
  q.ro = ro;
  if constexpr (NV == 7) {
    q.drh = CT(.667) * rk * (q.ypro * q.ypro) * drdh;
    q.ydrp = CT(1) / (CT(1) + CT(.667) * rk * q.ypro * drdp);
  } else {
    q.drh = q.ydrp = CT(0);
  }
  return q;
}

template <typename CT, int NV>
FF_DI void dd_syi_s(CT w[NV], const CT x[NV], const DdFrame<CT>& f, const DdScal<CT>& q) {
  CT z2 = f.nx * x[1] + f.ny * x[2] + f.nz * x[3];
  CT z3 = f.t21 * x[1] + f.t22 * x[2] + f.t23 * x[3];
  CT z4 = f.t31 * x[1] + f.t32 * x[2] + f.t33 * x[3];
  w[0] = x[0] - q.ypro * x[4];
  w[1] = q.roc * z2 + x[4];
  w[2] = z3;
  w[3] = z4;
  w[4] = -q.roc * z2 + x[4];
  if constexpr (NV == 7) { w[5] = x[5]; w[6] = x[6]; }
}

template <typename CT, int NV>
FF_DI void dd_sym1i_s(CT x[NV], const CT w[NV], const DdFrame<CT>& f, const DdScal<CT>& q) {
  CT dh = w[0] + q.pc2 * (w[1] + w[4]);
  CT x2i = q.proc * (w[1] - w[4]);
  CT x5 = CT(.5) * (w[1] + w[4]);
  x[0] = dh;
  if constexpr (NV == 5) {
    x[4] = x5;
  } else {
    x[4] = q.ydrp * (x5 - q.drh * q.ro * dh - CT(.667) * q.ro * w[5]);
    x[5] = w[5];
    x[6] = w[6];
  }
  x[1] = f.nx * x2i + f.t21 * w[2] + f.t31 * w[3];
  x[2] = f.ny * x2i + f.t22 * w[2] + f.t32 * w[3];
  x[3] = f.nz * x2i + f.t23 * w[2] + f.t33 * w[3];
}

template <typename CT, int NV, typename S>
FF_DI void dd_put_scal(CT* s, int stride, const DdScal<CT>& q) {
  s[S::ROC * stride] = q.roc; s[S::YPRO * stride] = q.ypro; s[S::PC2 * stride] = q.pc2; s[S::PROC * stride] = q.proc;
  if constexpr (NV == 7) { s[S::RO * stride] = q.ro; s[S::DRH * stride] = q.drh; s[S::YDRP * stride] = q.ydrp; }
}

template <typename CT, int NV, typename S>
FF_DI DdScal<CT> dd_get_scal(const CT* s, int stride) {
  DdScal<CT> q;
  q.roc = s[S::ROC * stride]; q.ypro = s[S::YPRO * stride]; q.pc2 = s[S::PC2 * stride]; q.proc = s[S::PROC * stride];
  if constexpr (NV == 7) { q.ro = s[S::RO * stride]; q.drh = s[S::DRH * stride]; q.ydrp = s[S::YDRP * stride]; }
  else { q.ro = q.drh = q.ydrp = CT(0); }
  return q;
}

// The raw values one producer step reads for cell K (storage index N):
// the cell's increments and flow values, the neighbour on the side the sweep
// goes next (PRED: K-1, CORR: K+1), the areas of faces K-1/2 and K+1/2 and
// the normals of face K-1/2 (PRED) and K+1/2.  Loaded one chunk ahead, so
// that their latency overlaps the arithmetic of the current chunk.
template <typename CT, int NV>
struct DdRaw {
  CT d[NV];
  CT dt1, vol, ro, c, u, v, w, mu, vol2, ro2, mu2, al, au, nxl, nyl, nzl, nxu, nyu, nzu, rk, drdp, drdh;
};

template <typename CT, int NV, bool UP>
FF_DI void dd_load(DdRaw<CT, NV>& r, const DevBlock& b, const ff_params& p, const DdLine& L, int K) {
  const size_t st = L.st, N = L.n0 + (size_t)(K - 1) * st, Nu = N + st, Q = UP ? Nu : N - st;
#pragma unroll
  for (int v = 0; v < NV; v++) r.d[v] = (CT)b.a[FF_DRO + v][N];
  r.dt1 = (CT)p.theta * (CT)__ldg(b.a[FF_DTL] + N);
  r.vol = (CT)__ldg(b.a[FF_VOL] + N); r.ro = (CT)__ldg(b.a[FF_RO] + N); r.c = (CT)__ldg(b.a[FF_C] + N);
  r.u = (CT)__ldg(b.a[FF_U] + N); r.v = (CT)__ldg(b.a[FF_V] + N); r.w = (CT)__ldg(b.a[FF_W] + N);
  // VIST + VIS of the cell and of the neighbour, summed as the reference
  // sums them: (VIST(N) + VIS(N)) + VIST(Q) + VIS(Q)
  r.mu = (CT)__ldg(b.a[FF_VIST] + N) + (CT)__ldg(b.a[FF_VIS] + N);
  r.vol2 = (CT)__ldg(b.a[FF_VOL] + Q); r.ro2 = (CT)__ldg(b.a[FF_RO] + Q);
  const CT vt2 = (CT)__ldg(b.a[FF_VIST] + Q), vs2 = (CT)__ldg(b.a[FF_VIS] + Q);
  r.mu2 = r.mu + vt2 + vs2;
  r.al = (CT)__ldg(L.A + N); r.au = (CT)__ldg(L.A + Nu);
  if (!UP) { r.nxl = (CT)__ldg(L.AX + N); r.nyl = (CT)__ldg(L.AY + N); r.nzl = (CT)__ldg(L.AZ + N); }
  r.nxu = (CT)__ldg(L.AX + Nu); r.nyu = (CT)__ldg(L.AY + Nu); r.nzu = (CT)__ldg(L.AZ + Nu);
  if constexpr (NV == 7) {
    r.rk = (CT)__ldg(b.a[FF_RK] + N); r.drdp = (CT)__ldg(b.a[FF_DRDP] + N); r.drdh = (CT)__ldg(b.a[FF_DRDH] + N);
  } else {
    r.rk = r.drdp = r.drdh = CT(0);
  }
}

// Producer side of PRED for cell K: the arithmetic of PRED/PREDKE and
// DIAG/DIAGKE that does not involve BD.
template <typename CT, int NV>
FF_DI void dd_pred_compute(CT* s, int stride, const DdRaw<CT, NV>& r, int idi, int K) {
  using S = DdPredSlots<NV>;
  const CT dt1 = r.dt1, vol = r.vol, c = r.c, al = r.al, au = r.au;
#pragma unroll
  for (int v = 0; v < NV; v++) s[(S::RHS + v) * stride] = vol * r.d[v];
  s[S::A * stride] = dt1 * au;
  const DdFrame<CT> fl = dd_frame<CT>(r.nxl, r.nyl, r.nzl);
  const DdFrame<CT> fu = dd_frame<CT>(r.nxu, r.nyu, r.nzu);
  dd_put_frame(s + S::FL * stride, stride, fl);
  dd_put_frame(s + S::FU * stride, stride, fu);
  dd_put_scal<CT, NV, S>(s, stride, dd_scal<CT, NV>(r.ro, c, r.rk, r.drdp, r.drdh));
  const CT rl1 = fl.nx * r.u + fl.ny * r.v + fl.nz * r.w, rl2 = rl1 + c, rl5 = rl1 - c;
  const CT ff = K == 1 ? CT(.25) : CT(.5);
  const CT cdiff = K <= idi ? CT(2) : CT(0);
  const CT rnum = ff * (vol + r.vol2) * (r.ro + r.ro2);
  const CT T = cdiff * al / rnum * r.mu2;
  s[S::X1 * stride] = dmax(-rl1, CT(0)) + T;
  s[S::X2 * stride] = dmax(-rl2, CT(0)) + T;
  s[S::X5 * stride] = dmax(-rl5, CT(0)) + T;
  const CT x1a = fabs(rl1) + T, x2a = fabs(rl2) + T, x5a = fabs(rl5) + T;
  const CT vr = NV == 7 ? vol + CT(1.e-21) : vol;
  s[S::R1 * stride] = CT(1) / (vr + dt1 * x1a * al);
  s[S::R2 * stride] = CT(1) / (vr + dt1 * x2a * al);
  s[S::R5 * stride] = CT(1) / (vr + dt1 * x5a * al);
  if constexpr (NV == 7) s[S::R6 * stride] = CT(1) / (vr + dt1 * (x1a * al));
  // DIAG: positive split eigenvalues of face K-1/2, negative of K+1/2
  const CT ucon = fu.nx * r.u + fu.ny * r.v + fu.nz * r.w;
  const CT rl2n = dmax(-(ucon + c), CT(0)), rl5n = dmax(-(ucon - c), CT(0)), rl1n = dmax(-ucon, CT(0));
  const CT dtv = dt1 / vr;
  s[S::F1 * stride] = CT(1) + dtv * (al * dmax(rl1, CT(0)) + au * rl1n);
  s[S::F2 * stride] = CT(1) + dtv * (al * dmax(rl2, CT(0)) + au * rl2n);
  s[S::F5 * stride] = CT(1) + dtv * (al * dmax(rl5, CT(0)) + au * rl5n);
}

// Consumer side of PRED + DIAG for one cell: the recurrence through BD.
template <typename CT, int NV>
FF_DI void dd_pred_consume(const CT* s, int stride, CT bd[NV], const DevBlock& b, size_t N) {
  using S = DdPredSlots<NV>;
  const CT a = s[S::A * stride];
  const DdFrame<CT> fl = dd_get_frame(s + S::FL * stride, stride);
  const DdScal<CT> q = dd_get_scal<CT, NV, S>(s, stride);
  CT bdx[NV], y[NV], out[NV];
#pragma unroll
  for (int v = 0; v < NV; v++) bdx[v] = a * bd[v] + s[(S::RHS + v) * stride];
  dd_syi_s<CT, NV>(y, bdx, fl, q);
  const CT r1 = s[S::R1 * stride];
  y[0] *= r1; y[1] *= s[S::R2 * stride]; y[2] *= r1; y[3] *= r1; y[4] *= s[S::R5 * stride];
  if constexpr (NV == 7) { const CT r6 = s[S::R6 * stride]; y[5] *= r6; y[6] *= r6; }
  dd_sym1i_s<CT, NV>(out, y, fl, q);
  dd_xmul<CT, NV>(y, s[S::X1 * stride], s[S::X2 * stride], s[S::X5 * stride]);
  dd_sym1i_s<CT, NV>(bd, y, fl, q);
  // DIAG
  const DdFrame<CT> fu = dd_get_frame(s + S::FU * stride, stride);
  CT z[NV];
  dd_syi_s<CT, NV>(z, out, fu, q);
  const CT f1 = s[S::F1 * stride];
  z[0] *= f1; z[1] *= s[S::F2 * stride]; z[2] *= f1; z[3] *= f1; z[4] *= s[S::F5 * stride];
  if constexpr (NV == 7) { z[5] *= f1; z[6] *= f1; }
  dd_sym1i_s<CT, NV>(out, z, fu, q);
#pragma unroll
  for (int v = 0; v < NV; v++) b.a[FF_DRO + v][N] = (double)out[v];
}

// Producer side of CORR for cell K.
template <typename CT, int NV>
FF_DI void dd_corr_compute(CT* s, int stride, const DdRaw<CT, NV>& r, int idi, int K) {
  using S = DdCorrSlots<NV>;
  const CT dt1 = r.dt1, vol = r.vol, c = r.c, au = r.au;
#pragma unroll
  for (int v = 0; v < NV; v++) s[(S::RHS + v) * stride] = vol * r.d[v];
  s[S::A * stride] = dt1 * r.al;
  const DdFrame<CT> fu = dd_frame<CT>(r.nxu, r.nyu, r.nzu);
  dd_put_frame(s + S::FU * stride, stride, fu);
  dd_put_scal<CT, NV, S>(s, stride, dd_scal<CT, NV>(r.ro, c, r.rk, r.drdp, r.drdh));
  const CT rl1 = fu.nx * r.u + fu.ny * r.v + fu.nz * r.w, rl2 = rl1 + c, rl5 = rl1 - c;
  const CT cdiff = K <= idi ? CT(2) : CT(0);
  const CT rnum = CT(.5) * (vol + r.vol2) * (r.ro + r.ro2);
  const CT T = cdiff * au / rnum * r.mu2;
  s[S::X1 * stride] = dmax(rl1, CT(0)) + T;
  s[S::X2 * stride] = dmax(rl2, CT(0)) + T;
  s[S::X5 * stride] = dmax(rl5, CT(0)) + T;
  const CT x1a = fabs(rl1) + T, x2a = fabs(rl2) + T, x5a = fabs(rl5) + T;
  const CT vr = NV == 7 ? vol + CT(1.e-21) : vol;
  s[S::R1 * stride] = CT(1) / (vr + dt1 * x1a * au);
  s[S::R2 * stride] = CT(1) / (vr + dt1 * x2a * au);
  s[S::R5 * stride] = CT(1) / (vr + dt1 * x5a * au);
  if constexpr (NV == 7) s[S::R6 * stride] = CT(1) / (vr + dt1 * (x1a * au));
}

template <typename CT, int NV>
FF_DI void dd_corr_consume(const CT* s, int stride, CT bd[NV], const DevBlock& b, size_t N) {
  using S = DdCorrSlots<NV>;
  const CT a = s[S::A * stride];
  const DdFrame<CT> fu = dd_get_frame(s + S::FU * stride, stride);
  const DdScal<CT> q = dd_get_scal<CT, NV, S>(s, stride);
  CT bdx[NV], y[NV], out[NV];
#pragma unroll
  for (int v = 0; v < NV; v++) bdx[v] = a * bd[v] + s[(S::RHS + v) * stride];
  dd_syi_s<CT, NV>(y, bdx, fu, q);
  const CT r1 = s[S::R1 * stride];
  y[0] *= r1; y[1] *= s[S::R2 * stride]; y[2] *= r1; y[3] *= r1; y[4] *= s[S::R5 * stride];
  if constexpr (NV == 7) { const CT r6 = s[S::R6 * stride]; y[5] *= r6; y[6] *= r6; }
  dd_sym1i_s<CT, NV>(out, y, fu, q);
#pragma unroll
  for (int v = 0; v < NV; v++) b.a[FF_DRO + v][N] = (double)out[v];
  dd_xmul<CT, NV>(y, s[S::X1 * stride], s[S::X2 * stride], s[S::X5 * stride]);
  dd_sym1i_s<CT, NV>(bd, y, fu, q);
}

// One sweep (PRED+DIAG if !UP, CORR if UP) of LPC lines per CTA: warp 0
// consumes (lane = line), the LPC*CH producer threads each take one cell of
// the chunk.  Step s of the sweep is cell K = n - s (PRED) or K = s + 1
// (CORR); chunk it holds steps it*CH .. it*CH+CH-1.  A producer loads the
// raw values of its cell of chunk it+1 before it computes chunk it.
template <typename CT, int NV, int LPC, int CH, bool UP>
__global__ void __launch_bounds__(32 + LPC * CH) k_ddadi_pc(DevBlock b, ff_params p, int dir) {
  static_assert(LPC <= 32 && (LPC * CH) % 32 == 0, "producer warps must be whole");
  constexpr int NS = UP ? DdCorrSlots<NV>::N : DdPredSlots<NV>::N;
  constexpr int SLOT = LPC * CH;
  extern __shared__ __align__(16) unsigned char dd_pc_raw[];
  CT* buf = reinterpret_cast<CT*>(dd_pc_raw);   // [2][NS][SLOT]
  const int line0 = blockIdx.x * LPC;
  DdLine L;
  if (!dd_line(b, p, dir, line0, L)) return;    // the whole CTA: no line (a grid of whole CTAs never has one)
  const int n = L.n;
  const size_t st = L.st;
  const int nch = (n + CH - 1) / CH;
  const bool cons = threadIdx.x < 32;
  int pl = threadIdx.x, pc = 0;
  if (!cons) {
    const int q = threadIdx.x - 32;
    if (dir == 1) { pc = q % CH; pl = q / CH; }   // i lines: lanes along the line (contiguous)
    else { pl = q % LPC; pc = q / LPC; }           // j, k lines: lanes across lines (contiguous)
  }
  const bool valid = pl < LPC && dd_line(b, p, dir, line0 + pl, L);
  auto cellK = [&](int s) { return UP ? s + 1 : n - s; };
  DdRaw<CT, NV> cur, nxt;
  if (!cons && valid && pc < n) dd_load<CT, NV, UP>(cur, b, p, L, cellK(pc));
  CT bd[NV];
#pragma unroll
  for (int v = 0; v < NV; v++) bd[v] = CT(0);
  for (int it = 0; it <= nch; it++) {
    if (!cons) {
      const int s = it * CH + pc, sn = s + CH;
      if (valid && sn < n) dd_load<CT, NV, UP>(nxt, b, p, L, cellK(sn));
      if (valid && s < n) {
        CT* sp = buf + (size_t)(it & 1) * NS * SLOT + pc * LPC + pl;
        if constexpr (UP) dd_corr_compute<CT, NV>(sp, SLOT, cur, L.idi, cellK(s));
        else dd_pred_compute<CT, NV>(sp, SLOT, cur, L.idi, cellK(s));
      }
      cur = nxt;
    } else if (valid && it >= 1) {
      const CT* cp = buf + (size_t)((it - 1) & 1) * NS * SLOT + pl;
      for (int c = 0; c < CH; c++) {
        const int s = (it - 1) * CH + c;
        if (s >= n) break;
        const size_t N = L.n0 + (size_t)(cellK(s) - 1) * st;
        if constexpr (UP) dd_corr_consume<CT, NV>(cp + c * LPC, SLOT, bd, b, N);
        else dd_pred_consume<CT, NV>(cp + c * LPC, SLOT, bd, b, N);
      }
    }
    __syncthreads();
  }
}

template <typename CT>
inline size_t ddadi_pc_smem_bytes(int nv, int lpc, int ch, bool up) {
  const int ns = up ? (nv == 7 ? DdCorrSlots<7>::N : DdCorrSlots<5>::N)
                    : (nv == 7 ? DdPredSlots<7>::N : DdPredSlots<5>::N);
  return (size_t)2 * ns * lpc * ch * sizeof(CT);
}
