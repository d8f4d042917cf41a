/*
 * CPU oracle, DDADI implicit stage (LUSGS=0, the reference's default).
 * TEST INFRASTRUCTURE ONLY (see finflo_oracle.c).  Included at the end of
 * finflo_oracle.c after finflo_oracle_sst.c, so that it shares their static
 * helpers.
 *
 * IMPS imps3.f:320-356 calls IMPSWE three times: k lines, then (after the
 * SORT38/SORT2 transposes that make the next direction the slowest index)
 * i lines, then j lines.  IMPSWE imps3.f:578-778 runs, for KMAX > 1 in its
 * rotated frame, the backward sweep PRED (imps4.f:788), the point factor
 * DIAG (imps4.f:911) and the forward sweep CORR (imps4.f:671) along every
 * line; for ITURB>=3 (JRIMP=0) PREDKE/DIAGKE/CORRKE (imps4.f:2084, 2235,
 * 1939) with SYIKE/SYM1KE.  The transposes only reorder the arrays, and the
 * lines of one direction are independent, so this file walks the lines of
 * each direction in place: the k lines with stride IL, i lines stride 1,
 * j lines stride IS, and the face arrays A3/A1/A2 of that direction, whose
 * entry N is the face between cell N - stride and cell N.
 *
 * Only interior lines are restated.  The reference also walks the ghost
 * columns of each plane (imps4.f:842 I = IN+1..JMAX*ISTRID); their
 * increments are zero and they never feed an interior cell.
 */

/* SYI / SYM1I imps4.f:10/46 (five equations) and SYIKE / SYM1KE
 * imps4.f:982/1034 (seven), split so that the sweeps can scale between. */
static void dd_syi(double *w, const double *x, int nv, double rk, double c, double ro, double drdp,
                   double drdh, double nx, double ny, double nz, double *t) {
  double a21, a22, a23, a31, a32, a33;
  surfvects(nx, ny, nz, &a21, &a22, &a23, &a31, &a32, &a33);
  t[0] = a21; t[1] = a22; t[2] = a23; t[3] = a31; t[4] = a32; t[5] = a33;
  double z1 = x[0], z5 = x[4];
  double z2 = nx * x[1] + ny * x[2] + nz * x[3];
  double z3 = a21 * x[1] + a22 * x[2] + a23 * x[3];
  double z4 = a31 * x[1] + a32 * x[2] + a33 * x[3];
  double roc = ro * c;
  if (nv == 5) {
    w[0] = z1 - z5 / ro;
  } else {
    double pc2 = 1. / ro;
    w[0] = z1 - pc2 * z5;
    w[5] = x[5];
    w[6] = x[6];
  }
  w[1] = roc * z2 + z5;
  w[2] = z3;
  w[3] = z4;
  w[4] = -roc * z2 + z5;
  (void)rk; (void)drdp; (void)drdh;
}

static void dd_sym1i(double *x, const double *w, int nv, double rk, double c, double ro, double drdp,
                     double drdh, double nx, double ny, double nz, const double *t) {
  double ypro = 1. / ro, pc2 = .5 * ypro, proc = pc2 / c;
  double dh = w[0] + pc2 * (w[1] + w[4]);
  double x2i = proc * (w[1] - w[4]), x3i = w[2], x4i = w[3];
  double x5 = .5 * (w[1] + w[4]);
  x[0] = dh;
  if (nv == 5) {
    x[4] = x5;
  } else {
    double drh = .667 * rk * (ypro * ypro) * drdh;
    double ydrp = 1. / (1. + .667 * rk * ypro * drdp);
    x[4] = ydrp * (x5 - drh * ro * dh - .667 * ro * w[5]);
    x[5] = w[5];
    x[6] = w[6];
  }
  x[1] = nx * x2i + t[0] * x3i + t[3] * x4i;
  x[2] = ny * x2i + t[1] * x3i + t[4] * x4i;
  x[3] = nz * x2i + t[2] * x3i + t[5] * x4i;
}

typedef struct {
  double *D[7];
  const double *VOL, *DTL, *U, *V, *W, *C, *RO, *VIS, *VIST, *RK, *DRDP, *DRDH;
  const double *A, *AX, *AY, *AZ;
  int nv, n, idi;
  size_t st;
  double theta;
} dd_line_t;

/* The scalars of cell N the transforms need. */
#define DD_CELL(L, N) \
  ((L)->nv == 7 ? (L)->RK[N] : 0.), (L)->C[N], (L)->RO[N], ((L)->nv == 7 ? (L)->DRDP[N] : 0.), \
      ((L)->nv == 7 ? (L)->DRDH[N] : 0.)

/* PRED imps4.f:788-905 / PREDKE imps4.f:2084-2229 on the line whose first
 * cell is n0: K = n .. 1, carry BD from cell K+1 through face K+1/2. */
static void dd_pred(const dd_line_t *L, size_t n0) {
  const int nv = L->nv;
  const size_t st = L->st;
  double bd[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int K = L->n; K >= 1; K--) {
    size_t N = n0 + (size_t)(K - 1) * st;
    double ff = .5;
    if (K == 1) ff = .25;
    double cdiff = K <= L->idi ? 2. : 0.;
    double dt1 = L->theta * L->DTL[N];
    double bdx[7], y[7], t[6];
    for (int v = 0; v < nv; v++) bdx[v] = dt1 * L->A[N + st] * bd[v] + L->VOL[N] * L->D[v][N];
    double nx = L->AX[N], ny = L->AY[N], nz = L->AZ[N];
    dd_syi(y, bdx, nv, DD_CELL(L, N), nx, ny, nz, t);
    double rl1 = nx * L->U[N] + ny * L->V[N] + nz * L->W[N] - 0.;
    double rl2 = rl1 + L->C[N], rl5 = rl1 - L->C[N];
    double rnum = ff * (L->VOL[N] + L->VOL[N - st]) * (L->RO[N] + L->RO[N - st]);
    double T = cdiff * L->A[N] / rnum * (L->VIST[N] + L->VIS[N] + L->VIST[N - st] + L->VIS[N - st]);
    double x1 = MAXD(-rl1, 0.) + T, x2 = MAXD(-rl2, 0.) + T, x5 = MAXD(-rl5, 0.) + T;
    double x1a = fabs(rl1) + T, x2a = fabs(rl2) + T, x5a = fabs(rl5) + T;
    if (nv == 5) {
      y[0] = y[0] / (L->VOL[N] + dt1 * x1a * L->A[N]);
      y[1] = y[1] / (L->VOL[N] + dt1 * x2a * L->A[N]);
      y[2] = y[2] / (L->VOL[N] + dt1 * x1a * L->A[N]);
      y[3] = y[3] / (L->VOL[N] + dt1 * x1a * L->A[N]);
      y[4] = y[4] / (L->VOL[N] + dt1 * x5a * L->A[N]);
    } else {
      const double vrel = 1.e-21;
      y[0] = y[0] / (L->VOL[N] + vrel + dt1 * x1a * L->A[N]);
      y[1] = y[1] / (L->VOL[N] + vrel + dt1 * x2a * L->A[N]);
      y[2] = y[2] / (L->VOL[N] + vrel + dt1 * x1a * L->A[N]);
      y[3] = y[3] / (L->VOL[N] + vrel + dt1 * x1a * L->A[N]);
      y[4] = y[4] / (L->VOL[N] + vrel + dt1 * x5a * L->A[N]);
      y[5] = y[5] / (L->VOL[N] + vrel + dt1 * (x1a * L->A[N] + 0.));
      y[6] = y[6] / (L->VOL[N] + vrel + dt1 * (x1a * L->A[N] + 0.));
    }
    double out[7];
    dd_sym1i(out, y, nv, DD_CELL(L, N), nx, ny, nz, t);
    for (int v = 0; v < nv; v++) L->D[v][N] = out[v];
    y[0] = x1 * y[0]; y[1] = x2 * y[1]; y[2] = x1 * y[2]; y[3] = x1 * y[3]; y[4] = x5 * y[4];
    if (nv == 7) { y[5] = x1 * y[5]; y[6] = x1 * y[6]; }
    dd_sym1i(bd, y, nv, DD_CELL(L, N), nx, ny, nz, t);
  }
}

/* DIAG imps4.f:911-971 / DIAGKE imps4.f:2235-2309 on one cell: the frame of
 * face K+1/2, positive split eigenvalues of face K-1/2, negative of K+1/2. */
static void dd_diag(const dd_line_t *L, size_t N) {
  const int nv = L->nv;
  const size_t st = L->st;
  double dtx = L->theta * L->DTL[N];
  double x[7], y[7], t[6];
  for (int v = 0; v < nv; v++) x[v] = L->D[v][N];
  double nx = L->AX[N + st], ny = L->AY[N + st], nz = L->AZ[N + st];
  dd_syi(y, x, nv, DD_CELL(L, N), nx, ny, nz, t);
  double c = L->C[N];
  double ucon = nx * L->U[N] + ny * L->V[N] + nz * L->W[N] - 0.;
  double rl2n = MAXD(-(ucon + c), 0.), rl5n = MAXD(-(ucon - c), 0.), rl1n = MAXD(-ucon, 0.);
  ucon = L->AX[N] * L->U[N] + L->AY[N] * L->V[N] + L->AZ[N] * L->W[N] - 0.;
  double rl2p = MAXD(ucon + c, 0.), rl5p = MAXD(ucon - c, 0.), rl1p = MAXD(ucon, 0.);
  double dt1 = nv == 5 ? dtx / L->VOL[N] : dtx / (L->VOL[N] + 1.e-21);
  const double a0 = L->A[N], a1 = L->A[N + st];
  y[0] = y[0] * (1. + dt1 * (a0 * rl1p + a1 * rl1n));
  y[1] = y[1] * (1. + dt1 * (a0 * rl2p + a1 * rl2n));
  y[2] = y[2] * (1. + dt1 * (a0 * rl1p + a1 * rl1n));
  y[3] = y[3] * (1. + dt1 * (a0 * rl1p + a1 * rl1n));
  y[4] = y[4] * (1. + dt1 * (a0 * rl5p + a1 * rl5n));
  if (nv == 7) {
    y[5] = y[5] * (1. + dt1 * (a0 * rl1p + a1 * rl1n + 0.));
    y[6] = y[6] * (1. + dt1 * (a0 * rl1p + a1 * rl1n + 0.));
  }
  double out[7];
  dd_sym1i(out, y, nv, DD_CELL(L, N), nx, ny, nz, t);
  for (int v = 0; v < nv; v++) L->D[v][N] = out[v];
}

/* CORR imps4.f:671-782 / CORRKE imps4.f:1939-2078: K = 1 .. n, carry BD from
 * cell K-1 through face K-1/2, frame of face K+1/2. */
static void dd_corr(const dd_line_t *L, size_t n0) {
  const int nv = L->nv;
  const size_t st = L->st;
  double bd[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int K = 1; K <= L->n; K++) {
    size_t N = n0 + (size_t)(K - 1) * st;
    double cdiff = K <= L->idi ? 2. : 0.;
    double dt1 = L->theta * L->DTL[N];
    double bdx[7], y[7], t[6];
    for (int v = 0; v < nv; v++) bdx[v] = dt1 * L->A[N] * bd[v] + L->VOL[N] * L->D[v][N];
    const size_t M = N + st;
    double nx = L->AX[M], ny = L->AY[M], nz = L->AZ[M];
    dd_syi(y, bdx, nv, DD_CELL(L, N), nx, ny, nz, t);
    double rl1 = nx * L->U[N] + ny * L->V[N] + nz * L->W[N] - 0.;
    double rl2 = rl1 + L->C[N], rl5 = rl1 - L->C[N];
    double rnum = .5 * (L->VOL[N] + L->VOL[M]) * (L->RO[N] + L->RO[M]);
    double T = cdiff * L->A[M] / rnum * (L->VIST[N] + L->VIS[N] + L->VIST[M] + L->VIS[M]);
    double x1 = MAXD(rl1, 0.) + T, x2 = MAXD(rl2, 0.) + T, x5 = MAXD(rl5, 0.) + T;
    double x1a = fabs(rl1) + T, x2a = fabs(rl2) + T, x5a = fabs(rl5) + T;
    if (nv == 5) {
      y[0] = y[0] / (L->VOL[N] + dt1 * x1a * L->A[M]);
      y[1] = y[1] / (L->VOL[N] + dt1 * x2a * L->A[M]);
      y[2] = y[2] / (L->VOL[N] + dt1 * x1a * L->A[M]);
      y[3] = y[3] / (L->VOL[N] + dt1 * x1a * L->A[M]);
      y[4] = y[4] / (L->VOL[N] + dt1 * x5a * L->A[M]);
    } else {
      const double vrel = 1.e-21;
      y[0] = y[0] / (L->VOL[N] + vrel + dt1 * x1a * L->A[M]);
      y[1] = y[1] / (L->VOL[N] + vrel + dt1 * x2a * L->A[M]);
      y[2] = y[2] / (L->VOL[N] + vrel + dt1 * x1a * L->A[M]);
      y[3] = y[3] / (L->VOL[N] + vrel + dt1 * x1a * L->A[M]);
      y[4] = y[4] / (L->VOL[N] + vrel + dt1 * x5a * L->A[M]);
      y[5] = y[5] / (L->VOL[N] + vrel + dt1 * (x1a * L->A[M] + 0.));
      y[6] = y[6] / (L->VOL[N] + vrel + dt1 * (x1a * L->A[M] + 0.));
    }
    double out[7];
    dd_sym1i(out, y, nv, DD_CELL(L, N), nx, ny, nz, t);
    for (int v = 0; v < nv; v++) L->D[v][N] = out[v];
    y[0] = x1 * y[0]; y[1] = x2 * y[1]; y[2] = x1 * y[2]; y[3] = x1 * y[3]; y[4] = x5 * y[4];
    if (nv == 7) { y[5] = x1 * y[5]; y[6] = x1 * y[6]; }
    dd_sym1i(bd, y, nv, DD_CELL(L, N), nx, ny, nz, t);
  }
}

/* IMPSWE imps3.f:578 for one direction (1 = i, 2 = j, 3 = k): PRED, DIAG
 * and CORR over every interior line, skipped when the line has one cell
 * (imps3.f:601 IF(KMAX > 1)).  The reference runs PRED over all lines
 * before DIAG and CORR; the lines are independent, so line by line is the
 * same arithmetic. */
static void dd_direction(orc_block *b, const ff_params *p, int nv, int dir) {
  dims_t d = dims_of(b);
  dd_line_t L;
  const int sl[7] = {FF_DRO, FF_DM, FF_DN, FF_DW, FF_DE, FF_DRK, FF_DEPS};
  for (int v = 0; v < 7; v++) L.D[v] = b->a[sl[v]];
  L.VOL = b->a[FF_VOL]; L.DTL = b->a[FF_DTL]; L.U = b->a[FF_U]; L.V = b->a[FF_V]; L.W = b->a[FF_W];
  L.C = b->a[FF_C]; L.RO = b->a[FF_RO]; L.VIS = b->a[FF_VIS]; L.VIST = b->a[FF_VIST];
  L.RK = b->a[FF_RK]; L.DRDP = b->a[FF_DRDP]; L.DRDH = b->a[FF_DRDH];
  L.nv = nv;
  L.theta = p->theta;
  int na, nb;
  if (dir == 1) {
    L.A = b->a[FF_A1]; L.AX = b->a[FF_A1XA]; L.AY = b->a[FF_A1YA]; L.AZ = b->a[FF_A1ZA];
    L.n = d.imax; L.idi = p->idi1; L.st = 1; na = d.jmax; nb = d.kmax;
  } else if (dir == 2) {
    L.A = b->a[FF_A2]; L.AX = b->a[FF_A2XA]; L.AY = b->a[FF_A2YA]; L.AZ = b->a[FF_A2ZA];
    L.n = d.jmax; L.idi = p->idi2; L.st = (size_t)d.is; na = d.imax; nb = d.kmax;
  } else {
    L.A = b->a[FF_A3]; L.AX = b->a[FF_A3XA]; L.AY = b->a[FF_A3YA]; L.AZ = b->a[FF_A3ZA];
    L.n = d.kmax; L.idi = p->idi3; L.st = (size_t)d.il; na = d.imax; nb = d.jmax;
  }
  if (L.n <= 1) return;
  for (int bb = 1; bb <= nb; bb++)
    for (int aa = 1; aa <= na; aa++) {
      size_t n0 = dir == 1 ? IX(d, 1, aa, bb) : (dir == 2 ? IX(d, aa, 1, bb) : IX(d, aa, bb, 1));
      dd_pred(&L, n0);
      for (int K = 1; K <= L.n; K++) dd_diag(&L, n0 + (size_t)(K - 1) * L.st);
      dd_corr(&L, n0);
    }
}

/* IMPS imps3.f:320-356: k lines, i lines, j lines. */
static void ddadi_sweeps(orc_block *b, const ff_params *p, int nv) {
  dd_direction(b, p, nv, 3);
  dd_direction(b, p, nv, 1);
  dd_direction(b, p, nv, 2);
}

void orc_ddadi(orc_block *b, const ff_params *p) { ddadi_sweeps(b, p, p->iturb >= 3 ? 7 : 5); }
