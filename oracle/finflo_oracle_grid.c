/* The reference's block set-up restated (test infrastructure: the checker of
 * the library's host and device set-up, never the thing measured):
 *
 *   GRIDEX / REFXYZ gluebm.f:1029, 1175  one reflected ghost node layer;
 *                                         edges and corners diagonally
 *   AREVC1 gluebm.f:1586 (GRID1B 1265)   face areas and unit normals, cell
 *                                         volumes (three passes) and centres
 *                                         of the cells 0..MAX+1
 *   D1D2D3 gluebm.f:2326                 cell thicknesses
 *   LUMPA1 / LUMPVS gluebm.f:2194, 2256  coarse faces, volumes, centres
 *   PICK_XYZ / WALL_DIST gluebm.f:9452,  wall distance: nearest of the wall
 *   9533 (DISTANCES 9136)                 points halfway between the first
 *                                         interior and ghost cell centres
 *   LUMP_DIST gluebm.f:9562              coarse wall distance
 *
 * Included by finflo_oracle.c.  Node arrays are [k][j][i] of the interior
 * nodes, (kmax+1)(jmax+1)(imax+1) values, i fastest. */

/* node (i, j, k) of the one-layer extended array, 1-based interior nodes
 * 1..n, ghosts 0 and n+1 */
#define EX(E, i, j, k) (E)[((size_t)(k) * (nj + 2) + (j)) * (ni + 2) + (i)]

static void gridex(const double *X, int ni, int nj, int nk, double *E) {
  for (int k = 1; k <= nk; k++)
    for (int j = 1; j <= nj; j++)
      for (int i = 1; i <= ni; i++) EX(E, i, j, k) = X[((size_t)(k - 1) * nj + (j - 1)) * ni + (i - 1)];
  /* faces (REFXYZ, three calls) */
  for (int j = 1; j <= nj; j++)
    for (int i = 1; i <= ni; i++) {
      EX(E, i, j, 0) = 2. * EX(E, i, j, 1) - EX(E, i, j, 2);
      EX(E, i, j, nk + 1) = 2. * EX(E, i, j, nk) - EX(E, i, j, nk - 1);
    }
  for (int k = 1; k <= nk; k++)
    for (int j = 1; j <= nj; j++) {
      EX(E, 0, j, k) = 2. * EX(E, 1, j, k) - EX(E, 2, j, k);
      EX(E, ni + 1, j, k) = 2. * EX(E, ni, j, k) - EX(E, ni - 1, j, k);
    }
  for (int k = 1; k <= nk; k++)
    for (int i = 1; i <= ni; i++) {
      EX(E, i, 0, k) = 2. * EX(E, i, 1, k) - EX(E, i, 2, k);
      EX(E, i, nj + 1, k) = 2. * EX(E, i, nj, k) - EX(E, i, nj - 1, k);
    }
  /* edges: along k, i, j, each diagonally in the other two directions */
  for (int k = 1; k <= nk; k++) {
    EX(E, 0, 0, k) = 2. * EX(E, 1, 1, k) - EX(E, 2, 2, k);
    EX(E, 0, nj + 1, k) = 2. * EX(E, 1, nj, k) - EX(E, 2, nj - 1, k);
    EX(E, ni + 1, 0, k) = 2. * EX(E, ni, 1, k) - EX(E, ni - 1, 2, k);
    EX(E, ni + 1, nj + 1, k) = 2. * EX(E, ni, nj, k) - EX(E, ni - 1, nj - 1, k);
  }
  for (int i = 1; i <= ni; i++) {
    EX(E, i, 0, 0) = 2. * EX(E, i, 1, 1) - EX(E, i, 2, 2);
    EX(E, i, 0, nk + 1) = 2. * EX(E, i, 1, nk) - EX(E, i, 2, nk - 1);
    EX(E, i, nj + 1, 0) = 2. * EX(E, i, nj, 1) - EX(E, i, nj - 1, 2);
    EX(E, i, nj + 1, nk + 1) = 2. * EX(E, i, nj, nk) - EX(E, i, nj - 1, nk - 1);
  }
  for (int j = 1; j <= nj; j++) {
    EX(E, 0, j, 0) = 2. * EX(E, 1, j, 1) - EX(E, 2, j, 2);
    EX(E, ni + 1, j, 0) = 2. * EX(E, ni, j, 1) - EX(E, ni - 1, j, 2);
    EX(E, 0, j, nk + 1) = 2. * EX(E, 1, j, nk) - EX(E, 2, j, nk - 1);
    EX(E, ni + 1, j, nk + 1) = 2. * EX(E, ni, j, nk) - EX(E, ni - 1, j, nk - 1);
  }
  /* corners */
  for (int c = 0; c < 8; c++) {
    int gi = c & 1 ? ni + 1 : 0, gj = c & 2 ? nj + 1 : 0, gk = c & 4 ? nk + 1 : 0;
    int i1 = c & 1 ? ni : 1, j1 = c & 2 ? nj : 1, k1 = c & 4 ? nk : 1;
    int i2 = c & 1 ? ni - 1 : 2, j2 = c & 2 ? nj - 1 : 2, k2 = c & 4 ? nk - 1 : 2;
    EX(E, gi, gj, gk) = 2. * EX(E, i1, j1, k1) - EX(E, i2, j2, k2);
  }
}

/* AREVC1 for the faces of direction dir (1, 2, 3) of the cells I, J, K in
 * 0..MAX+1 (1-based cells); the three passes in GRID1B's order accumulate
 * the volume (VSUM, VDIV) and the last one leaves the centres.  The pass's
 * (ISTR, JSTR, KSTR) are the directions (dir, dir+1, dir+2) cyclic; the
 * corners IT1..IT8 step by 0, KSTR, JSTR+KSTR, JSTR, ISTR, ISTR+KSTR,
 * ISTR+JSTR+KSTR, ISTR+JSTR. */
static void arevc1(orc_block *b, const double *EXn, const double *EYn, const double *EZn, int dir) {
  const int imax = b->imax, jmax = b->jmax, kmax = b->kmax;
  const int ni = imax + 1, nj = jmax + 1;
  const double vsum = dir == 1 ? 0. : 1., vdiv = dir == 3 ? 3. : 1.;
  double *AX = b->a[FF_A1XA + 4 * (dir - 1)], *AY = b->a[FF_A1YA + 4 * (dir - 1)];
  double *AZ = b->a[FF_A1ZA + 4 * (dir - 1)], *A = b->a[FF_A1 + 4 * (dir - 1)];
  const int istr = imax + 4, il = istr * (jmax + 4);
  int oa[3] = {0, 0, 0}, ob[3] = {0, 0, 0}, oc[3] = {0, 0, 0};
  oa[dir - 1] = 1;
  ob[dir % 3] = 1;
  oc[(dir + 1) % 3] = 1;
  const int off[8][3] = {{0, 0, 0},
                         {oc[0], oc[1], oc[2]},
                         {ob[0] + oc[0], ob[1] + oc[1], ob[2] + oc[2]},
                         {ob[0], ob[1], ob[2]},
                         {oa[0], oa[1], oa[2]},
                         {oa[0] + oc[0], oa[1] + oc[1], oa[2] + oc[2]},
                         {oa[0] + ob[0] + oc[0], oa[1] + ob[1] + oc[1], oa[2] + ob[2] + oc[2]},
                         {oa[0] + ob[0], oa[1] + ob[1], oa[2] + ob[2]}};
  const int cstep = dir == 1 ? 1 : (dir == 2 ? istr : il);
  for (int K = 0; K <= kmax + 1; K++)
    for (int J = 0; J <= jmax + 1; J++)
      for (int I = 0; I <= imax + 1; I++) {
        const size_t n0 = (size_t)(K + 1) * il + (size_t)(J + 1) * istr + (I + 1);
        double x[9], y[9], z[9];
        for (int q = 1; q <= 8; q++) {
          const int ii = I + off[q - 1][0], jj = J + off[q - 1][1], kk = K + off[q - 1][2];
          x[q] = EX(EXn, ii, jj, kk);
          y[q] = EX(EYn, ii, jj, kk);
          z[q] = EX(EZn, ii, jj, kk);
        }
        const double xce = .125 * (x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7] + x[8]);
        const double yce = .125 * (y[1] + y[2] + y[3] + y[4] + y[5] + y[6] + y[7] + y[8]);
        const double zce = .125 * (z[1] + z[2] + z[3] + z[4] + z[5] + z[6] + z[7] + z[8]);
        const double rdx = xce - .5 * (x[1] + x[2]), rdy = yce - .5 * (y[1] + y[2]), rdz = zce - .5 * (z[1] + z[2]);
        const double r2x = xce - .5 * (x[7] + x[8]), r2y = yce - .5 * (y[7] + y[8]), r2z = zce - .5 * (z[7] + z[8]);
        const double axx = 0.5 * ((z[3] - z[1]) * (y[4] - y[2]) - (y[3] - y[1]) * (z[4] - z[2]));
        const double ayy = 0.5 * ((x[3] - x[1]) * (z[4] - z[2]) - (z[3] - z[1]) * (x[4] - x[2]));
        const double azz = 0.5 * ((y[3] - y[1]) * (x[4] - x[2]) - (x[3] - x[1]) * (y[4] - y[2]));
        const double aa = sqrt(axx * axx + ayy * ayy + azz * azz);
        const double axx2 = -0.5 * ((z[7] - z[5]) * (y[8] - y[6]) - (y[7] - y[5]) * (z[8] - z[6]));
        const double ayy2 = -0.5 * ((x[7] - x[5]) * (z[8] - z[6]) - (z[7] - z[5]) * (x[8] - x[6]));
        const double azz2 = -0.5 * ((y[7] - y[5]) * (x[8] - x[6]) - (x[7] - x[5]) * (y[8] - y[6]));
        const double aa2 = sqrt(axx2 * axx2 + ayy2 * ayy2 + azz2 * azz2);
        const size_t n5 = n0 + cstep;
        AX[n0] = axx / (aa + 1.0E-20);
        AY[n0] = ayy / (aa + 1.0E-20);
        AZ[n0] = azz / (aa + 1.0E-20);
        AX[n5] = -axx2 / (aa2 + 1.0E-20);
        AY[n5] = -ayy2 / (aa2 + 1.0E-20);
        AZ[n5] = -azz2 / (aa2 + 1.0E-20);
        A[n0] = aa;
        A[n5] = aa2;
        b->a[FF_XC][n0] = xce;
        b->a[FF_YC][n0] = yce;
        b->a[FF_ZC][n0] = zce;
        b->a[FF_VOL][n0] = (vsum * b->a[FF_VOL][n0] + rdx * axx + rdy * ayy + rdz * azz + r2x * axx2 + r2y * ayy2 +
                            r2z * azz2) / vdiv;
      }
  /* zero-area faces keep the normal (1, 0, 0) */
  const int im = imax + 1 + (dir == 1), jm = jmax + 1 + (dir == 2), km = kmax + 1 + (dir == 3);
  for (int K = 0; K <= km; K++)
    for (int J = 0; J <= jm; J++)
      for (int I = 0; I <= im; I++) {
        const size_t n0 = (size_t)(K + 1) * il + (size_t)(J + 1) * istr + (I + 1);
        if (A[n0] < 1.E-20) { AX[n0] = 1.; AY[n0] = 0.; AZ[n0] = 0.; }
      }
}

/* Fine-level metrics of block b (its metric arrays written for the cells
 * AREVC1 covers, D1..D3 for the cells 0..MAX+1) from its interior nodes. */
void orc_grid_metrics(orc_block *b, const double *X, const double *Y, const double *Z) {
  const int ni = b->imax + 1, nj = b->jmax + 1, nk = b->kmax + 1;
  const size_t ne = (size_t)(ni + 2) * (nj + 2) * (nk + 2);
  double *E = malloc(3 * ne * sizeof(double));
  gridex(X, ni, nj, nk, E);
  gridex(Y, ni, nj, nk, E + ne);
  gridex(Z, ni, nj, nk, E + 2 * ne);
  for (int d = 1; d <= 3; d++) arevc1(b, E, E + ne, E + 2 * ne, d);
  free(E);
  const int istr = b->imax + 4, il = istr * (b->jmax + 4);
  const double eps = 1.E-20;
  for (int K = 0; K <= b->kmax + 1; K++)
    for (int J = 0; J <= b->jmax + 1; J++)
      for (int I = 0; I <= b->imax + 1; I++) {
        const size_t kk = (size_t)(K + 1) * il + (size_t)(J + 1) * istr + (I + 1);
        const double v = b->a[FF_VOL][kk];
        b->a[FF_D3][kk] = fmin(1.E4, (v + eps) / (b->a[FF_A3][kk] + b->a[FF_A3][kk + il] + eps) * 2.);
        b->a[FF_D2][kk] = fmin(1.E4, (v + eps) / (b->a[FF_A2][kk] + b->a[FF_A2][kk + istr] + eps) * 2.);
        b->a[FF_D1][kk] = fmin(1.E4, (v + eps) / (b->a[FF_A1][kk] + b->a[FF_A1][kk + 1] + eps) * 2.);
      }
}

/* LUMPA1 + LUMPVS (+ D1D2D3) of coarse block c from fine block f (interior
 * faces and cells of c), and LUMP_DIST of the wall distance. */
void orc_grid_lump(const orc_block *f, orc_block *c) {
  const int fs = f->imax + 4, fl = fs * (f->jmax + 4);
  const int cs = c->imax + 4, cl = cs * (c->jmax + 4);
#define FI(I, J, K) ((size_t)((K) + 1) * fl + (size_t)((J) + 1) * fs + ((I) + 1))
#define CI(I, J, K) ((size_t)((K) + 1) * cl + (size_t)((J) + 1) * cs + ((I) + 1))
  for (int dir = 1; dir <= 3; dir++) {
    const double *FA = f->a[FF_A1 + 4 * (dir - 1)], *FX = f->a[FF_A1XA + 4 * (dir - 1)];
    const double *FY = f->a[FF_A1YA + 4 * (dir - 1)], *FZ = f->a[FF_A1ZA + 4 * (dir - 1)];
    double *CA = c->a[FF_A1 + 4 * (dir - 1)], *CX = c->a[FF_A1XA + 4 * (dir - 1)];
    double *CY = c->a[FF_A1YA + 4 * (dir - 1)], *CZ = c->a[FF_A1ZA + 4 * (dir - 1)];
    /* the pass's second and third directions (LUMPA1's JSH, KSH) */
    const int bd = dir % 3, cd = (dir + 1) % 3;
    for (int K = 1; K <= c->kmax + (dir == 3); K++)
      for (int J = 1; J <= c->jmax + (dir == 2); J++)
        for (int I = 1; I <= c->imax + (dir == 1); I++) {
          const int fi[3] = {2 * I - 1, 2 * J - 1, 2 * K - 1};
          size_t it[4];
          for (int q = 0; q < 4; q++) {
            int o[3] = {0, 0, 0};
            if (q & 1) o[bd] = 1;
            if (q & 2) o[cd] = 1;
            it[q] = FI(fi[0] + o[0], fi[1] + o[1], fi[2] + o[2]);
          }
          const double axl = FA[it[0]] * FX[it[0]] + FA[it[1]] * FX[it[1]] + FA[it[2]] * FX[it[2]] + FA[it[3]] * FX[it[3]];
          const double ayl = FA[it[0]] * FY[it[0]] + FA[it[1]] * FY[it[1]] + FA[it[2]] * FY[it[2]] + FA[it[3]] * FY[it[3]];
          const double azl = FA[it[0]] * FZ[it[0]] + FA[it[1]] * FZ[it[1]] + FA[it[2]] * FZ[it[2]] + FA[it[3]] * FZ[it[3]];
          const double al = FA[it[0]] + FA[it[1]] + FA[it[2]] + FA[it[3]] + 1.E-20;
          const double axyzl = sqrt(axl * axl + ayl * ayl + azl * azl);
          const size_t n0 = CI(I, J, K);
          CX[n0] = axl / (axyzl + 1.E-20);
          CY[n0] = ayl / (axyzl + 1.E-20);
          CZ[n0] = azl / (axyzl + 1.E-20);
          if (axyzl < 1.E-20) CX[n0] = 1.;
          CA[n0] = al;
        }
  }
  for (int K = 1; K <= c->kmax; K++)
    for (int J = 1; J <= c->jmax; J++)
      for (int I = 1; I <= c->imax; I++) {
        const int i = 2 * I - 1, j = 2 * J - 1, k = 2 * K - 1;
        const size_t it[8] = {FI(i, j, k), FI(i, j + 1, k), FI(i, j, k + 1), FI(i, j + 1, k + 1),
                              FI(i + 1, j, k), FI(i + 1, j + 1, k), FI(i + 1, j, k + 1), FI(i + 1, j + 1, k + 1)};
        const double *V = f->a[FF_VOL];
        double vl = V[it[0]];
        for (int q = 1; q < 8; q++) vl = vl + V[it[q]];
        double cen[3];
        for (int d = 0; d < 3; d++) {
          const double *C = f->a[FF_XC + d];
          double s = V[it[0]] * C[it[0]];
          for (int q = 1; q < 8; q++) s = s + V[it[q]] * C[it[q]];
          cen[d] = s / vl;
        }
        const size_t n0 = CI(I, J, K);
        c->a[FF_VOL][n0] = vl;
        c->a[FF_XC][n0] = cen[0];
        c->a[FF_YC][n0] = cen[1];
        c->a[FF_ZC][n0] = cen[2];
        const double *DW = f->a[FF_DISTW];
        double ra = DW[it[0]];
        for (int q = 1; q < 8; q++) ra = ra + DW[it[q]];
        c->a[FF_DISTW][n0] = 0.125 * ra;
      }
  const double eps = 1.E-20;
  for (int K = 1; K <= c->kmax; K++)
    for (int J = 1; J <= c->jmax; J++)
      for (int I = 1; I <= c->imax; I++) {
        const size_t kk = CI(I, J, K);
        const double v = c->a[FF_VOL][kk];
        c->a[FF_D3][kk] = fmin(1.E4, (v + eps) / (c->a[FF_A3][kk] + c->a[FF_A3][kk + cl] + eps) * 2.);
        c->a[FF_D2][kk] = fmin(1.E4, (v + eps) / (c->a[FF_A2][kk] + c->a[FF_A2][kk + cs] + eps) * 2.);
        c->a[FF_D1][kk] = fmin(1.E4, (v + eps) / (c->a[FF_A1][kk] + c->a[FF_A1][kk + 1] + eps) * 2.);
      }
#undef FI
#undef CI
}

/* PICK_XYZ: the wall points of the solid patches (ICON(1) 8..10) of the
 * blocks, in block, patch and (second, first) in-face order; returns their
 * number, points in xyz[3 * n] (pass xyz = NULL to count). */
int orc_wall_points(orc_block **blk, int nblk, double *xyz) {
  int n = 0;
  for (int bi = 0; bi < nblk; bi++) {
    orc_block *b = blk[bi];
    dims_t d = dims_of(b);
    for (int ip = 0; ip < b->npatch; ip++) {
      const ff_patch *pa = &b->patch[ip];
      if (pa->ityp < 8 || pa->ityp > 10) continue;
      face_t fg = face_geom(&d, pa->iface);
      const long ls = (long)fg.idir * fg.s;
      for (int c = pa->r2a; c <= pa->r2b; c++)
        for (int a = pa->r1a; a <= pa->r1b; a++) {
          const size_t L = face_cell(&d, &fg, a, c);   /* first interior cell at the face */
          /* XC(KMI) + XC(KMA): the lower-index cell first */
          const size_t lo = ls > 0 ? L - ls : L, hi = ls > 0 ? L : L - ls;
          if (xyz) {
            xyz[3 * n + 0] = 0.5 * (b->a[FF_XC][lo] + b->a[FF_XC][hi]);
            xyz[3 * n + 1] = 0.5 * (b->a[FF_YC][lo] + b->a[FF_YC][hi]);
            xyz[3 * n + 2] = 0.5 * (b->a[FF_ZC][lo] + b->a[FF_ZC][hi]);
          }
          n++;
        }
    }
  }
  return n;
}

/* WALL_DIST: DISTW of every storage cell of b, the distance to the nearest
 * of the np wall points (squared distances compared, first minimum kept,
 * then the root). */
void orc_wall_distance(orc_block *b, const double *xyz, int np) {
  dims_t d = dims_of(b);
  const size_t nt = d.ntot;
  double *D = b->a[FF_DISTW];
  for (size_t i = 0; i < nt; i++) D[i] = 1.E+8;
  for (int ij = 0; ij < np; ij++)
    for (size_t i = 0; i < nt; i++) {
      const double dx = b->a[FF_XC][i] - xyz[3 * ij], dy = b->a[FF_YC][i] - xyz[3 * ij + 1];
      const double dz = b->a[FF_ZC][i] - xyz[3 * ij + 2];
      const double r = dx * dx + dy * dy + dz * dz;
      if (r < D[i]) D[i] = r;
    }
  for (size_t i = 0; i < nt; i++) D[i] = sqrt(D[i]);
}
#undef EX
