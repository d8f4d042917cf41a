// Block set-up on the device, the reference's construction (GRIVAL
// ns3c.f:5636 -> GRID1B gluebm.f:1265) in its order of operations, so that
// the result equals the host set-up (finflo_b200/grid.py, case.py) and the
// oracle's restatement to the bit:
//   - ghost nodes: the first layer as GRIDEX (gluebm.f:1029, REFXYZ 1175),
//     faces reflected x[-1] = 2 x[0] - x[1], edges and corners diagonally
//     x[-1,-1] = 2 x[0,0] - x[1,1]; further layers (the reference keeps
//     one) by mirror reflection along k, then j, then i;
//   - AREVC1 (gluebm.f:1586): per direction the face vectors from the
//     face's diagonals, areas and unit normals A*/(A + 1e-20) ((1, 0, 0)
//     for a vanishing face), the volume accumulated over the three passes
//     and the centre of the last pass; D1..D3 as D1D2D3 (2326);
//   - coarse levels: LUMPA1 (2194, area = sum of the four child areas,
//     normal = their area-weighted sum, normalised) and LUMPVS (2256);
//   - DISTW as DISTANCES (9136): the nearest of the wall points halfway
//     between the first interior and ghost cell centres of the solid
//     patches (PICK_XYZ 9452, WALL_DIST 9533), coarse interior cells the
//     mean of their children (LUMP_DIST 9562).
// Products, sums and quotients are written with the round-to-nearest
// intrinsics so that none is fused into a multiply-add.
#pragma once

struct GridDims {
  int ni, nj, nk;   // interior nodes per direction (IMAX+1, ...)
};

FF_DI double rm(double a, double b) { return __dmul_rn(a, b); }
FF_DI double ra(double a, double b) { return __dadd_rn(a, b); }
FF_DI double rs(double a, double b) { return __dsub_rn(a, b); }
FF_DI double rq(double a, double b) { return __ddiv_rn(a, b); }

// Node (i, j, k) of the extended node array (i in -ng .. ni+ng-1, ...) by
// mirror reflection in the order k, j, i.
FF_DI double node_k(const double* X, const GridDims& g, int i, int j, int k) {
  const size_t row = (size_t)(j)*g.ni + i, pl = (size_t)g.ni * g.nj;
  if (k < 0) return rs(2 * X[row], X[(size_t)(-k) * pl + row]);
  if (k >= g.nk) return rs(2 * X[(size_t)(g.nk - 1) * pl + row], X[(size_t)(2 * (g.nk - 1) - k) * pl + row]);
  return X[(size_t)k * pl + row];
}
FF_DI double node_jk(const double* X, const GridDims& g, int i, int j, int k) {
  if (j < 0) return rs(2 * node_k(X, g, i, 0, k), node_k(X, g, i, -j, k));
  if (j >= g.nj) return rs(2 * node_k(X, g, i, g.nj - 1, k), node_k(X, g, i, 2 * (g.nj - 1) - j, k));
  return node_k(X, g, i, j, k);
}
FF_DI double node_ijk(const double* X, const GridDims& g, int i, int j, int k) {
  if (i < 0) return rs(2 * node_jk(X, g, 0, j, k), node_jk(X, g, -i, j, k));
  if (i >= g.ni) return rs(2 * node_jk(X, g, g.ni - 1, j, k), node_jk(X, g, 2 * (g.ni - 1) - i, j, k));
  return node_jk(X, g, i, j, k);
}

// GRIDEX's first-layer edge and corner nodes (each index either the first
// ghost, -1 or n, or interior, and at least two of them ghosts): reflected
// diagonally through the first interior node; every other node by mirror.
FF_DI double node_ext(const double* X, const GridDims& g, int i, int j, int k) {
  const bool gi = i == -1 || i == g.ni, gj = j == -1 || j == g.nj, gk = k == -1 || k == g.nk;
  const bool ii = i >= 0 && i < g.ni, ij = j >= 0 && j < g.nj, ik = k >= 0 && k < g.nk;
  if ((int)gi + (int)gj + (int)gk >= 2 && (gi || ii) && (gj || ij) && (gk || ik)) {
    const int i1 = gi ? (i < 0 ? 0 : g.ni - 1) : i, i2 = gi ? (i < 0 ? 1 : g.ni - 2) : i;
    const int j1 = gj ? (j < 0 ? 0 : g.nj - 1) : j, j2 = gj ? (j < 0 ? 1 : g.nj - 2) : j;
    const int k1 = gk ? (k < 0 ? 0 : g.nk - 1) : k, k2 = gk ? (k < 0 ? 1 : g.nk - 2) : k;
    return rs(2 * X[((size_t)k1 * g.nj + j1) * g.ni + i1], X[((size_t)k2 * g.nj + j2) * g.ni + i2]);
  }
  return node_ijk(X, g, i, j, k);
}

// The extended nodes with ng ghost layers, (ni+2ng)(nj+2ng)(nk+2ng) per
// coordinate, i fastest.
__global__ void k_extend_nodes(const double* __restrict__ xyz, double* __restrict__ ext, GridDims g, int ng = 2) {
  const int ei = g.ni + 2 * ng, ej = g.nj + 2 * ng, ek = g.nk + 2 * ng;
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x, ne = (size_t)ei * ej * ek;
  if (n >= ne) return;
  const int i = (int)(n % ei) - ng, j = (int)((n / ei) % ej) - ng, k = (int)(n / ((size_t)ei * ej)) - ng;
  const size_t ni = (size_t)g.ni * g.nj * g.nk;
  for (int c = 0; c < 3; c++) ext[c * ne + n] = node_ext(xyz + c * ni, g, i, j, k);
}

struct V3 {
  double x, y, z;
};

// The extended node array's node (i, j, k) of a grid of ei x ej nodes per
// plane (ne nodes per coordinate).
struct ExtNodes {
  const double* e;
  size_t ne;
  int ei, ej;
  FF_DI V3 at(int i, int j, int k) const {
    const size_t n = ((size_t)k * ej + j) * ei + i;
    return V3{e[n], e[ne + n], e[2 * ne + n]};
  }
};

// AREVC1's face vector (AXX, AYY, AZZ) from the corners IT1..IT4.
FF_DI V3 face_vec(V3 p1, V3 p2, V3 p3, V3 p4) {
  return V3{rm(0.5, rs(rm(rs(p3.z, p1.z), rs(p4.y, p2.y)), rm(rs(p3.y, p1.y), rs(p4.z, p2.z)))),
            rm(0.5, rs(rm(rs(p3.x, p1.x), rs(p4.z, p2.z)), rm(rs(p3.z, p1.z), rs(p4.x, p2.x)))),
            rm(0.5, rs(rm(rs(p3.y, p1.y), rs(p4.x, p2.x)), rm(rs(p3.x, p1.x), rs(p4.y, p2.y))))};
}
FF_DI double vnorm(V3 s) { return __dsqrt_rn(ra(ra(rm(s.x, s.x), rm(s.y, s.y)), rm(s.z, s.z))); }

// One cell's AREVC1 results: low (IT0) and high (IT5) face vectors of each
// direction, the volume of the three passes and the centre of the last.
struct CellGeom {
  V3 lo[3], hi[3], cen;
  double vol;
};

// Cell whose low corner node is (i, j, k) of the extended array.
FF_DI CellGeom arevc1_cell(const ExtNodes& E, int i, int j, int k) {
  CellGeom g;
  double vol = 0.;
  for (int d = 0; d < 3; d++) {
    // the pass's (ISTR, JSTR, KSTR) = directions (d, d+1, d+2) cyclic;
    // corners IT1..IT8 at 0, KSTR, JSTR+KSTR, JSTR, ISTR, ISTR+KSTR,
    // ISTR+JSTR+KSTR, ISTR+JSTR
    int oa[3] = {0, 0, 0}, ob[3] = {0, 0, 0}, oc[3] = {0, 0, 0};
    oa[d] = 1;
    ob[(d + 1) % 3] = 1;
    oc[(d + 2) % 3] = 1;
    V3 p[8];
    p[0] = E.at(i, j, k);
    p[1] = E.at(i + oc[0], j + oc[1], k + oc[2]);
    p[2] = E.at(i + ob[0] + oc[0], j + ob[1] + oc[1], k + ob[2] + oc[2]);
    p[3] = E.at(i + ob[0], j + ob[1], k + ob[2]);
    p[4] = E.at(i + oa[0], j + oa[1], k + oa[2]);
    p[5] = E.at(i + oa[0] + oc[0], j + oa[1] + oc[1], k + oa[2] + oc[2]);
    p[6] = E.at(i + oa[0] + ob[0] + oc[0], j + oa[1] + ob[1] + oc[1], k + oa[2] + ob[2] + oc[2]);
    p[7] = E.at(i + oa[0] + ob[0], j + oa[1] + ob[1], k + oa[2] + ob[2]);
    V3 s = p[0];
    for (int q = 1; q < 8; q++) s = V3{ra(s.x, p[q].x), ra(s.y, p[q].y), ra(s.z, p[q].z)};
    const V3 xce{rm(0.125, s.x), rm(0.125, s.y), rm(0.125, s.z)};
    const V3 rd{rs(xce.x, rm(0.5, ra(p[0].x, p[1].x))), rs(xce.y, rm(0.5, ra(p[0].y, p[1].y))),
                rs(xce.z, rm(0.5, ra(p[0].z, p[1].z)))};
    const V3 rd2{rs(xce.x, rm(0.5, ra(p[6].x, p[7].x))), rs(xce.y, rm(0.5, ra(p[6].y, p[7].y))),
                 rs(xce.z, rm(0.5, ra(p[6].z, p[7].z)))};
    const V3 lo = face_vec(p[0], p[1], p[2], p[3]);
    const V3 hi = face_vec(p[4], p[5], p[6], p[7]);   // = -AXX2, the next cell's low face
    double v = d == 0 ? 0. : vol;
    v = ra(v, rm(rd.x, lo.x));
    v = ra(v, rm(rd.y, lo.y));
    v = ra(v, rm(rd.z, lo.z));
    v = ra(v, rm(rd2.x, -hi.x));
    v = ra(v, rm(rd2.y, -hi.y));
    v = ra(v, rm(rd2.z, -hi.z));
    vol = d == 2 ? rq(v, 3.0) : v;
    g.lo[d] = lo;
    g.hi[d] = hi;
    g.cen = xce;
  }
  g.vol = vol;
  return g;
}

// Area and unit normal of a face vector (AREVC1).
FF_DI void area_normal(V3 s, double& a, V3& n) {
  a = vnorm(s);
  const double den = ra(a, 1.0e-20);
  n = V3{rq(s.x, den), rq(s.y, den), rq(s.z, den)};
  if (a < 1.0e-20) n = V3{1., 0., 0.};
}

FF_DI double thickness(double vol, double alo, double ahi) {
  const double eps = 1e-20;
  return dmin(1e4, rm(rq(ra(vol, eps), ra(ra(alo, ahi), eps)), 2.0));
}

// Metrics of every storage cell (ghosts included) of the block from the
// extended nodes with 2 ghost layers.
__global__ void k_cell_metrics(DevBlock b, const double* __restrict__ ext) {
  const int is = b.imax + 4, js = b.jmax + 4, ks = b.kmax + 4;
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (size_t)b.ntot) return;
  const int i = (int)(n % is), j = (int)((n / is) % js), k = (int)(n / ((size_t)is * js));
  const ExtNodes E{ext, (size_t)(is + 1) * (js + 1) * (ks + 1), is + 1, js + 1};
  const CellGeom g = arevc1_cell(E, i, j, k);
  b.a[FF_XC][n] = g.cen.x;
  b.a[FF_YC][n] = g.cen.y;
  b.a[FF_ZC][n] = g.cen.z;
  b.a[FF_VOL][n] = g.vol;
  for (int d = 0; d < 3; d++) {
    double a, ah;
    V3 nr, nh;
    area_normal(g.lo[d], a, nr);
    area_normal(g.hi[d], ah, nh);
    b.a[FF_A1 + 4 * d][n] = a;
    b.a[FF_A1XA + 4 * d][n] = nr.x;
    b.a[FF_A1YA + 4 * d][n] = nr.y;
    b.a[FF_A1ZA + 4 * d][n] = nr.z;
    b.a[FF_D1 + d][n] = thickness(g.vol, a, ah);
  }
}

// Multigrid levels: per cell of a level with ng ghost layers ("raw",
// RW_N values a cell): the low and high face of each direction as area and
// unit normal, the volume and the centre; coarse levels lumped from the
// finer one level by level (ghost layers halved), each level then cropped
// to 2 ghost layers and finished (D1..D3) into its block.
struct RawDims {
  int ci, cj, ck;   // cells per direction including the ng ghost layers
  __host__ __device__ size_t n() const { return (size_t)ci * cj * ck; }
};
// RW_ALO + d: low-face area, RW_NLO + 3d + c: its normal; RW_AHI, RW_NHI the
// high face's; RW_VOL; RW_C + c
enum : int { RW_ALO = 0, RW_NLO = 3, RW_AHI = 12, RW_NHI = 15, RW_VOL = 24, RW_C = 25, RW_N = 28 };

__global__ void k_raw_metrics(const double* __restrict__ ext, double* __restrict__ raw, RawDims r) {
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x, nr = r.n();
  if (n >= nr) return;
  const int i = (int)(n % r.ci), j = (int)((n / r.ci) % r.cj), k = (int)(n / ((size_t)r.ci * r.cj));
  const ExtNodes E{ext, (size_t)(r.ci + 1) * (r.cj + 1) * (r.ck + 1), r.ci + 1, r.cj + 1};
  const CellGeom g = arevc1_cell(E, i, j, k);
  for (int d = 0; d < 3; d++) {
    double a, ah;
    V3 nr_, nh;
    area_normal(g.lo[d], a, nr_);
    area_normal(g.hi[d], ah, nh);
    raw[(size_t)(RW_ALO + d) * nr + n] = a;
    raw[(size_t)(RW_NLO + 3 * d + 0) * nr + n] = nr_.x;
    raw[(size_t)(RW_NLO + 3 * d + 1) * nr + n] = nr_.y;
    raw[(size_t)(RW_NLO + 3 * d + 2) * nr + n] = nr_.z;
    raw[(size_t)(RW_AHI + d) * nr + n] = ah;
    raw[(size_t)(RW_NHI + 3 * d + 0) * nr + n] = nh.x;
    raw[(size_t)(RW_NHI + 3 * d + 1) * nr + n] = nh.y;
    raw[(size_t)(RW_NHI + 3 * d + 2) * nr + n] = nh.z;
  }
  raw[(size_t)RW_VOL * nr + n] = g.vol;
  raw[(size_t)(RW_C + 0) * nr + n] = g.cen.x;
  raw[(size_t)(RW_C + 1) * nr + n] = g.cen.y;
  raw[(size_t)(RW_C + 2) * nr + n] = g.cen.z;
}

// One coarsening step: coarse cell (i, j, k) from the fine children
// (2i+a, 2j+b, 2k+c).  LUMPVS's child order: (i, j, k), (i, j+1, k),
// (i, j, k+1), (i, j+1, k+1), then the same at i+1; LUMPA1's four child
// faces of a face in direction d: offsets 0, +(d+1), +(d+2), +both.
__global__ void k_lump(const double* __restrict__ fr, RawDims f, double* __restrict__ cr, RawDims c) {
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x, nc = c.n(), nf = f.n();
  if (n >= nc) return;
  const int i = (int)(n % c.ci), j = (int)((n / c.ci) % c.cj), k = (int)(n / ((size_t)c.ci * c.cj));
  auto fidx = [&](int di, int dj, int dk) { return ((size_t)(2 * k + dk) * f.cj + (2 * j + dj)) * f.ci + (2 * i + di); };
  auto F = [&](int comp, size_t m) { return fr[(size_t)comp * nf + m]; };
  const int ord[8][3] = {{0, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0, 1, 1}, {1, 0, 0}, {1, 1, 0}, {1, 0, 1}, {1, 1, 1}};
  size_t m8[8];
  for (int q = 0; q < 8; q++) m8[q] = fidx(ord[q][0], ord[q][1], ord[q][2]);
  double vl = F(RW_VOL, m8[0]);
  for (int q = 1; q < 8; q++) vl = ra(vl, F(RW_VOL, m8[q]));
  cr[(size_t)RW_VOL * nc + n] = vl;
  for (int d = 0; d < 3; d++) {
    double s = rm(F(RW_VOL, m8[0]), F(RW_C + d, m8[0]));
    for (int q = 1; q < 8; q++) s = ra(s, rm(F(RW_VOL, m8[q]), F(RW_C + d, m8[q])));
    cr[(size_t)(RW_C + d) * nc + n] = rq(s, vl);
  }
  for (int d = 0; d < 3; d++) {
    const int bd = (d + 1) % 3, cd = (d + 2) % 3;
    for (int side = 0; side < 2; side++) {   // low faces from the children's low faces, high from high
      const int acomp = side ? RW_AHI : RW_ALO, ncomp = side ? RW_NHI : RW_NLO;
      size_t m4[4];
      for (int q = 0; q < 4; q++) {
        int o[3] = {0, 0, 0};
        o[d] = side;
        if (q & 1) o[bd] = 1;
        if (q & 2) o[cd] = 1;
        m4[q] = fidx(o[0], o[1], o[2]);
      }
      double v[3];
      for (int e = 0; e < 3; e++) {
        double t = rm(F(acomp + d, m4[0]), F(ncomp + 3 * d + e, m4[0]));
        for (int q = 1; q < 4; q++) t = ra(t, rm(F(acomp + d, m4[q]), F(ncomp + 3 * d + e, m4[q])));
        v[e] = t;
      }
      double al = F(acomp + d, m4[0]);
      for (int q = 1; q < 4; q++) al = ra(al, F(acomp + d, m4[q]));
      al = ra(al, 1.0e-20);
      const double axyzl = __dsqrt_rn(ra(ra(rm(v[0], v[0]), rm(v[1], v[1])), rm(v[2], v[2])));
      const double den = ra(axyzl, 1.0e-20);
      double nx = rq(v[0], den);
      const double ny = rq(v[1], den), nz = rq(v[2], den);
      if (axyzl < 1.0e-20) nx = 1.;
      cr[(size_t)(acomp + d) * nc + n] = al;
      cr[(size_t)(ncomp + 3 * d + 0) * nc + n] = nx;
      cr[(size_t)(ncomp + 3 * d + 1) * nc + n] = ny;
      cr[(size_t)(ncomp + 3 * d + 2) * nc + n] = nz;
    }
  }
}

// A level's metric slots from its raw arrays (ng ghost layers, cropped to 2).
__global__ void k_finish_metrics(DevBlock b, const double* __restrict__ raw, RawDims r, int ng) {
  const int is = b.imax + 4, js = b.jmax + 4;
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x, nr = r.n();
  if (n >= (size_t)b.ntot) return;
  const int i = (int)(n % is), j = (int)((n / is) % js), k = (int)(n / ((size_t)is * js));
  const int o = ng - 2;
  const size_t m = ((size_t)(k + o) * r.cj + (j + o)) * r.ci + (i + o);
  auto R = [&](int comp) { return raw[(size_t)comp * nr + m]; };
  const double vol = R(RW_VOL);
  b.a[FF_VOL][n] = vol;
  b.a[FF_XC][n] = R(RW_C);
  b.a[FF_YC][n] = R(RW_C + 1);
  b.a[FF_ZC][n] = R(RW_C + 2);
  for (int d = 0; d < 3; d++) {
    b.a[FF_A1 + 4 * d][n] = R(RW_ALO + d);
    b.a[FF_A1XA + 4 * d][n] = R(RW_NLO + 3 * d);
    b.a[FF_A1YA + 4 * d][n] = R(RW_NLO + 3 * d + 1);
    b.a[FF_A1ZA + 4 * d][n] = R(RW_NLO + 3 * d + 2);
    b.a[FF_D1 + d][n] = thickness(vol, R(RW_ALO + d), R(RW_AHI + d));
  }
}

// WALL_DIST: DISTW of every storage cell, the distance to the nearest of
// the wall points (3 values each), squared distances (dx^2 + dy^2) + dz^2
// compared starting from 1e8 (the least kept), then the root.  One thread
// per cell; the points staged through shared memory in tiles.
constexpr int WD_THREADS = 256, WD_TP = 512;
__global__ void __launch_bounds__(WD_THREADS) k_wall_distance(DevBlock b, const double* __restrict__ pts, int np) {
  __shared__ double sp[WD_TP * 3];
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = n < (size_t)b.ntot;
  const double x = ok ? b.a[FF_XC][n] : 0., y = ok ? b.a[FF_YC][n] : 0., z = ok ? b.a[FF_ZC][n] : 0.;
  double best = 1.e8;
  for (int t0 = 0; t0 < np; t0 += WD_TP) {
    const int nt = min(WD_TP, np - t0);
    __syncthreads();
    for (int q = threadIdx.x; q < nt * 3; q += blockDim.x) sp[q] = pts[(size_t)t0 * 3 + q];
    __syncthreads();
    if (ok)
      for (int t = 0; t < nt; t++) {
        const double dx = rs(x, sp[3 * t]), dy = rs(y, sp[3 * t + 1]), dz = rs(z, sp[3 * t + 2]);
        const double r = ra(ra(rm(dx, dx), rm(dy, dy)), rm(dz, dz));
        if (r < best) best = r;
      }
  }
  if (ok) b.a[FF_DISTW][n] = __dsqrt_rn(best);
}

// LUMP_DIST: the coarse block's interior cells, the mean of their eight
// children's DISTW (LUMPVS's order).
__global__ void k_lump_distw(DevBlock f, DevBlock c) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= c.imax * c.jmax * c.kmax) return;
  const int I = n % c.imax + 1, J = (n / c.imax) % c.jmax + 1, K = n / (c.imax * c.jmax) + 1;
  const int i = 2 * I - 1, j = 2 * J - 1, k = 2 * K - 1;
  const double* D = f.a[FF_DISTW];
  double s = D[ix(f, i, j, k)];
  s = ra(s, D[ix(f, i, j + 1, k)]);
  s = ra(s, D[ix(f, i, j, k + 1)]);
  s = ra(s, D[ix(f, i, j + 1, k + 1)]);
  s = ra(s, D[ix(f, i + 1, j, k)]);
  s = ra(s, D[ix(f, i + 1, j + 1, k)]);
  s = ra(s, D[ix(f, i + 1, j, k + 1)]);
  s = ra(s, D[ix(f, i + 1, j + 1, k + 1)]);
  c.a[FF_DISTW][ix(c, I, J, K)] = rm(0.125, s);
}
