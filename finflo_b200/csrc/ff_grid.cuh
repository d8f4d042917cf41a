// Block set-up on the device: the cell metrics from node coordinates and
// the wall distance DISTW.  This is the same construction as the project's
// host set-up (finflo_b200/grid.py compute_metrics, case.py wall_distance),
// moved to the GPU so that geometry sweeps do not wait on the host:
//   - ghost nodes by mirror extrapolation x[-m] = 2 x[0] - x[m], applied
//     along k, then j, then i (two layers per side);
//   - face vectors of every cell from the diagonals of the face,
//     0.5 (c11 - c00) x (c01 - c10), on the low side (A1/A2/A3 with unit
//     normals) and the high side;
//   - the volume from the divergence theorem over the six faces with the
//     face centroids, the cell centre as the mean of the 8 nodes, and the
//     thicknesses D1..D3 = min(1e4, (V + eps) / (A_low + A_high + eps) * 2)
//     of D1D2D3 (gluebm.f:2326);
//   - DISTW: the exact distance of every cell centre to the nearest point
//     of the wall triangles (each wall face split in two), brute force over
//     all triangles with the triangle list staged through shared memory.
#pragma once

struct GridDims {
  int ni, nj, nk;   // interior nodes per direction (IMAX+1, ...)
};

// Node (i, j, k) of the extended node array (i in -2 .. ni+1, ...) from the
// interior nodes X[(k * nj + j) * ni + i]: the reflections of the host
// construction, in its order (k first, then j, then i).
FF_DI double node_k(const double* X, const GridDims& g, int i, int j, int k) {
  const size_t row = (size_t)(j)*g.ni + i, pl = (size_t)g.ni * g.nj;
  if (k < 0) return 2 * X[row] - X[(size_t)(-k) * pl + row];
  if (k >= g.nk) return 2 * X[(size_t)(g.nk - 1) * pl + row] - X[(size_t)(2 * (g.nk - 1) - k) * pl + row];
  return X[(size_t)k * pl + row];
}
FF_DI double node_jk(const double* X, const GridDims& g, int i, int j, int k) {
  if (j < 0) return 2 * node_k(X, g, i, 0, k) - node_k(X, g, i, -j, k);
  if (j >= g.nj) return 2 * node_k(X, g, i, g.nj - 1, k) - node_k(X, g, i, 2 * (g.nj - 1) - j, k);
  return node_k(X, g, i, j, k);
}
FF_DI double node_ijk(const double* X, const GridDims& g, int i, int j, int k) {
  if (i < 0) return 2 * node_jk(X, g, 0, j, k) - node_jk(X, g, -i, j, k);
  if (i >= g.ni) return 2 * node_jk(X, g, g.ni - 1, j, k) - node_jk(X, g, 2 * (g.ni - 1) - i, j, k);
  return node_jk(X, g, i, j, k);
}

// The extended nodes with ng ghost layers, (ni+2ng)(nj+2ng)(nk+2ng) per
// coordinate, i fastest.
__global__ void k_extend_nodes(const double* __restrict__ xyz, double* __restrict__ ext, GridDims g, int ng = 2) {
  const int ei = g.ni + 2 * ng, ej = g.nj + 2 * ng, ek = g.nk + 2 * ng;
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x, ne = (size_t)ei * ej * ek;
  if (n >= ne) return;
  const int i = (int)(n % ei) - ng, j = (int)((n / ei) % ej) - ng, k = (int)(n / ((size_t)ei * ej)) - ng;
  const size_t ni = (size_t)g.ni * g.nj * g.nk;
  for (int c = 0; c < 3; c++) ext[c * ne + n] = node_ijk(xyz + c * ni, g, i, j, k);
}

struct V3 {
  double x, y, z;
};
FF_DI V3 v3(const double* ext, size_t ne, size_t n) { return V3{ext[n], ext[ne + n], ext[2 * ne + n]}; }
FF_DI V3 vsub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
FF_DI double vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// 0.5 (c11 - c00) x (c01 - c10)
FF_DI V3 face_vec(V3 c00, V3 c11, V3 c01, V3 c10) {
  V3 u = vsub(c11, c00), v = vsub(c01, c10);
  return V3{0.5 * (u.y * v.z - u.z * v.y), 0.5 * (u.z * v.x - u.x * v.z), 0.5 * (u.x * v.y - u.y * v.x)};
}
FF_DI V3 centroid4(V3 a, V3 b, V3 c, V3 d) {
  return V3{0.25 * (a.x + b.x + c.x + d.x), 0.25 * (a.y + b.y + c.y + d.y), 0.25 * (a.z + b.z + c.z + d.z)};
}

// Metrics of every storage cell (ghosts included) of the block.
__global__ void k_cell_metrics(DevBlock b, const double* __restrict__ ext) {
  const int is = b.imax + 4, js = b.jmax + 4, ks = b.kmax + 4;
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (size_t)b.ntot) return;
  const int i = (int)(n % is), j = (int)((n / is) % js), k = (int)(n / ((size_t)is * js));
  const int ei = is + 1, ej = js + 1;
  const size_t ne = (size_t)ei * ej * (ks + 1);
  auto P = [&](int dk, int dj, int di) { return v3(ext, ne, ((size_t)(k + dk) * ej + (j + dj)) * ei + (i + di)); };
  const V3 p000 = P(0, 0, 0), p001 = P(0, 0, 1), p010 = P(0, 1, 0), p011 = P(0, 1, 1);
  const V3 p100 = P(1, 0, 0), p101 = P(1, 0, 1), p110 = P(1, 1, 0), p111 = P(1, 1, 1);
  // faces on the low and high side of the cell (index order [k][j][i])
  const V3 si = face_vec(p000, p110, p100, p010), sih = face_vec(p001, p111, p101, p011);
  const V3 sj = face_vec(p000, p101, p001, p100), sjh = face_vec(p010, p111, p011, p110);
  const V3 sk = face_vec(p000, p011, p010, p001), skh = face_vec(p100, p111, p110, p101);
  const V3 ci = centroid4(p000, p100, p010, p110), cih = centroid4(p001, p101, p011, p111);
  const V3 cj = centroid4(p000, p100, p001, p101), cjh = centroid4(p010, p110, p011, p111);
  const V3 ck = centroid4(p000, p010, p001, p011), ckh = centroid4(p100, p110, p101, p111);
  const double vol = (vdot(cih, sih) - vdot(ci, si) + vdot(cjh, sjh) - vdot(cj, sj) + vdot(ckh, skh) - vdot(ck, sk)) / 3.0;
  const V3 c8[8] = {p000, p001, p010, p011, p100, p101, p110, p111};
  double cx = 0., cy = 0., cz = 0.;
  for (int q = 0; q < 8; q++) { cx = cx + c8[q].x; cy = cy + c8[q].y; cz = cz + c8[q].z; }
  b.a[FF_XC][n] = 0.125 * cx;
  b.a[FF_YC][n] = 0.125 * cy;
  b.a[FF_ZC][n] = 0.125 * cz;
  b.a[FF_VOL][n] = vol;
  const V3 lo[3] = {si, sj, sk}, hi[3] = {sih, sjh, skh};
  const double eps = 1e-20;
  for (int d = 0; d < 3; d++) {
    const double mag = sqrt(vdot(lo[d], lo[d])), safe = mag > 0. ? mag : 1.;
    b.a[FF_A1 + 4 * d][n] = mag;
    b.a[FF_A1XA + 4 * d][n] = lo[d].x / safe;
    b.a[FF_A1YA + 4 * d][n] = lo[d].y / safe;
    b.a[FF_A1ZA + 4 * d][n] = lo[d].z / safe;
    const double ah = sqrt(vdot(hi[d], hi[d]));
    b.a[FF_D1 + d][n] = dmin(1e4, (vol + eps) / (mag + ah + eps) * 2.0);
  }
}

// Multigrid levels (the host's mg_metrics): the fine level's face vectors,
// volumes and volume-weighted centres with NG = 2 * 2^(nlev-1) ghost
// layers ("raw" arrays, 22 values per cell: S1, S2, S3 low / high, VOL, C),
// lumped level by level (coarse volume = sum of the 8 children, coarse face
// vector = sum of the 4 child faces, centre volume-weighted, ghost layers
// halved), each level then cropped to 2 ghost layers and finished (areas,
// unit normals, D1..D3) into its block.
struct RawDims {
  int ci, cj, ck;   // cells per direction including the ng ghost layers
  __host__ __device__ size_t n() const { return (size_t)ci * cj * ck; }
};
enum : int { RW_S1 = 0, RW_S2 = 3, RW_S3 = 6, RW_S1H = 9, RW_S2H = 12, RW_S3H = 15, RW_VOL = 18, RW_C = 19, RW_N = 22 };

__global__ void k_raw_metrics(const double* __restrict__ ext, double* __restrict__ raw, RawDims r) {
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x, nr = r.n();
  if (n >= nr) return;
  const int i = (int)(n % r.ci), j = (int)((n / r.ci) % r.cj), k = (int)(n / ((size_t)r.ci * r.cj));
  const int ei = r.ci + 1, ej = r.cj + 1;
  const size_t ne = (size_t)ei * ej * (r.ck + 1);
  auto P = [&](int dk, int dj, int di) { return v3(ext, ne, ((size_t)(k + dk) * ej + (j + dj)) * ei + (i + di)); };
  const V3 p000 = P(0, 0, 0), p001 = P(0, 0, 1), p010 = P(0, 1, 0), p011 = P(0, 1, 1);
  const V3 p100 = P(1, 0, 0), p101 = P(1, 0, 1), p110 = P(1, 1, 0), p111 = P(1, 1, 1);
  const V3 f[6] = {face_vec(p000, p110, p100, p010), face_vec(p000, p101, p001, p100), face_vec(p000, p011, p010, p001),
                   face_vec(p001, p111, p101, p011), face_vec(p010, p111, p011, p110), face_vec(p100, p111, p110, p101)};
  const V3 ci = centroid4(p000, p100, p010, p110), cih = centroid4(p001, p101, p011, p111);
  const V3 cj = centroid4(p000, p100, p001, p101), cjh = centroid4(p010, p110, p011, p111);
  const V3 ck = centroid4(p000, p010, p001, p011), ckh = centroid4(p100, p110, p101, p111);
  const double vol = (vdot(cih, f[3]) - vdot(ci, f[0]) + vdot(cjh, f[4]) - vdot(cj, f[1]) + vdot(ckh, f[5]) - vdot(ck, f[2])) / 3.0;
  for (int q = 0; q < 6; q++) {
    raw[(size_t)(3 * q + 0) * nr + n] = f[q].x;
    raw[(size_t)(3 * q + 1) * nr + n] = f[q].y;
    raw[(size_t)(3 * q + 2) * nr + n] = f[q].z;
  }
  const V3 c8[8] = {p000, p001, p010, p011, p100, p101, p110, p111};
  double cx = 0., cy = 0., cz = 0.;
  for (int q = 0; q < 8; q++) { cx = cx + c8[q].x; cy = cy + c8[q].y; cz = cz + c8[q].z; }
  raw[(size_t)RW_VOL * nr + n] = vol;
  raw[(size_t)(RW_C + 0) * nr + n] = 0.125 * cx;
  raw[(size_t)(RW_C + 1) * nr + n] = 0.125 * cy;
  raw[(size_t)(RW_C + 2) * nr + n] = 0.125 * cz;
}

// One coarsening step: coarse cell (i, j, k) from the fine children
// (2i+a, 2j+b, 2k+c), in the host's summation order.
__global__ void k_lump(const double* __restrict__ fr, RawDims f, double* __restrict__ cr, RawDims c) {
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x, nc = c.n(), nf = f.n();
  if (n >= nc) return;
  const int i = (int)(n % c.ci), j = (int)((n / c.ci) % c.cj), k = (int)(n / ((size_t)c.ci * c.cj));
  auto F = [&](int comp, int dk, int dj, int di) {
    return fr[(size_t)comp * nf + ((size_t)(2 * k + dk) * f.cj + (2 * j + dj)) * f.ci + (2 * i + di)];
  };
  // the eight children in the order (k, j, i) = 000, 001, 010, 011, 100, ...
  auto csum = [&](auto val) {
    return val(0, 0, 0) + val(0, 0, 1) + val(0, 1, 0) + val(0, 1, 1) + val(1, 0, 0) + val(1, 0, 1) + val(1, 1, 0) +
           val(1, 1, 1);
  };
  const double vc = csum([&](int a, int bq, int cq) { return F(RW_VOL, a, bq, cq); });
  cr[(size_t)RW_VOL * nc + n] = vc;
  for (int d = 0; d < 3; d++)
    cr[(size_t)(RW_C + d) * nc + n] =
        csum([&](int a, int bq, int cq) { return F(RW_C + d, a, bq, cq) * F(RW_VOL, a, bq, cq); }) / vc;
  for (int d = 0; d < 3; d++) {
    // low faces: the four children on the low side of the direction
    cr[(size_t)(RW_S1 + d) * nc + n] = F(RW_S1 + d, 0, 0, 0) + F(RW_S1 + d, 0, 1, 0) + F(RW_S1 + d, 1, 0, 0) + F(RW_S1 + d, 1, 1, 0);
    cr[(size_t)(RW_S2 + d) * nc + n] = F(RW_S2 + d, 0, 0, 0) + F(RW_S2 + d, 0, 0, 1) + F(RW_S2 + d, 1, 0, 0) + F(RW_S2 + d, 1, 0, 1);
    cr[(size_t)(RW_S3 + d) * nc + n] = F(RW_S3 + d, 0, 0, 0) + F(RW_S3 + d, 0, 0, 1) + F(RW_S3 + d, 0, 1, 0) + F(RW_S3 + d, 0, 1, 1);
    cr[(size_t)(RW_S1H + d) * nc + n] = F(RW_S1H + d, 0, 0, 1) + F(RW_S1H + d, 0, 1, 1) + F(RW_S1H + d, 1, 0, 1) + F(RW_S1H + d, 1, 1, 1);
    cr[(size_t)(RW_S2H + d) * nc + n] = F(RW_S2H + d, 0, 1, 0) + F(RW_S2H + d, 0, 1, 1) + F(RW_S2H + d, 1, 1, 0) + F(RW_S2H + d, 1, 1, 1);
    cr[(size_t)(RW_S3H + d) * nc + n] = F(RW_S3H + d, 1, 0, 0) + F(RW_S3H + d, 1, 0, 1) + F(RW_S3H + d, 1, 1, 0) + F(RW_S3H + d, 1, 1, 1);
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
  const double vol = R(RW_VOL), eps = 1e-20;
  b.a[FF_VOL][n] = vol;
  b.a[FF_XC][n] = R(RW_C);
  b.a[FF_YC][n] = R(RW_C + 1);
  b.a[FF_ZC][n] = R(RW_C + 2);
  for (int d = 0; d < 3; d++) {
    const V3 lo{R(3 * d), R(3 * d + 1), R(3 * d + 2)}, hi{R(9 + 3 * d), R(10 + 3 * d), R(11 + 3 * d)};
    const double mag = sqrt(vdot(lo, lo)), safe = mag > 0. ? mag : 1.;
    b.a[FF_A1 + 4 * d][n] = mag;
    b.a[FF_A1XA + 4 * d][n] = lo.x / safe;
    b.a[FF_A1YA + 4 * d][n] = lo.y / safe;
    b.a[FF_A1ZA + 4 * d][n] = lo.z / safe;
    const double ah = sqrt(vdot(hi, hi));
    b.a[FF_D1 + d][n] = dmin(1e4, (vol + eps) / (mag + ah + eps) * 2.0);
  }
}

// Distance from p to the triangle (a, b, c): the closest point among the
// face interior, the three vertices and the three edges (the regions of
// the host construction).
FF_DI double tri_dist(V3 p, V3 a, V3 b, V3 c) {
  const V3 ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a), bp = vsub(p, b), cp = vsub(p, c);
  const double d1 = vdot(ab, ap), d2 = vdot(ac, ap), d3 = vdot(ab, bp), d4 = vdot(ac, bp);
  const double d5 = vdot(ab, cp), d6 = vdot(ac, cp);
  const double va = d3 * d6 - d5 * d4, vb = d5 * d2 - d1 * d6, vc = d1 * d4 - d3 * d2;
  auto dist = [&](V3 q) { V3 r = vsub(p, q); return sqrt(vdot(r, r)); };
  double best = dmin(dmin(dist(a), dist(b)), dist(c));
  const double sum = va + vb + vc;
  if (va >= 0. && vb >= 0. && vc >= 0.) {
    const double den = sum == 0. ? 1. : sum, v = vb / den, w = vc / den;
    best = dmin(best, dist(V3{a.x + ab.x * v + ac.x * w, a.y + ab.y * v + ac.y * w, a.z + ab.z * v + ac.z * w}));
  }
  auto clamp01 = [](double t) { return dmin(1., dmax(0., t)); };
  const double tab = clamp01(d1 - d3 != 0. ? d1 / (d1 - d3) : 0.);
  const double tac = clamp01(d2 - d6 != 0. ? d2 / (d2 - d6) : 0.);
  const double den_bc = (d4 - d3) + (d5 - d6);
  const double tbc = clamp01(den_bc != 0. ? (d4 - d3) / den_bc : 0.);
  const V3 bc = vsub(c, b);
  best = dmin(best, dist(V3{a.x + ab.x * tab, a.y + ab.y * tab, a.z + ab.z * tab}));
  best = dmin(best, dist(V3{a.x + ac.x * tac, a.y + ac.y * tac, a.z + ac.z * tac}));
  best = dmin(best, dist(V3{b.x + bc.x * tbc, b.y + bc.y * tbc, b.z + bc.z * tbc}));
  return best;
}

// DISTW of every storage cell: one thread per cell, the triangles (9
// values each: a, b, c) staged through shared memory in tiles of TT.
constexpr int WD_THREADS = 256, WD_TT = 256;
__global__ void __launch_bounds__(WD_THREADS) k_wall_distance(DevBlock b, const double* __restrict__ tri, int ntri) {
  __shared__ double st[WD_TT * 9];
  const size_t n = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = n < (size_t)b.ntot;
  const V3 p = ok ? V3{b.a[FF_XC][n], b.a[FF_YC][n], b.a[FF_ZC][n]} : V3{0., 0., 0.};
  double best = 1e300;
  for (int t0 = 0; t0 < ntri; t0 += WD_TT) {
    const int nt = min(WD_TT, ntri - t0);
    __syncthreads();
    for (int q = threadIdx.x; q < nt * 9; q += blockDim.x) st[q] = tri[(size_t)t0 * 9 + q];
    __syncthreads();
    if (ok)
      for (int t = 0; t < nt; t++) {
        const double* s = st + 9 * t;
        best = dmin(best, tri_dist(p, V3{s[0], s[1], s[2]}, V3{s[3], s[4], s[5]}, V3{s[6], s[7], s[8]}));
      }
  }
  if (ok) b.a[FF_DISTW][n] = ntri > 0 ? best : 1.0e3;
}

// DISTW with pruning.  The triangles come in tiles of WD_TT consecutive
// triangles (the wall list is ordered along the wall surface, so a tile is
// a compact patch) with their bounding boxes; a CTA takes an 8 x 8 x 4
// brick of cells, orders the tiles by the distance between their box and
// the brick's box, and stops at the first tile farther than the largest
// distance its cells have found so far.  Same result as k_wall_distance.
constexpr int WD_BI = 8, WD_BJ = 8, WD_BK = 4;
__global__ void __launch_bounds__(WD_THREADS) k_wall_distance_pruned(DevBlock b, const double* __restrict__ tri, int ntri,
                                                                     const double* __restrict__ tbox, int ntile) {
  extern __shared__ double wd_smem[];
  double* st = wd_smem;                         // [WD_TT * 9] one tile of triangles
  double* lb = st + WD_TT * 9;                  // [ntile] squared box distances
  int* order = reinterpret_cast<int*>(lb + ntile);   // [ntile]
  __shared__ double red[2][WD_THREADS / 32][3];
  __shared__ double cta_best2;
  const int is = b.imax + 4, js = b.jmax + 4, ks = b.kmax + 4;
  const int nbi = (is + WD_BI - 1) / WD_BI, nbj = (js + WD_BJ - 1) / WD_BJ;
  const int bi = blockIdx.x % nbi, bj = (blockIdx.x / nbi) % nbj, bk = blockIdx.x / (nbi * nbj);
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int i = bi * WD_BI + t % WD_BI, j = bj * WD_BJ + (t / WD_BI) % WD_BJ, k = bk * WD_BK + t / (WD_BI * WD_BJ);
  const bool ok = i < is && j < js && k < ks;
  const size_t n = ((size_t)k * js + j) * is + i;
  const V3 p = ok ? V3{b.a[FF_XC][n], b.a[FF_YC][n], b.a[FF_ZC][n]} : V3{0., 0., 0.};
  // the brick's box
  double lo[3] = {ok ? p.x : 1e300, ok ? p.y : 1e300, ok ? p.z : 1e300};
  double hi[3] = {ok ? p.x : -1e300, ok ? p.y : -1e300, ok ? p.z : -1e300};
  for (int c = 0; c < 3; c++)
    for (int o = 16; o > 0; o >>= 1) {
      lo[c] = dmin(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
      hi[c] = dmax(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
    }
  if (lane == 0)
    for (int c = 0; c < 3; c++) { red[0][wid][c] = lo[c]; red[1][wid][c] = hi[c]; }
  __syncthreads();
  for (int c = 0; c < 3; c++) {
    lo[c] = red[0][0][c]; hi[c] = red[1][0][c];
    for (int w = 1; w < WD_THREADS / 32; w++) { lo[c] = dmin(lo[c], red[0][w][c]); hi[c] = dmax(hi[c], red[1][w][c]); }
  }
  // squared distance between the brick's box and each tile's box
  for (int q = t; q < ntile; q += WD_THREADS) {
    double d2 = 0.;
    for (int c = 0; c < 3; c++) {
      const double gap = dmax(0., dmax(tbox[q * 6 + c] - hi[c], lo[c] - tbox[q * 6 + 3 + c]));
      d2 += gap * gap;
    }
    lb[q] = d2;
  }
  __syncthreads();
  // tiles in increasing box distance (rank sort; ties by index)
  for (int q = t; q < ntile; q += WD_THREADS) {
    int r = 0;
    const double v = lb[q];
    for (int u = 0; u < ntile; u++) r += (lb[u] < v) || (lb[u] == v && u < q);
    order[r] = q;
  }
  if (t == 0) cta_best2 = 1e300;
  __syncthreads();
  double best = 1e300;
  for (int r = 0; r < ntile; r++) {
    const int q = order[r];
    if (lb[q] > cta_best2) break;   // every later tile is farther than every cell's best
    const int t0 = q * WD_TT, nt = min(WD_TT, ntri - t0);
    for (int e = t; e < nt * 9; e += WD_THREADS) st[e] = tri[(size_t)t0 * 9 + e];
    __syncthreads();
    if (ok)
      for (int u = 0; u < nt; u++) {
        const double* s = st + 9 * u;
        best = dmin(best, tri_dist(p, V3{s[0], s[1], s[2]}, V3{s[3], s[4], s[5]}, V3{s[6], s[7], s[8]}));
      }
    // the brick's largest best distance (squared), for the stop test
    double m = ok ? best * best : 0.;
    for (int o = 16; o > 0; o >>= 1) m = dmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) red[0][wid][0] = m;
    __syncthreads();
    if (t == 0) {
      double mm = red[0][0][0];
      for (int w = 1; w < WD_THREADS / 32; w++) mm = dmax(mm, red[0][w][0]);
      cta_best2 = mm;
    }
    __syncthreads();
  }
  if (ok) b.a[FF_DISTW][n] = best;
}

inline size_t wd_pruned_smem(int ntile) { return (size_t)WD_TT * 9 * sizeof(double) + (size_t)ntile * (sizeof(double) + sizeof(int)); }
