// LU-SGS sweep as a pipelined tile wavefront (one thread-block cluster).
//
// The (j,k) lines of a block are cut into tiles of 16 x TK lines, one tile
// per CTA of the cluster (at most 16 tiles).  Thread (lj, lk) owns the
// i-line (J, K) and at hyperplane m handles the cell I = m - J - K.  As in
// the reference (PREDGS imps4.f:345 / CORRGS imps4.f:76) every solved cell
// produces the split-Jacobian products for its three downstream neighbours:
//   * the i product stays in the thread's registers (its own line);
//   * j and k products of lines inside the tile go through shared memory
//     (double-buffered by plane parity, two __syncthreads per plane);
//   * products of the tile's edge lines are written straight into the
//     downstream tile's shared memory (DSMEM), into a ring of RING slots.
// Tiles are synchronised point to point, not by a cluster-wide barrier: a
// producer arrives (release, cluster scope) on the consumer's "full"
// mbarrier of the slot once its CTA has written it; the consumer arrives on
// the producer's "empty" mbarrier once its CTA has read it, which frees the
// slot for reuse RING planes later.  Each CTA therefore only waits for its
// upstream tiles' previous plane, and the tiles run as a pipeline.  The
// triangular system is the reference's (incl. PREDGS's dropped i+1 coupling
// in row J = JMAX), so the result equals the line and hyperplane sweeps up
// to rounding.
//
// Every wait is bounded: on time-out the error word is set, the remaining
// waits give up at once, and every CTA still reaches the final cluster
// barrier, so no CTA exits while another may still access its shared memory.
// With STAGE each thread's next-plane sweep data is copied by cp.async into
// its own shared-memory slots while the current plane finishes.
#pragma once

constexpr int PTJ = 16;       // lines of a tile along j (consecutive in the sweep layout)
constexpr int PRING = 8;      // ring slots of the edge products

struct PipeGeom {
  int ntj, ntk;     // tiles along j and k (ntj * ntk <= 16 = the cluster)
};

// Shared memory of k_lusgs_pipe<..., TK, STAGE>.
__host__ __device__ inline size_t pipe_smem_bytes(int nv, int tk, size_t elem, bool stage) {
  const size_t thr = (size_t)PTJ * tk;
  size_t b = 2 * 2 * (size_t)nv * thr * elem;                    // in-tile j and k products, 2 planes
  b += (size_t)PRING * nv * (tk + PTJ) * elem;                   // rings: j edge (tk lines), k edge (16)
  if (stage) b += (size_t)LSTAGE * thr * elem;                    // staged sweep data
  return b + 2 * PRING * 8 + 64;                                  // full / empty mbarriers
}

FF_DI uint32_t pipe_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

FF_DI void pipe_mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Arrive on the mbarrier at the same offset in the shared memory of CTA
// `rank` of the cluster (release at cluster scope: the data this CTA wrote
// before is visible to whoever completes the wait).
FF_DI void pipe_remote_arrive(uint32_t local_bar, int rank) {
  uint32_t ra;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(ra) : "r"(local_bar), "r"(rank));
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(ra) : "memory");
}

FF_DI bool pipe_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait; gives up at once when the error word is already set.
FF_DI void pipe_wait(uint32_t bar, uint32_t parity, int* err) {
  for (long it = 0; it < (1L << 24); it++) {
    if (pipe_try_wait(bar, parity)) return;
    if ((it & 255) == 0 && *((volatile int*)err)) return;
  }
  atomicExch(err, 2);
}

template <typename CT, int NV, int TK, bool STAGE>
__global__ void __launch_bounds__(PTJ* TK) k_lusgs_pipe(DevBlock b, const CT* __restrict__ sw, CT* dwp, int upper,
                                                          PipeGeom pg, int* err) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  constexpr int NT = PTJ * TK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  CT* pj = reinterpret_cast<CT*>(smem_raw);      // [2][NV][NT] j products of in-tile lines
  CT* pk = pj + 2 * NV * NT;                      // [2][NV][NT] k products
  CT* rj = pk + 2 * NV * NT;                      // [RING][NV][TK]  j products from the upstream j tile
  CT* rk = rj + PRING * NV * TK;                  // [RING][NV][PTJ] k products from the upstream k tile
  CT* my = rk + PRING * NV * PTJ + threadIdx.x;   // stage [LSTAGE][NT]
  unsigned char* bars_raw = smem_raw + pipe_smem_bytes(NV, TK, sizeof(CT), STAGE) - 2 * PRING * 8 - 64;
  uint64_t* full = reinterpret_cast<uint64_t*>(bars_raw);
  uint64_t* empty = full + PRING;
  const int IMAX = b.imax, JMAX = b.jmax, KMAX = b.kmax;
  const int W = IMAX + JMAX - 1;
  const size_t ns = sw_size(IMAX, JMAX, KMAX);
  const int rank = (int)cluster.block_rank();
  const int tid = threadIdx.x, lj = tid % PTJ, lk = tid / PTJ;
  const int tj = rank % pg.ntj, tk = rank / pg.ntj;
  const int J = tj * PTJ + lj + 1, K = tk * TK + lk + 1;
  const bool own = J <= JMAX && K <= KMAX;
  const int nplanes = IMAX + JMAX + KMAX - 2;
  // neighbour tiles in sweep order
  const int up_j = upper ? (tj < pg.ntj - 1 ? rank + 1 : -1) : (tj > 0 ? rank - 1 : -1);
  const int up_k = upper ? (tk < pg.ntk - 1 ? rank + pg.ntj : -1) : (tk > 0 ? rank - pg.ntj : -1);
  const int dn_j = upper ? (tj > 0 ? rank - 1 : -1) : (tj < pg.ntj - 1 ? rank + 1 : -1);
  const int dn_k = upper ? (tk > 0 ? rank - pg.ntj : -1) : (tk < pg.ntk - 1 ? rank + pg.ntj : -1);
  const int n_up = (up_j >= 0) + (up_k >= 0), n_dn = (dn_j >= 0) + (dn_k >= 0);
  // this line's upstream neighbours: in the tile, or at the tile edge
  const bool hj = upper ? (J < JMAX) : (J > 1);
  const bool hk = upper ? (K < KMAX) : (K > 1);
  const bool edge_in_j = upper ? (lj == PTJ - 1) : (lj == 0);    // the j neighbour is in the upstream tile
  const bool edge_in_k = upper ? (lk == TK - 1) : (lk == 0);
  const bool edge_out_j = upper ? (lj == 0) : (lj == PTJ - 1);   // this line feeds the downstream tile
  const bool edge_out_k = upper ? (lk == 0) : (lk == TK - 1);
  const int nb_j = upper ? tid + 1 : tid - 1, nb_k = upper ? tid + PTJ : tid - PTJ;
  CT* rj_dn = dn_j >= 0 ? cluster.map_shared_rank(rj, dn_j) : rj;
  CT* rk_dn = dn_k >= 0 ? cluster.map_shared_rank(rk, dn_k) : rk;
  if (tid == 0) {
    for (int q = 0; q < PRING; q++) {
      pipe_mbar_init(pipe_smem_u32(full + q), (uint32_t)max(n_up, 1));
      pipe_mbar_init(pipe_smem_u32(empty + q), (uint32_t)max(n_dn, 1));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  auto plane_cell = [&](int s, int& I, size_t& S) {
    const int m = upper ? IMAX + JMAX + KMAX - s : 3 + s;
    I = m - J - K;
    S = ((size_t)(K - 1) * W + (m - K - 2)) * JMAX + (J - 1);
    return own && I >= 1 && I <= IMAX;
  };
  if (STAGE) {
    int I;
    size_t S;
    if (plane_cell(0, I, S)) lines_stage<CT, NV>(my, NT, sw, dwp, ns, S, upper);
  }
  cluster.sync();   // barriers initialised everywhere
  CT yd[NV];
#pragma unroll
  for (int v = 0; v < NV; v++) yd[v] = CT(0);
  for (int s = 0; s < nplanes; s++) {
    const int slot = s % PRING, pslot = (s + PRING - 1) % PRING;
    // the upstream tiles' products of plane s-1 (warp 0), and a free slot s
    // downstream (warp 1), waited for in parallel
    if (tid == 0 && s >= 1 && n_up > 0) pipe_wait(pipe_smem_u32(full + pslot), (uint32_t)(((s - 1) / PRING) & 1), err);
    if (tid == 32 && s >= PRING && n_dn > 0)
      pipe_wait(pipe_smem_u32(empty + slot), (uint32_t)(((s / PRING) - 1) & 1), err);
    __syncthreads();
    const int bin = (s & 1) ^ 1, bout = s & 1;   // in-tile products: read plane s-1, write plane s
    int I;
    size_t S;
    if (plane_cell(s, I, S)) {
      if (STAGE) cp_async_wait_all();
      auto cd_ = [&](int c) -> CT {
        if (STAGE) return my[c * NT];
        return c < SW_N ? __ldg(sw + c * ns + S) : dwp[(c - SW_N) * ns + S];
      };
      // PREDGS drops the i+1 coupling of row J = JMAX unless bit 2 of upper
      // (predgs_full) asks for it; PRKEGS does not drop it
      const bool hy = upper ? (I < IMAX && (NV == 7 || J < JMAX || (upper & 2))) : (I > 1);
      CT bd[NV], ck[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) {
        bd[v] = !hj ? CT(0) : (edge_in_j ? rj[(pslot * NV + v) * TK + lk] : pj[(bin * NV + v) * NT + nb_j]);
        ck[v] = !hk ? CT(0) : (edge_in_k ? rk[(pslot * NV + v) * PTJ + lj] : pk[(bin * NV + v) * NT + nb_k]);
        if (!hy) yd[v] = CT(0);
      }
      const CT dt1 = cd_(SW_DT1), vol = cd_(SW_VOL), fd = upper ? CT(1) : cd_(SW_FD);
      const CT a1 = cd_(SW_A1), a2 = cd_(SW_A2), a3 = cd_(SW_A3);
      const CT scinv = cd_(SW_SCINV), scinp = cd_(SW_SCINP);
      CT res[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) {
        CT cdv = cd_(SW_N + v) * fd;
        CT x = upper ? (-dt1 * a3 * ck[v] + vol * cdv) : (dt1 * a3 * ck[v] + vol * cdv);
        x = upper ? x - dt1 * (a1 * yd[v] + a2 * bd[v]) : x + dt1 * (a1 * yd[v] + a2 * bd[v]);
        res[v] = x * (v == 4 ? scinp : scinv);
        dwp[v * ns + S] = res[v];
      }
      CT sc[5];
#pragma unroll
      for (int c = 0; c < (NV == 7 ? 5 : 3); c++) sc[c] = cd_(SW_SC + c);
      const CT ro = NV == 7 ? cd_(SW_RO) : CT(0);
#pragma unroll
      for (int d = 0; d < 3; d++) {
        CT f[3], l[3], out[NV];
#pragma unroll
        for (int c = 0; c < 3; c++) f[c] = cd_(SW_F + 3 * d + c);
#pragma unroll
        for (int e = 0; e < 3; e++) l[e] = cd_(SW_L + 3 * d + e);
        nb_product_pre<CT, NV>(out, res, f, sc, ro, l[0], l[1], l[2]);
        if (d == 0) {
#pragma unroll
          for (int v = 0; v < NV; v++) yd[v] = out[v];
        } else if (d == 1) {
#pragma unroll
          for (int v = 0; v < NV; v++) {
            pj[(bout * NV + v) * NT + tid] = out[v];
            if (edge_out_j && dn_j >= 0) rj_dn[(slot * NV + v) * TK + lk] = out[v];
          }
        } else {
#pragma unroll
          for (int v = 0; v < NV; v++) {
            pk[(bout * NV + v) * NT + tid] = out[v];
            if (edge_out_k && dn_k >= 0) rk_dn[(slot * NV + v) * PTJ + lj] = out[v];
          }
        }
      }
    }
    if (STAGE && s + 1 < nplanes) {   // this thread's next-plane data, in flight across the barriers
      int I2;
      size_t S2;
      if (plane_cell(s + 1, I2, S2)) lines_stage<CT, NV>(my, NT, sw, dwp, ns, S2, upper);
    }
    __syncthreads();
    // slot s is written in the downstream tiles; slot s-1 here is read: one
    // release-arrive per neighbour, each from its own warp, so they overlap
    if ((tid & 31) == 0) {
      const int w = tid >> 5;
      if (w == 0 && dn_j >= 0) pipe_remote_arrive(pipe_smem_u32(full + slot), dn_j);
      if (w == 1 && dn_k >= 0) pipe_remote_arrive(pipe_smem_u32(full + slot), dn_k);
      if (w == 2 && s >= 1 && up_j >= 0) pipe_remote_arrive(pipe_smem_u32(empty + pslot), up_j);
      if (w == 3 && s >= 1 && up_k >= 0) pipe_remote_arrive(pipe_smem_u32(empty + pslot), up_k);
    }
  }
  cluster.sync();   // no CTA leaves while another may still reach its shared memory
}
