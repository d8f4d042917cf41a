// Allocation-free variant of the LU-SGS implicit stage (ff_imps_noalloc).
//
// Who needs it: callers that must not allocate device memory while they run.
// Examples are a host code that has already handed all device memory to its
// own pool allocator and forbids further cudaMalloc calls, an application
// that runs under a hard per-process memory cap fixed at start-up, or a code
// path that is not allowed to synchronise the device (cudaMalloc and cudaFree
// can synchronise).  Such a caller owns the block's arrays itself and passes
// their device addresses in; this entry point then runs TIME3, LOCDT, COPR,
// PREDGS, DIAGGS, CORRGS and DRO/CP (the same kernels as ff_imps) without
// creating a context and without calling cudaMalloc, cudaFree or any
// allocating library routine.
//
// The LU-SGS coefficients and the grid-barrier words that ff_imps keeps in
// per-context buffers live here in one file-scope __device__ array of fixed
// size.  Every GPU that loads the library holds that array (about 10 MB)
// until the process exits.  Its maximum block size is FF_NOALLOC_MAX_NTOT
// cells including the two ghost layers; larger blocks are rejected with
// FF_ERR_SIZE before any work is queued.
//
// This file is compiled as part of ff_gpu.cu's translation unit (included at
// its end), so it shares the kernels with the context-based entry points.

#define FF_NOALLOC_BAR_WORDS 64   // doubles reserved for the barrier words

// Scratch: NCOEF coefficient arrays of FF_NOALLOC_MAX_NTOT doubles, then the
// barrier words {count, generation, error, sticky error}.  The sticky word
// collects the time-outs of every call since the caller last asked for the
// status (level = 0).  In host code the name below is
// only a host-side stand-in for the array; its device address comes from
// cudaGetSymbolAddress in noalloc_setup().
static __device__ __align__(256) double ff_noalloc_scratch[ff::NCOEF * (size_t)FF_NOALLOC_MAX_NTOT + FF_NOALLOC_BAR_WORDS];

namespace {

struct NoallocDevice {
  int ready;
  double* scratch;   // device address of ff_noalloc_scratch on this device
  int sm_count;
  int coop_per_sm;
};
constexpr int kMaxDevices = 64;
NoallocDevice g_noalloc[kMaxDevices];

// Once per device, with that device current: resolve the device address of
// the scratch array and the cooperative occupancy of the sweep kernel.
int noalloc_setup(int dev) {
  NoallocDevice& d = g_noalloc[dev];
  if (d.ready) return 0;
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, ff_noalloc_scratch) != cudaSuccess || !p) return FF_ERR_CUDA;
  int sms = 0, per_sm = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return FF_ERR_CUDA;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (ff::k_lusgs_sweep_basic<double, 5>), 256, 0) != cudaSuccess ||
      per_sm < 1)
    return FF_ERR_CUDA;
  d.scratch = (double*)p;
  d.sm_count = sms;
  d.coop_per_sm = per_sm;
  d.ready = 1;
  return 0;
}

// Start of a call, in stream order: fold the previous call's time-out flag
// into the sticky word, then clear the barrier words for this call's sweeps.
__global__ void k_noalloc_begin(unsigned* bar) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    bar[3] |= bar[2];
    bar[0] = 0u;
    bar[1] = 0u;
    bar[2] = 0u;
  }
}

// level = 0: wait for `stream`, then report and clear the time-out flags of
// the calls queued on it so far.
int noalloc_status(cudaStream_t st) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FF_ERR_CUDA;
  int rc = noalloc_setup(dev);
  if (rc) return rc;
  unsigned* bar = (unsigned*)(g_noalloc[dev].scratch + ff::NCOEF * (size_t)FF_NOALLOC_MAX_NTOT);
  unsigned w[2] = {0u, 0u};
  if (cudaMemcpyAsync(w, bar + 2, sizeof(w), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return FF_ERR_CUDA;
  if (!(w[0] | w[1])) return 0;
  if (cudaMemsetAsync(bar + 2, 0, sizeof(w), st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
    return FF_ERR_CUDA;
  return FF_ERR_TIMEOUT;
}

}  // namespace

extern "C" int ff_imps_noalloc(int imax, int jmax, int kmax, const ff_params* prm,
                               double* const* slots, int level, void* stream) {
  if (level == 0) return noalloc_status((cudaStream_t)stream);
  if (imax < 2 || jmax < 2 || kmax < 1 || !prm || !slots || (level != 1 && level != 2 && level != 3))
    return FF_ERR_ARG;
  if (prm->iturb >= 3) return FF_ERR_ARG;   // five-equation (laminar) implicit stage only
  // the LU-SGS sweeps here run in FP64 only; the DDADI branch honours FP32
  if (prm->lusgs_fp32 && !prm->ddadi) return FF_ERR_ARG;
  long ntot = (long)(imax + 4) * (jmax + 4) * (kmax + 4);
  if (ntot > FF_NOALLOC_MAX_NTOT) return FF_ERR_SIZE;
  static const int needed[] = {FF_RO, FF_E, FF_P, FF_U, FF_V, FF_W, FF_C, FF_VIS, FF_CP, FF_DRDP, FF_DRDH,
                               FF_VIST, FF_DRO, FF_DM, FF_DN, FF_DW, FF_DE, FF_DTL, FF_A1, FF_A1XA,
                               FF_A1YA, FF_A1ZA, FF_A2, FF_A2XA, FF_A2YA, FF_A2ZA, FF_A3, FF_A3XA,
                               FF_A3YA, FF_A3ZA, FF_VOL};
  for (int s : needed)
    if (!slots[s]) return FF_ERR_ARG;
  // the five increment arrays must be back to back (ntot apart), as the
  // sweep kernel addresses them from DRO
  for (int v = 1; v < 5; v++)
    if (slots[FF_DRO + v] != slots[FF_DRO] + (size_t)v * ntot) return FF_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FF_ERR_CUDA;
  int rc = noalloc_setup(dev);
  if (rc) return rc;
  const NoallocDevice& nd = g_noalloc[dev];
  cudaStream_t st = (cudaStream_t)stream;

  DevBlock db{};
  db.imax = imax; db.jmax = jmax; db.kmax = kmax;
  db.is = imax + 4; db.il = (imax + 4) * (jmax + 4); db.ntot = (int)ntot;
  db.npatch = 0; db.patch = nullptr;
  for (int s = 0; s < FF_NSLOTS; s++) db.a[s] = slots[s];

  double* coef = nd.scratch;
  unsigned* bar = (unsigned*)(nd.scratch + ff::NCOEF * (size_t)FF_NOALLOC_MAX_NTOT);
  int* err = (int*)(bar + 2);
  // every call shares the array: the barrier words must start at zero, and
  // an earlier call's time-out moves to the sticky word
  k_noalloc_begin<<<1, 32, 0, st>>>(bar);

  int ncell = imax * jmax * kmax;
  ff_params p = *prm;
  double cfl = level == 1 ? p.cfl : p.cfll;
  k_time3_copr<<<(ncell + 127) / 128, 128, 0, st>>>(db, p, cfl);
  if (p.ddadi) {   // DDADI (LUSGS=0): k, i, j line sweeps, no scratch
    const int dirs[3] = {3, 1, 2};
    for (int d : dirs) {
      const int n = d == 1 ? imax : (d == 2 ? jmax : kmax);
      if (n <= 1) continue;
      if (p.lusgs_fp32) ddadi_pc_launch<float, 5>(st, db, p, d, ncell / n, 1);
      else ddadi_pc_launch<double, 5>(st, db, p, d, ncell / n, 1);
    }
    k_fin_divide<<<(int)((ntot + 255) / 256), 256, 0, st>>>(db, 0);
    if (cudaGetLastError() != cudaSuccess) return FF_ERR_CUDA;
    return 0;
  }
  long widest = (long)jmax * kmax;
  int nb = (int)min((long)nd.coop_per_sm * nd.sm_count, max(1L, (widest + 255) / 256));
  double* dw = slots[FF_DRO];
  for (int upper = 1; upper >= 0; upper--) {
    k_lusgs_coef<double><<<(ncell + 127) / 128, 128, 0, st>>>(db, p, coef, upper);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nb);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int uflag = upper && p.predgs_full ? (upper | 2) : upper;
    if (cudaLaunchKernelEx(&cfg, k_lusgs_sweep_basic<double, 5>, db, (const double*)coef, dw, uflag, bar, err) != cudaSuccess)
      return FF_ERR_CUDA;
  }
  k_fin_divide<<<(int)((ntot + 255) / 256), 256, 0, st>>>(db, 0);
  if (cudaGetLastError() != cudaSuccess) return FF_ERR_CUDA;
  return 0;
}
