// noalloc.cu -- tmd_neighbor_list_noalloc: the full neighbor list built with
// no device allocation at all.
//
// Who needs it: host programs that give a library no device memory of its
// own, because they account for every byte through their own pool or have
// reserved the whole device up front (a cudaMalloc inside the library would
// then fail or break their accounting).  Those callers pass the positions and
// the output rows in memory they own; the cell-binning scratch below is the
// only other memory the call touches.  The call is synchronous: it waits for
// its stream and reads a status word back to the host, so it must be made
// outside any stream capture.
//
// The scratch is one static device array of 4 MiB that every GPU loading this
// library keeps until the process exits.  Its device address is looked up
// once per device (cudaGetSymbolAddress) with that device current; host code
// must never pass the array's name itself to a kernel, because on the host
// that name is only a stand-in, not a device address.  All calls share the
// array and it keeps the last call's contents, so everything that must start
// at zero is cleared on the stream first, and calls whose work overlaps on the
// GPU race with each other.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/tmd_b200.h"
#include "tmd_kernels.h"

namespace tmd {

// kernels of neighbor.cu, reused unchanged
__global__ void k_nb_zero(int ncell, int *cell_count, const int *flag);
__global__ void k_nb_scan(int ncell, const int *__restrict__ cell_count,
                          int *__restrict__ cell_start, int *__restrict__ cell_cursor,
                          const int *flag);
__global__ void k_nb_fill(int n, const int *__restrict__ cell_of, int *__restrict__ cell_cursor,
                          int *__restrict__ cell_atoms, const int *flag);
__global__ void k_nb_cellsort(int ncell, const int *__restrict__ cell_start,
                              int *__restrict__ cell_atoms, const int *flag);
__global__ void k_nb_build(int n, const double *__restrict__ x, BoxP box, BinP bin,
                           const int *__restrict__ cell_of, const int *__restrict__ cell_start,
                           const int *__restrict__ cell_atoms, double cutsq, int cap,
                           uint32_t *__restrict__ tmp, int *__restrict__ nraw, int *status,
                           int *maxneed, const int *flag);
__global__ void k_set_flag(int *flag);
size_t nb_build_smem(int threads);
void set_last_error(const std::string &msg);

namespace {

constexpr int kScratchInts = 1 << 20;  // 4 MiB
constexpr int kHead = 64;              // flag, status[2], maxneed, padding

static_assert(kHead + 2 * TMD_NOALLOC_MAX_ATOMS + 3 * TMD_NOALLOC_MAX_CELLS + 1 <= kScratchInts,
              "no-alloc scratch too small for its stated limits");

__device__ __align__(256) int g_scratch[kScratchInts];

std::mutex g_mu;
int *g_addr[64] = {nullptr};  // device address of g_scratch per device

// Bin atoms by fractional coordinate without moving them; an atom outside the
// cell is an error here (the caller's positions are read-only).  As in the
// system build (k_nb_bin), a periodic axis needs 0 <= f < 1 and a
// non-periodic one 0 <= f <= 1 (an atom on a shrink-wrapped upper face is in).
__global__ void k_bin_inplace(int n, const double *__restrict__ x, BoxP box, BinP bin,
                              int *__restrict__ cell_of, int *__restrict__ cell_count,
                              int *status) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double dx = x[3 * i] - box.lo[0], dy = x[3 * i + 1] - box.lo[1],
           dz = x[3 * i + 2] - box.lo[2];
    double f[3];
    f[2] = dz / box.zprd;
    f[1] = (dy - f[2] * box.yz) / box.yprd;
    f[0] = (dx - f[1] * box.xy - f[2] * box.xz) / box.xprd;
    int c3[3];
    for (int a = 0; a < 3; a++) {
      if (f[a] < 0.0 || (box.pbc[a] ? f[a] >= 1.0 : f[a] > 1.0)) atomicOr(status, kStatusOutside);
      int q = (int)floor(f[a] * bin.nb[a]);
      q = q < 0 ? 0 : (q >= bin.nb[a] ? bin.nb[a] - 1 : q);
      c3[a] = q;
    }
    int c = (c3[2] * bin.nb[1] + c3[1]) * bin.nb[0] + c3[0];
    cell_of[i] = c;
    atomicAdd(&cell_count[c], 1);
  }
}

int fail(int code, const std::string &m) {
  set_last_error(m);
  return code;
}

}  // namespace
}  // namespace tmd

using namespace tmd;

extern "C" int tmd_neighbor_list_noalloc(const double *x_dev, int n, const double box[9],
                                         const int pbc[3], double cut, int cap,
                                         int *counts_dev, unsigned int *rows_dev,
                                         void *stream) {
  if (!box || !pbc || n < 0 || (n > 0 && (!x_dev || !counts_dev || !rows_dev)))
    return fail(TMD_ERR_ARG, "null argument");
  if (n > TMD_NOALLOC_MAX_ATOMS)
    return fail(TMD_ERR_CAPACITY, "n = " + std::to_string(n) + " exceeds the no-alloc limit of " +
                                      std::to_string(TMD_NOALLOC_MAX_ATOMS) + " atoms");
  if (!(cut > 0) || cap < 1) return fail(TMD_ERR_ARG, "cut and cap must be positive");
  if (!(box[3] > 0 && box[4] > 0 && box[5] > 0)) return fail(TMD_ERR_ARG, "box lengths must be > 0");
  if (n == 0) return TMD_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return fail(TMD_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 64)
    return fail(TMD_ERR_ARG, "device index " + std::to_string(dev) +
                                 " exceeds the no-alloc address table (64 devices)");
  int *base = nullptr;
  {
    // set-up, once per device, with that device current
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess || !p)
        return fail(TMD_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_addr[dev] = static_cast<int *>(p);
    }
    base = g_addr[dev];
  }
  // cell geometry: bins slightly wider than cut/2, stencil covering cut
  BoxP b{};
  b.lo[0] = box[0]; b.lo[1] = box[1]; b.lo[2] = box[2];
  b.xprd = box[3]; b.yprd = box[4]; b.zprd = box[5];
  b.xy = box[6]; b.xz = box[7]; b.yz = box[8];
  for (int a = 0; a < 3; a++) b.pbc[a] = pbc[a] ? 1 : 0;
  b.triclinic = (b.xy != 0.0 || b.xz != 0.0 || b.yz != 0.0) ? 1 : 0;
  double av[3] = {b.xprd, 0, 0}, bv[3] = {b.xy, b.yprd, 0}, cv[3] = {b.xz, b.yz, b.zprd};
  auto cross = [](const double *u, const double *v, double *o) {
    o[0] = u[1] * v[2] - u[2] * v[1];
    o[1] = u[2] * v[0] - u[0] * v[2];
    o[2] = u[0] * v[1] - u[1] * v[0];
  };
  double V = b.xprd * b.yprd * b.zprd, t[3], w[3];
  cross(bv, cv, t); w[0] = V / std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  cross(cv, av, t); w[1] = V / std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  cross(av, bv, t); w[2] = V / std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  BinP bin{};
  long ncell = 1;
  for (int a = 0; a < 3; a++) {
    int nb = (int)std::floor(w[a] / (0.5 * cut * (1.0 + 1e-6)));
    nb = nb < 1 ? 1 : (nb > 1024 ? 1024 : nb);
    int ns = (int)std::ceil(cut * (1.0 + 1e-9) / (w[a] / nb));
    if (!b.pbc[a] && ns > nb) ns = nb;
    if (ns < 1) ns = 1;
    if (b.pbc[a] && (ns + nb - 1) / nb > kShiftR + 1)
      return fail(TMD_ERR_ARG, "periodic cell is too small for the cutoff");
    bin.nb[a] = nb;
    bin.ns[a] = ns;
    ncell *= nb;
  }
  while (ncell > TMD_NOALLOC_MAX_CELLS) {
    int a = (bin.nb[0] >= bin.nb[1] && bin.nb[0] >= bin.nb[2]) ? 0 : (bin.nb[1] >= bin.nb[2] ? 1 : 2);
    bin.nb[a] = (bin.nb[a] + 1) / 2;
    bin.ns[a] = (int)std::ceil(cut * (1.0 + 1e-9) / (w[a] / bin.nb[a]));
    if (!b.pbc[a] && bin.ns[a] > bin.nb[a]) bin.ns[a] = bin.nb[a];
    ncell = (long)bin.nb[0] * bin.nb[1] * bin.nb[2];
  }
  bin.ncell = (int)ncell;
  // carve the scratch array
  int *flag = base, *status = base + 1, *maxneed = base + 3;
  int *cell_of = base + kHead;
  int *cell_atoms = cell_of + TMD_NOALLOC_MAX_ATOMS;
  int *cell_count = cell_atoms + TMD_NOALLOC_MAX_ATOMS;
  int *cell_cursor = cell_count + TMD_NOALLOC_MAX_CELLS;
  int *cell_start = cell_cursor + TMD_NOALLOC_MAX_CELLS;  // ncell + 1 entries
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int T = 256, kMaxGrid = 148 * 8;
  auto grid = [&](long g) { return (int)(g < 1 ? 1 : (g > kMaxGrid ? kMaxGrid : g)); };
  // the array keeps the previous call's contents: clear what must start at zero
  e = cudaMemsetAsync(status, 0, 3 * sizeof(int), st);
  if (e != cudaSuccess) return fail(TMD_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  k_set_flag<<<1, 1, 0, st>>>(flag);
  k_nb_zero<<<grid((bin.ncell + T - 1) / T), T, 0, st>>>(bin.ncell, cell_count, flag);
  k_bin_inplace<<<grid((n + T - 1) / T), T, 0, st>>>(n, x_dev, b, bin, cell_of, cell_count, status);
  k_nb_scan<<<1, 1024, 0, st>>>(bin.ncell, cell_count, cell_start, cell_cursor, flag);
  k_nb_fill<<<grid((n + T - 1) / T), T, 0, st>>>(n, cell_of, cell_cursor, cell_atoms, flag);
  k_nb_cellsort<<<grid((bin.ncell + T - 1) / T), T, 0, st>>>(bin.ncell, cell_start, cell_atoms, flag);
  k_nb_build<<<grid(((long)n * 32 + T - 1) / T), T, nb_build_smem(T), st>>>(
      n, x_dev, b, bin, cell_of, cell_start, cell_atoms, cut * cut, cap,
      reinterpret_cast<uint32_t *>(rows_dev), counts_dev, status, maxneed, flag);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(TMD_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  int h[3] = {0, 0, 0};
  e = cudaMemcpyAsync(h, status, 3 * sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(TMD_ERR_CUDA, std::string("status read: ") + cudaGetErrorString(e));
  if (h[0] & kStatusOutside)
    return fail(TMD_ERR_ARG, "atom outside the cell (wrap positions into it first)");
  if (h[0] & kStatusLaunch) return fail(TMD_ERR_CUDA, "neighbor build launched without its shared memory");
  if (h[0] & kStatusShift) return fail(TMD_ERR_ARG, "periodic cell is too small for the cutoff");
  if (h[0] & kStatusOverflow)
    return fail(TMD_ERR_CAPACITY, "a row needs " + std::to_string(h[2]) + " entries, cap is " +
                                      std::to_string(cap));
  return TMD_OK;
}
