// impz_static.cu -- the charge deposit without any device allocation.
//
// Some callers may not allocate device memory while they run: a host code
// whose GPU memory is all handed out by its own pool or arena (it would be
// bypassed, and the allocation can fail in the middle of a run), or a timed
// loop that cannot take the device-wide synchronization cudaMalloc and
// cudaFree imply.  impz_deposit_static serves them: the caller passes the
// particles and the output grid in device memory it owns, and the only
// scratch, the int64 fixed-point accumulator of the deposit, is a fixed
// array in this library's device image (IMPZ_STATIC_MAX_CELLS nodes, 4 MiB),
// held by every GPU that loads the library until the process exits.
//
// The arithmetic is that of the bunch deposit (k_deposit): the z->t frame
// conversion and loss test of conv1st, the CIC cell and weights of
// deposit_BeamBunch, the same fixed-point quanta with the remainder on the
// largest corner, with the quantum chosen from this call's n; for a bunch
// created with the same n and the same geometry the grid equals
// impz_deposit's bit for bit.  Sums go straight to the accumulator with
// 64-bit atomics (integer adds: the result does not depend on their order).
//
// Compiled with --fmad=false like the other FP64 kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "../../include/impz_b200.h"
#include "impz_host.h"
#include "impz_launch.h"

#define IMPZ_NS noalloc
#include "impz_particle.cuh"

namespace impz {
namespace noalloc {

// The deposit's accumulator, one int64 per grid node.  Every call on a device
// uses the same array, and it keeps the last call's sums: each call clears
// the nodes it uses before depositing.
static __device__ __align__(256) unsigned long long g_static_rho[IMPZ_STATIC_MAX_CELLS];

struct StaticDepositArgs {
  const double* col[6];  // x, px, y, py, ph, pt (Pts1 rows 1..6), device
  long long n;
  double gam, rad, xl, scale;
  int nx, ny, nz, fixbits;
  Geom g;
};

__global__ void k_static_clear(unsigned long long* acc, long long G) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < G;
       i += (long long)gridDim.x * blockDim.x)
    acc[i] = 0ull;
}

// conv1st z->t frame and loss test, deposit_BeamBunch cell, weights and the
// int64 quanta of k_deposit; 64-bit global reductions per corner.  A
// particle outside the caller's box (far outside included: cell_inside does
// not overflow) is skipped, as deposit_BeamBunch skips it.
__global__ void __launch_bounds__(256) k_static_deposit(StaticDepositArgs a,
                                                        unsigned long long* acc) {
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long long P = (long long)nx * ny;
  const double scale = ldexp(1.0, a.fixbits);
  const unsigned long long unit = 1ull << a.fixbits;
  const double magic = 6755399441055744.0;  // 1.5 * 2^52: round to nearest even
  const long long magic_bits = 0x4338000000000000ll;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
       i += (long long)gridDim.x * blockDim.x) {
    Particle p;
    p.x = a.col[0][i]; p.px = a.col[1][i]; p.y = a.col[2][i];
    p.py = a.col[3][i]; p.ph = a.col[4][i]; p.pt = a.col[5][i];
    const TFrame t = to_tframe(p, a.gam, a.rad, a.xl);
    if (t.lost) continue;
    const Cell c = cic_cell(t.xt, t.yt, t.zt, a.g);
    if (!cell_inside(c, nx, ny, nz)) continue;
    const double ab = c.ab, cd = c.cd, ef = c.ef;
    // corner order of deposit_BeamBunch (BeamBunch.f90:3749-3763)
    const double w8[8] = {ab * cd * ef,
                          ab * (1.0 - cd) * ef,
                          ab * (1.0 - cd) * (1.0 - ef),
                          ab * cd * (1.0 - ef),
                          (1.0 - ab) * cd * (1.0 - ef),
                          (1.0 - ab) * (1.0 - cd) * (1.0 - ef),
                          (1.0 - ab) * (1.0 - cd) * ef,
                          (1.0 - ab) * cd * ef};
    int big = 0;
    double wbig = w8[0];
#pragma unroll
    for (int k = 1; k < 8; k++)
      if (w8[k] > wbig) { wbig = w8[k]; big = k; }
    unsigned long long qv[8];
    unsigned long long sum7 = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const double sh = __dadd_rn(__dmul_rn(w8[k], scale), magic);
      qv[k] = (k == big) ? 0ull : (unsigned long long)(__double_as_longlong(sh) - magic_bits);
      sum7 += qv[k];
    }
#pragma unroll
    for (int k = 0; k < 8; k++)
      if (k == big) qv[k] = unit - sum7;
    const long long cc = lin_cell(c, nx, ny);
    const long long node[8] = {cc, cc + nx, cc + nx + P, cc + P, cc + 1 + P, cc + 1 + nx + P,
                               cc + 1 + nx, cc + 1};
#pragma unroll
    for (int k = 0; k < 8; k++) atomicAdd(acc + node[k], qv[k]);
  }
}

// chgdens = sum of quanta * weight * 2^-fixbits, as impz_deposit forms it
__global__ void k_static_finish(const unsigned long long* acc, long long G, double scale,
                                double* out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < G;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (double)(long long)acc[i] * scale;
}

// Device address of g_static_rho and the device's SM count, looked up once
// per device.  In host code the name g_static_rho is only a host-side
// stand-in for the symbol, so the kernels are always given this address,
// never the name.  The cached address belongs to the device's current
// context: a cudaDeviceReset would invalidate it, so the library must not be
// used across one.
constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
unsigned long long* g_addr[kMaxDevices] = {nullptr};
int g_sms[kMaxDevices] = {0};

int scratch_address(unsigned long long** out, int* sms) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return report_cuda_error(e, "impz_deposit_static: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return IMPZ_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> g(g_addr_mu);
  if (!g_addr[dev]) {
    int n_sm = 0;
    e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return report_cuda_error(e, "impz_deposit_static: SM count");
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_rho);
    if (e != cudaSuccess) return report_cuda_error(e, "impz_deposit_static: cudaGetSymbolAddress");
    g_addr[dev] = (unsigned long long*)p;
    g_sms[dev] = n_sm > 0 ? n_sm : 1;
  }
  *out = g_addr[dev];
  *sms = g_sms[dev];
  return IMPZ_OK;
}

}  // namespace noalloc
}  // namespace impz

extern "C" int impz_deposit_static(const double* x, const double* px, const double* y,
                                   const double* py, const double* ph, const double* pt,
                                   long long n, double gam, double piperad, double piperad2,
                                   double freq, double weight, const double range[6], int nx,
                                   int ny, int nz, double* chgdens, void* stream) {
  using namespace impz;
  using namespace impz::noalloc;
  if (nx < 2 || ny < 2 || nz < 2 || n < 0 || !range || !chgdens || !(freq > 0)) return IMPZ_ERR_ARG;
  const long long G = (long long)nx * ny * nz;
  if (G > IMPZ_STATIC_MAX_CELLS) return IMPZ_ERR_LIMIT;
  if (n > 0 && (!x || !px || !y || !py || !ph || !pt)) return IMPZ_ERR_ARG;
  unsigned long long* acc = nullptr;
  int sms = 1;
  int r = scratch_address(&acc, &sms);
  if (r) return r;
  StaticDepositArgs a;
  const double* cols[6] = {x, px, y, py, ph, pt};
  for (int c = 0; c < 6; c++) a.col[c] = cols[c];
  a.n = n;
  a.gam = gam;
  a.rad = (piperad + piperad2) / 2;       // as impz_sc_prepare forms it
  a.xl = make_phys(freq).Scxl;
  a.nx = nx; a.ny = ny; a.nz = nz;
  int l = 0;
  while ((1ll << l) < n + 1) l++;
  a.fixbits = std::min(40, 62 - l);       // the bunch's rule, l = ceil(log2(n + 1))
  a.scale = weight * std::ldexp(1.0, -a.fixbits);
  // update_CompDom's mesh sizes for this box, as the device computes them
  const int mesh[3] = {nx, ny, nz};
  for (int k = 0; k < 3; k++) {
    a.g.ptrange[2 * k] = a.g.ptrange[2 * k + 1] = 0.0;
    a.g.range[2 * k] = range[2 * k];
    a.g.range[2 * k + 1] = range[2 * k + 1];
    a.g.h[k] = (range[2 * k + 1] - range[2 * k]) / (double)(mesh[k] - 1);
    a.g.hi[k] = 1.0 / a.g.h[k];
    if (!(a.g.h[k] > 0.0) || !std::isfinite(a.g.hi[k])) return IMPZ_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int gclear = (int)std::min<long long>((G + 255) / 256, (long long)sms * 8);
  k_static_clear<<<gclear, 256, 0, s>>>(acc, G);
  if (n > 0) {
    const int gdep = (int)std::min<long long>((n + 255) / 256, (long long)sms * 16);
    k_static_deposit<<<gdep, 256, 0, s>>>(a, acc);
  }
  k_static_finish<<<gclear, 256, 0, s>>>(acc, G, a.scale, chgdens);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return report_cuda_error(e, "impz_deposit_static: launch");
  return IMPZ_OK;
}
