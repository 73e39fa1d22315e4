// Launch wrappers of the open-boundary Poisson solve (impz_poisson.cuh).
// Compiled with --fmad=false: the Green-function corners and differences
// keep the reference's rounding; the FFT passes lose nothing by it.
#include "impz_launch.h"
#include "impz_poisson.cuh"

namespace impz {

static int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) l++;
  return l;
}

static PoissonDims dims_of(const PoissonBuffers& b) {
  PoissonDims d;
  d.nx = b.nx; d.ny = b.ny; d.nz = b.nz;
  d.lx = ilog2(2 * b.nx); d.ly = ilog2(2 * b.ny); d.lz = ilog2(2 * b.nz);
  return d;
}

template <typename T>
static size_t xy_smem(int nx, int ny) {
  return sizeof(typename Cplx<T>::type) *
         ((size_t)(ny / 2) * line_pitch(2 * nx) + (size_t)(nx + 1) * line_pitch(2 * ny) + nx +
          ny);
}
#ifndef IMPZ_XY_PARTS
#define IMPZ_XY_PARTS 1
#endif
#ifndef IMPZ_XY_THREADS
#define IMPZ_XY_THREADS 512
#endif
template <typename T>
static size_t xyf_smem(int nx, int ny, int parts) {
  return sizeof(typename Cplx<T>::type) *
         ((size_t)(ny / 2) * line_pitch(2 * nx) +
          (size_t)((nx + 1 + parts - 1) / parts) * line_pitch(2 * ny) + nx + ny);
}

// largest dynamic shared memory one block may opt into on this device
static size_t smem_optin() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return (size_t)v;
}
template <typename T>
static size_t z_smem(int nz, int tkx) {
  return sizeof(typename Cplx<T>::type) * ((size_t)tkx * line_pitch(2 * nz) + nz);
}
// z lines per block: 8, fewer when long lines do not fit (FP32 at
// 64x64x128: 31.5 us per launch with 8 lines, 40.3 with 16, 32.0 with 4)
template <typename T>
static int ztile(int nz) {
  int t = 8;
  while (t > 1 && z_smem<T>(nz, t) > smem_optin()) t /= 2;
  return t;
}
static const int kDctLines = 16;
template <typename T>
static size_t dct_smem(int n, int lines) {
  return sizeof(typename Cplx<T>::type) * ((size_t)(lines / 2) * line_pitch(2 * n) + n);
}
template <typename T>
static int dct_lines(int n) {
  int t = kDctLines;
  while (t > 2 && dct_smem<T>(n, t) > smem_optin()) t /= 2;
  return t;
}

// k_green_xy: the line pairs of the longer of its two transforms, both
// twiddle sets and the (nx+1)(ny+1) plane
template <typename T>
static size_t green_xy_smem(int nx, int ny) {
  const size_t lx = (size_t)((ny + 2) / 2) * line_pitch(2 * nx);
  const size_t ly = (size_t)((nx + 2) / 2) * line_pitch(2 * ny);
  return sizeof(typename Cplx<T>::type) * ((lx > ly ? lx : ly) + nx + ny) +
         sizeof(T) * (size_t)(nx + 1) * (ny + 1);
}

// true when every Poisson kernel fits the device's shared memory
template <typename T>
bool poisson_fits(int nx, int ny, int nz) {
  const size_t lim = smem_optin();
  return xy_smem<T>(nx, ny) <= lim && xyf_smem<T>(nx, ny, 1) <= lim && z_smem<T>(nz, 1) <= lim &&
         dct_smem<T>(nz, 2) <= lim && green_xy_smem<T>(nx, ny) <= lim;
}

template <typename K>
static cudaError_t allow_smem(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

static int grid_for(long long work, int block) {
  long long g = (work + block - 1) / block;
  if (g > 148 * 16) g = 148 * 16;
  return (int)(g < 1 ? 1 : g);
}

// One DCT-I pass of length n+1 over ninner x nouter lines, as many lines
// per block as fit in shared memory (16 for the usual sizes).
template <typename TI, typename T, int TL>
static cudaError_t dct_pass_t(const TI* in, T* out, int n, long long es, long long ls, int ninner,
                              long long os, int nouter, double scale,
                              const typename Cplx<T>::type* tw, cudaStream_t s) {
  auto kern = k_dct1<TI, T, T, TL>;
  const size_t sm = dct_smem<T>(n, TL);
  cudaError_t e = allow_smem(kern, sm);
  if (e != cudaSuccess) return e;
  dim3 g((ninner + TL - 1) / TL, nouter);
  kern<<<g, 256, sm, s>>>(in, out, ilog2(2 * n), es, ls, ninner, os, scale, tw);
  return cudaGetLastError();
}
template <typename TI, typename T>
static cudaError_t dct_pass(const TI* in, T* out, int n, long long es, long long ls, int ninner,
                            long long os, int nouter, double scale,
                            const typename Cplx<T>::type* tw, cudaStream_t s) {
  switch (dct_lines<T>(n)) {
    case 16: return dct_pass_t<TI, T, 16>(in, out, n, es, ls, ninner, os, nouter, scale, tw, s);
    case 8: return dct_pass_t<TI, T, 8>(in, out, n, es, ls, ninner, os, nouter, scale, tw, s);
    case 4: return dct_pass_t<TI, T, 4>(in, out, n, es, ls, ninner, os, nouter, scale, tw, s);
    default: return dct_pass_t<TI, T, 2>(in, out, n, es, ls, ninner, os, nouter, scale, tw, s);
  }
}

template <typename T, int TKX>
static cudaError_t zconv_t(const PoissonBuffers& b, const PoissonDims& d, cudaStream_t s) {
  typedef typename Cplx<T>::type C;
  const size_t sz = z_smem<T>(b.nz, TKX);
  cudaError_t e = allow_smem(k_fft_z_conv<T, TKX>, sz);
  if (e != cudaSuccess) return e;
  dim3 gz((b.nx + 1 + TKX - 1) / TKX, 2 * b.ny);
  return launch_pdl(k_fft_z_conv<T, TKX>, gz, dim3(256), sz, s, d, (C*)b.spec,
                    (const T*)b.ghat, (const C*)b.twz);
}

// The Green function: FP64 corners, then per z plane the FP64 8-corner
// difference (it cancels catastrophically, Field.f90:420-428) and the DCT-I
// along x and y in the convolution's type T (FP64 in the plain form, FP32 in
// the FP32-convolution form), then the DCT-I along z.
template <typename T>
cudaError_t launch_green(const PoissonBuffers& b, cudaStream_t s) {
  typedef typename Cplx<T>::type C;
  const int nx = b.nx, ny = b.ny, nz = b.nz;
  const long long nc = (long long)(nx + 2) * (ny + 2) * (nz + 2);
  k_igf_corners<<<grid_for(nc, 256), 256, 0, s>>>(nx, ny, nz, b.st, b.F);
  const size_t sm = green_xy_smem<T>(nx, ny);
  cudaError_t e = allow_smem(k_green_xy<T>, sm);
  if (e != cudaSuccess) return e;
  k_green_xy<T><<<nz + 1, IMPZ_GREEN_THREADS, sm, s>>>(nx, ny, ilog2(2 * nx), ilog2(2 * ny), b.F,
                                                       (T*)b.ghat, (const C*)b.twx,
                                                       (const C*)b.twy);
  const long long gx = nx + 1, gxy = (long long)(nx + 1) * (ny + 1);
  const double scale = 1.0 / ((double)(2 * nx) * (double)(2 * ny) * (double)(2 * nz));
  T* work = (T*)b.ghat;
  // along z: lines i (inner) x j (outer, stride gx); points stride gxy
  if ((e = dct_pass<T, T>(work, work, nz, gxy, 1, nx + 1, gx, ny + 1, scale, (const C*)b.twz,
                          s)) != cudaSuccess)
    return e;
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_conv_forward(const PoissonBuffers& b, cudaStream_t s) {
  typedef typename Cplx<T>::type C;
  const PoissonDims d = dims_of(b);
  cudaError_t e;
  const size_t sm = xyf_smem<T>(b.nx, b.ny, IMPZ_XY_PARTS);
  if ((e = allow_smem(k_fft_xy_fwd<T, IMPZ_XY_PARTS>, sm)) != cudaSuccess) return e;
  return launch_pdl(k_fft_xy_fwd<T, IMPZ_XY_PARTS>, dim3(IMPZ_XY_PARTS, b.nz),
                    dim3(IMPZ_XY_THREADS), sm, s, d, (const unsigned long long*)b.rho, b.qscale,
                    (C*)b.spec, (const C*)b.twx, (const C*)b.twy);
}

template <typename T>
cudaError_t launch_conv_rest(const PoissonBuffers& b, cudaStream_t s) {
  typedef typename Cplx<T>::type C;
  const PoissonDims d = dims_of(b);
  cudaError_t e;
  const size_t sxy = xy_smem<T>(b.nx, b.ny);
  if ((e = allow_smem(k_fft_xy_inv<T>, sxy)) != cudaSuccess) return e;
  int zt = ztile<T>(b.nz);
  if (b.ztile > 0 && b.ztile < zt && (b.ztile & (b.ztile - 1)) == 0) zt = b.ztile;
  switch (zt) {
    case 16: e = zconv_t<T, 16>(b, d, s); break;
    case 8: e = zconv_t<T, 8>(b, d, s); break;
    case 4: e = zconv_t<T, 4>(b, d, s); break;
    case 2: e = zconv_t<T, 2>(b, d, s); break;
    default: e = zconv_t<T, 1>(b, d, s); break;
  }
  if (e != cudaSuccess) return e;
  return launch_pdl(k_fft_xy_inv<T>, dim3(b.nz), dim3(512), sxy, s, d, (const C*)b.spec,
                    (T*)b.phi, (const C*)b.twx, (const C*)b.twy);
}

template <typename T>
cudaError_t launch_convolve(const PoissonBuffers& b, cudaStream_t s) {
  cudaError_t e = launch_conv_forward<T>(b, s);
  if (e != cudaSuccess) return e;
  return launch_conv_rest<T>(b, s);
}

template <typename T>
cudaError_t launch_efield(const PoissonBuffers& b, cudaStream_t s) {
  const long long G = (long long)b.nx * b.ny * b.nz;
  return launch_pdl(k_efield<T>, dim3(grid_for(G, 256)), dim3(256), 0, s, b.nx, b.ny, b.nz,
                    (const T*)b.phi, (const DevState*)b.st, (T*)b.efield, b.rho, b.wake,
                    b.wake_line);
}

// ---- groups: the same solve for several bunches of one grid size, one
// launch per kernel (PoissonMember array `mem` in device memory)
static int group_grid(long long work, int block, int nmem) {
  long long g = (work + block - 1) / block;
  const long long cap = (148 * 16 + nmem - 1) / nmem;
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
}

template <typename TI, typename T, int TL>
static cudaError_t dct_group_t(int axis, int n, long long es, long long ls, int ninner,
                               long long os, int nouter, double scale,
                               const PoissonMember* mem, int nmem, cudaStream_t s) {
  auto kern = k_dct1_group<TI, T, T, TL>;
  const size_t sm = dct_smem<T>(n, TL);
  cudaError_t e = allow_smem(kern, sm);
  if (e != cudaSuccess) return e;
  dim3 g((ninner + TL - 1) / TL, nouter, nmem);
  kern<<<g, 256, sm, s>>>(axis, ilog2(2 * n), es, ls, ninner, os, scale, mem);
  return cudaGetLastError();
}
template <typename TI, typename T>
static cudaError_t dct_group(int axis, int n, long long es, long long ls, int ninner, long long os,
                             int nouter, double scale, const PoissonMember* mem, int nmem,
                             cudaStream_t s) {
  switch (dct_lines<T>(n)) {
    case 16: return dct_group_t<TI, T, 16>(axis, n, es, ls, ninner, os, nouter, scale, mem, nmem, s);
    case 8: return dct_group_t<TI, T, 8>(axis, n, es, ls, ninner, os, nouter, scale, mem, nmem, s);
    case 4: return dct_group_t<TI, T, 4>(axis, n, es, ls, ninner, os, nouter, scale, mem, nmem, s);
    default: return dct_group_t<TI, T, 2>(axis, n, es, ls, ninner, os, nouter, scale, mem, nmem, s);
  }
}

template <typename T>
cudaError_t launch_green_group(int nx, int ny, int nz, const PoissonMember* mem, int nmem,
                               cudaStream_t s) {
  const long long nc = (long long)(nx + 2) * (ny + 2) * (nz + 2);
  k_igf_corners_group<<<dim3(group_grid(nc, 256, nmem), nmem), 256, 0, s>>>(nx, ny, nz, mem);
  const size_t sm = green_xy_smem<T>(nx, ny);
  cudaError_t e = allow_smem(k_green_xy_group<T>, sm);
  if (e != cudaSuccess) return e;
  k_green_xy_group<T><<<dim3(nz + 1, nmem), IMPZ_GREEN_THREADS, sm, s>>>(
      nx, ny, ilog2(2 * nx), ilog2(2 * ny), mem);
  const long long gx = nx + 1, gxy = (long long)(nx + 1) * (ny + 1);
  const double scale = 1.0 / ((double)(2 * nx) * (double)(2 * ny) * (double)(2 * nz));
  if ((e = dct_group<T, T>(2, nz, gxy, 1, nx + 1, gx, ny + 1, scale, mem, nmem, s)) !=
      cudaSuccess)
    return e;
  return cudaGetLastError();
}

template <typename T, int TKX>
static cudaError_t zconv_group_t(const PoissonDims& d, const PoissonMember* mem, int nmem,
                                 cudaStream_t s) {
  const size_t sz = z_smem<T>(d.nz, TKX);
  cudaError_t e = allow_smem(k_fft_z_conv_group<T, TKX>, sz);
  if (e != cudaSuccess) return e;
  dim3 gz((d.nx + 1 + TKX - 1) / TKX, 2 * d.ny, nmem);
  return launch_pdl(k_fft_z_conv_group<T, TKX>, gz, dim3(256), sz, s, d, mem);
}

template <typename T>
cudaError_t launch_conv_group_forward(int nx, int ny, int nz, const PoissonMember* mem, int nmem,
                                      cudaStream_t s) {
  PoissonBuffers pb;
  pb.nx = nx; pb.ny = ny; pb.nz = nz;
  const PoissonDims d = dims_of(pb);
  cudaError_t e;
  const size_t sm = xyf_smem<T>(nx, ny, IMPZ_XY_PARTS);
  if ((e = allow_smem(k_fft_xy_fwd_group<T, IMPZ_XY_PARTS>, sm)) != cudaSuccess) return e;
  return launch_pdl(k_fft_xy_fwd_group<T, IMPZ_XY_PARTS>, dim3(IMPZ_XY_PARTS, nz, nmem),
                    dim3(IMPZ_XY_THREADS), sm, s, d, mem);
}

// the z convolution (needs G-hat) and the inverse transform
template <typename T>
cudaError_t launch_conv_group_rest(int nx, int ny, int nz, const PoissonMember* mem, int nmem,
                                   cudaStream_t s) {
  PoissonBuffers pb;
  pb.nx = nx; pb.ny = ny; pb.nz = nz;
  const PoissonDims d = dims_of(pb);
  cudaError_t e;
  switch (ztile<T>(nz)) {
    case 16: e = zconv_group_t<T, 16>(d, mem, nmem, s); break;
    case 8: e = zconv_group_t<T, 8>(d, mem, nmem, s); break;
    case 4: e = zconv_group_t<T, 4>(d, mem, nmem, s); break;
    case 2: e = zconv_group_t<T, 2>(d, mem, nmem, s); break;
    default: e = zconv_group_t<T, 1>(d, mem, nmem, s); break;
  }
  if (e != cudaSuccess) return e;
  const size_t sxy = xy_smem<T>(nx, ny);
  if ((e = allow_smem(k_fft_xy_inv_group<T>, sxy)) != cudaSuccess) return e;
  return launch_pdl(k_fft_xy_inv_group<T>, dim3(nz, nmem), dim3(512), sxy, s, d, mem);
}

template <typename T>
cudaError_t launch_efield_group(int nx, int ny, int nz, const PoissonMember* mem, int nmem,
                                cudaStream_t s) {
  const long long G = (long long)nx * ny * nz;
  return launch_pdl(k_efield_group<T>, dim3(group_grid(G, 256, nmem), nmem), dim3(256), 0, s, nx,
                    ny, nz, mem);
}

template cudaError_t launch_green_group<double>(int, int, int, const PoissonMember*, int,
                                                cudaStream_t);
template cudaError_t launch_green_group<float>(int, int, int, const PoissonMember*, int,
                                               cudaStream_t);
template <typename T>
cudaError_t launch_conv_group(int nx, int ny, int nz, const PoissonMember* mem, int nmem,
                              cudaStream_t s) {
  cudaError_t e = launch_conv_group_forward<T>(nx, ny, nz, mem, nmem, s);
  if (e != cudaSuccess) return e;
  return launch_conv_group_rest<T>(nx, ny, nz, mem, nmem, s);
}

template cudaError_t launch_conv_group<double>(int, int, int, const PoissonMember*, int,
                                               cudaStream_t);
template cudaError_t launch_conv_group<float>(int, int, int, const PoissonMember*, int,
                                              cudaStream_t);
template cudaError_t launch_conv_group_forward<double>(int, int, int, const PoissonMember*, int,
                                                       cudaStream_t);
template cudaError_t launch_conv_group_forward<float>(int, int, int, const PoissonMember*, int,
                                                      cudaStream_t);
template cudaError_t launch_conv_group_rest<double>(int, int, int, const PoissonMember*, int,
                                                    cudaStream_t);
template cudaError_t launch_conv_group_rest<float>(int, int, int, const PoissonMember*, int,
                                                   cudaStream_t);
template cudaError_t launch_efield_group<double>(int, int, int, const PoissonMember*, int,
                                                 cudaStream_t);
template cudaError_t launch_efield_group<float>(int, int, int, const PoissonMember*, int,
                                               cudaStream_t);
template cudaError_t launch_green<double>(const PoissonBuffers&, cudaStream_t);
template cudaError_t launch_green<float>(const PoissonBuffers&, cudaStream_t);
template cudaError_t launch_convolve<double>(const PoissonBuffers&, cudaStream_t);
template cudaError_t launch_conv_forward<double>(const PoissonBuffers&, cudaStream_t);
template cudaError_t launch_conv_forward<float>(const PoissonBuffers&, cudaStream_t);
template cudaError_t launch_conv_rest<double>(const PoissonBuffers&, cudaStream_t);
template cudaError_t launch_conv_rest<float>(const PoissonBuffers&, cudaStream_t);
template cudaError_t launch_convolve<float>(const PoissonBuffers&, cudaStream_t);
template cudaError_t launch_efield<double>(const PoissonBuffers&, cudaStream_t);
template cudaError_t launch_efield<float>(const PoissonBuffers&, cudaStream_t);
template bool poisson_fits<double>(int, int, int);
template bool poisson_fits<float>(int, int, int);

}  // namespace impz
