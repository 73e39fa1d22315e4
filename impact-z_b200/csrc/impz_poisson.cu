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
         ((size_t)(ny / 2) * (2 * nx) + (size_t)(nx + 1) * (2 * ny + 1) + nx + ny);
}
template <typename T>
static int ztile() { return sizeof(T) == 8 ? 8 : 16; }
template <typename T>
static size_t z_smem(int nz) {
  return sizeof(typename Cplx<T>::type) * ((size_t)ztile<T>() * (2 * nz + 1) + nz);
}
static const int kDctLines = 16;
template <typename T>
static size_t dct_smem(int n) {
  return sizeof(typename Cplx<T>::type) * ((size_t)(kDctLines / 2) * (2 * n + 1) + n);
}

template <typename T>
size_t poisson_smem_max(int nx, int ny, int nz) {
  size_t m = xy_smem<T>(nx, ny);
  m = m > z_smem<T>(nz) ? m : z_smem<T>(nz);
  int nmax = nx > ny ? nx : ny;
  nmax = nmax > nz ? nmax : nz;
  return m > dct_smem<T>(nmax) ? m : dct_smem<T>(nmax);
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

// The Green function: FP64 corners and 8-corner difference (the difference
// cancels catastrophically, Field.f90:420-428), then three DCT-I passes in
// the convolution's type T (FP64 in the plain form, FP32 in the
// FP32-convolution form, whose first pass converts the FP64 octant).
template <typename T>
cudaError_t launch_green(const PoissonBuffers& b, cudaStream_t s) {
  typedef typename Cplx<T>::type C;
  const int nx = b.nx, ny = b.ny, nz = b.nz;
  const long long nc = (long long)(nx + 2) * (ny + 2) * (nz + 2);
  const long long ng = (long long)(nx + 1) * (ny + 1) * (nz + 1);
  k_igf_corners<<<grid_for(nc, 256), 256, 0, s>>>(nx, ny, nz, b.st, b.F);
  k_igf_green<<<grid_for(ng, 256), 256, 0, s>>>(nx, ny, nz, b.F, b.Gt);
  const long long gx = nx + 1, gxy = (long long)(nx + 1) * (ny + 1);
  const double scale = 1.0 / ((double)(2 * nx) * (double)(2 * ny) * (double)(2 * nz));
  T* work = (T*)b.ghat;
  cudaError_t e;
  // along x: lines j (inner, stride gx) x k (outer); points contiguous
  {
    auto kern = k_dct1<double, T, T, kDctLines>;
    const size_t sm = dct_smem<T>(nx);
    if ((e = allow_smem(kern, sm)) != cudaSuccess) return e;
    dim3 g((ny + 1 + kDctLines - 1) / kDctLines, nz + 1);
    kern<<<g, 256, sm, s>>>(b.Gt, work, ilog2(2 * nx), 1, gx, ny + 1, gxy, 1.0, (const C*)b.twx);
  }
  // along y: lines i (inner, stride 1) x k (outer); points stride gx
  {
    auto kern = k_dct1<T, T, T, kDctLines>;
    const size_t sm = dct_smem<T>(ny);
    if ((e = allow_smem(kern, sm)) != cudaSuccess) return e;
    dim3 g((nx + 1 + kDctLines - 1) / kDctLines, nz + 1);
    kern<<<g, 256, sm, s>>>(work, work, ilog2(2 * ny), gx, 1, nx + 1, gxy, 1.0, (const C*)b.twy);
  }
  // along z: lines i (inner) x j (outer, stride gx); points stride gxy
  {
    auto kern = k_dct1<T, T, T, kDctLines>;
    const size_t sm = dct_smem<T>(nz);
    if ((e = allow_smem(kern, sm)) != cudaSuccess) return e;
    dim3 g((nx + 1 + kDctLines - 1) / kDctLines, ny + 1);
    kern<<<g, 256, sm, s>>>(work, work, ilog2(2 * nz), gxy, 1, nx + 1, gx, scale,
                            (const C*)b.twz);
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_conv_forward(const PoissonBuffers& b, cudaStream_t s) {
  typedef typename Cplx<T>::type C;
  const PoissonDims d = dims_of(b);
  cudaError_t e;
  const size_t sxy = xy_smem<T>(b.nx, b.ny);
  if ((e = allow_smem(k_fft_xy_fwd<T>, sxy)) != cudaSuccess) return e;
  k_fft_xy_fwd<T><<<b.nz, 512, sxy, s>>>(d, b.rho, b.st, b.qscale, (C*)b.spec,
                                         (const C*)b.twx, (const C*)b.twy);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_conv_rest(const PoissonBuffers& b, cudaStream_t s) {
  typedef typename Cplx<T>::type C;
  const PoissonDims d = dims_of(b);
  cudaError_t e;
  const size_t sxy = xy_smem<T>(b.nx, b.ny);
  if ((e = allow_smem(k_fft_xy_inv<T>, sxy)) != cudaSuccess) return e;
  const int tk = ztile<T>();
  const size_t sz = z_smem<T>(b.nz);
  dim3 gz((b.nx + 1 + tk - 1) / tk, 2 * b.ny);
  if (tk == 8) {
    if ((e = allow_smem(k_fft_z_conv<T, 8>, sz)) != cudaSuccess) return e;
    k_fft_z_conv<T, 8><<<gz, 256, sz, s>>>(d, (C*)b.spec, (const T*)b.ghat, (const C*)b.twz);
  } else {
    if ((e = allow_smem(k_fft_z_conv<T, 16>, sz)) != cudaSuccess) return e;
    k_fft_z_conv<T, 16><<<gz, 256, sz, s>>>(d, (C*)b.spec, (const T*)b.ghat, (const C*)b.twz);
  }
  k_fft_xy_inv<T><<<b.nz, 512, sxy, s>>>(d, (const C*)b.spec, (T*)b.phi, (const C*)b.twx,
                                         (const C*)b.twy);
  return cudaGetLastError();
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
  k_efield<T><<<grid_for(G, 256), 256, 0, s>>>(b.nx, b.ny, b.nz, (const T*)b.phi, b.st,
                                                (T*)b.efield);
  return cudaGetLastError();
}

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
template size_t poisson_smem_max<double>(int, int, int);
template size_t poisson_smem_max<float>(int, int, int);

}  // namespace impz
