// impz_poisson.cuh -- open-boundary Poisson solve on the device.
//
// Restates openBC3D + greenf1tIntnew (src/Appl/Field.f90:239-519): Hockney's
// doubled-grid convolution phi = IFFT(FFT(rho_padded) * FFT(G_even)) with the
// integrated Green's function G, then kick1's finite-difference field
// (src/Appl/BeamBunch.f90:1784-2005).  Any correct FFT reproduces the
// reference's FFTPACK convolution to rounding, so the transforms here are the
// project's own shared-memory radix-2 kernels laid out for the doubled grid:
//
//   xy-forward  one block per z plane: int64 charge -> real, R2C along x
//               (two real rows packed into one complex FFT of length 2Nx),
//               C2C along y (length 2Ny, upper half zero), spectrum plane out
//   z-convolve  one block per (ky, tile of kx): C2C along z (length 2Nz,
//               upper half zero), times the real even G-hat, inverse C2C,
//               only the Nz planes the crop needs are written back
//   xy-inverse  one block per z plane < Nz: inverse C2C along y, C2R along x,
//               potential plane out (only Nx x Ny of the doubled grid)
//
// G is even in every direction, so its transform is real and is computed as
// three DCT-I passes over the octant (Nx+1)(Ny+1)(Nz+1) (two lines packed
// into one complex FFT: even real sequences have real transforms).  The
// 1/(n1 n2 n3) inverse normalisation of Field.f90:321-323 is folded into G-hat.
//
// Spectrum layout in HBM: S[z][ky][kx], kx fastest, (Nx+1) x 2Ny x Nz complex.
// Forward passes use decimation in frequency (natural in, bit-reversed out)
// and inverse passes decimation in time (bit-reversed in, natural out), so no
// pass ever permutes data explicitly.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "impz_common.h"
#include "impz_device.cuh"

namespace impz {

template <typename T> struct Cplx;
template <> struct Cplx<double> { typedef double2 type; };
template <> struct Cplx<float> { typedef float2 type; };

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}

__device__ __forceinline__ int bitrev(int v, int logn) {
  return (int)(__brev((unsigned)v) >> (32 - logn));
}

// Lines in shared memory keep one spare slot after every eight elements:
// element j of a line sits at sw(j).  The butterfly groups read eight
// elements a fixed spacing apart, and at the small spans consecutive
// threads start eight elements apart, which without the spare slots would
// put 16 threads of a warp on the same banks.
__device__ __forceinline__ int sw(int j) { return j + (j >> 3); }
// line pitch (in elements) for lines of n >= 8 elements: odd, past sw(n-1)
__host__ __device__ constexpr int line_pitch(int n) { return n + n / 8 + 1; }

// Radix-2 butterflies over `nlines` lines in shared memory; element j of
// line l sits at buf[l*lstride + sw(j)].  tw[k] = exp(-2 pi i k / n), k < n/2.
// DIF: natural order in, bit-reversed out.  DIT: bit-reversed in, natural out.
// Up to three consecutive radix-2 stages act on the 2^NS elements spaced by
// the narrowest span, so each thread runs them in registers (one barrier and
// one shared-memory round trip per NS stages); the butterflies, twiddles and output order are those of plain
// radix-2.  Within a group, a stage with pair distance se uses only se
// distinct twiddles: element e pairs at position k + (e mod se) q, so the se
// twiddles are loaded once per stage and shared by its butterflies.
template <typename C>
__device__ __forceinline__ C twid(const C* tw, int idx, int sign) {
  C w = tw[idx];
  if (sign > 0) w.y = -w.y;
  return w;
}

// stages with half-spans 2^lh, 2^(lh-1), .., 2^(lh-NS+1) (DIF)
template <typename C, int NS>
__device__ __forceinline__ void dif_group(C* L, int o, int logn, int lh, int k, int sign,
                                          const C* tw) {
  constexpr int E = 1 << NS;
  const int q = 1 << (lh - NS + 1);  // spacing of the E elements
  C v[E];
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = L[sw(o + k + e * q)];
#pragma unroll
  for (int m = 0; m < NS; m++) {
    const int se = E >> (m + 1);      // pair distance; 2^(lh-m) = se * q
    const int tsh = logn - 1 - (lh - m);
    C w[E / 2];
#pragma unroll
    for (int j = 0; j < se; j++) w[j] = twid(tw, (k + j * q) << tsh, sign);
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (e & se) continue;
      const C u = v[e], t = v[e + se];
      v[e] = cadd(u, t);
      v[e + se] = cmul(csub(u, t), w[e & (se - 1)]);
    }
  }
#pragma unroll
  for (int e = 0; e < E; e++) L[sw(o + k + e * q)] = v[e];
}

// stages with half-spans 2^lh, .., 2^(lh+NS-1) (DIT)
template <typename C, int NS>
__device__ __forceinline__ void dit_group(C* L, int o, int logn, int lh, int k, int sign,
                                          const C* tw) {
  constexpr int E = 1 << NS;
  const int q = 1 << lh;
  C v[E];
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = L[sw(o + k + e * q)];
#pragma unroll
  for (int m = 0; m < NS; m++) {
    const int se = 1 << m;            // pair distance; 2^(lh+m) = se * q
    const int tsh = logn - 1 - (lh + m);
    C w[E / 2];
#pragma unroll
    for (int j = 0; j < se; j++) w[j] = twid(tw, (k + j * q) << tsh, sign);
#pragma unroll
    for (int e = 0; e < E; e++) {
      if (e & se) continue;
      const C u = v[e], t = cmul(v[e + se], w[e & (se - 1)]);
      v[e] = cadd(u, t);
      v[e + se] = csub(u, t);
    }
  }
#pragma unroll
  for (int e = 0; e < E; e++) L[sw(o + k + e * q)] = v[e];
}

// widest group: three stages (four for FP32 lines spent more registers than
// the fewer rounds saved)
#ifndef IMPZ_FFT_NS_F32
#define IMPZ_FFT_NS_F32 3
#endif
template <typename C>
struct MaxStages { static constexpr int value = sizeof(C) == 8 ? IMPZ_FFT_NS_F32 : 3; };

template <typename C>
__device__ void fft_dif(C* buf, int logn, int nlines, int lstride, int sign, const C* tw) {
  constexpr int MS = MaxStages<C>::value;
  int lh = logn - 1;
  while (lh >= 0) {
    const int ns = lh + 1 >= MS ? MS : lh + 1;
    const int lper = lh - ns + 1;            // log2 of the groups per block
    const int lngl = logn - ns;              // log2 of the groups per line
    const int total = nlines << lngl;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int l = b >> lngl, r = b & ((1 << lngl) - 1);
      const int o = (r >> lper) << (lh + 1), k = r & ((1 << lper) - 1);
      C* Lp = buf + l * lstride;
      if (MS >= 4 && ns == 4) dif_group<C, (MS >= 4 ? 4 : 1)>(Lp, o, logn, lh, k, sign, tw);
      else if (ns == 3) dif_group<C, 3>(Lp, o, logn, lh, k, sign, tw);
      else if (ns == 2) dif_group<C, 2>(Lp, o, logn, lh, k, sign, tw);
      else dif_group<C, 1>(Lp, o, logn, lh, k, sign, tw);
    }
    __syncthreads();
    lh -= ns;
  }
}

template <typename C>
__device__ void fft_dit(C* buf, int logn, int nlines, int lstride, int sign, const C* tw) {
  constexpr int MS = MaxStages<C>::value;
  int lh = 0;
  while (lh < logn) {
    const int ns = (logn - lh) >= MS ? MS : logn - lh;
    const int lngl = logn - ns;
    const int total = nlines << lngl;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int l = b >> lngl, r = b & ((1 << lngl) - 1);
      const int o = (r >> lh) << (lh + ns), k = r & ((1 << lh) - 1);
      C* Lp = buf + l * lstride;
      if (MS >= 4 && ns == 4) dit_group<C, (MS >= 4 ? 4 : 1)>(Lp, o, logn, lh, k, sign, tw);
      else if (ns == 3) dit_group<C, 3>(Lp, o, logn, lh, k, sign, tw);
      else if (ns == 2) dit_group<C, 2>(Lp, o, logn, lh, k, sign, tw);
      else dit_group<C, 1>(Lp, o, logn, lh, k, sign, tw);
    }
    __syncthreads();
    lh += ns;
  }
}

// copies n/2 twiddles into shared memory (whole block, no barrier)
template <typename C>
__device__ __forceinline__ void stage_tw(C* dst, const C* __restrict__ src, int n) {
  for (int e = threadIdx.x; e < n / 2; e += blockDim.x) dst[e] = src[e];
}

struct PoissonDims {
  int nx, ny, nz;
  int lx, ly, lz;  // log2 of the doubled lengths 2nx, 2ny, 2nz
};

// ---------------------------------------------------------------------
// xy-forward: PARTS blocks per z plane k < nz (one by default: splitting a
// plane measured slower at 64x64).  Each block transforms all the plane's
// rows along x and then unpacks, transforms along y and stores its own share
// of the nx+1 kx lines.  The charge is cleared later, by k_efield (not by
// stores interleaved with the transform's loads).
// smem: Z[ny/2][2nx] (packed row pairs) and Tm[own kx][2ny] (y lines).
template <typename T, int PARTS>
__device__ __forceinline__ void fft_xy_fwd_body(const PoissonDims& d,
                                                const unsigned long long* __restrict__ rho,
                                                double qscale, typename Cplx<T>::type* __restrict__ S,
                                                const typename Cplx<T>::type* __restrict__ twx,
                                                const typename Cplx<T>::type* __restrict__ twy,
                                                const int bx, const int by) {
  typedef typename Cplx<T>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  griddep_wait();
  const int nx = d.nx, ny = d.ny, n1 = 2 * nx, n2 = 2 * ny, w = nx + 1;
  const int zp = line_pitch(n1), tp = line_pitch(n2);  // x-line and y-line pitches
  const int hy = ny / 2;
  const int part = bx, k = by;
  const int kx_lo = w * part / PARTS, nown = w * (part + 1) / PARTS - kx_lo;
  C* Z = reinterpret_cast<C*>(smem_raw);
  C* Tm = Z + hy * zp;
  C* twxs = Tm + ((w + PARTS - 1) / PARTS) * tp;
  C* twys = twxs + n1 / 2;
  stage_tw(twxs, twx, n1);
  stage_tw(twys, twy, n2);
  const size_t plane = (size_t)nx * ny * k;
  // load two real rows per complex line, natural order, zero padded
  for (int e = threadIdx.x; e < hy * n1; e += blockDim.x) {
    const int l = e >> d.lx, j = e & (n1 - 1);
    C z;
    z.x = 0; z.y = 0;
    if (j < nx) {
      const size_t ia = plane + (size_t)l * nx + j, ib = plane + (size_t)(l + hy) * nx + j;
      z.x = (T)((double)(long long)rho[ia] * qscale);
      z.y = (T)((double)(long long)rho[ib] * qscale);
    }
    Z[l * zp + sw(j)] = z;
  }
  __syncthreads();
  fft_dif<C>(Z, d.lx, hy, zp, -1, twxs);
  // unpack: row a = (Z(k)+conj(Z(n1-k)))/2, row b = (Z(k)-conj(Z(n1-k)))/(2i),
  // own kx, into y lines Tm[kx - kx_lo][y] (natural y, zero padded to 2ny)
  for (int e = threadIdx.x; e < nown * n2; e += blockDim.x) {
    const int kl = e >> d.ly, y = e & (n2 - 1);
    const int kx = kx_lo + kl;
    C v;
    v.x = 0; v.y = 0;
    if (y < ny) {
      const int l = y < hy ? y : y - hy;
      const C* L = Z + l * zp;
      const C zk = L[sw(bitrev(kx, d.lx))];
      const C zm = L[sw(bitrev((n1 - kx) & (n1 - 1), d.lx))];
      if (y < hy) {
        v.x = (T)0.5 * (zk.x + zm.x);
        v.y = (T)0.5 * (zk.y - zm.y);
      } else {
        v.x = (T)0.5 * (zk.y + zm.y);
        v.y = (T)0.5 * (zm.x - zk.x);
      }
    }
    Tm[kl * tp + sw(y)] = v;
  }
  __syncthreads();
  fft_dif<C>(Tm, d.ly, nown, tp, -1, twys);
  // store S[k][ky][kx] for the own kx, (ky, kl) walked with a carry
  C* Sk = S + (size_t)k * n2 * w + kx_lo;
  {
    const int dky = blockDim.x / nown, dkl = blockDim.x - dky * nown;
    int ky = threadIdx.x / nown, kl = threadIdx.x - ky * nown;
    for (int e = threadIdx.x; e < nown * n2; e += blockDim.x) {
      Sk[(size_t)ky * w + kl] = Tm[kl * tp + sw(bitrev(ky, d.ly))];
      kl += dkl;
      ky += dky;
      if (kl >= nown) { kl -= nown; ky++; }
    }
  }
}

template <typename T, int PARTS>
__global__ void k_fft_xy_fwd(PoissonDims d, const unsigned long long* __restrict__ rho,
                             double qscale, typename Cplx<T>::type* __restrict__ S,
                             const typename Cplx<T>::type* __restrict__ twx,
                             const typename Cplx<T>::type* __restrict__ twy) {
  fft_xy_fwd_body<T, PARTS>(d, rho, qscale, S, twx, twy, blockIdx.x, blockIdx.y);
}

// the same for every bunch of a group of one grid size: blockIdx.z = member
template <typename T, int PARTS>
__global__ void k_fft_xy_fwd_group(PoissonDims d, const PoissonMember* __restrict__ mem) {
  typedef typename Cplx<T>::type C;
  const PoissonMember& m = mem[blockIdx.z];
  fft_xy_fwd_body<T, PARTS>(d, m.rho, m.qscale, (C*)m.spec, (const C*)m.twx, (const C*)m.twy,
                            blockIdx.x, blockIdx.y);
}

// z-convolve: block = (tile of TKX kx values, one ky).
template <typename T, int TKX>
__device__ __forceinline__ void fft_z_conv_body(const PoissonDims& d,
                                                typename Cplx<T>::type* __restrict__ S,
                                                const T* __restrict__ ghat,
                                                const typename Cplx<T>::type* __restrict__ twz,
                                                const int bx, const int by) {
  typedef typename Cplx<T>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  griddep_wait();
  const int nx = d.nx, ny = d.ny, nz = d.nz, n2 = 2 * ny, n3 = 2 * nz;
  const int lp = line_pitch(n3);
  C* L = reinterpret_cast<C*>(smem_raw);
  C* twzs = L + TKX * lp;
  stage_tw(twzs, twz, n3);
  const int kx0 = bx * TKX;
  const int ky = by;
  const int ntk = min(TKX, nx + 1 - kx0);
  const size_t pstride = (size_t)n2 * (nx + 1);  // one z plane of S
  C* base = S + (size_t)ky * (nx + 1) + kx0;
  for (int e = threadIdx.x; e < TKX * n3; e += blockDim.x) {
    const int z = e / TKX, t = e - z * TKX;
    C v;
    v.x = 0; v.y = 0;
    if (z < nz && t < ntk) v = base[(size_t)z * pstride + t];
    L[t * lp + sw(z)] = v;
  }
  __syncthreads();
  fft_dif<C>(L, d.lz, TKX, lp, -1, twzs);
  // multiply by G-hat (bit-reversed positions); G-hat octant [kz'][ky'][kx]
  const int kyp = ky <= ny ? ky : n2 - ky;
  const size_t gy = (size_t)(nx + 1), gz = (size_t)(nx + 1) * (ny + 1);
  for (int e = threadIdx.x; e < TKX * n3; e += blockDim.x) {
    const int t = e >> d.lz, pos = e & (n3 - 1);
    if (t >= ntk) continue;
    const int kz = bitrev(pos, d.lz);
    const int kzp = kz <= nz ? kz : n3 - kz;
    const T gv = ghat[(size_t)kzp * gz + (size_t)kyp * gy + kx0 + t];
    C& v = L[t * lp + sw(pos)];
    v.x *= gv;
    v.y *= gv;
  }
  __syncthreads();
  fft_dit<C>(L, d.lz, TKX, lp, +1, twzs);
  for (int e = threadIdx.x; e < TKX * nz; e += blockDim.x) {
    const int z = e / TKX, t = e - z * TKX;
    if (t < ntk) base[(size_t)z * pstride + t] = L[t * lp + sw(z)];
  }
}

template <typename T, int TKX>
__global__ void k_fft_z_conv(PoissonDims d, typename Cplx<T>::type* __restrict__ S,
                             const T* __restrict__ ghat,
                             const typename Cplx<T>::type* __restrict__ twz) {
  fft_z_conv_body<T, TKX>(d, S, ghat, twz, blockIdx.x, blockIdx.y);
}

template <typename T, int TKX>
__global__ void k_fft_z_conv_group(PoissonDims d, const PoissonMember* __restrict__ mem) {
  typedef typename Cplx<T>::type C;
  const PoissonMember& m = mem[blockIdx.z];
  fft_z_conv_body<T, TKX>(d, (C*)m.spec, (const T*)m.ghat, (const C*)m.twz, blockIdx.x,
                          blockIdx.y);
}

// xy-inverse: one block per z plane k < nz; phi out (nx, ny, nz) real.
template <typename T>
__device__ __forceinline__ void fft_xy_inv_body(const PoissonDims& d,
                                                const typename Cplx<T>::type* __restrict__ S,
                                                T* __restrict__ phi,
                                                const typename Cplx<T>::type* __restrict__ twx,
                                                const typename Cplx<T>::type* __restrict__ twy,
                                                const int bx) {
  typedef typename Cplx<T>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  griddep_wait();
  const int nx = d.nx, ny = d.ny, n1 = 2 * nx, n2 = 2 * ny;
  const int zp = line_pitch(n1), tp = line_pitch(n2);
  const int hy = ny / 2;
  C* Z = reinterpret_cast<C*>(smem_raw);
  C* Tm = Z + hy * zp;
  C* twxs = Tm + (nx + 1) * tp;
  C* twys = twxs + n1 / 2;
  stage_tw(twxs, twx, n1);
  stage_tw(twys, twy, n2);
  const int k = bx;
  const C* Sk = S + (size_t)k * n2 * (nx + 1);
  // y lines in bit-reversed order for the DIT inverse
  {
    const int w = nx + 1, dky = blockDim.x / w, dkx = blockDim.x - dky * w;
    int ky = threadIdx.x / w, kx = threadIdx.x - ky * w;
    for (int e = threadIdx.x; e < w * n2; e += blockDim.x) {
      Tm[kx * tp + sw(bitrev(ky, d.ly))] = Sk[e];
      kx += dkx;
      ky += dky;
      if (kx >= w) { kx -= w; ky++; }
    }
  }
  __syncthreads();
  fft_dit<C>(Tm, d.ly, nx + 1, tp, +1, twys);
  // C2R along x for row pairs (y, y+ny/2), y < ny/2: Z(kx) = Xa(kx) + i Xb(kx),
  // with X(n1-kx) = conj(X(kx)); placed bit-reversed for the DIT inverse
  for (int e = threadIdx.x; e < hy * n1; e += blockDim.x) {
    const int l = e >> d.lx, kk = e & (n1 - 1);
    const int kxs = kk <= nx ? kk : n1 - kk;
    C xa = Tm[kxs * tp + sw(l)], xb = Tm[kxs * tp + sw(l + hy)];
    if (kk > nx) { xa.y = -xa.y; xb.y = -xb.y; }
    C z;
    z.x = xa.x - xb.y;
    z.y = xa.y + xb.x;
    Z[l * zp + sw(bitrev(kk, d.lx))] = z;
  }
  __syncthreads();
  fft_dit<C>(Z, d.lx, hy, zp, +1, twxs);
  T* ph = phi + (size_t)nx * ny * k;
  for (int e = threadIdx.x; e < nx * ny; e += blockDim.x) {
    const int y = e >> (d.lx - 1), x = e & (nx - 1);
    const C v = Z[(y < hy ? y : y - hy) * zp + sw(x)];
    ph[e] = y < hy ? v.x : v.y;
  }
}

template <typename T>
__global__ void k_fft_xy_inv(PoissonDims d, const typename Cplx<T>::type* __restrict__ S,
                             T* __restrict__ phi,
                             const typename Cplx<T>::type* __restrict__ twx,
                             const typename Cplx<T>::type* __restrict__ twy) {
  fft_xy_inv_body<T>(d, S, phi, twx, twy, blockIdx.x);
}

template <typename T>
__global__ void k_fft_xy_inv_group(PoissonDims d, const PoissonMember* __restrict__ mem) {
  typedef typename Cplx<T>::type C;
  const PoissonMember& m = mem[blockIdx.y];
  fft_xy_inv_body<T>(d, (const C*)m.spec, (T*)m.phi, (const C*)m.twx, (const C*)m.twy,
                     blockIdx.x);
}

// ---------------------------------------------------------------------
// greenf1tIntnew corner antiderivative (Field.f90:392-418), FP64, at the
// (nx+2)(ny+2)(nz+2) corners v = (i-1)h - h/2.
__device__ __forceinline__ void igf_corners_body(int nx, int ny, int nz, const DevState* st,
                                                 double* F) {
  const int ax = nx + 2, ay = ny + 2, az = nz + 2;
  const long long total = (long long)ax * ay * az;
  const double hx = st->geom.h[0], hy = st->geom.h[1], hz = st->geom.h[2];
  const double hxyz = hx * hy * hz;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(e % ax);
    const int j0 = (int)((e / ax) % ay);
    const int k0 = (int)(e / ((long long)ax * ay));
    const double v1 = (double)i0 * hx - hx / 2;
    const double v2 = (double)j0 * hy - hy / 2;
    const double v3 = (double)k0 * hz - hz / 2;
    const double rr = sqrt(v1 * v1 + v2 * v2 + v3 * v3);
    const double aa = -(v3 * v3 * atan(v1 * v2 / (v3 * rr)) / 2);
    const double bb = -(v2 * v2 * atan(v1 * v3 / (v2 * rr)) / 2);
    const double cc = -(v1 * v1 * atan(v2 * v3 / (v1 * rr)) / 2);
    const double dd = v2 * v3 * log(v1 + rr);
    const double ee = v1 * v3 * log(v2 + rr);
    const double ff = v1 * v2 * log(v3 + rr);
    const double gg2 = aa + bb + cc + dd + ee + ff;
    F[e] = gg2 / hxyz;
  }
}

__global__ void k_igf_corners(int nx, int ny, int nz, const DevState* st, double* F) {
  igf_corners_body(nx, ny, nz, st, F);
}

__global__ void k_igf_corners_group(int nx, int ny, int nz, const PoissonMember* __restrict__ mem) {
  const PoissonMember& m = mem[blockIdx.y];
  igf_corners_body(nx, ny, nz, m.st, m.F);
}

// The Green octant one z plane per block: the 8-corner difference of plane
// k (Field.f90:420-428, FP64: it cancels catastrophically), rounded to the
// convolution's type T, then its DCT-I along x and along y in shared memory
// (rows, then columns, two lines per complex FFT of length 2n), written to
// plane k of G-hat; the z pass follows.  One pass over the corners and one
// write of the plane instead of a difference kernel and two strided DCT
// passes through global memory.  lx, ly: log2(2 nx), log2(2 ny).
// smem: the line pairs of the longer transform, the twiddles of both, and
// the plane P[(ny+1)][(nx+1)] (T).
template <typename T>
__device__ __forceinline__ void green_xy_body(int nx, int ny, int lx, int ly,
                                              const double* __restrict__ F, T* __restrict__ ghat,
                                              const typename Cplx<T>::type* __restrict__ twx,
                                              const typename Cplx<T>::type* __restrict__ twy,
                                              const int k) {
  typedef typename Cplx<T>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int gx = nx + 1, gy = ny + 1, ax = nx + 2, ay = ny + 2;
  const int lpx = line_pitch(2 * nx), lpy = line_pitch(2 * ny);
  const int npx = (gy + 1) / 2;  // row pairs (j, j + npx) for the x transform
  const int npy = (gx + 1) / 2;  // column pairs (i, i + npy) for the y transform
  C* L = reinterpret_cast<C*>(smem_raw);
  C* twxs = L + max(npx * lpx, npy * lpy);
  C* twys = twxs + nx;
  T* P = reinterpret_cast<T*>(twys + ny);
  stage_tw(twxs, twx, 2 * nx);
  stage_tw(twys, twy, 2 * ny);
  const double* F0 = F + (size_t)ax * ay * k;  // corner planes k and k + 1
  const double* F1 = F0 + (size_t)ax * ay;
#pragma unroll 4
  for (int e = threadIdx.x; e < gx * gy; e += blockDim.x) {
    const int j = e / gx, i = e - j * gx;
#define IMPZ_F(p, a, b) __ldg(p + (a) + (size_t)ax * (b))
    const double v = IMPZ_F(F1, i + 1, j + 1) - IMPZ_F(F1, i, j + 1) - IMPZ_F(F1, i + 1, j) +
                     IMPZ_F(F1, i, j) - IMPZ_F(F0, i + 1, j + 1) + IMPZ_F(F0, i, j + 1) +
                     IMPZ_F(F0, i + 1, j) - IMPZ_F(F0, i, j);
#undef IMPZ_F
    P[e] = (T)v;
  }
  __syncthreads();
  // along x: row t with row t + npx (real and imaginary parts)
  for (int e = threadIdx.x; e < npx * 2 * nx; e += blockDim.x) {
    const int m = e / npx, t = e - m * npx;
    const int mm = m <= nx ? m : 2 * nx - m;
    C v;
    v.x = P[t * gx + mm];
    v.y = t + npx < gy ? P[(t + npx) * gx + mm] : (T)0;
    L[t * lpx + sw(m)] = v;
  }
  __syncthreads();
  fft_dif<C>(L, lx, npx, lpx, -1, twxs);
  for (int e = threadIdx.x; e < npx * gx; e += blockDim.x) {
    const int m = e / npx, t = e - m * npx;
    const C v = L[t * lpx + sw(bitrev(m, lx))];
    P[t * gx + m] = v.x;
    if (t + npx < gy) P[(t + npx) * gx + m] = v.y;
  }
  __syncthreads();
  // along y: column t with column t + npy
  for (int e = threadIdx.x; e < npy * 2 * ny; e += blockDim.x) {
    const int m = e / npy, t = e - m * npy;
    const int mm = m <= ny ? m : 2 * ny - m;
    C v;
    v.x = P[mm * gx + t];
    v.y = t + npy < gx ? P[mm * gx + t + npy] : (T)0;
    L[t * lpy + sw(m)] = v;
  }
  __syncthreads();
  fft_dif<C>(L, ly, npy, lpy, -1, twys);
  T* out = ghat + (size_t)gx * gy * k;
  for (int e = threadIdx.x; e < npy * gy; e += blockDim.x) {
    const int m = e / npy, t = e - m * npy;
    const C v = L[t * lpy + sw(bitrev(m, ly))];
    out[(size_t)m * gx + t] = v.x;
    if (t + npy < gx) out[(size_t)m * gx + t + npy] = v.y;
  }
}

#ifndef IMPZ_GREEN_THREADS
#define IMPZ_GREEN_THREADS 512
#endif
template <typename T>
__global__ void __launch_bounds__(IMPZ_GREEN_THREADS)
    k_green_xy(int nx, int ny, int lx, int ly, const double* __restrict__ F, T* __restrict__ ghat,
               const typename Cplx<T>::type* __restrict__ twx,
               const typename Cplx<T>::type* __restrict__ twy) {
  green_xy_body<T>(nx, ny, lx, ly, F, ghat, twx, twy, blockIdx.x);
}

template <typename T>
__global__ void __launch_bounds__(IMPZ_GREEN_THREADS)
    k_green_xy_group(int nx, int ny, int lx, int ly, const PoissonMember* __restrict__ mem) {
  typedef typename Cplx<T>::type C;
  const PoissonMember& m = mem[blockIdx.y];
  green_xy_body<T>(nx, ny, lx, ly, m.F, (T*)m.ghat, (const C*)m.twx, (const C*)m.twy,
                   blockIdx.x);
}

// DCT-I (transform of the even extension) along one axis of the octant.
// Lines have n+1 points spaced by `es`; TL lines spaced by `ls` are handled
// by one block (consecutive inner lines for coalescing), outer lines are
// spaced by `os`.  Pairs of lines share one complex FFT of length 2n in the
// compute type CT.  Reads `in` (TI), writes `out` (TO, may alias `in`: each
// block owns its lines) times `scale`.
template <typename TI, typename TO, typename CT, int TL>
__device__ __forceinline__ void dct1_body(const TI* in, TO* out, int logn, long long es,
                                          long long ls, int ninner, long long os, double scale,
                                          const typename Cplx<CT>::type* __restrict__ tw,
                                          const int bx, const int by) {
  typedef typename Cplx<CT>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* L = reinterpret_cast<C*>(smem_raw);
  const int n = 1 << (logn - 1);  // octant points - 1
  const int n2 = 2 * n;
  const int lp = line_pitch(n2);
  C* tws = L + (TL / 2) * lp;
  stage_tw(tws, tw, n2);
  const int l0 = bx * TL;
  const int nl = min(TL, ninner - l0);
  const long long off = (long long)by * os + (long long)l0 * ls;
  const TI* ib = in + off;
  TO* ob = out + off;
  // pair line t with line t + TL/2 (real and imaginary parts)
  const int np = TL / 2;
  for (int e = threadIdx.x; e < np * n2; e += blockDim.x) {
    const int m = e / np, t = e - m * np;  // t fastest for coalescing
    const int mm = m <= n ? m : n2 - m;
    C v;
    v.x = t < nl ? (CT)ib[(long long)t * ls + mm * es] : (CT)0;
    v.y = t + np < nl ? (CT)ib[(long long)(t + np) * ls + mm * es] : (CT)0;
    L[t * lp + sw(m)] = v;
  }
  __syncthreads();
  fft_dif<C>(L, logn, np, lp, -1, tws);
  for (int e = threadIdx.x; e < np * (n + 1); e += blockDim.x) {
    const int m = e / np, t = e - m * np;
    const C v = L[t * lp + sw(bitrev(m, logn))];
    if (t < nl) ob[(long long)t * ls + m * es] = (TO)((double)v.x * scale);
    if (t + np < nl) ob[(long long)(t + np) * ls + m * es] = (TO)((double)v.y * scale);
  }
}

template <typename TI, typename TO, typename CT, int TL>
__global__ void k_dct1(const TI* in, TO* out, int logn, long long es, long long ls, int ninner,
                       long long os, double scale,
                       const typename Cplx<CT>::type* __restrict__ tw) {
  dct1_body<TI, TO, CT, TL>(in, out, logn, es, ls, ninner, os, scale, tw, blockIdx.x, blockIdx.y);
}

// pass `axis` (0: x from the FP64 octant Gt into G-hat, 1: y, 2: z in place
// on G-hat) for every member of a group: blockIdx.z = member
template <typename TI, typename TO, typename CT, int TL>
__global__ void k_dct1_group(int axis, int logn, long long es, long long ls, int ninner,
                             long long os, double scale, const PoissonMember* __restrict__ mem) {
  typedef typename Cplx<CT>::type C;
  const PoissonMember& m = mem[blockIdx.z];
  const TI* in = (const TI*)m.ghat;  // x and y are done by k_green_xy_group
  const C* tw = (const C*)(axis == 0 ? m.twx : axis == 1 ? m.twy : m.twz);
  dct1_body<TI, TO, CT, TL>(in, (TO*)m.ghat, logn, es, ls, ninner, os, scale, tw, blockIdx.x,
                            blockIdx.y);
}

// ---------------------------------------------------------------------
// kick1_BeamBunch finite differences (BeamBunch.f90:1784-2005), one rank,
// open BC: centred inside, one-sided on the faces.  Out: {Ex,Ey,Ez,0}.
// Also clears the charge grid (its last reader, the forward transform, is
// done) for the next deposit.  With a wake (read-in or CSR), adds its
// per-plane field wake = {dEx, dEy, dEz}[nz] to every node of the plane
// (kick1wake, BeamBunch.f90:5015-5033) and clears the wake's line sums.
template <typename T>
__device__ __forceinline__ void efield_body(int nx, int ny, int nz, const T* __restrict__ phi,
                                            const DevState* st, T* __restrict__ E,
                                            unsigned long long* __restrict__ rho,
                                            const double* __restrict__ wake,
                                            unsigned long long* __restrict__ wake_line) {
  griddep_wait();
  if (wake_line)
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 3 * nz; e += gridDim.x * blockDim.x)
      wake_line[e] = 0ull;
  const long long G = (long long)nx * ny * nz;
  const T hxi = (T)st->geom.hi[0], hyi = (T)st->geom.hi[1], hzi = (T)st->geom.hi[2];
  const T half = (T)0.5;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < G;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % nx);
    const int j = (int)((e / nx) % ny);
    const int k = (int)(e / ((long long)nx * ny));
    const long long sy = nx, sz = (long long)nx * ny;
    T ex, ey, ez;
    if (i == 0) ex = hxi * (phi[e] - phi[e + 1]);
    else if (i == nx - 1) ex = hxi * (phi[e - 1] - phi[e]);
    else ex = half * hxi * (phi[e - 1] - phi[e + 1]);
    if (j == 0) ey = hyi * (phi[e] - phi[e + sy]);
    else if (j == ny - 1) ey = hyi * (phi[e - sy] - phi[e]);
    else ey = half * hyi * (phi[e - sy] - phi[e + sy]);
    if (k == 0) ez = hzi * (phi[e] - phi[e + sz]);
    else if (k == nz - 1) ez = hzi * (phi[e - sz] - phi[e]);
    else ez = half * hzi * (phi[e - sz] - phi[e + sz]);
    if (wake) {
      ex = ex + (T)wake[k];
      ey = ey + (T)wake[nz + k];
      ez = ez + (T)wake[2 * nz + k];
    }
    rho[e] = 0ull;  // the next deposit accumulates into a cleared charge grid
    T* o = E + 4 * e;
    o[0] = ex;
    o[1] = ey;
    o[2] = ez;
    o[3] = (T)0;
  }
}

template <typename T>
__global__ void k_efield(int nx, int ny, int nz, const T* __restrict__ phi,
                         const DevState* st, T* __restrict__ E,
                         unsigned long long* __restrict__ rho,
                         const double* __restrict__ wake,
                         unsigned long long* __restrict__ wake_line) {
  efield_body<T>(nx, ny, nz, phi, st, E, rho, wake, wake_line);
}

template <typename T>
__global__ void k_efield_group(int nx, int ny, int nz, const PoissonMember* __restrict__ mem) {
  const PoissonMember& m = mem[blockIdx.y];
  efield_body<T>(nx, ny, nz, (const T*)m.phi, m.st, (T*)m.efield, m.rho, nullptr, nullptr);
}

}  // namespace impz
