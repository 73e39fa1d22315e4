// impz_launch.h -- host-side launch wrappers of the sm_100a kernels.
#pragma once
#include <cuda_runtime.h>

#include "impz_common.h"

namespace impz {

// Launches `kernel` on `s` with programmatic stream serialization: its grid
// may be scheduled while the stream's previous kernel drains, which hides
// the launch gap; the kernel calls griddep_wait() before it reads what that
// kernel wrote.
template <typename... KP, typename... A>
inline cudaError_t launch_pdl(void (*kernel)(KP...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t s, A... args) {
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr.val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KP>(args)...);
}

#ifndef IMPZ_ADV_BLOCK
#define IMPZ_ADV_BLOCK 256
#endif
#ifndef IMPZ_ADV_U
#define IMPZ_ADV_U 2
#endif
#ifndef IMPZ_ADV_PREFETCH
#define IMPZ_ADV_PREFETCH 0
#endif
#ifndef IMPZ_ADV_MINB
#define IMPZ_ADV_MINB 2
#endif
#ifndef IMPZ_DEP_BLOCK
#define IMPZ_DEP_BLOCK 256
#endif
#ifndef IMPZ_DEP_PPT
#define IMPZ_DEP_PPT 4
#endif
#ifndef IMPZ_DEP_MINB
#define IMPZ_DEP_MINB 4
#endif
#define IMPZ_SCAN_THREADS 256  // x 16 cells: 4096 cells (one scan block) per block

#define IMPZ_DECLARE_PARTICLE_LAUNCHERS(NS)                                              \
  namespace NS {                                                                         \
  cudaError_t launch_advance(const AdvanceArgs& a, bool f32, bool light, int grid,       \
                             cudaStream_t s);                                            \
  cudaError_t launch_deposit(const DepositArgs& a, int grid, cudaStream_t s);            \
  cudaError_t launch_wake(const WakeArgs& a, int grid, cudaStream_t s);                  \
  cudaError_t prepare_wake();                                                            \
  cudaError_t launch_scan(int* counts, int* cursor, int* bsum, long long total,          \
                          DevState* st, cudaStream_t s);                                 \
  int max_blocks_advance(bool f32);                                                      \
  cudaError_t launch_advance_packed(const AdvanceArgs* args, const int* offs, int nmem,  \
                                    int blocks, bool f32, bool light, bool species,      \
                                    cudaStream_t s);                                     \
  cudaError_t launch_deposit_packed(const DepositArgs* args, const int* offs, int nmem,  \
                                    int blocks, bool species, cudaStream_t s);            \
  cudaError_t launch_scan_packed(const ScanArgs* args, const int* offs, int nmem, int blocks, \
                                 cudaStream_t s);                                         \
  int max_blocks_deposit();                                                              \
  cudaError_t launch_species_count(const DepositArgs& a, int test_loss, int nspecies,    \
                                   int* counts, int grid, cudaStream_t s);               \
  }
IMPZ_DECLARE_PARTICLE_LAUNCHERS(exact)
IMPZ_DECLARE_PARTICLE_LAUNCHERS(fast)

// Poisson solve (T = double for the FP64 form, float for the FP32 form)
struct PoissonBuffers {
  int nx, ny, nz;
  unsigned long long* rho;  // int64 charge, cleared by the forward pass
  double qscale;            // grid value of one fixed-point quantum
  void* spec;               // (nx+1)*2ny*nz complex T
  double* F;                // (nx+2)(ny+2)(nz+2) IGF corners
  void* ghat;               // (nx+1)(ny+1)(nz+1) T
  void* phi;                // nx*ny*nz T
  void* efield;             // 4*nx*ny*nz T
  const void* twx;          // twiddles of length 2nx, 2ny, 2nz in T
  const void* twy;
  const void* twz;
  const double2* tw64x;     // FP64 twiddles for the DCT of G
  const double2* tw64y;
  const double2* tw64z;
  DevState* st;
  const double* wake;       // per-plane {dEx, dEy, dEz}[nz] added to E, or null
  unsigned long long* wake_line;  // the wake's [3][nz] line sums, cleared with the charge
  int ztile;                // z lines per block of the z convolution (0: the largest that fits)
};

template <typename T>
cudaError_t launch_green(const PoissonBuffers& b, cudaStream_t s);
template <typename T>
cudaError_t launch_convolve(const PoissonBuffers& b, cudaStream_t s);
// the convolution split at the point where G-hat is first needed
template <typename T>
cudaError_t launch_conv_forward(const PoissonBuffers& b, cudaStream_t s);
template <typename T>
cudaError_t launch_conv_rest(const PoissonBuffers& b, cudaStream_t s);
template <typename T>
cudaError_t launch_efield(const PoissonBuffers& b, cudaStream_t s);
// the same solve for nmem bunches of one grid size (PoissonMember array in
// device memory), one launch per kernel for the whole group
template <typename T>
cudaError_t launch_green_group(int nx, int ny, int nz, const PoissonMember* mem, int nmem,
                               cudaStream_t s);
template <typename T>
cudaError_t launch_conv_group(int nx, int ny, int nz, const PoissonMember* mem, int nmem,
                              cudaStream_t s);
template <typename T>
cudaError_t launch_efield_group(int nx, int ny, int nz, const PoissonMember* mem, int nmem,
                                cudaStream_t s);
// launch_conv_group split where G-hat is first needed
template <typename T>
cudaError_t launch_conv_group_forward(int nx, int ny, int nz, const PoissonMember* mem, int nmem,
                                      cudaStream_t s);
template <typename T>
cudaError_t launch_conv_group_rest(int nx, int ny, int nz, const PoissonMember* mem, int nmem,
                                   cudaStream_t s);
// true when every Poisson kernel of the form fits the device's shared memory
template <typename T>
bool poisson_fits(int nx, int ny, int nz);

// Records a CUDA failure for impz_last_cuda_error and returns IMPZ_ERR_CUDA
// (for translation units other than the C-ABI core).
int report_cuda_error(cudaError_t e, const char* where);

}  // namespace impz
