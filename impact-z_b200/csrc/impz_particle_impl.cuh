// Kernel instantiation and launch wrappers for one numerical form
// (included by impz_particle_exact.cu and impz_particle_fast.cu).
#include "impz_launch.h"
#include "impz_particle.cuh"

namespace impz {
namespace IMPZ_NS {

static const size_t kDepSmem = (size_t)3 * IMPZ_DEP_TILE * sizeof(unsigned int);

static const size_t kAdvSmem = (size_t)(IMPZ_ADV_BLOCK / 32) * 32 * 37 * sizeof(double);

template <bool F32, bool LIGHT, bool SP>
static cudaError_t adv_attr() {
  static cudaError_t once = cudaFuncSetAttribute(
      k_advance<IMPZ_ADV_BLOCK, F32, IMPZ_ADV_U, LIGHT, SP>,
      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kAdvSmem);
  return once;
}

template <bool F32, bool LIGHT, bool SP>
static cudaError_t launch_adv_t(const AdvanceArgs& a, int grid, cudaStream_t s) {
  cudaError_t e = adv_attr<F32, LIGHT, SP>();
  if (e != cudaSuccess) return e;
  return launch_pdl(k_advance<IMPZ_ADV_BLOCK, F32, IMPZ_ADV_U, LIGHT, SP>, dim3(grid),
                    dim3(IMPZ_ADV_BLOCK), kAdvSmem, s, a);
}

template <bool F32, bool LIGHT>
static cudaError_t launch_adv_sp(const AdvanceArgs& a, int grid, cudaStream_t s) {
  return a.sp_in ? launch_adv_t<F32, LIGHT, true>(a, grid, s)
                 : launch_adv_t<F32, LIGHT, false>(a, grid, s);
}

cudaError_t launch_advance(const AdvanceArgs& a, bool f32, bool light, int grid, cudaStream_t s) {
  if (f32) return light ? launch_adv_sp<true, true>(a, grid, s) : launch_adv_sp<true, false>(a, grid, s);
  return light ? launch_adv_sp<false, true>(a, grid, s) : launch_adv_sp<false, false>(a, grid, s);
}

template <bool F32, bool LIGHT, bool SP>
static cudaError_t launch_adv_packed_t(const AdvanceArgs* args, const int* offs, int nmem,
                                       int blocks, cudaStream_t s) {
  auto kern = k_advance_packed<IMPZ_ADV_BLOCK, F32, IMPZ_ADV_U, LIGHT, SP>;
  static cudaError_t once =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kAdvSmem);
  if (once != cudaSuccess) return once;
  return launch_pdl(kern, dim3(blocks), dim3(IMPZ_ADV_BLOCK), kAdvSmem, s, args, offs, nmem);
}

template <bool F32, bool LIGHT>
static cudaError_t launch_adv_packed_sp(const AdvanceArgs* args, const int* offs, int nmem,
                                        int blocks, bool species, cudaStream_t s) {
  return species ? launch_adv_packed_t<F32, LIGHT, true>(args, offs, nmem, blocks, s)
                 : launch_adv_packed_t<F32, LIGHT, false>(args, offs, nmem, blocks, s);
}

cudaError_t launch_advance_packed(const AdvanceArgs* args, const int* offs, int nmem, int blocks,
                                  bool f32, bool light, bool species, cudaStream_t s) {
  if (f32)
    return light ? launch_adv_packed_sp<true, true>(args, offs, nmem, blocks, species, s)
                 : launch_adv_packed_sp<true, false>(args, offs, nmem, blocks, species, s);
  return light ? launch_adv_packed_sp<false, true>(args, offs, nmem, blocks, species, s)
               : launch_adv_packed_sp<false, false>(args, offs, nmem, blocks, species, s);
}

template <bool SP>
static cudaError_t dep_attr() {
  static cudaError_t once = cudaFuncSetAttribute(
      k_deposit<IMPZ_DEP_BLOCK, IMPZ_DEP_PPT, SP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
      (int)kDepSmem);
  return once;
}

template <bool SP>
static cudaError_t launch_dep_packed_t(const DepositArgs* args, const int* offs, int nmem,
                                      int blocks, cudaStream_t s) {
  auto kern = k_deposit_packed<IMPZ_DEP_BLOCK, IMPZ_DEP_PPT, SP>;
  static cudaError_t once =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDepSmem);
  if (once != cudaSuccess) return once;
  return launch_pdl(kern, dim3(blocks), dim3(IMPZ_DEP_BLOCK), kDepSmem, s, args, offs, nmem);
}

cudaError_t launch_deposit_packed(const DepositArgs* args, const int* offs, int nmem, int blocks,
                                  bool species, cudaStream_t s) {
  return species ? launch_dep_packed_t<true>(args, offs, nmem, blocks, s)
                 : launch_dep_packed_t<false>(args, offs, nmem, blocks, s);
}

cudaError_t launch_scan_packed(const ScanArgs* args, const int* offs, int nmem, int blocks,
                               cudaStream_t s) {
  k_scan_packed<IMPZ_SCAN_THREADS><<<blocks, IMPZ_SCAN_THREADS, 0, s>>>(
      args, offs, nmem);
  return cudaGetLastError();
}

template <bool SP>
static cudaError_t launch_dep_t(const DepositArgs& a, int grid, cudaStream_t s) {
  cudaError_t e = dep_attr<SP>();
  if (e != cudaSuccess) return e;
  return launch_pdl(k_deposit<IMPZ_DEP_BLOCK, IMPZ_DEP_PPT, SP>, dim3(grid), dim3(IMPZ_DEP_BLOCK),
                    kDepSmem, s, a);
}

cudaError_t launch_deposit(const DepositArgs& a, int grid, cudaStream_t s) {
  return a.sp_in ? launch_dep_t<true>(a, grid, s) : launch_dep_t<false>(a, grid, s);
}

#define IMPZ_WAKE_BLOCK 256
static const size_t kWakeSmemMax = (size_t)6 * 4096 * sizeof(double);

cudaError_t prepare_wake() {
  static cudaError_t once = cudaFuncSetAttribute(
      k_wake_field, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWakeSmemMax);
  return once;
}

cudaError_t launch_wake(const WakeArgs& a, int grid, cudaStream_t s) {
  cudaError_t once = prepare_wake();
  if (once != cudaSuccess) return once;
  if (a.nz < 2 || (size_t)6 * a.nz * sizeof(double) > kWakeSmemMax) return cudaErrorInvalidValue;
  k_wake_line<IMPZ_WAKE_BLOCK><<<grid, IMPZ_WAKE_BLOCK, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_wake_field<<<(a.nz + 255) / 256, 256, (size_t)6 * a.nz * sizeof(double), s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_scan(int* counts, int* cursor, int* bsum, long long total, DevState* st,
                        cudaStream_t s) {
  const long long nb = (total + (1ll << IMPZ_SCAN_LOG) - 1) >> IMPZ_SCAN_LOG;
  k_scan<IMPZ_SCAN_THREADS><<<(int)nb, IMPZ_SCAN_THREADS, 0, s>>>(counts, cursor, bsum, total, st);
  return cudaGetLastError();
}

cudaError_t launch_species_count(const DepositArgs& a, int test_loss, int nspecies, int* counts,
                                 int grid, cudaStream_t s) {
  k_species_count<256><<<grid, 256, 0, s>>>(a, test_loss, nspecies, counts);
  return cudaGetLastError();
}

int max_blocks_advance(bool f32) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // the full multi-species instantiation bounds the others (at most its registers)
  if (f32) {
    adv_attr<true, false, true>();
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per, k_advance<IMPZ_ADV_BLOCK, true, IMPZ_ADV_U, false, true>, IMPZ_ADV_BLOCK, kAdvSmem);
  } else {
    adv_attr<false, false, true>();
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per, k_advance<IMPZ_ADV_BLOCK, false, IMPZ_ADV_U, false, true>, IMPZ_ADV_BLOCK, kAdvSmem);
  }
  return sms * (per > 0 ? per : 1);
}

int max_blocks_deposit() {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  dep_attr<true>();
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_deposit<IMPZ_DEP_BLOCK, IMPZ_DEP_PPT, true>,
                                                IMPZ_DEP_BLOCK, kDepSmem);
  return sms * (per > 0 ? per : 1);
}

}  // namespace IMPZ_NS
}  // namespace impz
