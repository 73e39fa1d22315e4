// impz_device.cuh -- device helpers shared by the kernel headers.
#pragma once
#include <cuda_runtime.h>

namespace impz {

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization (launch_pdl) may be scheduled while the previous kernel on
// its stream drains; it waits here, before reading anything that kernel
// wrote.  For an ordinary launch this returns at once.
__device__ __forceinline__ void griddep_wait() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

}  // namespace impz
