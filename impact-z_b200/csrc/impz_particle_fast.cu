// FP32-convolution form of the particle kernels: contraction allowed.
#define IMPZ_NS fast
// maps and kick may use reciprocals and rsqrt instead of IEEE divisions
#define IMPZ_FASTMATH 1
#include "impz_particle_impl.cuh"
