// FP32-convolution form of the particle kernels: contraction allowed.
#define IMPZ_NS fast
#include "impz_particle_impl.cuh"
