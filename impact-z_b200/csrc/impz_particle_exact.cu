// Plain FP64 form of the particle kernels: compiled with --fmad=false so
// every FP64 operation rounds like the reference's x86-64 build.
#define IMPZ_NS exact
#include "impz_particle_impl.cuh"
