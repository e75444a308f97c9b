// fused_d.cu -- the FP64 fused stage and edge-strip kernels (every configuration and RK mode).
#include "fused_tu.cuh"

template struct chswe::FusedTU<double>;
