// fused_f.cu -- the FP32 fused stage and edge-strip kernels (every configuration and RK mode).
#include "fused_tu.cuh"

template struct chswe::FusedTU<float>;
