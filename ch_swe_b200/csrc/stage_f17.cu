// stage_f17.cu -- the FP32 stage and contravariant kernels for tiles of at most
// 17 x 17 points (every blocks-per-SM, runs, SBP-order and operator variant).
#include "swe_stage_tu.cuh"

template struct chswe::StageTU<float, 17>;
