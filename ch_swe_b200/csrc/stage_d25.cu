// stage_d25.cu -- the FP64 stage and contravariant kernels for tiles of at most
// 25 x 25 points (every blocks-per-SM, runs, SBP-order and operator variant).
#include "swe_stage_tu.cuh"

template struct chswe::StageTU<double, 25>;
