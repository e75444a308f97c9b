// group_f.cu -- the FP32 group launches (several contexts' RK4 stages as one grid
// per kernel).
#include "group_tu.cuh"

template struct chswe::GroupTU<float>;
