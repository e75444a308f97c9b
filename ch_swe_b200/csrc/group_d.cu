// group_d.cu -- the FP64 group launches (several contexts' RK4 stages as one grid
// per kernel).
#include "group_tu.cuh"

template struct chswe::GroupTU<double>;
