#pragma once
// GraphOne's archi/thrust/thrust.h: the same names, provided by
// archi/archi.cuh.
#include "GraphOne/archi/archi.cuh"
