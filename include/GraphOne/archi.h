#pragma once
// GraphOne's archi.h: the same names, provided by
// archi/archi.cuh, archi/blas/spmv/spmv.h.
#include "GraphOne/archi/archi.cuh"
#include "GraphOne/archi/blas/spmv/spmv.h"
