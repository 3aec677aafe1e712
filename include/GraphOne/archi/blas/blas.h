#pragma once
// GraphOne's archi/blas/blas.h (its SpMV part; SpMM and GEMM serve the GNN domain): the same names, provided by
// archi/blas/spmv/spmv.h.
#include "GraphOne/archi/blas/spmv/spmv.h"
