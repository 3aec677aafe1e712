#pragma once
// GraphOne API on libgraphone_b200: include this header, write a ComponentX,
// a BlasFunctor or AdvanceFunctor and a frontier, and call Run (reference:
// graph_one.h).  Kernels are compiled for sm_100a; link with
// -lgraphone_b200.

#include <thrust/functional.h>
#include <thrust/iterator/counting_iterator.h>

#include "GraphOne/type.hpp"
#include "GraphOne/macros.h"
#include "GraphOne/utils/string.hpp"
#include "GraphOne/utils/limits.hpp"
#include "GraphOne/utils/log.hpp"
#include "GraphOne/utils/cli.hpp"
#include "GraphOne/base/buffer.h"
#include "GraphOne/archi/archi.cuh"
#include "GraphOne/archi/blas/spmv/spmv.h"
#include "GraphOne/loader/loader.h"
#include "GraphOne/graph/graph.h"
#include "GraphOne/base/component.h"
#include "GraphOne/frontier/frontier.h"
#include "GraphOne/engine/advance_gc.h"
#include "GraphOne/engine/blas_gc.h"
#include "GraphOne/base/run.h"
