// ref_prelude.h -- forced include (-include) for every build of the
// reference's sources here (oracle/build_ref.sh, baseline/build_ref_gpu.sh).
// It includes, before the reference's own headers, the standard and Thrust
// headers whose content CUDA 8 brought in transitively (FLT_MAX, DBL_MAX,
// thrust::count ...).  Included first, they are also read before src/types.h
// defines float_t as a macro (types.h:69), which would otherwise break the C++
// library's own float_t in <cmath>.
#pragma once
#include <cassert>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cuda_runtime.h>
#include <thrust/count.h>
#include <thrust/device_ptr.h>
#include <thrust/device_vector.h>
#include <thrust/extrema.h>
#include <thrust/functional.h>
#include <thrust/reduce.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>
