/* Pre-included before the reference's math header when building the pin harness (test
 * infrastructure).  CUDA 12 removed texture references; the header's unused helper
 * fetch_double(texture<int2,1>, int) still names them, so this declares a stand-in type
 * with no behaviour.  Nothing in the harness calls it. */
#pragma once
#include <cuda_runtime.h>
template <class T, int D = 1, int M = 0> struct texture {};
template <class T, int D, int M> __device__ int2 tex1Dfetch(texture<T, D, M>, int)
{
    return make_int2(0, 0);
}
