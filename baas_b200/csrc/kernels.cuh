// Small helper kernels shared by the C ABI entry points.
#pragma once

#include "device_common.cuh"

namespace baas {

// x[r * ldx + row] = sentinel for every right-hand side r: arms the value-as-flag slots of a
// sweep's output before the sweep kernel runs.
template <typename T>
__global__ void k_fill_sentinel(T *x, int n, int nrhs, int ldx) {
    const long long total = (long long)n * nrhs;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / n, row = i - r * n;
        x[r * ldx + row] = Sent<T>::value();
    }
}

}  // namespace baas
