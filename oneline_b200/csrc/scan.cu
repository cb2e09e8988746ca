// Exclusive scan of the columns of a small row-major matrix of per-tile
// counts: one block of 1024 threads per column; thread t owns a contiguous run
// of rows, so the column is read and written once, in order.
#include <cuda_runtime.h>

#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

__global__ void __launch_bounds__(1024) scan_columns_kernel(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                                                            uint32_t *__restrict__ totals, uint32_t rows, uint32_t stride) {
    __shared__ uint32_t warp_sum[32];
    const uint32_t c = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t per = (rows + 1023) / 1024;
    const uint32_t lo = min(rows, tid * per), hi = min(rows, lo + per);
    uint32_t sum = 0;
    for (uint32_t r = lo; r < hi; r++) sum += in[(size_t)r * stride + c];
    uint32_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if ((int)lane >= o) inc += t;
    }
    if (lane == 31) warp_sum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sum[lane], wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, wi, o);
            if ((int)lane >= o) wi += t;
        }
        warp_sum[lane] = wi - w;  // exclusive over warps
        if (lane == 31 && totals) totals[c] = wi;
    }
    __syncthreads();
    uint32_t run = warp_sum[warp] + inc - sum;
    for (uint32_t r = lo; r < hi; r++) {
        uint32_t v = in[(size_t)r * stride + c];
        out[(size_t)r * stride + c] = run;
        run += v;
    }
}

cudaError_t launch_scan_columns(const uint32_t *in, uint32_t *out, uint32_t *totals, uint32_t rows, uint32_t cols,
                                uint32_t stride, cudaStream_t st) {
    if (rows == 0 || cols == 0) return cudaSuccess;
    scan_columns_kernel<<<cols, 1024, 0, st>>>(in, out, totals, rows, stride);
    return cudaGetLastError();
}

}  // namespace ol
