// Exclusive scan of the columns of a small row-major matrix of per-tile
// counts ([rows][stride], first `cols` columns): one block of 1024 threads
// per column. Thread t owns a contiguous run of rows; all of its loads are
// issued before any is used, so the scan costs about two memory round trips
// however many tiles there are.
#include <cuda_runtime.h>

#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

constexpr uint32_t SC_THREADS = 1024;
constexpr uint32_t SC_BATCH = 16;  // rows loaded per batch, per thread

__global__ void __launch_bounds__(SC_THREADS) scan_columns_kernel(const uint32_t *__restrict__ in,
                                                                  uint32_t *__restrict__ out,
                                                                  uint32_t *__restrict__ totals, uint32_t rows,
                                                                  uint32_t stride) {
    __shared__ uint32_t warp_sum[32];
    const uint32_t c = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t per = (rows + SC_THREADS - 1) / SC_THREADS;
    const uint32_t lo = min(rows, tid * per), hi = min(rows, lo + per);
    uint32_t sum = 0;
    for (uint32_t r0 = lo; r0 < hi; r0 += SC_BATCH) {
        uint32_t v[SC_BATCH];
#pragma unroll
        for (uint32_t i = 0; i < SC_BATCH; i++) v[i] = r0 + i < hi ? __ldg(in + (size_t)(r0 + i) * stride + c) : 0u;
#pragma unroll
        for (uint32_t i = 0; i < SC_BATCH; i++) sum += v[i];
    }
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
    for (uint32_t r0 = lo; r0 < hi; r0 += SC_BATCH) {
        uint32_t v[SC_BATCH];
#pragma unroll
        for (uint32_t i = 0; i < SC_BATCH; i++) v[i] = r0 + i < hi ? __ldg(in + (size_t)(r0 + i) * stride + c) : 0u;
#pragma unroll
        for (uint32_t i = 0; i < SC_BATCH; i++) {
            if (r0 + i < hi) out[(size_t)(r0 + i) * stride + c] = run;
            run += v[i];
        }
    }
}

cudaError_t launch_scan_columns(const uint32_t *in, uint32_t *out, uint32_t *totals, uint32_t rows, uint32_t cols,
                                uint32_t stride, cudaStream_t st) {
    if (rows == 0 || cols == 0) return cudaSuccess;
    scan_columns_kernel<<<cols, SC_THREADS, 0, st>>>(in, out, totals, rows, stride);
    return cudaGetLastError();
}

}  // namespace ol
