// Exclusive scan of the columns of a small column-major matrix of per-tile
// counts: column c holds `rows` u32 at in + c * ld (ld a multiple of 4, the
// base 16-byte aligned). Block (k, c) owns rows [4096k, 4096k + 4096) of column
// c: it sums the rows before its chunk itself (coalesced 16-byte loads of data
// the producing kernel just left in L2), scans its own chunk and writes it. No
// block waits on another; the last chunk's block writes the column total.
#include <cuda_runtime.h>

#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

constexpr uint32_t SC_THREADS = 1024;
constexpr uint32_t SC_CHUNK = SC_THREADS * 4;  // rows per block

__global__ void __launch_bounds__(SC_THREADS) scan_columns_kernel(const uint32_t *__restrict__ in,
                                                                  uint32_t *__restrict__ out,
                                                                  uint32_t *__restrict__ totals, uint32_t rows,
                                                                  uint32_t ld) {
    __shared__ uint32_t red[SC_THREADS / 32];
    __shared__ uint32_t scan[SC_THREADS / 32];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t chunk = blockIdx.x, c = blockIdx.y;
    const uint32_t *col = in + (size_t)c * ld;
    uint32_t *ocol = out + (size_t)c * ld;
    const uint32_t r0 = chunk * SC_CHUNK;

    // this thread's four rows of the chunk
    const uint32_t r = r0 + tid * 4;
    uint4 v;
    if (r + 3 < rows) {
        v = __ldg(reinterpret_cast<const uint4 *>(col + r));
    } else {
        v.x = r < rows ? __ldg(col + r) : 0u;
        v.y = r + 1 < rows ? __ldg(col + r + 1) : 0u;
        v.z = r + 2 < rows ? __ldg(col + r + 2) : 0u;
        v.w = 0u;
    }
    // rows before the chunk (whole chunks: all in range)
    uint32_t before = 0;
    const uint4 *cv = reinterpret_cast<const uint4 *>(col);
    const uint32_t nvec = r0 / 4;
    uint32_t i = tid;
    for (; i + 3 * SC_THREADS < nvec; i += 4 * SC_THREADS) {
        uint4 a = __ldg(cv + i), b = __ldg(cv + i + SC_THREADS), d = __ldg(cv + i + 2 * SC_THREADS),
              e = __ldg(cv + i + 3 * SC_THREADS);
        before += (a.x + a.y + a.z + a.w) + (b.x + b.y + b.z + b.w) + (d.x + d.y + d.z + d.w) + (e.x + e.y + e.z + e.w);
    }
    for (; i < nvec; i += SC_THREADS) {
        uint4 a = __ldg(cv + i);
        before += a.x + a.y + a.z + a.w;
    }
    const uint32_t mine = v.x + v.y + v.z + v.w;
    // warp sums of `before`, warp inclusive scan of `mine`
    uint32_t inc = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if ((int)lane >= o) inc += t;
        before += __shfl_xor_sync(0xFFFFFFFFu, before, o);
    }
    if (lane == 31) scan[warp] = inc;
    if (lane == 0) red[warp] = before;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = scan[lane], wi = w, b = red[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, wi, o);
            if ((int)lane >= o) wi += t;
            b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
        }
        scan[lane] = b + wi - w;  // chunk prefix + exclusive over warps
        if (lane == 31 && totals && chunk + 1 == gridDim.x) totals[c] = b + wi;
    }
    __syncthreads();
    uint32_t run = scan[warp] + inc - mine;
    uint4 o;
    o.x = run;
    o.y = run + v.x;
    o.z = o.y + v.y;
    o.w = o.z + v.z;
    if (r + 3 < rows) {
        *reinterpret_cast<uint4 *>(ocol + r) = o;
    } else {
        if (r < rows) ocol[r] = o.x;
        if (r + 1 < rows) ocol[r + 1] = o.y;
        if (r + 2 < rows) ocol[r + 2] = o.z;
    }
}

cudaError_t launch_scan_columns(const uint32_t *in, uint32_t *out, uint32_t *totals, uint32_t rows, uint32_t cols,
                                uint32_t ld, cudaStream_t st) {
    if (rows == 0 || cols == 0) return cudaSuccess;
    dim3 grid((rows + SC_CHUNK - 1) / SC_CHUNK, cols);
    scan_columns_kernel<<<grid, SC_THREADS, 0, st>>>(in, out, totals, rows, ld); OL_LAUNCHED();
    return cudaGetLastError();
}

}  // namespace ol
