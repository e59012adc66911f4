// nbg_grid.cu — device uniform grid over quantised int32 coordinates.
//
// Replaces the reference's KD3 build on the query side (PointView::build3dIndex,
// pdal/PointView.cpp:264-290) and the fork's Morton-key CUB sort
// (src/index/SpatialIndexKernels.cu:1772-1906).  The build is a single-digit
// radix (counting) sort keyed by the linear cell index:
//   1. bbox      min/max of the raw coordinates (warp reductions + atomics)
//   2. config    cell size and grid dims chosen on the device (no host sync)
//   3. count     cell key per point, histogram of keys
//   4. scan      exclusive prefix sum of the histogram = cell start table
//   5. scatter   points into cell order as float4 {x, y, z, id} relative to
//                the tile minimum (exact: extents < 2^24 raw units)
// Within-cell order is not fixed; no output depends on it (neighbour sets
// are exact, covariance sums are exact integers).
#include <cub/cub.cuh>

#include "nbg_common.cuh"
#include "nbg_internal.h"

namespace nbg {

__global__ void bbox_init_kernel(int32_t* bb) {
    if (threadIdx.x < 3) bb[threadIdx.x] = INT32_MAX;
    else if (threadIdx.x < 6) bb[threadIdx.x] = INT32_MIN;
}

__global__ void bbox_kernel(const int32_t* __restrict__ x, const int32_t* __restrict__ y,
                            const int32_t* __restrict__ z, uint64_t n, int32_t* bb) {
    int32_t lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX};
    int32_t hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        int32_t v[3] = {x[i], y[i], z[i]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            lo[d] = min(lo[d], v[d]);
            hi[d] = max(hi[d], v[d]);
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        lo[d] = __reduce_min_sync(0xffffffffu, lo[d]);
        hi[d] = __reduce_max_sync(0xffffffffu, hi[d]);
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            atomicMin(&bb[d], lo[d]);
            atomicMax(&bb[3 + d], hi[d]);
        }
    }
}

// Cell edge c = ceil(cell_factor * r_k), r_k the radius holding k1 points
// on a surface of the tile's planar density; grown until the table fits.
__global__ void grid_config_kernel(const int32_t* bb, uint64_t n, int k1, float cell_factor,
                                   uint64_t ncells_cap, int32_t fixed_cell, GridParams* gp) {
    GridParams g;
    g.minx = bb[0];
    g.miny = bb[1];
    g.minz = bb[2];
    g.maxx = bb[3];
    g.maxy = bb[4];
    g.maxz = bb[5];
    double ex = (double)g.maxx - g.minx + 1.0;
    double ey = (double)g.maxy - g.miny + 1.0;
    double ez = (double)g.maxz - g.minz + 1.0;
    double c;
    if (fixed_cell > 0) {
        c = fixed_cell;
    } else {
        double rho2 = (double)n / (ex * ey);
        double r = sqrt((double)k1 / (3.14159265358979 * rho2));
        c = ceil((double)cell_factor * r);
    }
    if (c < 1.0) c = 1.0;
    g.cap_hit = 0;
    for (;;) {
        double gx = floor((ex - 1.0) / c) + 1.0;
        double gy = floor((ey - 1.0) / c) + 1.0;
        double gz = floor((ez - 1.0) / c) + 1.0;
        if (gx * gy * gz <= (double)ncells_cap) {
            g.gx = (int32_t)gx;
            g.gy = (int32_t)gy;
            g.gz = (int32_t)gz;
            break;
        }
        c = ceil(c * 1.25 + 1.0);
        g.cap_hit = 1;
    }
    g.cell = (int32_t)c;
    g.ncells = (uint32_t)g.gx * (uint32_t)g.gy * (uint32_t)g.gz;
    *gp = g;
}

__global__ void cell_count_kernel(const int32_t* __restrict__ x, const int32_t* __restrict__ y,
                                  const int32_t* __restrict__ z, uint64_t n,
                                  const GridParams* __restrict__ gpp, uint32_t* __restrict__ keys,
                                  uint32_t* __restrict__ counts) {
    const GridParams g = *gpp;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t cx = (uint32_t)(x[i] - g.minx) / (uint32_t)g.cell;
        uint32_t cy = (uint32_t)(y[i] - g.miny) / (uint32_t)g.cell;
        uint32_t cz = (uint32_t)(z[i] - g.minz) / (uint32_t)g.cell;
        uint32_t key = (cz * (uint32_t)g.gy + cy) * (uint32_t)g.gx + cx;
        keys[i] = key;
        atomicAdd(&counts[key], 1u);
    }
}

__global__ void cell_scatter_kernel(const int32_t* __restrict__ x, const int32_t* __restrict__ y,
                                    const int32_t* __restrict__ z, uint64_t n,
                                    const GridParams* __restrict__ gpp,
                                    const uint32_t* __restrict__ keys, uint32_t* __restrict__ cursor,
                                    float4* __restrict__ sorted) {
    const GridParams g = *gpp;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t pos = atomicAdd(&cursor[keys[i]], 1u);
        float4 r;
        r.x = (float)(x[i] - g.minx);
        r.y = (float)(y[i] - g.miny);
        r.z = (float)(z[i] - g.minz);
        r.w = __uint_as_float((uint32_t)i);
        sorted[pos] = r;
    }
}

static int grid_blocks(uint64_t n, int threads, int sms) {
    uint64_t b = (n + threads - 1) / threads;
    uint64_t cap = (uint64_t)sms * 8;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// Builds the grid of `t` on `stream`.  Scratch: keys (n), counts (cap+1).
int build_grid(Context* ctx, Tile* t, int k1, cudaStream_t stream) {
    const uint64_t n = t->n;
    const int sms = ctx->sm_count;
    bbox_init_kernel<<<1, 32, 0, stream>>>(t->bbox);
    bbox_kernel<<<grid_blocks(n, 256, sms), 256, 0, stream>>>(t->x, t->y, t->z, n, t->bbox);
    grid_config_kernel<<<1, 1, 0, stream>>>(t->bbox, n, k1, t->cell_factor, t->ncells_cap,
                                            t->fixed_cell, t->gp);
    if (cudaMemsetAsync(t->cell_start, 0, (t->ncells_cap + 1) * sizeof(uint32_t), stream))
        return NBG_ERR_CUDA;
    cell_count_kernel<<<grid_blocks(n, 256, sms), 256, 0, stream>>>(t->x, t->y, t->z, n, t->gp,
                                                                   t->keys, t->cell_start);
    size_t tmp = t->scan_tmp_bytes;
    if (cub::DeviceScan::ExclusiveSum(t->scan_tmp, tmp, t->cell_start, t->cell_start,
                                      (int)(t->ncells_cap + 1), stream) != cudaSuccess)
        return NBG_ERR_CUDA;
    if (cudaMemcpyAsync(t->cursor, t->cell_start, (t->ncells_cap + 1) * sizeof(uint32_t),
                        cudaMemcpyDeviceToDevice, stream))
        return NBG_ERR_CUDA;
    cell_scatter_kernel<<<grid_blocks(n, 256, sms), 256, 0, stream>>>(
        t->x, t->y, t->z, n, t->gp, t->keys, t->cursor, t->sorted);
    NBG_LAUNCHED(7);  // five grid kernels + the two kernels of the scan
    return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
}

size_t scan_temp_bytes(uint64_t items) {
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (int)items);
    return bytes;
}

}  // namespace nbg
