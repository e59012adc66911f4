// nbg_grid.cu — column-compacted device grid over quantised int32 coordinates.
//
// Replaces the reference's KD3 build on the query side (PointView::build3dIndex,
// pdal/PointView.cpp:264-290) and the fork's Morton-key CUB sort
// (src/index/SpatialIndexKernels.cu:1772-1906).
//
// Airborne point clouds are 2.5-dimensional with walls, vegetation and wires:
// a dense 3D cell table over the tile's bounding box is mostly empty, and
// capping it forces cells far larger than the neighbourhoods.  Here every
// (cx, cy) column keeps a dense run of cells over its own occupied z-range
// only:
//   colinfo[col] = {base, zmin, zmax}      (one 16-byte load per column)
//   cell (cx, cy, cz) -> table entry base + cz - zmin, for zmin <= cz <= zmax
//   cstart[entry]     first point of the cell in the sorted point array
// so a query finds any cell with two dependent loads and scans, per column,
// one contiguous z-run of cells.  The build is a counting sort keyed by the
// table entry:
//   1. bbox      min/max of the raw coordinates
//   2. config    cell edge from the planar density, grid dims (device)
//   3. zrange    per-column min/max cell layer (atomics)
//   4. bases     exclusive scan of the column extents -> table size T
//   5. count     table entry per point, histogram
//   6. scan      exclusive scan of the histogram -> cstart
//   7. scatter   points into cell order as float4 {x, y, z, id} relative to
//                the tile minimum (exact: extents < 2^24)
// Within-cell order is not fixed; no output depends on it (neighbour sets are
// exact, covariance sums are exact integers).
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

// Cell edge c = ceil(cell_factor * r_k), r_k the radius holding k1 points on
// a surface of the tile's planar density; grown only when the column count
// exceeds the directory.
__global__ void grid_config_kernel(const int32_t* bb, uint64_t n, int k1, float cell_factor,
                                   uint64_t cols_cap, int32_t fixed_cell, GridParams* gp) {
    GridParams g;
    g.minx = bb[0];
    g.miny = bb[1];
    g.minz = bb[2];
    g.maxx = bb[3];
    g.maxy = bb[4];
    g.maxz = bb[5];
    const double ex = (double)g.maxx - g.minx + 1.0;
    const double ey = (double)g.maxy - g.miny + 1.0;
    const double ez = (double)g.maxz - g.minz + 1.0;
    double c;
    if (fixed_cell > 0) {
        c = fixed_cell;
    } else {
        const double rho2 = (double)n / (ex * ey);
        const double r = sqrt((double)k1 / (3.14159265358979 * rho2));
        c = ceil((double)cell_factor * r);
    }
    if (c < 1.0) c = 1.0;
    g.cap_hit = 0;
    for (;;) {
        const double gx = floor((ex - 1.0) / c) + 1.0;
        const double gy = floor((ey - 1.0) / c) + 1.0;
        if (gx * gy <= (double)cols_cap) {
            g.gx = (int32_t)gx;
            g.gy = (int32_t)gy;
            g.gz = (int32_t)(floor((ez - 1.0) / c) + 1.0);
            break;
        }
        c = ceil(c * 1.25 + 1.0);
        g.cap_hit = 1;
    }
    g.cell = (int32_t)c;
    g.ncols = (uint32_t)g.gx * (uint32_t)g.gy;
    *gp = g;
}

__global__ void col_init_kernel(uint32_t ncols_cap, int4* __restrict__ colinfo) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncols_cap;
         c += gridDim.x * blockDim.x)
        colinfo[c] = make_int4(0, INT32_MAX, -1, 0);
}

__global__ void col_zrange_kernel(const int32_t* __restrict__ x, const int32_t* __restrict__ y,
                                  const int32_t* __restrict__ z, uint64_t n,
                                  const GridParams* __restrict__ gpp, int4* __restrict__ colinfo) {
    const GridParams g = *gpp;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t cx = (uint32_t)(x[i] - g.minx) / (uint32_t)g.cell;
        const uint32_t cy = (uint32_t)(y[i] - g.miny) / (uint32_t)g.cell;
        const int cz = (int)((uint32_t)(z[i] - g.minz) / (uint32_t)g.cell);
        int4* ci = &colinfo[cy * (uint32_t)g.gx + cx];
        atomicMin(&ci->y, cz);
        atomicMax(&ci->z, cz);
    }
}

__global__ void col_extent_kernel(const GridParams* __restrict__ gpp,
                                  const int4* __restrict__ colinfo, uint32_t* __restrict__ ext) {
    const uint32_t ncols = gpp->ncols;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c <= ncols;
         c += gridDim.x * blockDim.x) {
        uint32_t e = 0;
        if (c < ncols) {
            const int4 ci = colinfo[c];
            e = ci.z >= ci.y ? (uint32_t)(ci.z - ci.y + 1) : 0u;
        }
        ext[c] = e;
    }
}

__global__ void col_base_kernel(const GridParams* __restrict__ gpp, const uint32_t* __restrict__ ext,
                                int4* __restrict__ colinfo, uint32_t* __restrict__ table_size) {
    const uint32_t ncols = gpp->ncols;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c <= ncols;
         c += gridDim.x * blockDim.x) {
        if (c < ncols) colinfo[c].x = (int)ext[c];
        else *table_size = ext[c];
    }
}

// Table entry of every point and the per-entry histogram.  An entry at or
// beyond `entries` (a table too small for this grid: only the build that does
// not read the table size first can see one) sets bit 2 of cap_hit and is
// dropped; the caller rebuilds such a grid.
__global__ void cell_count_kernel(const int32_t* __restrict__ x, const int32_t* __restrict__ y,
                                  const int32_t* __restrict__ z, uint64_t n, GridParams* gpp,
                                  const int4* __restrict__ colinfo, uint32_t* __restrict__ keys,
                                  uint32_t* __restrict__ counts, uint64_t entries) {
    const GridParams g = *gpp;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t cx = (uint32_t)(x[i] - g.minx) / (uint32_t)g.cell;
        const uint32_t cy = (uint32_t)(y[i] - g.miny) / (uint32_t)g.cell;
        const int cz = (int)((uint32_t)(z[i] - g.minz) / (uint32_t)g.cell);
        const int4 ci = colinfo[cy * (uint32_t)g.gx + cx];
        const uint32_t key = (uint32_t)ci.x + (uint32_t)(cz - ci.y);
        if ((uint64_t)key >= entries) {
            keys[i] = 0xFFFFFFFFu;
            atomicOr(&gpp->cap_hit, 2u);
            continue;
        }
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
        if (keys[i] == 0xFFFFFFFFu) continue;
        const uint32_t pos = atomicAdd(&cursor[keys[i]], 1u);
        float4 r;
        r.x = (float)(x[i] - g.minx);
        r.y = (float)(y[i] - g.miny);
        r.z = (float)(z[i] - g.minz);
        r.w = __uint_as_float((uint32_t)i);
        sorted[pos] = r;
    }
}

static int grid_blocks(uint64_t n, int threads, int sms, int per_sm = 8) {
    uint64_t b = (n + threads - 1) / threads;
    uint64_t cap = (uint64_t)sms * per_sm;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// Bytes of CUB scan storage for `items` entries.
size_t grid_temp_bytes(uint64_t items) {
    size_t b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (int)items);
    return b + 256;
}

// Builds the grid of `t` on `stream`.  One host synchronisation reads the
// table size T (sum of the column extents); the table grows when needed.
int build_grid(Context* ctx, Tile* t, int k1, cudaStream_t stream) {
    const uint64_t n = t->n;
    const int sms = ctx->sm_count;
    const int nb = grid_blocks(n, 256, sms);
    // the scatter waits on a returned atomic per point: more resident threads
    // keep more of those round trips in flight
    const int sb = grid_blocks(n, 256, sms, 32);
    bbox_init_kernel<<<1, 32, 0, stream>>>(t->bbox);
    bbox_kernel<<<nb, 256, 0, stream>>>(t->x, t->y, t->z, n, t->bbox);
    grid_config_kernel<<<1, 1, 0, stream>>>(t->bbox, n, k1, t->cell_factor, t->cols_cap,
                                            t->fixed_cell, t->gp);
    const int cb = grid_blocks(t->cols_cap + 1, 256, sms);
    col_init_kernel<<<cb, 256, 0, stream>>>((uint32_t)t->cols_cap, t->colinfo);
    col_zrange_kernel<<<nb, 256, 0, stream>>>(t->x, t->y, t->z, n, t->gp, t->colinfo);
    col_extent_kernel<<<cb, 256, 0, stream>>>(t->gp, t->colinfo, t->ext);
    size_t tmp = t->grid_tmp_bytes;
    if (cub::DeviceScan::ExclusiveSum(t->grid_tmp, tmp, t->ext, t->ext, (int)(t->cols_cap + 1),
                                      stream))
        return NBG_ERR_CUDA;
    col_base_kernel<<<cb, 256, 0, stream>>>(t->gp, t->ext, t->colinfo, t->table_dev);
    uint32_t T = 0;
    if (cudaMemcpyAsync(&T, t->table_dev, 4, cudaMemcpyDeviceToHost, stream) ||
        cudaStreamSynchronize(stream))
        return NBG_ERR_CUDA;
    if ((uint64_t)T + 1 > t->table_cap) {
        int rc = grid_grow_table(ctx, t, (uint64_t)T + 1);
        if (rc) return rc;
    }
    t->table_size = T;
    if (cudaMemsetAsync(t->cstart, 0, ((size_t)T + 1) * sizeof(uint32_t), stream))
        return NBG_ERR_CUDA;
    cell_count_kernel<<<nb, 256, 0, stream>>>(t->x, t->y, t->z, n, t->gp, t->colinfo, t->keys,
                                              t->cstart, (uint64_t)T + 1);
    tmp = t->grid_tmp_bytes;
    if (cub::DeviceScan::ExclusiveSum(t->grid_tmp, tmp, t->cstart, t->cstart, (int)(T + 1),
                                      stream))
        return NBG_ERR_CUDA;
    if (cudaMemcpyAsync(t->cursor, t->cstart, ((size_t)T + 1) * sizeof(uint32_t),
                        cudaMemcpyDeviceToDevice, stream))
        return NBG_ERR_CUDA;
    cell_scatter_kernel<<<sb, 256, 0, stream>>>(t->x, t->y, t->z, n, t->gp, t->keys, t->cursor,
                                                t->sorted);
    // bbox (2), config, col init, zrange, extent, scan (2), bases, count, scan (2), scatter
    NBG_LAUNCHED(13);
    return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
}

// The same build without reading the table size on the host (no
// synchronisation, so it can be captured in a CUDA graph): the histogram and
// its scan cover the whole table capacity.  A grid whose table would not fit
// sets bit 2 of cap_hit; the caller rebuilds it with build_grid.
int build_grid_async(Context* ctx, Tile* t, int k1, cudaStream_t stream) {
    const uint64_t n = t->n;
    const int sms = ctx->sm_count;
    const int nb = grid_blocks(n, 256, sms);
    // the scatter waits on a returned atomic per point: more resident threads
    // keep more of those round trips in flight
    const int sb = grid_blocks(n, 256, sms, 32);
    const uint64_t entries = t->table_cap - 1;  // cstart needs entries + 1 slots
    bbox_init_kernel<<<1, 32, 0, stream>>>(t->bbox);
    bbox_kernel<<<nb, 256, 0, stream>>>(t->x, t->y, t->z, n, t->bbox);
    grid_config_kernel<<<1, 1, 0, stream>>>(t->bbox, n, k1, t->cell_factor, t->cols_cap,
                                            t->fixed_cell, t->gp);
    const int cb = grid_blocks(t->cols_cap + 1, 256, sms);
    col_init_kernel<<<cb, 256, 0, stream>>>((uint32_t)t->cols_cap, t->colinfo);
    col_zrange_kernel<<<nb, 256, 0, stream>>>(t->x, t->y, t->z, n, t->gp, t->colinfo);
    col_extent_kernel<<<cb, 256, 0, stream>>>(t->gp, t->colinfo, t->ext);
    size_t tmp = t->grid_tmp_bytes;
    if (cub::DeviceScan::ExclusiveSum(t->grid_tmp, tmp, t->ext, t->ext, (int)(t->cols_cap + 1),
                                      stream))
        return NBG_ERR_CUDA;
    col_base_kernel<<<cb, 256, 0, stream>>>(t->gp, t->ext, t->colinfo, t->table_dev);
    if (cudaMemsetAsync(t->cstart, 0, (size_t)(entries + 1) * sizeof(uint32_t), stream))
        return NBG_ERR_CUDA;
    cell_count_kernel<<<nb, 256, 0, stream>>>(t->x, t->y, t->z, n, t->gp, t->colinfo, t->keys,
                                              t->cstart, entries);
    tmp = t->grid_tmp_bytes;
    if (cub::DeviceScan::ExclusiveSum(t->grid_tmp, tmp, t->cstart, t->cstart, (int)(entries + 1),
                                      stream))
        return NBG_ERR_CUDA;
    if (cudaMemcpyAsync(t->cursor, t->cstart, (size_t)(entries + 1) * sizeof(uint32_t),
                        cudaMemcpyDeviceToDevice, stream))
        return NBG_ERR_CUDA;
    cell_scatter_kernel<<<sb, 256, 0, stream>>>(t->x, t->y, t->z, n, t->gp, t->keys, t->cursor,
                                                t->sorted);
    NBG_LAUNCHED(13);
    t->table_size = entries;
    return cudaGetLastError() == cudaSuccess ? NBG_OK : NBG_ERR_CUDA;
}

}  // namespace nbg
