// nbg_las.cu — direct LAS ingest: the public header block and the point
// records' raw X/Y/Z decoded on the device into a tile.
//
// Replaces the reader step of the fork's LAS path (records mapped and decoded
// on the device: src/io/las/LasKernels.cu:266-321, src/pdal/PdgNeighborhood.cpp:
// 1115-1192).  The coordinates stay the LAS file's own int32 values, scaled by
// the header's scale and offset, so the reference sees raw*scale+offset in
// double exactly as its LAS reader gives them.  Layout facts follow the ASPRS
// LAS 1.0-1.4 specification: the header fields at fixed offsets below, and
// every point record format (0-10) beginning with X, Y, Z as little-endian
// int32 at bytes 0, 4, 8.
#include <cuda_runtime.h>

#include <cstring>

#include "nbg_internal.h"

namespace nbg {

namespace {

template <class T>
T rd(const unsigned char* b, size_t off) {
    T v;
    std::memcpy(&v, b + off, sizeof(T));
    return v;
}

// Records (any alignment) -> x, y, z.
__global__ void las_decode_kernel(const unsigned char* __restrict__ rec, uint64_t n, uint32_t rl,
                                  int32_t* __restrict__ x, int32_t* __restrict__ y,
                                  int32_t* __restrict__ z) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned char* p = rec + i * rl;
        uint32_t v[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            v[d] = (uint32_t)p[4 * d] | ((uint32_t)p[4 * d + 1] << 8) | ((uint32_t)p[4 * d + 2] << 16) |
                   ((uint32_t)p[4 * d + 3] << 24);
        x[i] = (int32_t)v[0];
        y[i] = (int32_t)v[1];
        z[i] = (int32_t)v[2];
    }
}

}  // namespace

}  // namespace nbg

using namespace nbg;

extern "C" int nbg_las_header(const void* bytes, size_t size, nbg_las_info* info) {
    if (!bytes || !info) return NBG_ERR_INVALID;
    std::memset(info, 0, sizeof(*info));
    const unsigned char* b = (const unsigned char*)bytes;
    if (size < 227 || std::memcmp(b, "LASF", 4) != 0) return NBG_ERR_INVALID;
    info->version_major = b[24];
    info->version_minor = b[25];
    const uint16_t header_size = rd<uint16_t>(b, 94);
    info->offset_to_points = rd<uint32_t>(b, 96);
    const uint8_t fmt = b[104];
    info->compressed = (fmt & 0xC0) ? 1 : 0;  // LAZ marks compression in the top bits
    info->point_format = (uint8_t)(fmt & 0x3F);
    info->point_record_length = rd<uint16_t>(b, 105);
    uint64_t count = rd<uint32_t>(b, 107);
    if (info->version_major == 1 && info->version_minor >= 4 && header_size >= 255 && size >= 255) {
        const uint64_t c64 = rd<uint64_t>(b, 247);
        if (c64) count = c64;
    }
    info->point_count = count;
    for (int d = 0; d < 3; ++d) {
        info->scale[d] = rd<double>(b, 131 + 8 * d);
        info->offset[d] = rd<double>(b, 155 + 8 * d);
        info->max[d] = rd<double>(b, 179 + 16 * d);
        info->min[d] = rd<double>(b, 187 + 16 * d);
    }
    if (info->point_format > 10 || info->point_record_length < 12) return NBG_ERR_INVALID;
    return NBG_OK;
}

extern "C" int nbg_tile_upload_las(nbg_context* h, const void* records, uint64_t n,
                                   uint32_t record_length, int32_t on_device, const double scale[3],
                                   const double offset[3], void* stream_v, nbg_tile** out) {
    if (!h || !out) return NBG_ERR_INVALID;
    Context* ctx = &h->c;
    std::lock_guard<std::mutex> lock(ctx->mu);
    *out = nullptr;
    if (n && !records) return fail(ctx, NBG_ERR_INVALID, "null record buffer");
    if (record_length < 12) return fail(ctx, NBG_ERR_INVALID, "LAS point records hold at least X, Y, Z");
    nbg_tile* th = nullptr;
    int rc = tile_alloc(ctx, n, scale, offset, &th);
    if (rc) return rc;
    Tile* t = &th->t;
    cudaStream_t stream = (cudaStream_t)stream_v;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, ctx->sm_count * 8));
    if (n && on_device) {
        las_decode_kernel<<<grid, 256, 0, stream>>>((const unsigned char*)records, n, record_length,
                                                     t->x, t->y, t->z);
        NBG_LAUNCHED(1);
        if (cudaGetLastError() != cudaSuccess) rc = fail(ctx, NBG_ERR_CUDA, "LAS decode launch");
    } else if (n) {
        // host records: staged in chunks of whole records through device scratch
        const uint64_t chunk_recs = std::max<uint64_t>(1, ((uint64_t)64 << 20) / record_length);
        const uint64_t chunk_bytes = chunk_recs * record_length;
        unsigned char* stage = nullptr;
        rc = ctx_alloc(ctx, (void**)&stage, chunk_bytes);
        for (uint64_t b = 0; !rc && b < n; b += chunk_recs) {
            const uint64_t m = std::min(chunk_recs, n - b);
            rc = host_to_device(ctx, stage, (const unsigned char*)records + b * record_length,
                                m * record_length, stream);
            if (rc) break;
            las_decode_kernel<<<grid, 256, 0, stream>>>(stage, m, record_length, t->x + b, t->y + b,
                                                         t->z + b);
            NBG_LAUNCHED(1);
            if (cudaGetLastError() != cudaSuccess) rc = fail(ctx, NBG_ERR_CUDA, "LAS decode launch");
        }
        // the scratch may be reused only once the last decode has read it
        if (cudaStreamSynchronize(stream) != cudaSuccess && !rc) rc = fail(ctx, NBG_ERR_CUDA, "LAS decode");
        if (stage) ctx_free(ctx, stage, chunk_bytes);
    }
    if (rc) {
        tile_destroy(ctx, th);
        return rc;
    }
    *out = th;
    return NBG_OK;
}
