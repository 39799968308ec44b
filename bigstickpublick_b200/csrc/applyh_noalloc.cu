// bsg_applyh_noalloc: applyH on host vectors without any device allocation.
//
// Some callers of this library cannot allocate device memory at the point
// where they need a matvec: hosts whose device memory is handed out by a
// fixed-budget pool owned by another component (the pool takes the free
// memory at start-up, so a later cudaMalloc fails or steals from it), and
// Fortran/C drivers that must not grow the device footprint after set-up.
// bsg_applyh with host pointers stages vin/vout in device buffers that it
// allocates on first use; this entry point stages them instead in one
// file-scope __device__ array of fixed size that exists from the moment the
// library is loaded on a device until the process exits.
//
// Limits and contract:
//  * each staged vector (dim * nb * element size) must fit in
//    BSG_NOALLOC_MAX_VECTOR_BYTES; larger calls are rejected with
//    BSG_ERR_ARG before anything is copied;
//  * the call is synchronous: it copies vin in, runs the matvec and copies
//    vout back on the context's stream, then waits for that stream (a stream
//    that cannot be waited on gets BSG_ERR_ARG before anything is queued);
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, with that device current);
//  * the row tiles of the context are used when an earlier bsg_applyh or
//    bsg_lanczos call on the context built them; otherwise the tile list is
//    written into the same static array, which holds at most
//    kTileBytes / sizeof(Tile) = 65536 row tiles (a context with more gets
//    BSG_ERR_ARG; an applyH made on it during set-up, when allocation is
//    still allowed, caches its tiles and lifts the limit);
//  * every call on every context of the process shares the array and leaves
//    its contents behind; the kernel writes every output element, so nothing
//    needs clearing, but two calls that overlap on the GPU (other host threads
//    or other streams) race on the array.

#include <cstring>
#include <mutex>
#include <vector>

#include "bsg_internal.h"

namespace {

constexpr size_t kVecBytes = BSG_NOALLOC_MAX_VECTOR_BYTES;
constexpr size_t kTileBytes = 1u << 20;  // 65536 row tiles
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[2 * kVecBytes + kTileBytes];

std::mutex g_mu;
void *g_addr[kMaxDevices] = {nullptr};

// device address of g_noalloc_scratch on the current device (set-up on the
// first call per device)
int scratch_address(bsg_ctx *ctx, void **out) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (ctx->device < 0 || ctx->device >= kMaxDevices)
        return bsg::set_err(ctx, BSG_ERR_ARG, "bsg_applyh_noalloc: device ordinal out of range");
    if (!g_addr[ctx->device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return bsg::cuda_check(ctx, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_addr[ctx->device] = p;
    }
    *out = g_addr[ctx->device];
    return BSG_OK;
}

thread_local unsigned char *t_tile_region = nullptr;
thread_local cudaStream_t t_stream = nullptr;
thread_local bsg::TileSet t_static_tiles;

// the context's cached tiles when present, else the list written into the
// static array (no device allocation either way)
const bsg::TileSet *static_tiles(bsg_ctx *ctx, int tp) {
    auto it = ctx->tiles.find(tp);
    if (it != ctx->tiles.end()) return &it->second;
    std::vector<bsg::Tile> tiles;
    bsg::build_tile_list(ctx, tp, tiles);
    const size_t bytes = tiles.size() * sizeof(bsg::Tile);
    if (bytes > kTileBytes) {
        bsg::set_err(ctx, BSG_ERR_ARG,
                     "bsg_applyh_noalloc: " + std::to_string(tiles.size()) + " row tiles exceed the static array's " +
                         std::to_string(kTileBytes / sizeof(bsg::Tile)) +
                         "; an applyH on this context during set-up caches its tiles and lifts the limit");
        return nullptr;
    }
    cudaError_t e = cudaMemcpyAsync(t_tile_region, tiles.data(), bytes, cudaMemcpyHostToDevice, t_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t_stream);
    if (e != cudaSuccess) {
        bsg::cuda_check(ctx, e, "bsg_applyh_noalloc tile upload");
        return nullptr;
    }
    t_static_tiles.buf.p = t_tile_region;
    t_static_tiles.buf.bytes = kTileBytes;
    t_static_tiles.ntiles = (int32_t)tiles.size();
    return &t_static_tiles;
}

}  // namespace

extern "C" int bsg_applyh_noalloc(bsg_ctx *ctx, const void *vin, void *vout, int nb, int prec, int flags) {
    if (!ctx) return BSG_ERR_ARG;
    if (!vin || !vout || nb < 1 || nb > 64 || (prec != BSG_PREC_FP32 && prec != BSG_PREC_FP64))
        return bsg::set_err(ctx, BSG_ERR_ARG, "bsg_applyh_noalloc: bad arguments");
    if (flags & BSG_DEVICE_PTRS)
        return bsg::set_err(ctx, BSG_ERR_ARG, "bsg_applyh_noalloc takes host vectors only");
    const size_t bytes = (size_t)ctx->dim * (size_t)nb * (prec == BSG_PREC_FP32 ? 4u : 8u);
    if (bytes > kVecBytes)
        return bsg::set_err(ctx, BSG_ERR_ARG,
                            "bsg_applyh_noalloc: a vector of " + std::to_string(bytes) +
                                " bytes exceeds the static staging limit of " + std::to_string(kVecBytes) + " bytes");
    int st = bsg::cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (st) return st;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if ((st = bsg::cuda_check(ctx, cudaStreamIsCapturing(ctx->stream, &cap), "cudaStreamIsCapturing"))) return st;
    if (cap != cudaStreamCaptureStatusNone)
        return bsg::set_err(ctx, BSG_ERR_ARG,
                            "bsg_applyh_noalloc synchronizes its stream and cannot run while the stream is captured");
    void *base = nullptr;
    if ((st = scratch_address(ctx, &base))) return st;
    unsigned char *in = (unsigned char *)base, *out = in + kVecBytes;
    t_tile_region = in + 2 * kVecBytes;
    t_stream = ctx->stream;
    const int acc = (flags & BSG_ACCUMULATE) ? 1 : 0;
    cudaStream_t s = ctx->stream;
    st = bsg::cuda_check(ctx, cudaMemcpyAsync(in, vin, bytes, cudaMemcpyHostToDevice, s), "H2D vin");
    if (!st && acc) st = bsg::cuda_check(ctx, cudaMemcpyAsync(out, vout, bytes, cudaMemcpyHostToDevice, s), "H2D vout");
    if (!st) st = bsg::launch_applyh(ctx, in, out, nb, prec, acc, s, static_tiles);
    if (!st) st = bsg::cuda_check(ctx, cudaMemcpyAsync(vout, out, bytes, cudaMemcpyDeviceToHost, s), "D2H vout");
    if (!st) st = bsg::cuda_check(ctx, cudaStreamSynchronize(s), "bsg_applyh_noalloc sync");
    return st;
}
