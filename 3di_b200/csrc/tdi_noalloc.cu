// Visibility of one frame without any device allocation (tdi_raster_noalloc in tdi.h).
//
// Some callers of this library cannot call cudaMalloc: a plugin hosted by an application
// that owns every byte of device memory through its own pool and only lends out buffers,
// code that runs with a device-memory budget fixed before it starts, or a per-frame loop
// that must not stall on the allocator. tdi_batch_raster needs a batch, and a batch
// allocates its working set. This entry point takes the frame's projected vertices and
// triangles and writes the fragment list into buffers the caller already owns; its own
// working memory -- the 64-bit depth-key buffer of the 256x256 crop and one fragment count
// per triangle -- is a fixed array compiled into the library's device image.
//
// Limits and sharing rules:
//  * at most NOALLOC_MAX_TRIANGLES (131,072) triangles; larger meshes are rejected;
//  * the array costs 640 KiB on every device that loads the library, until the process ends;
//  * every call on a device uses the same array. Each call first resets the depth keys, so
//    nothing carries over between calls, but two calls whose kernels overlap on the GPU
//    (different streams, or different host threads) race on the array and give undefined
//    fragments. Serialise calls on one stream.
//  * the triangle corners are caller-owned device memory that the host cannot check: a
//    triangle with a corner outside [0, n_vertices) is skipped on the device before any
//    vertex is read and the call's flags get TDI_FLAG_BAD_INDEX;
//  * every call looks up the array's device address (cudaGetSymbolAddress, which allocates
//    nothing) with the caller's device current, so a device reset between calls is safe. The
//    first call on a device also loads the library's device code there; make that first call
//    before any stream capture begins.

namespace tdi {

constexpr int NOALLOC_MAX_TRIANGLES = 131072;
constexpr int NA_RC = 8;          // blocks of the frame's cluster
constexpr int NA_WARPS = 32;      // warps per block

struct NoAllocScratch {
    unsigned long long zbuf[NPIX];                 // depth keys of the crop (512 KiB)
    uint8_t tri_cnt[NOALLOC_MAX_TRIANGLES];        // fragments per triangle (128 KiB)
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// The batch raster's algorithm for a single frame, as one cluster: same fragment order, same
// slot order, same owner rule, with the scratch above and the caller's output arrays (16-byte records: pixel | owner<<31,
// triangle, float bits of alpha and beta).
__global__ void __cluster_dims__(NA_RC, 1, 1) __launch_bounds__(1024)
k_raster_noalloc(const float *xp, const float *yp, const float *zc, const int32_t *tl, int V, int T,
                 int x0, int y0, NoAllocScratch *scr, int32_t *frags, int capacity,
                 int32_t *count, uint32_t *flags_out)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    __shared__ uint32_t s_cnt[NA_WARPS][NTMP];
    __shared__ uint32_t s_off[NA_WARPS][NTMP];
    __shared__ uint32_t s_blk[NTMP];
    __shared__ int s_bbox[4];
    __shared__ uint32_t s_flags;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    DModel dm{};
    dm.T = T;
    dm.tl = tl;
    unsigned long long *zb = scr->zbuf;
    uint8_t *cnt8 = scr->tri_cnt;
    if (tid == 0) {
        s_flags = 0;
        s_bbox[0] = s_bbox[2] = 1 << 30;
        s_bbox[1] = s_bbox[3] = -1;
    }
    // the array keeps the previous call's keys: reset them (every key below compares smaller)
    for (int p = rank * 1024 + tid; p < NPIX; p += NA_RC * 1024) zb[p] = ~0ull;
    __threadfence();
    cluster.sync();
    const uint32_t tag = 0;
    const int gwarps = NA_RC * NA_WARPS;
    const int per_warp = ((T + gwarps * 32 - 1) / (gwarps * 32)) * 32;
    const int t_begin = (rank * NA_WARPS + warp) * per_warp;
    const int t_end = min(T, t_begin + per_warp);
    uint32_t flags = 0;
    int bx0 = 1 << 30, bx1 = -1, by0 = 1 << 30, by1 = -1;

    for (int base = t_begin; base < t_end; base += 32) {
        const int idx = base + lane;
        if (idx < t_end) {
            // corners outside the vertex arrays: the triangle has no fragments and no vertex
            // is read; the passes below skip it through its zero count
            const bool ok = (uint32_t)tl[idx] < (uint32_t)V && (uint32_t)tl[T + idx] < (uint32_t)V &&
                            (uint32_t)tl[2 * T + idx] < (uint32_t)V;
            uint16_t pix[NTMP]; float al[NTMP], be[NTMP];
            int nf = 0;
            if (ok) nf = tri_fragments(dm, xp, yp, idx, x0, y0, pix, al, be, flags);
            else flags |= FLAG_BAD_INDEX;
            cnt8[idx] = (uint8_t)nf;
            if (nf) {
                const float Z = zc[tl[idx]];
                if (!(Z > 0.0f)) flags |= FLAG_OUT_OF_DOMAIN;
                const unsigned long long key = zkey(tag, Z, idx);
                for (int r = 0; r < nf; ++r) atomicMin(zb + pix[r], key);
            }
        }
    }
    __threadfence();
    cluster.sync();

    uint32_t cnt[NTMP] = {0, 0, 0, 0};
    for (int base = t_begin; base < t_end; base += 32) {
        const int idx = base + lane;
        bool sv[NTMP] = {false, false, false, false};
        if (idx < t_end && cnt8[idx]) {
            uint16_t pix[NTMP]; float al[NTMP], be[NTMP];
            uint32_t fl2 = 0;
            const int nf = tri_fragments(dm, xp, yp, idx, x0, y0, pix, al, be, fl2);
            const uint32_t zbits = __float_as_uint(zc[tl[idx]]) & 0x7FFFFFFFu;
            for (int r = 0; r < nf; ++r)
                sv[r] = survives(__ldcg(zb + pix[r]), tag, zbits) && !(r == 0 && idx == 0);
        }
#pragma unroll
        for (int r = 0; r < NTMP; ++r) cnt[r] += __popc(__ballot_sync(0xffffffffu, sv[r]));
    }
    if (lane == 0)
        for (int r = 0; r < NTMP; ++r) s_cnt[warp][r] = cnt[r];
    __syncthreads();
    if (tid < NTMP) {
        uint32_t tot = 0;
        for (int w = 0; w < NA_WARPS; ++w) { s_off[w][tid] = tot; tot += s_cnt[w][tid]; }
        s_blk[tid] = tot;
    }
    cluster.sync();
    uint32_t rowbase[NTMP], blkoff[NTMP];
    {
        uint32_t tot[NTMP] = {0, 0, 0, 0};
        for (int q = 0; q < NA_RC; ++q) {
            const uint32_t *rb = cluster.map_shared_rank(s_blk, q);
            for (int r = 0; r < NTMP; ++r) {
                const uint32_t v = rb[r];
                if (q == rank) blkoff[r] = tot[r];
                tot[r] += v;
            }
        }
        uint32_t acc = 0;
        for (int r = 0; r < NTMP; ++r) { rowbase[r] = acc; acc += tot[r]; }
        if (tid == 0 && rank == 0) {
            *count = (int32_t)min(acc, (uint32_t)capacity);
            uint32_t fl = 0;
            if (acc > (uint32_t)capacity) fl |= FLAG_OVERFLOW;
            if (acc < 1000u || acc > 52000u) fl |= FLAG_RENDER_SKIPPED;
            if (acc > 25600u) fl |= FLAG_OUT_OF_DOMAIN;
            atomicOr(&s_flags, fl);
        }
    }

    uint32_t run[NTMP] = {0, 0, 0, 0};
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int base = t_begin; base < t_end; base += 32) {
        const int idx = base + lane;
        bool sv[NTMP] = {false, false, false, false};
        bool own[NTMP] = {false, false, false, false};
        uint16_t pix[NTMP]; float al[NTMP], be[NTMP];
        if (idx < t_end && cnt8[idx]) {
            uint32_t fl2 = 0;
            const int nf = tri_fragments(dm, xp, yp, idx, x0, y0, pix, al, be, fl2);
            const float Z = zc[tl[idx]];
            const uint32_t zbits = __float_as_uint(Z) & 0x7FFFFFFFu;
            const unsigned long long mykey = zkey(tag, Z, idx);
            for (int r = 0; r < nf; ++r) {
                const unsigned long long k = __ldcg(zb + pix[r]);
                sv[r] = survives(k, tag, zbits) && !(r == 0 && idx == 0);
                own[r] = (k == mykey);
            }
        }
#pragma unroll
        for (int r = 0; r < NTMP; ++r) {
            const unsigned mask = __ballot_sync(0xffffffffu, sv[r]);
            if (sv[r]) {
                const uint32_t pos = rowbase[r] + blkoff[r] + s_off[warp][r] + run[r] + __popc(mask & lt_mask);
                if (pos < (uint32_t)capacity) {
                    int32_t *o = frags + (size_t)pos * 4;
                    o[0] = (int32_t)((uint32_t)pix[r] | (own[r] ? 0x80000000u : 0u));
                    o[1] = idx;
                    o[2] = __float_as_int(al[r]);
                    o[3] = __float_as_int(be[r]);
                }
                const int px = pix[r] >> 8, py = pix[r] & 255;
                bx0 = min(bx0, px); bx1 = max(bx1, px);
                by0 = min(by0, py); by1 = max(by1, py);
            }
            run[r] += __popc(mask);
        }
    }
    if (flags) atomicOr(&s_flags, flags);
    if (bx1 >= 0) {
        atomicMin(&s_bbox[0], bx0); atomicMax(&s_bbox[1], bx1);
        atomicMin(&s_bbox[2], by0); atomicMax(&s_bbox[3], by1);
    }
    cluster.sync();
    if (tid == 0 && rank == 0) {
        int bb[4] = {1 << 30, -1, 1 << 30, -1};
        uint32_t fl = 0;
        for (int q = 0; q < NA_RC; ++q) {
            const int *rb = cluster.map_shared_rank(s_bbox, q);
            bb[0] = min(bb[0], rb[0]); bb[1] = max(bb[1], rb[1]);
            bb[2] = min(bb[2], rb[2]); bb[3] = max(bb[3], rb[3]);
            fl |= *cluster.map_shared_rank(&s_flags, q);
        }
        if (bb[1] >= 0 && (bb[0] < 1 || bb[1] > DIM - 2 || bb[2] < 1 || bb[3] > DIM - 2))
            fl |= FLAG_OUT_OF_DOMAIN;
        *flags_out = fl;
    }
    cluster.sync();
}

}  // namespace tdi

extern "C" tdi_status tdi_raster_noalloc(const float *xp, const float *yp, const float *zc,
                                         const int32_t *triangles, int32_t n_vertices,
                                         int32_t n_triangles, int32_t x0, int32_t y0,
                                         int32_t *fragments, int32_t capacity, int32_t *count,
                                         uint32_t *flags, void *stream)
{
    using namespace tdi;
    if (!xp || !yp || !zc || !triangles || !fragments || !count || !flags)
        return fail(TDI_ERR_INVALID, "tdi_raster_noalloc: null pointer");
    if (n_vertices <= 0 || n_triangles <= 0 || capacity <= 0)
        return fail(TDI_ERR_INVALID, "tdi_raster_noalloc: sizes must be positive");
    if (n_triangles > NOALLOC_MAX_TRIANGLES)
        return fail(TDI_ERR_CAPACITY, "tdi_raster_noalloc: at most 131072 triangles (fixed working array)");
    // The array's name is only a host-side stand-in: the kernel needs its address on the
    // current device, looked up on every call (no allocation; valid after a device reset).
    NoAllocScratch *scr = nullptr;
    cudaError_t e0 = cudaGetSymbolAddress((void **)&scr, g_noalloc_scratch);
    if (e0 != cudaSuccess)
        return fail(TDI_ERR_CUDA, std::string("tdi_raster_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e0));
    k_raster_noalloc<<<NA_RC, 1024, 0, (cudaStream_t)stream>>>(xp, yp, zc, triangles, n_vertices, n_triangles,
                                                            x0, y0, scr, fragments, capacity, count, flags);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(TDI_ERR_CUDA, std::string("tdi_raster_noalloc: launch: ") + cudaGetErrorString(e));
    return TDI_OK;
}
