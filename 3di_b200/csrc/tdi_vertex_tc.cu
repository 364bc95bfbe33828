// Vertex stage on the 5th-generation tensor cores (tdi_fit_config.vertex_stage = 1).
//
// The batched vertex stage is the product [3V x K] . [K x F] of the expression basis with the
// coefficients of the frames that render (renderer.cu:806-861 forms it per frame with
// cublasSgemv), followed per vertex and frame by the mean shape, the camera transform and the
// projection. Here the product runs on tcgen05: every FP32 value is split exactly into three
// BF16 pieces (the basis once, when the model is created; the coefficients per launch) and the
// six products hh, hm, mh, mm, hl, lh are accumulated in FP32 in tensor memory (the omitted
// ml, lm, ll are at or below 2^-24 of the product). The sum order differs from the exact
// stage's sequential fused multiply-add chain, so vertex positions agree with it to FP32
// accumulation error, not bit for bit: this is the mixed-precision mode of the fit.
//
// One block per SM, persistent over vertex tiles of 32 vertices for a tile of 128 frames:
// the tensor-core tile is M = 128 rows (x, y, z rows of the 32 vertices and 32 rows that are
// never read) by N = 128 frames by K (the coefficients, padded to a multiple of 16).
//   warp 16, one thread: bulk copies of the pre-split basis tiles (46 KB) into two buffers,
//     the 30 MMAs of a tile into one of two tensor-memory accumulators, commits;
//   warps 0-15: the epilogue -- tensor memory -> shared memory (x, y, z of each vertex and
//     frame; warp w reads lane group w % 4, frame quarter w / 4), then mean + product,
//     rotation, translation and projection per vertex and frame, written as the exact stage
//     writes them (geometry and projection records). Sixteen warps keep enough stores in
//     flight; the stage is bound by those stores.
// The copy of tile j + 2, the MMAs of tile j + 1 and the epilogue of tile j overlap. Every
// mbarrier wait gives up after about a second: the block sets the batch's error word, waits
// (again bounded) for its copies and MMAs in flight and frees its tensor memory.

namespace tdi {

constexpr int VC_V = 32;                          // vertices per tile
constexpr int VC_F = 128;                         // frames per block (the MMA's N)
constexpr int VC_M = 128;                         // accumulator rows (x, y, z rows + 32 unused)
constexpr int VC_EPI_WARPS = 16;                  // four per tensor-memory lane group
constexpr int VC_THREADS = (VC_EPI_WARPS + 1) * 32;
constexpr int VC_MAXK = 80;                       // coefficients supported (K padded to 16)
constexpr int VC_ROWGROUPS = 3 * VC_V / 8;        // 12 groups of 8 rows hold data
constexpr int VC_TMEM_COLS = 2 * VC_F;            // two accumulators

__host__ __device__ __forceinline__ int vc_k16(int K) { return (K + 15) & ~15; }
// bytes of one BF16 piece of a basis tile: 12 row groups x K/8 core matrices of 128 bytes
__host__ __device__ __forceinline__ int vc_piece(int K) { return VC_ROWGROUPS * (vc_k16(K) / 8) * 128; }
__host__ __device__ __forceinline__ int vc_tile_bytes(int K) { return 3 * vc_piece(K); }
// a tile buffer: the three pieces and the tail that the MMA's unused rows 96-127 of the last
// piece address (their values never reach a read accumulator row)
__host__ __device__ __forceinline__ int vc_abuf(int K) { return 3 * vc_piece(K) + 4 * (vc_k16(K) / 8) * 128; }
__host__ __device__ __forceinline__ int vc_bpiece(int K) { return (VC_F / 8) * (vc_k16(K) / 8) * 128; }
__host__ __device__ __forceinline__ size_t vc_smem(int K)
{
    return (size_t)2 * vc_abuf(K) + 3 * (size_t)vc_bpiece(K) + (size_t)3 * VC_F * VC_V * sizeof(float) +
           (size_t)VC_F * VT_FR * sizeof(float);
}

// Byte offset of element (row r, column k) in a K-major, no-swizzle operand whose core
// matrices (8 rows x 8 BF16) are ordered K-fastest: the layout umma_desc(lbo 128, sbo KG*128)
// describes.
__host__ __device__ __forceinline__ uint32_t vc_off(int r, int k, int KG)
{
    return (uint32_t)((r >> 3) * KG + (k >> 3)) * 128u + (uint32_t)(r & 7) * 16u + (uint32_t)(k & 7) * 2u;
}

// The pre-split basis: per vertex tile t, per piece p (hi, mid, lo), rows 32c + i = coordinate c
// of vertex 32t + i (zero past the last vertex), one thread per (tile, row, k pair).
__global__ void k_split_basis(DModel m, int ntiles, __nv_bfloat16 *out)
{
    const int K16 = vc_k16(m.K), KG = K16 / 8, piece = vc_piece(m.K);
    const size_t total = (size_t)ntiles * 3 * VC_V * (K16 / 2);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int kp = (int)(i % (K16 / 2));
        const size_t rest = i / (K16 / 2);
        const int r = (int)(rest % (3 * VC_V));
        const int t = (int)(rest / (3 * VC_V));
        const int c = r / VC_V, v = t * VC_V + (r % VC_V);
        uint8_t *tile = reinterpret_cast<uint8_t *>(out) + (size_t)t * 3 * piece;
        __nv_bfloat16 h[2], mm[2], l[2];
        for (int u = 0; u < 2; ++u) {
            const int k = 2 * kp + u;
            const float x = (v < m.V && k < m.K) ? m.E[((size_t)v * 3 + c) * m.KP + k] : 0.0f;
            split3(x, h[u], mm[u], l[u]);
        }
        const uint32_t o = vc_off(r, 2 * kp, KG);
        *reinterpret_cast<uint32_t *>(tile + o) = pack2(h[0], h[1]);
        *reinterpret_cast<uint32_t *>(tile + piece + o) = pack2(mm[0], mm[1]);
        *reinterpret_cast<uint32_t *>(tile + 2 * piece + o) = pack2(l[0], l[1]);
    }
}

__device__ __forceinline__ void vc_bar_sync_epi()
{
    asm volatile("bar.sync 1, %0;" :: "n"(VC_EPI_WARPS * 32) : "memory");
}

__global__ void __launch_bounds__(VC_THREADS, 1) k_vertex_tc(DModel m, DBatch b, const __nv_bfloat16 *Etc)
{
    extern __shared__ __align__(1024) uint8_t vcsm[];
    const int K = m.K, K16 = vc_k16(K), KG = K16 / 8;
    const int ABUF = vc_abuf(K), BPIECE = vc_bpiece(K), TILE = vc_tile_bytes(K), PIECE = vc_piece(K);
    uint8_t *Ab = vcsm;                                    // [2][ABUF]
    uint8_t *Bb = Ab + 2 * ABUF;                           // [3][BPIECE]
    float *Ex = reinterpret_cast<float *>(Bb + 3 * BPIECE);   // [3][VC_F][VC_V]
    float *Fs = Ex + 3 * VC_F * VC_V;                      // [VC_F][VT_FR]
    __shared__ int s_render[VC_F], s_frame[VC_F];
    __shared__ int s_any;
    __shared__ volatile int s_abort;                       // set by the producer
    __shared__ int s_epi_abort;                            // set by epilogue warps before a barrier only
    __shared__ int s_tma, s_mma;                           // tiles copied / multiplied (producer)
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t s_full[2], s_mma_bar[2], s_free[2];

    const int ntiles = (m.V + VC_V - 1) / VC_V;
    const int rc = b.rcount[0];
    const int ftiles = (rc + VC_F - 1) / VC_F;
    if (ftiles == 0) return;
    const int groups = max(1, min(ntiles, (int)gridDim.x / ftiles));
    if ((int)blockIdx.x >= ftiles * groups) return;
    const int gy = blockIdx.x / ftiles;
    const int f0 = (blockIdx.x - gy * ftiles) * VC_F;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool producer = warp == VC_EPI_WARPS;
    if (tid == 0) { s_any = 0; s_abort = 0; s_epi_abort = 0; s_tma = 0; s_mma = 0; }
    __syncthreads();
    if (tid < VC_F) {
        const int ai = f0 + tid;
        const int f = ai < rc ? b.rlist[ai] : -1;
        const int r = f >= 0 && b.ctl[f].render;
        s_frame[tid] = f;
        s_render[tid] = r;
        if (r) {
            s_any = 1;
            if (gy == 0) prof_count(b, KID_VERTEX);
        }
    }
    __syncthreads();
    if (!s_any) return;                                    // uniform: nothing allocated yet
    const uint32_t full0 = smem_addr(&s_full[0]), mma0 = smem_addr(&s_mma_bar[0]), free0 = smem_addr(&s_free[0]);
    if (producer) {
        // the whole warp allocates the two accumulators
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_addr(&s_tmem)), "r"(VC_TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        if (lane == 0) {
            for (int i = 0; i < 2; ++i) {
                mbar_init(full0 + 8u * i, 1);
                mbar_init(mma0 + 8u * i, 1);
                mbar_init(free0 + 8u * i, 1);
            }
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    } else {
        // coefficients of the block's frames: three BF16 pieces in the B operand's layout
        // (rows = frames), and the per-frame rotation, translation and camera
        for (int i = tid; i < VC_F * (K16 / 2); i += VC_EPI_WARPS * 32) {
            const int fl = i / (K16 / 2), kp = i - fl * (K16 / 2);
            const int f = s_frame[fl];
            __nv_bfloat16 h[2], mm[2], l[2];
            for (int u = 0; u < 2; ++u) {
                const int k = 2 * kp + u;
                const float x = (f >= 0 && k < K) ? b.xe[(size_t)f * m.KTP + k] : 0.0f;
                split3(x, h[u], mm[u], l[u]);
            }
            const uint32_t o = vc_off(fl, 2 * kp, KG);
            *reinterpret_cast<uint32_t *>(Bb + o) = pack2(h[0], h[1]);
            *reinterpret_cast<uint32_t *>(Bb + BPIECE + o) = pack2(mm[0], mm[1]);
            *reinterpret_cast<uint32_t *>(Bb + 2 * BPIECE + o) = pack2(l[0], l[1]);
        }
        for (int i = tid; i < VC_F * VT_FR; i += VC_EPI_WARPS * 32) {
            const int fl = i / VT_FR, j = i - fl * VT_FR;
            const int f = s_frame[fl];
            float v = 0.0f;
            if (f >= 0) v = j < 9 ? b.R[f * 9 + j] : j < 12 ? b.xe[(size_t)f * m.KTP + K + (j - 9)] : b.cam[f * 4 + (j - 12)];
            Fs[i] = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // B is read by the MMAs
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;

    if (producer) {
        if (lane == 0) {
            const uint32_t abase = smem_addr(Ab), bbase = smem_addr(Bb);
            const uint32_t idesc = umma_idesc_bf16(VC_M, VC_F);
            const uint32_t sbo = (uint32_t)KG * 128u, lbo = 128u;
            auto copy_tile = [&](int j) {
                const int t = gy + j * groups;
                const uint32_t bar = full0 + 8u * (uint32_t)(j & 1);
                mbar_expect_tx(bar, (uint32_t)TILE);
                bulk_g2s(abase + (uint32_t)(j & 1) * (uint32_t)ABUF,
                         reinterpret_cast<const uint8_t *>(Etc) + (size_t)t * TILE, (uint32_t)TILE, bar);
                s_tma = j + 1;
            };
            for (int j = 0; j < 2 && gy + j * groups < ntiles; ++j) copy_tile(j);
            for (int j = 0;; ++j) {
                const int t = gy + j * groups;
                if (t >= ntiles || s_abort) break;
                const int buf = j & 1;
                bool ok = mbar_wait(full0 + 8u * buf, (uint32_t)((j >> 1) & 1));
                if (ok && j >= 2) ok = mbar_wait(free0 + 8u * buf, (uint32_t)(((j - 2) >> 1) & 1));
                if (!ok) { s_abort = 1; atomicOr(b.err, 4); break; }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(buf * VC_F);
                const uint32_t a0 = abase + (uint32_t)(buf * ABUF);
                for (int ks = 0; ks < KG / 2; ++ks) {
                    const uint32_t o = (uint32_t)ks * 256u;
                    const uint64_t ah = umma_desc(a0 + o, lbo, sbo);
                    const uint64_t am = umma_desc(a0 + (uint32_t)PIECE + o, lbo, sbo);
                    const uint64_t al = umma_desc(a0 + 2u * (uint32_t)PIECE + o, lbo, sbo);
                    const uint64_t bh = umma_desc(bbase + o, lbo, sbo);
                    const uint64_t bm = umma_desc(bbase + (uint32_t)BPIECE + o, lbo, sbo);
                    const uint64_t bl = umma_desc(bbase + 2u * (uint32_t)BPIECE + o, lbo, sbo);
                    umma_bf16(d, ah, bh, idesc, ks > 0 ? 1u : 0u);
                    umma_bf16(d, ah, bm, idesc, 1u);
                    umma_bf16(d, am, bh, idesc, 1u);
                    umma_bf16(d, am, bm, idesc, 1u);
                    umma_bf16(d, ah, bl, idesc, 1u);
                    umma_bf16(d, al, bh, idesc, 1u);
                }
                umma_commit(mma0 + 8u * buf);
                s_mma = j + 1;
                // refill this buffer with tile j + 2 once the MMAs above have read it
                if (gy + (j + 2) * groups < ntiles) {
                    if (!mbar_wait(mma0 + 8u * buf, (uint32_t)((j >> 1) & 1))) { s_abort = 1; atomicOr(b.err, 4); break; }
                    copy_tile(j + 2);
                }
            }
        }
    } else {
        const int lg = warp & 3, qt = warp >> 2;           // tensor-memory lane group, frame quarter
        for (int j = 0;; ++j) {
            const int t = gy + j * groups;
            if (t >= ntiles) break;
            const int buf = j & 1;
            const int v = t * VC_V + lane;
            float mx = 0.0f, my = 0.0f, mz = 0.0f, tx = 0.0f;
            if (v < m.V) { mx = m.mean[v]; my = m.mean[m.V + v]; mz = m.mean[2 * m.V + v]; tx = m.tex[v]; }
            const bool w = mbar_wait(mma0 + 8u * buf, (uint32_t)((j >> 1) & 1));
            if (!__all_sync(0xffffffffu, w)) {
                if (lane == 0) { s_epi_abort = 1; s_abort = 1; atomicOr(b.err, 4); }
            }
            vc_bar_sync_epi();
            // s_epi_abort is written only before this barrier, so every epilogue thread reads the
            // same value (a producer-side failure reaches the epilogue as a wait that gave up)
            if (s_epi_abort) break;
            tc_fence_after();
            if (lg < 3) {
                // rows 32 lg + lane: coordinate lg of vertex `lane`, frames of this quarter
                constexpr int QF = VC_F / 4;
                const uint32_t taddr = tmem + ((uint32_t)(32 * lg) << 16) + (uint32_t)(buf * VC_F + qt * QF);
#pragma unroll
                for (int cb = 0; cb < QF; cb += 16) {
                    float vv[16];
                    tmem_ld16(taddr + (uint32_t)cb, vv);
#pragma unroll
                    for (int i = 0; i < 16; ++i) Ex[(lg * VC_F + qt * QF + cb + i) * VC_V + lane] = vv[i];
                }
            }
            tc_fence_before();
            vc_bar_sync_epi();
            if (tid == 0) mbar_arrive(free0 + 8u * buf);   // the accumulator may be overwritten
            if (v < m.V) {
                for (int fl = warp; fl < VC_F; fl += VC_EPI_WARPS) {
                    if (!s_render[fl]) continue;
                    const int f = s_frame[fl];
                    const float *R = Fs + fl * VT_FR, *tau = R + 9, *cam = R + 12;
                    const float X0 = mx + Ex[(0 * VC_F + fl) * VC_V + lane];
                    const float Y0 = my + Ex[(1 * VC_F + fl) * VC_V + lane];
                    const float Z0 = mz + Ex[(2 * VC_F + fl) * VC_V + lane];
                    const float X3 = ((R[0] * X0 + R[3] * Y0) + R[6] * Z0) + tau[0];
                    const float Y3 = ((R[1] * X0 + R[4] * Y0) + R[7] * Z0) + tau[1];
                    const float Z3 = ((R[2] * X0 + R[5] * Y0) + R[8] * Z0) + tau[2];
                    b.geo[(size_t)f * m.V + v] = make_float4(X0, Y0, Z0, tx);
                    b.proj[(size_t)f * m.V + v] = make_float4((cam[0] * X3) / Z3 + cam[2], (cam[1] * Y3) / Z3 + cam[3], Z3, 0.0f);
                }
            }
            vc_bar_sync_epi();                             // shared staging is free for the next tile
        }
    }
    tc_fence_before();
    __syncthreads();
    if (producer) {
        if (lane == 0) {
            // bounded waits for the copies and MMAs this block issued and has not seen finish
            // (after an abort), so that shared and tensor memory are released idle
            for (int j = max(0, s_tma - 2); j < s_tma; ++j) mbar_wait(full0 + 8u * (uint32_t)(j & 1), (uint32_t)((j >> 1) & 1));
            if (s_mma > 0) mbar_wait(mma0 + 8u * (uint32_t)((s_mma - 1) & 1), (uint32_t)(((s_mma - 1) >> 1) & 1));
        }
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(VC_TMEM_COLS) : "memory");
    }
}

}  // namespace tdi
