// Normal equations on the 5th-generation tensor cores (tdi_fit_config.normal_eq = 1).
//
// H = tau * sum_k r_k r_k^T and g = -tau * sum_k w_k r_k over the 2N rows r_k of
// d(gx/|g|)/dtheta and d(gy/|g|)/dtheta with weights w_k = gxs_n, gys_n
// (derivative_computer.cu:157-163 forms them with four cublasSgemm calls). The row matrix is
// extended by one column holding w_k, so that g is the last column of the same product.
// Every FP32 value is split exactly into three BF16 pieces, x = h + m + l (8 significant bits
// each), and the six products hh, hm, mh, mm, hl, lh of each row pair are accumulated in FP32
// in tensor memory by tcgen05.mma (the omitted ml, lm, ll are at or below 2^-24 of the
// product). The chunk sums (256 fragments each) are added in FP64 in chunk order. The error
// is that of FP32 accumulation over one chunk, the same class as the reference's
// cublasSgemm; the upper triangle of each chunk sum is used, so H is symmetric.
//
// One block per (frame, chunk loop): 8 warps build 32 fragments' rows at a time into one
// shared-memory stage (K-major BF16 core matrices, no swizzle), thread 0 issues 24 MMAs
// (M=128 x N x K=16, four K slices) and commits them to an mbarrier that the next build
// waits on. Three blocks share an SM (128 tensor-memory columns each). Every mbarrier wait
// gives up after about a second: the block sets the batch's error word, waits once more for
// its MMAs and frees its tensor memory before it leaves.

namespace tdi {

constexpr int TC_THREADS = 256;
constexpr int TC_SUB = 32;                        // fragments per stage
constexpr int TC_KS = 2 * TC_SUB;                 // K rows per stage (x row, y row per fragment)
constexpr int TC_M = 128;                         // accumulator rows (parameters, zero padded)
constexpr int TC_MAXN = 128;                      // accumulator columns at most
constexpr int TC_PIECE = TC_M * TC_KS * 2;        // bytes of one BF16 piece of a stage (16 KB)
constexpr int TC_SMEM = 3 * TC_PIECE;             // dynamic shared memory: hi, mid, lo pieces
constexpr int TC_TMEM_COLS = 128;                 // the accumulator
constexpr int TC_BPF = 32;                        // blocks per frame (each loops over chunks)
static_assert(TC_THREADS == NE_CH, "one thread per fragment of a chunk");

// accumulator columns: the parameters and the weight column, rounded up to 16
__host__ __device__ __forceinline__ int tc_cols(int KT) { return (KT + 1 + 15) & ~15; }

// pitch of a chunk partial: the parameters and the weight column, rounded up to 4
__host__ __device__ __forceinline__ int tc_pitch(int KT) { return (KT + 1 + 3) & ~3; }

// bytes of one chunk partial: the upper triangle of the chunk sum, transposed, [PK][PK]
__host__ __device__ __forceinline__ size_t tc_part_bytes(int KT)
{
    return (size_t)tc_pitch(KT) * tc_pitch(KT) * sizeof(float);
}

// Shared-memory matrix descriptor, K-major, no swizzle: core matrices of 8 rows x 16 bytes;
// lbo = byte step between the two 8-element K halves, sbo = byte step between 8-row groups.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, both K-major, M x N.
__device__ __forceinline__ uint32_t umma_idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 :: "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc) : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive FP32 columns of this warp's 32 TMEM lanes (one row per thread).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                   "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Exact split of x into three BF16 pieces (hi, mid, lo), packed per piece with the y value
// of the same fragment and column (K rows 2q and 2q+1 are adjacent in a core matrix).
__device__ __forceinline__ void split3(float x, __nv_bfloat16 &h, __nv_bfloat16 &mm, __nv_bfloat16 &l)
{
    h = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(h);
    mm = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(mm);
    l = __float2bfloat16_rn(r2);
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 a, __nv_bfloat16 b)
{
    return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

template <int GRP>
__global__ void __launch_bounds__(TC_THREADS, 3) k_normal_eq_tc(DModel m, DBatch b)
{
    if ((int)blockIdx.y >= active_n(b)) return;
    const int f = b.act[blockIdx.y];
    const FrameCtl &ctl = b.ctl[f];
    if (!ctl.need_jac) return;
    const int N = ctl.N;
    const int nch = (N + NE_CH - 1) / NE_CH;
    if ((int)blockIdx.x >= nch) return;                  // the whole block leaves together
    if (blockIdx.x == 0 && threadIdx.x == 0) prof_count(b, KID_NORMAL_EQ);
    extern __shared__ __align__(1024) uint8_t tcsm[];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_tmem;
    __shared__ ChunkHead hd;
    const int KTP = m.KTP, KT = m.KT;
    const int NN = tc_cols(KT), PK = tc_pitch(KT);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t bar = smem_addr(&s_bar);

    // zero the three pieces once: rows a > KT stay zero
    for (int i = tid; i < TC_SMEM / 16; i += TC_THREADS)
        reinterpret_cast<uint4 *>(tcsm)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_addr(&s_tmem)), "r"(TC_TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = umma_idesc_bf16(TC_M, NN);
    const uint32_t sbase = smem_addr(tcsm);

    const float *Jf = b.J + (size_t)f * NMAX * KTP;
    const int32_t *nb = b.nb + (size_t)f * 4 * NMAX;
    const float *fg = b.fgrad + (size_t)f * 5 * NMAX;
    const size_t pbytes = tc_part_bytes(KT);
    uint8_t *part_base = reinterpret_cast<uint8_t *>(b.ne_part) + (size_t)f * NE_MAXCH * pbytes;
    // build mapping: thread -> fragment q of the stage, columns a = 8*g + (lane & 7)
    const int a_low = lane & 7, q_me = 4 * warp + (lane >> 3);
    uint32_t phase = 0;
    bool ok = true;

    for (int ch = blockIdx.x; ch < nch && ok; ch += gridDim.x) {
        const int c0 = ch * NE_CH, cnt = min(N, c0 + NE_CH) - c0;
        const int nsub = (cnt + TC_SUB - 1) / TC_SUB;
        __syncthreads();                          // the previous chunk is done with hd
        chunk_head(hd, fg, nb, c0, cnt);
        __syncthreads();
        for (int it = 0; it < nsub; ++it) {
            const int ql = q_me, q = it * TC_SUB + ql;
            float v[GRP][4];
            chunk_prefetch<GRP>(v, hd, Jf, KT, KTP, q, cnt, a_low);
            if (it > 0) {
                // the previous stage's MMAs must have read the pieces before they are
                // rewritten; the outcome of the wait is made uniform over the block
                const bool w = mbar_wait(bar, phase);
                if (!__syncthreads_and(w)) { ok = false; break; }
                phase ^= 1u;
            }
            {
                const bool live = q < cnt;
                const float pre = hd.pre[q], diffx = hd.dx[q], diffy = hd.dy[q];
                const uint32_t kofs = (uint32_t)(ql >> 2) * 128u + (uint32_t)(a_low * 16 + (ql & 3) * 4);
#pragma unroll
                for (int g = 0; g < GRP; ++g) {
                    const int a = 8 * g + a_low;
                    if (a > KT) continue;
                    float ox = 0.0f, oy = 0.0f;
                    if (live) {
                        if (a < KT) chain_value(v[g], pre, diffx, diffy, ox, oy);
                        else { ox = (float)hd.w[2 * q]; oy = (float)hd.w[2 * q + 1]; }
                    }
                    __nv_bfloat16 xh, xm, xl, yh, ym, yl;
                    split3(ox, xh, xm, xl);
                    split3(oy, yh, ym, yl);
                    const uint32_t off = (uint32_t)g * (TC_KS / 8) * 128u + kofs;
                    *reinterpret_cast<uint32_t *>(tcsm + off) = pack2(xh, yh);
                    *reinterpret_cast<uint32_t *>(tcsm + TC_PIECE + off) = pack2(xm, ym);
                    *reinterpret_cast<uint32_t *>(tcsm + 2 * TC_PIECE + off) = pack2(xl, yl);
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                tc_fence_after();
                const uint32_t sbo = (TC_KS / 8) * 128u, lbo = 128u;
#pragma unroll
                for (int ks = 0; ks < TC_KS / 16; ++ks) {
                    const uint32_t o = (uint32_t)ks * 256u;
                    const uint64_t ah = umma_desc(sbase + o, lbo, sbo);
                    const uint64_t am = umma_desc(sbase + TC_PIECE + o, lbo, sbo);
                    const uint64_t al = umma_desc(sbase + 2 * TC_PIECE + o, lbo, sbo);
                    umma_bf16(tmem, ah, ah, idesc, (it > 0 || ks > 0) ? 1u : 0u);
                    umma_bf16(tmem, ah, am, idesc, 1u);
                    umma_bf16(tmem, am, ah, idesc, 1u);
                    umma_bf16(tmem, am, am, idesc, 1u);
                    umma_bf16(tmem, ah, al, idesc, 1u);
                    umma_bf16(tmem, al, ah, idesc, 1u);
                }
                umma_commit(bar);
            }
        }
        if (!ok) break;
        // the chunk sum is complete
        {
            const bool w = mbar_wait(bar, phase);
            if (!__syncthreads_and(w)) { ok = false; break; }
            phase ^= 1u;
        }
        tc_fence_after();
        // upper triangle (a <= c), stored transposed so that lanes (rows a) write contiguously
        float *P = reinterpret_cast<float *>(part_base + (size_t)ch * pbytes);
        if (warp < 4) {
            const int a = 32 * warp + lane;
            const uint32_t lanebits = (uint32_t)(32 * warp) << 16;
            for (int cb = 0; cb < NN; cb += 16) {
                float v0[16];
                tmem_ld16(tmem + lanebits + (uint32_t)cb, v0);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int c = cb + i;
                    if (a <= c && c < PK) P[(size_t)c * PK + a] = v0[i];
                }
            }
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    if (!ok) {
        if (tid == 0) atomicOr(b.err, 1);
        // let MMAs still in flight finish before the tensor memory is released
        mbar_wait(bar, phase);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TC_TMEM_COLS) : "memory");
    }
}

// H = tau * (sum over chunks, in order, of the chunk sums) in FP64; g from the weight column.
// TC_RBLOCKS blocks per frame, each over a slice of the entries; the chunk values of an entry
// are loaded eight at a time.
constexpr int TC_RBLOCKS = 4;

__global__ void __launch_bounds__(256) k_normal_eq_tc_reduce(DModel m, DBatch b)
{
    if ((int)blockIdx.y >= active_n(b)) return;
    const int f = b.act[blockIdx.y];
    const FrameCtl &ctl = b.ctl[f];
    if (!ctl.need_jac) return;
    const int KTP = m.KTP, KT = m.KT, PK = tc_pitch(KT);
    const int nch = (ctl.N + NE_CH - 1) / NE_CH;
    const size_t pstride = tc_part_bytes(KT) / sizeof(float);
    const float *base = reinterpret_cast<const float *>(b.ne_part) + (size_t)f * NE_MAXCH * pstride;
    const double tau = 25.0;
    float *H = b.H + (size_t)f * KTP * KTP;
    // entry (a, c), a <= c <= KT, sits at [c][a]; consecutive threads take consecutive a
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < (KT + 1) * PK; e += gridDim.x * blockDim.x) {
        const int c = e / PK, a = e - c * PK;
        if (a > c) continue;
        const float *p = base + (size_t)c * PK + a;
        double s = 0.0;
        int q = 0;
        for (; q + 8 <= nch; q += 8) {
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = p[(size_t)(q + u) * pstride];
#pragma unroll
            for (int u = 0; u < 8; ++u) s += (double)v[u];
        }
        for (; q < nch; ++q) s += (double)p[(size_t)q * pstride];
        if (c < KT) {
            const float v = (float)(tau * s);
            H[(size_t)a * KTP + c] = v;
            H[(size_t)c * KTP + a] = v;
        } else if (a < KT) {
            b.g[(size_t)f * KTP + a] = (float)(-tau * s);
        }
    }
}

}  // namespace tdi
