// cnn_tc.cu -- the network's 32-input-channel 5x5 convolutions on the fifth-generation tensor cores, with
// warp-specialised roles: TMA into a ring of input rows, one thread issuing tcgen05.mma into tensor memory, and
// four epilogue warps. For sm_100a.
//
// Work: output tiles of 4 rows x 128 pixels. A CTA takes a contiguous range of tiles down 128-pixel strips, so
// consecutive tiles share 4 of their 8 input rows: the ring holds 3 blocks of 4 input rows, and a tile that
// continues its predecessor's strip loads one new block.
//   warp 0 (one thread): per block, 4 rows x 2 channel planes as eight TMA tile loads (box 16 channels x 132
//     pixels, 32-byte swizzle, zero fill outside the image) into a free ring slot; they complete on the slot's
//     `full` barrier.
//   warp 1: allocates the tensor memory (2 accumulator sets x 4 rows x C columns, C = output channels); one
//     thread waits for the tile's two blocks and a free accumulator set and issues 80 MMAs (M = 128 pixels,
//     K = 16: one tap's 16 channels): per (input row, tap column, channel half), ONE MMA for all the tile's output
//     rows that read that slice, N = their number x C (the weights staged ky-fastest make their B blocks
//     consecutive rows; the accumulators in reverse row order make their D blocks consecutive columns). It
//     commits to the set's `tfull` barrier and to the `empty` barrier of each block no later tile reads.
//   warps 2-5: wait on `tfull`, read their 32 tensor-memory lanes (pixels) with tcgen05.ld and clear them (the
//     MMAs only accumulate), write bias + ReLU to bf16, or fp32, or the gradient times the ReLU mask, and arrive
//     on the set's `tempty` barrier.
// Every wait is bounded: on expiry the CTA sets ST_TIMEOUT and every role leaves its loop; the CTA then waits
// (bounded) for its copies and MMAs in flight before it frees the tensor memory.
//
// Operand layouts (K-major, 32-byte swizzle): an input row is two planes (channels 0-15, 16-31) of 132 pixels x
// 32 bytes; the A operand of output row r, tap (ky, kx) and channel half kc starts at input row r + ky, plane kc,
// pixel kx. The weights: per k step (tap, half), N rows of 32 bytes.
#include "cnn.cuh"

namespace vf {

namespace {

constexpr int TC_THREADS = 192;
constexpr int TC_M = 128;                  // pixels per MMA
constexpr int TC_TR = 4;                   // output rows per tile
constexpr int TC_PIX = TC_M + 4;           // pixels per staged input row
constexpr int TC_RING = 3;                 // ring blocks of TC_TR input rows
constexpr int TC_KSTEPS = CNN_TAPS * 2;    // 16-channel k steps
constexpr int TC_PLANE = (TC_PIX * 32 + 255) / 256 * 256;   // 4352: one channel half of one input row
constexpr int TC_ROWB = 2 * TC_PLANE;
constexpr int TC_BLOCKB = TC_TR * TC_ROWB;
constexpr uint32_t TC_BOX_BYTES = 16 * TC_PIX * 2;         // one TMA box: 16 channels x 132 pixels of bf16
constexpr int TC_SPINS = 1 << 22;          // mbarrier polls before a role gives up

template <int NMMA>
struct TcLayout {
    static constexpr int B_BYTES = TC_KSTEPS * NMMA * 32;
    static constexpr int NBAR = 2 * TC_RING + 4 + 1;   // full[3], empty[3], tfull[2], tempty[2], done
    static constexpr int SMEM = TC_RING * TC_BLOCKB + B_BYTES + NBAR * 8 + 16 + 1024;
    static constexpr int TCOLS = 2 * TC_TR * NMMA <= 128 ? 128 : 256;   // two accumulator sets
};

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp16(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

// K-major operand in the 32-byte swizzle: 8-row groups 256 bytes apart, version 1, layout type 6.
__device__ __forceinline__ uint64_t desc_sw32(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3fff) | ((uint64_t)1 << 16) | ((uint64_t)(256 >> 4) << 32) | (1ull << 46) |
           (6ull << 61);
}

__host__ __device__ constexpr uint32_t sw32(uint32_t r, uint32_t h) { return r * 32 + ((h ^ ((r >> 2) & 1)) << 4); }

// kind::f16 instruction descriptor: fp32 accumulate, bf16 A and B, both K-major.
__host__ __device__ constexpr uint32_t idesc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase of `parity`; on expiry sets the status and the CTA's abort flag.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_cta, uint32_t* status) {
    for (int spin = 0; spin < TC_SPINS; spin++) {
        if (mbar_try(bar, parity)) return true;
        if ((spin & 1023) == 1023 && *abort_cta) return false;
    }
    set_status(status, ST_TIMEOUT);
    *abort_cta = 1;
    return false;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// D += A B (the accumulators start at zero: the epilogue clears what it reads).
__device__ __forceinline__ void umma_acc(uint32_t tmem, uint64_t a, uint64_t b, uint32_t id) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.eq.b32 p, 0, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(id));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 32; k++) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

// Zeros into 32 (or 16) consecutive fp32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_zero32(uint32_t taddr) {
    const uint32_t z = 0;
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
        "%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1};" ::"r"(taddr),
        "r"(z)
        : "memory");
}

__device__ __forceinline__ void tmem_zero16(uint32_t taddr) {
    const uint32_t z = 0;
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
        "%1};" ::"r"(taddr),
        "r"(z)
        : "memory");
}

template <int NMMA>
__device__ __forceinline__ void tmem_zero(uint32_t taddr) {
    if constexpr (NMMA == 32) tmem_zero32(taddr);
    else tmem_zero16(taddr);
}

// The tile sequence of a CTA: tiles [t0, t1) of (sample, 128-pixel strip, 4-row quad), quads fastest.
struct TileSeq {
    int xs_n, qy_n;
    __device__ void at(int t, int& b, int& x0, int& y0) const {
        const int qy = t % qy_n, r = t / qy_n;
        y0 = qy * TC_TR;
        x0 = (r % xs_n) * TC_M;
        b = r / xs_n;
    }
    // whether tile t continues tile t - 1's strip (so shares its last input block)
    __device__ bool continues(int t, int t0) const { return t > t0 && t % qy_n != 0; }
};

}  // namespace

template <int NMMA, int COUT, int MODE>
__global__ void __launch_bounds__(TC_THREADS, 1) k_conv_tc(ConvArgs a, const __grid_constant__ CUtensorMap tmap,
                                                            uint32_t* status) {
    using L = TcLayout<NMMA>;
    constexpr int K = conv_k(32);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024 - (su32(smem_raw) & 1023)) & 1023);
    const uint32_t ring = su32(smem);                    // TC_RING blocks
    const uint32_t wts = ring + TC_RING * TC_BLOCKB;     // [k step][NMMA rows x 32 B]
    const uint32_t bars = wts + L::B_BYTES;              // mbarriers
    const uint32_t full = bars, empty = bars + 8 * TC_RING, tfull = bars + 16 * TC_RING, tempty = tfull + 16,
                   done = tempty + 16;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + TC_RING * TC_BLOCKB + L::B_BYTES + L::NBAR * 8);
    __shared__ volatile int abort_cta;
    __shared__ float bias_s[32];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // the weights once (cp.async into the swizzled K-major layout), barriers, tensor memory
    for (int i = tid; i < NMMA * (K / 8); i += TC_THREADS) {
        const int co = i / (K / 8), c = i % (K / 8), step = c / 2, half = c % 2;
        const int tap = step / 2, kc = step % 2, ky = tap / 5, kx = tap % 5;
        const int blk = (kx * 2 + kc) * 5 + ky;   // ky fastest
        cp16(wts + blk * NMMA * 32 + sw32(co, half), co < COUT ? a.w + (int64_t)co * K + c * 8 : a.w,
             co < COUT ? 16u : 0u);
    }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (tid < 32) bias_s[tid] = (MODE != CONV_GRAD_MASK && a.bias && tid < a.bias_n) ? a.bias[tid] : 0.0f;
    if (tid == 0) {
        for (int q = 0; q < TC_RING; q++) {
            mbar_init(full + 8 * q, 1);
            mbar_init(empty + 8 * q, 1);
        }
        for (int q = 0; q < 2; q++) {
            mbar_init(tfull + 8 * q, 1);
            mbar_init(tempty + 8 * q, 4);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_cta = 0;
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                     "r"(L::TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    if (warp >= 2) {   // both accumulator sets start at zero (the MMAs only accumulate)
        for (int c = 0; c < 2 * TC_TR; c++) tmem_zero<NMMA>(tmem + ((uint32_t)((warp & 3) * 32) << 16) + c * NMMA);
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    const int H = a.H, W = a.W;
    const TileSeq seq{(W + TC_M - 1) / TC_M, (H + TC_TR - 1) / TC_TR};
    const int total = a.B * seq.xs_n * seq.qy_n;
    const int t0 = (int)((int64_t)blockIdx.x * total / gridDim.x);
    const int t1 = (int)((int64_t)(blockIdx.x + 1) * total / gridDim.x);
    int issued_blocks = 0;   // producer: blocks whose copies were issued

    if (warp == 0 && lane == 0) {
        // ---- producer
        int n = 0;
        for (int t = t0; t < t1 && !abort_cta; t++) {
            int b, x0, y0;
            seq.at(t, b, x0, y0);
            const bool cont = seq.continues(t, t0);
            for (int k = cont ? 1 : 0; k < 2; k++, n++) {
                const int slot = n % TC_RING;
                if (n >= TC_RING && !mbar_wait(empty + 8 * slot, (uint32_t)((n / TC_RING - 1) & 1), &abort_cta, status))
                    break;
                const uint32_t fb = full + 8 * slot;
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb),
                             "r"(8u * TC_BOX_BYTES)
                             : "memory");
                const int row0 = y0 - 2 + 4 * k;
                for (int r = 0; r < TC_TR; r++)
                    for (int pl = 0; pl < 2; pl++) {
                        const uint32_t dst = ring + slot * TC_BLOCKB + r * TC_ROWB + pl * TC_PLANE;
                        asm volatile(
                            "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
                            "%3, %4, %5}], [%6];" ::"r"(dst),
                            "l"(&tmap), "r"(pl * 16), "r"(x0 - 2), "r"(row0 + r), "r"(b), "r"(fb)
                            : "memory");
                    }
                issued_blocks = n + 1;
            }
        }
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issue
        int fb = 0, i = 0;
        for (int t = t0; t < t1 && !abort_cta; t++, i++) {
            const bool cont = seq.continues(t, t0);
            fb = i == 0 ? 0 : cont ? fb + 1 : fb + 2;
            if (!cont && !mbar_wait(full + 8 * (fb % TC_RING), (uint32_t)((fb / TC_RING) & 1), &abort_cta, status)) break;
            if (!mbar_wait(full + 8 * ((fb + 1) % TC_RING), (uint32_t)(((fb + 1) / TC_RING) & 1), &abort_cta, status))
                break;
            const int set = i & 1;
            if (i >= 2 && !mbar_wait(tempty + 8 * set, (uint32_t)((i / 2 - 1) & 1), &abort_cta, status)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // descriptors are linear in the start address (16-byte units in the low bits, no carry below 256 KB):
            // each MMA's is the tile's block or weight base plus a compile-time offset
            const uint64_t d0 = desc_sw32(ring + (fb % TC_RING) * TC_BLOCKB);
            const uint64_t d1 = desc_sw32(ring + ((fb + 1) % TC_RING) * TC_BLOCKB);
            const uint64_t dw = desc_sw32(wts);
            const uint32_t acc = tmem + set * TC_TR * NMMA;
            // input row ir, tap column kx, channel half kc: one MMA for every output row orow = ir - ky of the
            // tile that reads the slice. The weights are staged ky-fastest, so the n taps' B blocks are n * NMMA
            // consecutive rows, and the accumulators lie in reverse row order, so the rows' D blocks are
            // consecutive columns: N = n * NMMA.
#pragma unroll
            for (int ir = 0; ir < TC_TR + 4; ir++) {
                constexpr int last = TC_TR - 1;
                const int ky0 = ir - last > 0 ? ir - last : 0, ky1 = ir < 4 ? ir : 4;
                const int n = ky1 - ky0 + 1;
                const uint32_t id = idesc(TC_M, n * NMMA);
                const uint32_t d = acc + (last - (ir - ky0)) * NMMA;
#pragma unroll
                for (int kx = 0; kx < 5; kx++)
#pragma unroll
                    for (int kc = 0; kc < 2; kc++)
                        umma_acc(d, (ir < 4 ? d0 : d1) + (uint64_t)((((ir & 3) * TC_ROWB) + kc * TC_PLANE + kx * 32) >> 4),
                                 dw + (uint64_t)((((kx * 2 + kc) * 5 + ky0) * NMMA * 32) >> 4), id);
            }
            umma_commit(tfull + 8 * set);
            umma_commit(empty + 8 * (fb % TC_RING));   // no later tile reads this tile's first block
            const bool last_of_run = t + 1 == t1 || !seq.continues(t + 1, t0);
            if (last_of_run) umma_commit(empty + 8 * ((fb + 1) % TC_RING));
        }
        umma_commit(done);   // arrives when every MMA this thread issued has completed
    } else if (warp >= 2) {
        // ---- epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31
        const int q = warp & 3;
        int i = 0;
        for (int t = t0; t < t1 && !abort_cta; t++, i++) {
            const int set = i & 1;
            if (!mbar_wait(tfull + 8 * set, (uint32_t)((i / 2) & 1), &abort_cta, status)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            int b, x0, y0;
            seq.at(t, b, x0, y0);
            const int px = x0 + q * 32 + lane;
#pragma unroll 1
            for (int orow = 0; orow < TC_TR; orow++) {
                const int py = y0 + orow;
                // row orow's accumulator: reverse row order within the set; cleared once read
                const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (set * TC_TR + TC_TR - 1 - orow) * NMMA;
                if constexpr (NMMA == 32) {
                    float v[32];
                    tmem_ld32(taddr, v);
                    tmem_zero32(taddr);
                    if (px >= W || py >= H) continue;
                    const int64_t pix = ((int64_t)b * H + py) * W + px;
                    __align__(16) __nv_bfloat16 o[32];
                    if constexpr (MODE == CONV_RELU) {
#pragma unroll
                        for (int c = 0; c < 32; c++) o[c] = __float2bfloat16_rn(fmaxf(v[c] + bias_s[c], 0.0f));
                    } else {
                        __align__(16) __nv_bfloat16 mk[32];
#pragma unroll
                        for (int u = 0; u < 4; u++)
                            reinterpret_cast<uint4*>(mk)[u] = reinterpret_cast<const uint4*>(a.mask + pix * 32)[u];
#pragma unroll
                        for (int c = 0; c < 32; c++)
                            o[c] = __float2bfloat16_rn(__bfloat162float(mk[c]) > 0.0f ? v[c] : 0.0f);
                    }
#pragma unroll
                    for (int u = 0; u < 4; u++)
                        reinterpret_cast<uint4*>(a.out_b + pix * 32)[u] = reinterpret_cast<const uint4*>(o)[u];
                } else {
                    float v[16];
                    tmem_ld16(taddr, v);
                    tmem_zero16(taddr);
                    if (px >= W || py >= H) continue;
                    const int64_t pix = ((int64_t)b * H + py) * W + px;
                    __align__(16) float o[8];
#pragma unroll
                    for (int c = 0; c < 8; c++) o[c] = v[c] + bias_s[c];
                    reinterpret_cast<float4*>(a.out_f + pix * 8)[0] = reinterpret_cast<const float4*>(o)[0];
                    reinterpret_cast<float4*>(a.out_f + pix * 8)[1] = reinterpret_cast<const float4*>(o)[1];
                }
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty + 8 * set);
        }
    }

    // ---- teardown: nothing in flight may outlive the CTA's shared and tensor memory
    __syncwarp();
    if (warp == 0 && lane == 0 && abort_cta) {
        // every issued block's copies land before the shared memory goes (bounded)
        for (int n = max(0, issued_blocks - TC_RING); n < issued_blocks; n++)
            for (int spin = 0; spin < TC_SPINS && !mbar_try(full + 8 * (n % TC_RING), (uint32_t)((n / TC_RING) & 1));
                 spin++) {
            }
    }
    if (warp == 1 && lane == 0) {
        for (int spin = 0; spin < TC_SPINS && !mbar_try(done, 0u); spin++) {
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(L::TCOLS));
}

const void* conv_tc_kernel(int cout, int mode) {
    if (cout == 32 && mode == CONV_RELU) return (const void*)k_conv_tc<32, 32, CONV_RELU>;
    if (cout == 8 && mode == CONV_LINEAR) return (const void*)k_conv_tc<16, 8, CONV_LINEAR>;
    if (cout == 32 && mode == CONV_GRAD_MASK) return (const void*)k_conv_tc<32, 32, CONV_GRAD_MASK>;
    return nullptr;
}

size_t conv_tc_smem(int cout) { return cout == 8 ? TcLayout<16>::SMEM : TcLayout<32>::SMEM; }

cudaError_t launch_conv_tc(int cout, int mode, const ConvArgs& a, uint32_t* status, cudaStream_t s) {
    const void* k = conv_tc_kernel(cout, mode);
    EncodeTiled enc = tensor_map_encoder();
    if (!k || !enc) return cudaErrorInvalidValue;
    // the input as a 4-D tensor (channels, x, y, sample); a box is 16 channels x 132 pixels of one row
    CUtensorMap map;
    const cuuint64_t dims[4] = {32, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.B};
    const cuuint64_t strides[3] = {64, (cuuint64_t)a.W * 64, (cuuint64_t)a.H * a.W * 64};
    const cuuint32_t box[4] = {16, TC_PIX, 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void*)a.in, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    const int total = a.B * ((a.W + TC_M - 1) / TC_M) * ((a.H + TC_TR - 1) / TC_TR);
    const int grid = total < sm_count() ? total : sm_count();
    void* args[] = {const_cast<ConvArgs*>(&a), &map, &status};
    return cudaLaunchKernel(k, dim3(grid), dim3(TC_THREADS), args, conv_tc_smem(cout), s);
}

}  // namespace vf
