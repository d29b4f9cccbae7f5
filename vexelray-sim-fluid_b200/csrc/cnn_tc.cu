// cnn_tc.cu -- the network's 32-input-channel 5x5 convolutions on the fifth-generation tensor cores, with
// warp-specialised roles: TMA into a ring of input rows, one thread issuing tcgen05.mma into tensor memory, and
// eight epilogue warps. For sm_100a.
//
// Work: output tiles of 4 rows x 128 pixels. A CTA takes a contiguous range of tiles down 128-pixel strips, so
// consecutive tiles share 4 of their 8 input rows: the ring holds blocks of 4 input rows (4 blocks for 32 input
// channels, 6 for 8), and a tile that continues its predecessor's strip loads one new block.
//   warp 0 (one thread): per block, one TMA tile load per input row (box: the row's channels x 132 or 136 pixels,
//     zero fill outside the image) into a free ring slot, ahead of the MMAs by up to the ring's depth; they
//     complete on the slot's `full` barrier.
//   warp 1: allocates the tensor memory (2 accumulator sets x 4 rows x C columns, C = output channels); one
//     thread waits for the tile's two blocks and a free accumulator set and issues 80 MMAs (M = 128 pixels,
//     K = 16: one tap's 16 channels): per (input row, tap column, channel half), ONE MMA for all the tile's output
//     rows that read that slice, N = their number x C (the weights staged ky-fastest make their B blocks
//     consecutive rows; the accumulators in reverse row order make their D blocks consecutive columns). It
//     commits to the set's `tfull` barrier and to the `empty` barrier of each block no later tile reads.
//   warps 2-9: wait on `tfull`; warp w reads tensor-memory lanes 32 (w % 4) .. + 31 (its pixels) and half of the
//     columns (channels), the tile's four rows with one wait, clears them (the MMAs only accumulate), writes bias
//     + ReLU to bf16, or fp32, or the gradient times the ReLU mask, and arrives on the set's `tempty` barrier.
// Every wait is bounded: on expiry the CTA sets ST_TIMEOUT and every role leaves its loop; the CTA then waits
// (bounded) for its copies and MMAs in flight before it frees the tensor memory.
//
// Operand layouts (K-major, 32-byte swizzle): an input row is two planes (channels 0-15, 16-31) of 132 pixels x
// 32 bytes; the A operand of output row r, tap (ky, kx) and channel half kc starts at input row r + ky, plane kc,
// pixel kx. The weights: per k step (tap, half), N rows of 32 bytes.
#include "cnn.cuh"

namespace vf {

namespace {

constexpr int TC_THREADS = 320;          // warp 0 TMA, warp 1 MMA, warps 2-9 epilogue
constexpr int TC_M = 128;                  // pixels per MMA
constexpr int TC_TR = 4;                   // output rows per tile
constexpr int TC_SPINS = 1 << 22;          // mbarrier polls before a role gives up

// The staged geometry by input channels. 32: an input row is two planes (channels 0-15, 16-31) of 132 pixels x
// 32 bytes in the 32-byte swizzle; a k step is (tap, channel half). 8: one unswizzled plane of 136 pixels x 16
// bytes; a k step is the taps (ky, 2p) and (ky, 2p + 1), p = 0..2 (the sixth tap, kx = 5, has zero weights and
// reads pixel 130 + 127 at most).
#ifndef TC_WIDE
#define TC_WIDE 1   // 32 input channels: A in 64-byte rows (64-byte swizzle), B in 128-byte rows (128-byte swizzle)
#endif

template <int CIN, int NMMA>
struct TcLayout {
    static constexpr bool SWZ = CIN == 32;
    static constexpr bool WIDE = SWZ && TC_WIDE;
    static constexpr int PIX = SWZ ? TC_M + 4 : TC_M + 8;
    static constexpr int PLANES = SWZ && !WIDE ? 2 : 1;
    static constexpr int CH = WIDE ? 32 : SWZ ? 16 : 8;                        // channels per TMA box
    static constexpr int PLANE = WIDE  ? (PIX * 64 + 511) / 512 * 512
                                 : SWZ ? (PIX * 32 + 255) / 256 * 256
                                       : (PIX * 16 + 127) / 128 * 128;
    static constexpr int ROWB = PLANES * PLANE;
    static constexpr int BLOCKB = TC_TR * ROWB;
    static constexpr uint32_t BOX_BYTES = CH * PIX * 2;
    static constexpr int KSTEPS = SWZ ? CNN_TAPS * 2 : 5 * 3;
    static constexpr int B_BYTES = WIDE ? 3 * 5 * NMMA * 128 : KSTEPS * NMMA * 32;   // WIDE: 3 tap pairs
    static constexpr int RING = SWZ ? 4 : 6;           // ring blocks of TC_TR input rows (as many as fit)
    static constexpr int NBAR = 2 * RING + 4 + 1;      // full[RING], empty[RING], tfull[2], tempty[2], done
    static constexpr int SMEM = RING * BLOCKB + B_BYTES + NBAR * 8 + 16 + 1024;
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

// K-major operand without swizzle: 8-row core matrices of 16-byte rows, LBO between the two k halves, SBO between
// 8-row groups.
__device__ __forceinline__ uint64_t desc_plain(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | (1ull << 46);
}

// K-major operands in the 64-byte and 128-byte swizzles (8-row groups 512 and 1024 bytes apart).
__device__ __forceinline__ uint64_t desc_sw64(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3fff) | ((uint64_t)1 << 16) | ((uint64_t)(512 >> 4) << 32) | (1ull << 46) |
           (4ull << 61);
}

__device__ __forceinline__ uint64_t desc_sw128(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3fff) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
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



// CW consecutive fp32 columns of this thread's tensor-memory lane, without the wait (tmem_wait_ld after a batch).
template <int CW>
__device__ __forceinline__ void tmem_ld_nowait(uint32_t taddr, uint32_t (&r)[CW]) {
    if constexpr (CW == 16) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
            "%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
    } else {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                     : "r"(taddr));
    }
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

template <int CW>
__device__ __forceinline__ void tmem_zero_cols(uint32_t taddr) {
    const uint32_t z = 0;
    if constexpr (CW == 16) {
        asm volatile(
            "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
            "%1};" ::"r"(taddr),
            "r"(z)
            : "memory");
    } else {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1};" ::"r"(taddr), "r"(z)
                     : "memory");
    }
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

template <int CIN, int NMMA, int COUT, int MODE>
__global__ void __launch_bounds__(TC_THREADS, 1) k_conv_tc(ConvArgs a, const __grid_constant__ CUtensorMap tmap,
                                                            uint32_t* status) {
    using L = TcLayout<CIN, NMMA>;
    constexpr int K = conv_k(CIN);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024 - (su32(smem_raw) & 1023)) & 1023);
    constexpr int TC_RING = L::RING;
    const uint32_t ring = su32(smem);                    // TC_RING blocks
    const uint32_t wts = ring + TC_RING * L::BLOCKB;     // the weights (layout below)
    const uint32_t bars = wts + L::B_BYTES;              // mbarriers
    const uint32_t full = bars, empty = bars + 8 * TC_RING, tfull = bars + 16 * TC_RING, tempty = tfull + 16,
                   done = tempty + 16;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + TC_RING * L::BLOCKB + L::B_BYTES + L::NBAR * 8);
    __shared__ volatile int abort_cta;
    __shared__ float bias_s[32];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // the weights once (cp.async), ky fastest so that consecutive taps' blocks are consecutive rows; 32 input
    // channels: per (kx, half kc, ky) NMMA swizzled rows of 32 bytes; 8: per (pair p, half h, ky) NMMA rows of
    // 16 bytes (tap ky * 5 + 2p + h, the zero tap 25 where 2p + h = 5); then barriers and tensor memory
    if constexpr (L::WIDE) {
        // per tap pair P = kx / 2: NMMA x 5 rows (ky fastest) of 128 bytes = [tap (ky, 2P) | tap (ky, 2P + 1)],
        // 16-byte chunk q of row r at chunk q ^ (r % 8) (the 128-byte swizzle; pair blocks 1024-byte aligned)
        for (int i = tid; i < NMMA * (K / 8); i += TC_THREADS) {
            const int co = i / (K / 8), c = i % (K / 8), tap = c / 4, g = c % 4, ky = tap / 5, kx = tap % 5;
            const int r = ky * NMMA + co, q = (kx & 1) * 4 + g;
            cp16(wts + (kx / 2) * 5 * NMMA * 128 + r * 128 + ((q ^ (r & 7)) << 4),
                 co < COUT ? a.w + (int64_t)co * K + c * 8 : a.w, co < COUT ? 16u : 0u);
        }
    } else if constexpr (L::SWZ) {
        for (int i = tid; i < NMMA * (K / 8); i += TC_THREADS) {
            const int co = i / (K / 8), c = i % (K / 8), step = c / 2, half = c % 2;
            const int tap = step / 2, kc = step % 2, ky = tap / 5, kx = tap % 5;
            const int blk = (kx * 2 + kc) * 5 + ky;
            cp16(wts + blk * NMMA * 32 + sw32(co, half), co < COUT ? a.w + (int64_t)co * K + c * 8 : a.w,
                 co < COUT ? 16u : 0u);
        }
    } else {
        for (int i = tid; i < 3 * 2 * 5 * NMMA; i += TC_THREADS) {
            const int co = i % NMMA, ky = (i / NMMA) % 5, h = (i / (5 * NMMA)) % 2, pr = i / (10 * NMMA);
            const int kx = 2 * pr + h, tap = kx <= 4 ? ky * 5 + kx : CNN_TAPS;
            cp16(wts + i * 16, co < COUT ? a.w + (int64_t)co * K + tap * 8 : a.w, co < COUT ? 16u : 0u);
        }
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
            mbar_init(tempty + 8 * q, 8);
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
    constexpr int CW = NMMA / 2;   // accumulator columns per epilogue warp: warps 2-5 the first half, 6-9 the second
    if (warp >= 2) {   // both accumulator sets start at zero (the MMAs only accumulate)
        const uint32_t base = tmem + ((uint32_t)((warp & 3) * 32) << 16) + ((warp - 2) >> 2) * CW;
        for (int c = 0; c < 2 * TC_TR; c++) tmem_zero_cols<CW>(base + c * NMMA);
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
                             "r"((uint32_t)(TC_TR * L::PLANES) * L::BOX_BYTES)
                             : "memory");
                const int row0 = y0 - 2 + 4 * k;
                for (int r = 0; r < TC_TR; r++)
                    for (int pl = 0; pl < L::PLANES; pl++) {
                        const uint32_t dst = ring + slot * L::BLOCKB + r * L::ROWB + pl * L::PLANE;
                        asm volatile(
                            "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
                            "%3, %4, %5}], [%6];" ::"r"(dst),
                            "l"(&tmap), "r"(pl * L::CH), "r"(x0 - 2), "r"(row0 + r), "r"(b), "r"(fb)
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
            const uint32_t r0 = ring + (fb % TC_RING) * L::BLOCKB, r1 = ring + ((fb + 1) % TC_RING) * L::BLOCKB;
            const uint32_t acc = tmem + set * TC_TR * NMMA;
            // input row ir and one k-step slice: ONE MMA for every output row orow = ir - ky of the tile that reads
            // the slice: the weights are staged ky-fastest, so the n taps' B blocks are n * NMMA consecutive rows,
            // and the accumulators lie in reverse row order, so the rows' D blocks are consecutive: N = n * NMMA.
            // Descriptors are linear in the start address (16-byte units in the low bits, no carry below 256 KB),
            // so each is a base plus a compile-time offset.
#ifndef TC_ORDER
#define TC_ORDER 1   // 1: consecutive MMAs alternate between the tile's first and last input rows
#endif
            // one MMA of input row ir and k slice (kx or pair p, channel half kc)
            auto mma = [&](int ir, int kx, int kc) {
                constexpr int last = TC_TR - 1;
                const int ky0 = ir - last > 0 ? ir - last : 0, ky1 = ir < 4 ? ir : 4;
                const int n = ky1 - ky0 + 1;
                const uint32_t id = idesc(TC_M, n * NMMA);
                const uint32_t d = acc + (last - (ir - ky0)) * NMMA;
                const uint32_t row = (ir < 4 ? r0 : r1) + (ir & 3) * L::ROWB;
                if constexpr (L::WIDE) {
                    // A: pixel rows of 64 bytes, channel half kc at +32; B: the pair block of kx, its half at
                    // +64 (kx odd), channel half at +32
                    umma_acc(d, desc_sw64(row) + (uint64_t)((kx * 64 + kc * 32) >> 4),
                             desc_sw128(wts) + (uint64_t)(((kx / 2) * 5 * NMMA * 128 + ky0 * NMMA * 128 + (kx & 1) * 64 +
                                                           kc * 32) >> 4),
                             id);
                } else if constexpr (L::SWZ) {
                    umma_acc(d, desc_sw32(row) + (uint64_t)((kc * L::PLANE + kx * 32) >> 4),
                             desc_sw32(wts) + (uint64_t)((((kx * 2 + kc) * 5 + ky0) * NMMA * 32) >> 4), id);
                } else {
                    // A: pixels at 16-byte rows, the pair's second tap one pixel (16 bytes) on; B: per pair p = kx,
                    // half 0 then half 1 (5 * NMMA rows each)
                    umma_acc(d, desc_plain(row, 16, 128) + (uint64_t)((2 * kx * 16) >> 4),
                             desc_plain(wts, 5 * NMMA * 16, 128) + (uint64_t)(((kx * 10 * NMMA + ky0 * NMMA) * 16) >> 4),
                             id);
                }
            };
            constexpr int KX = L::SWZ ? 5 : 3, KC = L::SWZ ? 2 : 1;
            if constexpr (TC_ORDER) {
                // consecutive MMAs on accumulators that overlap as little as possible (rows 0,7,1,6,2,5,3,4)
#pragma unroll
                for (int kx = 0; kx < KX; kx++)
#pragma unroll
                    for (int kc = 0; kc < KC; kc++)
#pragma unroll
                        for (int j = 0; j < TC_TR + 4; j++) mma((j & 1) ? TC_TR + 3 - j / 2 : j / 2, kx, kc);
            } else {
#pragma unroll
                for (int ir = 0; ir < TC_TR + 4; ir++)
#pragma unroll
                    for (int kx = 0; kx < KX; kx++)
#pragma unroll
                        for (int kc = 0; kc < KC; kc++) mma(ir, kx, kc);
            }
            umma_commit(tfull + 8 * set);
            umma_commit(empty + 8 * (fb % TC_RING));   // no later tile reads this tile's first block
            const bool last_of_run = t + 1 == t1 || !seq.continues(t + 1, t0);
            if (last_of_run) umma_commit(empty + 8 * ((fb + 1) % TC_RING));
        }
        umma_commit(done);   // arrives when every MMA this thread issued has completed
    } else if (warp >= 2) {
        // ---- epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 (its 32 pixels), columns
        //      hh * CW .. + CW - 1 (hh = 0 for warps 2-5, 1 for 6-9): the tile's four rows loaded before one wait
        const int q = warp & 3, hh = (warp - 2) >> 2;
        int i = 0;
        for (int t = t0; t < t1 && !abort_cta; t++, i++) {
            const int set = i & 1;
            if (!mbar_wait(tfull + 8 * set, (uint32_t)((i / 2) & 1), &abort_cta, status)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            int b, x0, y0;
            seq.at(t, b, x0, y0);
            const int px = x0 + q * 32 + lane;
            // row orow's accumulator lies at reverse position TC_TR - 1 - orow of the set
            const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + set * TC_TR * NMMA + hh * CW;
            uint32_t v[TC_TR][CW];
#pragma unroll
            for (int orow = 0; orow < TC_TR; orow++) tmem_ld_nowait<CW>(base + (TC_TR - 1 - orow) * NMMA, v[orow]);
            tmem_wait_ld();
#pragma unroll
            for (int orow = 0; orow < TC_TR; orow++) tmem_zero_cols<CW>(base + (TC_TR - 1 - orow) * NMMA);
            const int c0 = hh * CW;   // this warp's first output channel
#pragma unroll
            for (int orow = 0; orow < TC_TR; orow++) {
                const int py = y0 + orow;
                if (px >= W || py >= H) continue;
                const int64_t pix = ((int64_t)b * H + py) * W + px;
                if constexpr (NMMA == 32) {
                    __align__(16) __nv_bfloat16 o[CW];
                    if constexpr (MODE == CONV_RELU) {
#pragma unroll
                        for (int c = 0; c < CW; c++)
                            o[c] = __float2bfloat16_rn(fmaxf(__uint_as_float(v[orow][c]) + bias_s[c0 + c], 0.0f));
                    } else {
                        __align__(16) __nv_bfloat16 mk[CW];
#pragma unroll
                        for (int u = 0; u < CW / 8; u++)
                            reinterpret_cast<uint4*>(mk)[u] = reinterpret_cast<const uint4*>(a.mask + pix * 32 + c0)[u];
#pragma unroll
                        for (int c = 0; c < CW; c++)
                            o[c] = __float2bfloat16_rn(__bfloat162float(mk[c]) > 0.0f ? __uint_as_float(v[orow][c]) : 0.0f);
                    }
#pragma unroll
                    for (int u = 0; u < CW / 8; u++)
                        reinterpret_cast<uint4*>(a.out_b + pix * 32 + c0)[u] = reinterpret_cast<const uint4*>(o)[u];
                } else if (hh == 0) {   // 8 output channels: the second half holds the MMA's padding only
                    __align__(16) float o[8];
#pragma unroll
                    for (int c = 0; c < 8; c++) o[c] = __uint_as_float(v[orow][c]) + bias_s[c];
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

const void* conv_tc_kernel(int cin, int cout, int mode) {
    if (cin == 32 && cout == 32 && mode == CONV_RELU) return (const void*)k_conv_tc<32, 32, 32, CONV_RELU>;
    if (cin == 32 && cout == 8 && mode == CONV_LINEAR) return (const void*)k_conv_tc<32, 16, 8, CONV_LINEAR>;
    if (cin == 32 && cout == 32 && mode == CONV_GRAD_MASK) return (const void*)k_conv_tc<32, 32, 32, CONV_GRAD_MASK>;
    if (cin == 8 && cout == 32 && mode == CONV_RELU) return (const void*)k_conv_tc<8, 32, 32, CONV_RELU>;
    if (cin == 8 && cout == 32 && mode == CONV_GRAD_MASK) return (const void*)k_conv_tc<8, 32, 32, CONV_GRAD_MASK>;
    return nullptr;
}

size_t conv_tc_smem(int cin, int cout) {
    if (cin == 8) return TcLayout<8, 32>::SMEM;
    return cout == 8 ? TcLayout<32, 16>::SMEM : TcLayout<32, 32>::SMEM;
}

cudaError_t launch_conv_tc(int cin, int cout, int mode, const ConvArgs& a, uint32_t* status, cudaStream_t s) {
    const void* k = conv_tc_kernel(cin, cout, mode);
    EncodeTiled enc = tensor_map_encoder();
    if (!k || !enc) return cudaErrorInvalidValue;
    // the input as a 4-D tensor (channels, x, y, sample); a box is one plane's channels x the staged pixels of a row
    const bool swz = cin == 32, wide = swz && TC_WIDE;
    CUtensorMap map;
    const cuuint64_t px = (cuuint64_t)cin * 2;
    const cuuint64_t dims[4] = {(cuuint64_t)cin, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.B};
    const cuuint64_t strides[3] = {px, (cuuint64_t)a.W * px, (cuuint64_t)a.H * a.W * px};
    const cuuint32_t box[4] = {swz ? (cuuint32_t)TcLayout<32, 32>::CH : (cuuint32_t)TcLayout<8, 32>::CH,
                               swz ? (cuuint32_t)TcLayout<32, 32>::PIX : (cuuint32_t)TcLayout<8, 32>::PIX, 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void*)a.in, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE,
            wide ? CU_TENSOR_MAP_SWIZZLE_64B : swz ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    const int total = a.B * ((a.W + TC_M - 1) / TC_M) * ((a.H + TC_TR - 1) / TC_TR);
    const int grid = total < sm_count() ? total : sm_count();   // one CTA per SM (the register file allows no more)
    void* args[] = {const_cast<ConvArgs*>(&a), &map, &status};
    return cudaLaunchKernel(k, dim3(grid), dim3(TC_THREADS), args, conv_tc_smem(cin, cout), s);
}

}  // namespace vf
