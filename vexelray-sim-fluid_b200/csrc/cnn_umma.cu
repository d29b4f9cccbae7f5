// cnn_umma.cu -- the network's 5x5 convolutions on the fifth-generation tensor cores: tcgen05.mma
// (kind::f16, bf16 operands from shared memory, fp32 accumulators in tensor memory), for sm_100a.
//
// A CTA of 4 warps owns a tile of TR output rows x 128 pixels (TR = 4: four independent accumulators, whose MMAs
// are issued interleaved). Per tile:
//   1. the TR + 4 input rows it reads (132 pixels each, zeros outside the grid) are copied (cp.async, zero fill)
//      into shared memory in a K-major layout. 32 input channels: two planes per row (channels 0-15, 16-31), each
//      pixel a 32-byte row in the 32-byte swizzle; the A operand of tap (ky, kx) and channels [16 kc, 16 kc + 16)
//      for output row r starts at row r + ky, plane kc, pixel kx (8-row groups 256 bytes apart). 8 input channels:
//      no swizzle, 16 bytes per pixel; a 16-wide k step is two taps and LBO is the distance between their views.
//   2. one thread issues the TR x (k steps) MMAs, M = 128 pixels, N = output channels, K = 16, accumulating
//      into TR column blocks of the CTA's tensor memory, then tcgen05.commit arrives on an mbarrier;
//   3. every thread waits on the mbarrier (a bounded wait: on expiry it sets the status word and the CTA stops),
//      then warp w reads tensor-memory lanes 32w..32w+31 (its 32 pixels) with tcgen05.ld, and writes them: bias
//      and ReLU to bf16, or fp32, or the gradient times the ReLU mask of the forward activation.
// The weights (K-major per output channel, the same canonical layout) are staged once per CTA; the grid is
// persistent, and each CTA runs two stages: tile t+1's MMAs run while the CTA writes tile t and copies tile t+2.
#include "cnn.cuh"

namespace vf {

namespace {

constexpr int UM_THREADS = 128;
constexpr int UM_M = 128;                 // pixels per MMA (one output row's tile)
#ifndef UMMA_ROWS
#define UMMA_ROWS 4
#endif
constexpr int UM_TR = UMMA_ROWS;          // output rows per tile (independent accumulators per stage)
constexpr int UM_ROWS = UM_TR + 4;        // staged input rows
constexpr int UM_PIX = UM_M + 4;          // staged pixels per input row
constexpr int UM_SPINS = 1 << 20;         // mbarrier polls before a tile gives up

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// An asynchronous 16-byte copy global -> shared; src_bytes 0 fills the destination with zeros (src unread).
__device__ __forceinline__ void cp16(uint32_t dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ void cp_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

#ifndef UMMA_BASE_OFFSET
#define UMMA_BASE_OFFSET 0   // 1: the descriptors of swizzled operands carry their start's row phase (address bits 7-9)
#endif

// Shared-memory matrix descriptor: start, LBO, SBO in 16-byte units; version 1; no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | (1ull << 46);
}

// The same for a K-major operand in the 32-byte swizzle: rows of 32 bytes (one 16-wide k step of bf16) whose two
// 16-byte halves are exchanged where address bit 7 is set; 8-row groups 256 bytes apart.
__device__ __forceinline__ uint64_t smem_desc_sw32(uint32_t addr) {
    uint64_t d = smem_desc(addr, 16, 256) | (6ull << 61);
    if (UMMA_BASE_OFFSET) d |= (uint64_t)((addr >> 7) & 7) << 49;
    return d;
}

// Byte offset of 16-byte half h of 32-byte row r in the 32-byte swizzle (block base 256-byte aligned).
__host__ __device__ constexpr uint32_t sw32(uint32_t r, uint32_t h) { return r * 32 + ((h ^ ((r >> 2) & 1)) << 4); }

// Instruction descriptor of kind::f16: fp32 accumulator, bf16 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
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

// 32 consecutive fp32 columns of this thread's tensor-memory lane.
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

// Operand layouts. 32 input channels: the 32-byte swizzle, each staged row as two planes (channels 0-15, 16-31)
// of 132 pixels x 32 bytes, every plane 256-byte aligned. 8 input channels: no swizzle (a k step's two halves
// are two taps, 16-byte rows), one plane of 132 pixels x 16 bytes.
template <int CIN, int NMMA>
struct UmmaLayout {
    static constexpr bool SWZ = CIN == 32;
    static constexpr int KSTEPS = CIN == 8 ? 13 : CNN_TAPS * CIN / 16;   // 16-wide k steps per output row
    static constexpr int NG = CIN / 8;                                   // 8-channel groups per input pixel
    static constexpr int PLANE = SWZ ? (UM_PIX * 32 + 255) / 256 * 256 : UM_PIX * 16;
    static constexpr int ROW_BYTES = SWZ ? 2 * PLANE : UM_PIX * 16;      // one staged input row
    static constexpr int A_BYTES = UM_ROWS * ROW_BYTES;                  // one stage (two are kept)
    static constexpr int B_BYTES = KSTEPS * 2 * NMMA * 16;               // weights, K-major
    static constexpr int SMEM = 2 * A_BYTES + B_BYTES + 64 + 1024;       // + barriers, tmem address, alignment
    static constexpr int TCOLS = 2 * UM_TR * NMMA <= 32    ? 32
                                : 2 * UM_TR * NMMA <= 64  ? 64
                                : 2 * UM_TR * NMMA <= 128 ? 128
                                                          : 256;   // two stages of accumulators
};

}  // namespace

size_t conv_umma_smem(int cin, int nmma) {
    if (cin == 8) return nmma == 32 ? UmmaLayout<8, 32>::SMEM : UmmaLayout<8, 16>::SMEM;
    return nmma == 32 ? UmmaLayout<32, 32>::SMEM : UmmaLayout<32, 16>::SMEM;
}

int conv_umma_tmem_cols(int cin, int nmma) {
    if (cin == 8) return nmma == 32 ? UmmaLayout<8, 32>::TCOLS : UmmaLayout<8, 16>::TCOLS;
    return nmma == 32 ? UmmaLayout<32, 32>::TCOLS : UmmaLayout<32, 16>::TCOLS;
}

// CIN input channels, NMMA = the MMA's N (output channels, padded to 16 or 32), COUT = channels of the output
// buffer, MODE as k_conv. Two stages: tile t+1's MMAs run on the tensor core while the CTA writes tile t out of
// tensor memory and copies tile t+2's rows in.
template <int CIN, int NMMA, int COUT, int MODE>
__global__ void __launch_bounds__(UM_THREADS) k_conv_umma(ConvArgs a, uint32_t* status) {
    using L = UmmaLayout<CIN, NMMA>;
    constexpr int K = conv_k(CIN);
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024 - (su32(smem_raw) & 1023)) & 1023);   // 1024-byte aligned operands
    unsigned char* A = smem;                                    // 2 stages of UM_ROWS staged rows
    unsigned char* Bw = smem + 2 * L::A_BYTES;                  // [KSTEPS][2][NMMA][16 B]
    uint64_t* bar = reinterpret_cast<uint64_t*>(Bw + L::B_BYTES);   // one per stage
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);
    __shared__ int abort_cta;
    __shared__ float bias_s[32];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int H = a.H, W = a.W;
    const uint32_t a_base = su32(A), b_base = su32(Bw);

    // the weights, once: element (co, k) of the [cout][K] matrix -> k step k/16, half (k%16)/8, row co
    for (int i = tid; i < NMMA * (K / 8); i += UM_THREADS) {
        const int co = i / (K / 8), c = i % (K / 8);   // 8-element chunk c of row co
        const int step = c / 2, half = c % 2;
        const uint32_t dst = L::SWZ ? b_base + step * NMMA * 32 + sw32(co, half)
                                    : b_base + ((step * 2 + half) * NMMA + co) * 16;
        cp16(dst, co < COUT ? a.w + (int64_t)co * K + c * 8 : a.w, co < COUT ? 16u : 0u);
    }
    if (tid < 32) bias_s[tid] = (MODE != CONV_GRAD_MASK && a.bias && tid < a.bias_n) ? a.bias[tid] : 0.0f;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(bar)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(bar + 1)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_cta = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                     "r"(L::TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = idesc_bf16(UM_M, NMMA);
    // the MMAs' operand descriptors for stage 0 (a stage's are these plus its offset): A per (output row, k step),
    // B per k step
    __shared__ uint64_t desc_a[UM_TR * L::KSTEPS], desc_b[L::KSTEPS];
    for (int i = tid; i < UM_TR * L::KSTEPS; i += UM_THREADS) {
        const int orow = i / L::KSTEPS, s = i % L::KSTEPS;
        uint32_t a_addr, lbo;
        if constexpr (CIN == 8) {
            const int t0 = 2 * s, t1 = min(2 * s + 1, CNN_TAPS - 1);
            a_addr = a_base + (orow + t0 / 5) * L::ROW_BYTES + (t0 % 5) * 16;
            const uint32_t a1 = a_base + (orow + t1 / 5) * L::ROW_BYTES + (t1 % 5) * 16;
            lbo = a1 - a_addr;
        } else {
            const int tap = s / (CIN / 16), kc = s % (CIN / 16);
            a_addr = a_base + (orow + tap / 5) * L::ROW_BYTES + kc * L::PLANE + (tap % 5) * 32;
            lbo = 0;
        }
        if constexpr (L::SWZ) {
            desc_a[i] = smem_desc_sw32(a_addr);
            if (orow == 0) desc_b[s] = smem_desc_sw32(b_base + s * NMMA * 32);
        } else {
            desc_a[i] = smem_desc(a_addr, lbo, 128);
            if (orow == 0) desc_b[s] = smem_desc(b_base + s * 2 * NMMA * 16, NMMA * 16, 128);
        }
    }
    __syncthreads();

    const int tx_n = (W + UM_M - 1) / UM_M, ty_n = (H + UM_TR - 1) / UM_TR;
    const int total = a.B * tx_n * ty_n;
    auto coords = [&](int tile, int& b, int& x0, int& y0) {
        b = tile / (tx_n * ty_n);
        const int r = tile % (tx_n * ty_n);
        x0 = (r % tx_n) * UM_M;
        y0 = (r / tx_n) * UM_TR;
    };
    // copies tile `tile`'s input rows y0-2 .. y0+TR+1, pixels x0-2 .. x0+129 (zeros outside) into stage st
    auto stage = [&](int tile, int st) {
        int b, x0, y0;
        coords(tile, b, x0, y0);
        const uint32_t dst = a_base + st * L::A_BYTES;
        for (int i = tid; i < UM_ROWS * UM_PIX * L::NG; i += UM_THREADS) {
            const int g = i % L::NG, p = (i / L::NG) % UM_PIX, row = i / (L::NG * UM_PIX);
            const int gx = x0 + p - 2, gy = y0 + row - 2;
            const bool in = gx >= 0 && gx < W && gy >= 0 && gy < H;
            const __nv_bfloat16* src = in ? a.in + (((int64_t)b * H + gy) * W + gx) * CIN + g * 8 : a.in;
            const uint32_t off = L::SWZ ? (g >> 1) * L::PLANE + sw32(p, g & 1) : (g * UM_PIX + p) * 16;
            cp16(dst + row * L::ROW_BYTES + off, src, in ? 16u : 0u);
        }
    };
    // waits for this thread's copies, makes every thread's visible to the tensor core, then one thread issues
    // stage st's MMAs into accumulator set st and commits them to bar[st]
    auto issue = [&](int st) {
        cp_wait_all();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            const uint64_t shift = (uint64_t)(st * L::A_BYTES) >> 4;   // the stage's offset in the descriptors' units
            // the rows' accumulations interleaved, so consecutive MMAs are independent
            const uint32_t acc0 = tmem + st * UM_TR * NMMA;
#pragma unroll
            for (int orow = 0; orow < UM_TR; orow++)
                umma(acc0 + orow * NMMA, desc_a[orow * L::KSTEPS] + shift, desc_b[0], idesc, 0u);
#pragma unroll 1
            for (int s = 1; s < L::KSTEPS; s++) {
                const uint64_t bd = desc_b[s];
#pragma unroll
                for (int orow = 0; orow < UM_TR; orow++)
                    umma(acc0 + orow * NMMA, desc_a[orow * L::KSTEPS + s] + shift, bd, idesc, 1u);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             su32(bar + st))
                         : "memory");
        }
    };
    // waits (bounded) for stage st's MMAs; false (and the status set) if they did not signal in time
    uint32_t phase[2] = {0, 0};
    auto wait_mma = [&](int st) {
        bool done = false;
        for (int spin = 0; spin < UM_SPINS; spin++) {
            if (mbar_try(su32(bar + st), phase[st])) {
                done = true;
                break;
            }
        }
        if (!done) {
            set_status(status, ST_TIMEOUT);
            atomicExch(&abort_cta, 1);
        }
        __syncthreads();
        if (abort_cta) return false;
        phase[st] ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        return true;
    };
    // writes tile `tile` out of accumulator set st
    auto epilogue = [&](int tile, int st) {
        int b, x0, y0;
        coords(tile, b, x0, y0);
        const int px = x0 + warp * 32 + (tid & 31);
#pragma unroll 1
        for (int orow = 0; orow < UM_TR; orow++) {
            const int py = y0 + orow;
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (st * UM_TR + orow) * NMMA;
            if constexpr (NMMA == 32) {
                float v[32];
                tmem_ld32(taddr, v);
                if (px >= W || py >= H) continue;
                const int64_t pix = ((int64_t)b * H + py) * W + px;
                __align__(16) __nv_bfloat16 o[32];
                if constexpr (MODE == CONV_RELU) {
#pragma unroll
                    for (int c = 0; c < 32; c++) o[c] = __float2bfloat16_rn(fmaxf(v[c] + bias_s[c], 0.0f));
                } else {
                    __align__(16) __nv_bfloat16 mk[32];
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        reinterpret_cast<uint4*>(mk)[q] = reinterpret_cast<const uint4*>(a.mask + pix * 32)[q];
#pragma unroll
                    for (int c = 0; c < 32; c++) o[c] = __float2bfloat16_rn(__bfloat162float(mk[c]) > 0.0f ? v[c] : 0.0f);
                }
#pragma unroll
                for (int q = 0; q < 4; q++)
                    reinterpret_cast<uint4*>(a.out_b + pix * 32)[q] = reinterpret_cast<const uint4*>(o)[q];
            } else {
                float v[16];
                tmem_ld16(taddr, v);
                if (px >= W || py >= H) continue;
                const int64_t pix = ((int64_t)b * H + py) * W + px;
                __align__(16) float o[8];
#pragma unroll
                for (int c = 0; c < 8; c++) o[c] = v[c] + bias_s[c];
                reinterpret_cast<float4*>(a.out_f + pix * 8)[0] = reinterpret_cast<const float4*>(o)[0];
                reinterpret_cast<float4*>(a.out_f + pix * 8)[1] = reinterpret_cast<const float4*>(o)[1];
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();   // accumulator set st is free again
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    };

    // the pipeline over this CTA's tiles t0, t0 + G, ...: MMAs of k+1 overlap the epilogue of k and the copies of k+2
    const int first = blockIdx.x, G = gridDim.x;
    int pending = -1;   // the stage whose MMAs are in flight and not yet waited for
    if (first < total) {
        stage(first, 0);
        issue(0);
        pending = 0;
    }
    int k = 0;
    for (int tile = first; tile < total; tile += G, k++) {
        const int st = k & 1, nx = (k + 1) & 1;
        const int next = tile + G;
        if (next < total) {
            stage(next, nx);   // stage nx was last read by tile k-1's MMAs, waited for in the last iteration
            issue(nx);
        }
        const bool ok = wait_mma(st);
        pending = next < total ? nx : -1;
        if (!ok) break;
        epilogue(tile, st);
    }
    __syncthreads();
    if (abort_cta) {
        // MMAs that never signalled may still be running: give each stage a bounded while before the memory goes
        for (int q = 0; q < 2; q++)
            for (int spin = 0; spin < UM_SPINS && !mbar_try(su32(bar + q), phase[q]); spin++) {
            }
    } else if (pending >= 0) {
        // unreachable in a complete pass (every issued stage is waited for); kept as a bounded guard
        for (int spin = 0; spin < UM_SPINS && !mbar_try(su32(bar + pending), phase[pending]); spin++) {
        }
    }
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(L::TCOLS));
}

const void* conv_umma_kernel(int cin, int cout, int mode) {
    if (cin == 8 && cout == 32 && mode == CONV_RELU) return (const void*)k_conv_umma<8, 32, 32, CONV_RELU>;
    if (cin == 32 && cout == 32 && mode == CONV_RELU) return (const void*)k_conv_umma<32, 32, 32, CONV_RELU>;
    if (cin == 32 && cout == 8 && mode == CONV_LINEAR) return (const void*)k_conv_umma<32, 16, 8, CONV_LINEAR>;
    if (cin == 8 && cout == 32 && mode == CONV_GRAD_MASK) return (const void*)k_conv_umma<8, 32, 32, CONV_GRAD_MASK>;
    if (cin == 32 && cout == 32 && mode == CONV_GRAD_MASK) return (const void*)k_conv_umma<32, 32, 32, CONV_GRAD_MASK>;
    return nullptr;
}

// The dynamic shared memory a launch asks for: the kernel's own, raised where needed so that no more CTAs are
// resident on an SM than its 512 tensor-memory columns can serve at once (a CTA whose allocation had to wait for
// another CTA's release would idle until that persistent CTA finished).
size_t conv_umma_smem_for(int cin, int cout) {
    const int nmma = cout == 8 ? 16 : 32;
    const size_t own = conv_umma_smem(cin, nmma);
    const int cap = 512 / conv_umma_tmem_cols(cin, nmma);
    int dev = 0, per_sm = 0, reserved = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess) {
        cudaGetLastError();
        return own;
    }
    const long long floor_for_cap = (long long)per_sm / (cap + 1) - reserved + 16;   // cap + 1 CTAs no longer fit
    const size_t need = floor_for_cap > 0 ? (size_t)((floor_for_cap + 15) / 16 * 16) : 0;
    return own > need ? own : need;
}

cudaError_t launch_conv_umma(int cin, int cout, int mode, int grid, const ConvArgs& a, uint32_t* status,
                             cudaStream_t s) {
    const void* k = conv_umma_kernel(cin, cout, mode);
    if (!k) return cudaErrorInvalidValue;
    void* args[] = {const_cast<ConvArgs*>(&a), &status};
    return cudaLaunchKernel(k, dim3(grid), dim3(UM_THREADS), args, conv_umma_smem_for(cin, cout), s);
}

}  // namespace vf
