// cnn_kernels.cu -- the network's 5x5 convolutions as implicit GEMMs on the tensor cores (mma.sync
// m16n8k16, bf16 in, fp32 accumulate), for sm_100a.
//
// Forward (and backward data, which is the same convolution over the output gradient with the weights
// transposed and mirrored): a CTA of 8 warps owns a 32 x 8 pixel output tile; the tile's 36 x 12 input
// halo is staged in shared memory (16-byte channel chunks XOR-swizzled by pixel so that the 8 rows of an
// ldmatrix hit distinct banks) and the whole weight matrix stays resident for the CTA's life (persistent
// grid). Warp w computes output row w: two m16 tiles of pixels by all output channels, the k loop over
// 25 taps x input channels (a 16-wide k step is 16 channels of one tap, or 8 channels of two taps when
// the input has 8).
//
// The default is the row-blocked kernel (k_conv_rows): a warp computes 16 pixels of four output rows, so
// each A fragment it loads from shared memory serves every output row that reads that input row (up to
// five, one per ky) and each B fragment four rows. With 32 input and output channels ldmatrix traffic per
// pixel falls from 6.25 to 2.8 fragments. With 8 input channels a k step pairs the taps (ky, 2p) and
// (ky, 2p + 1), p = 0..2, so that the pairs stay within one kernel row; the sixth tap's A rows read zeros.
//
// Weight gradient: dW[co][tap][ci] = sum over pixels of dy[p][co] * x[p + tap][ci], a GEMM with M = output
// channels, N = taps x input channels, K = pixels. Both operands come from shared memory through
// ldmatrix.trans (pixels are their rows there); warps split the (tap, m tile) units, each accumulating in
// registers over every tile the persistent CTA visits, and add into the fp32 gradient once at the end.
#include "cnn.cuh"

namespace vf {

namespace {

constexpr int TW = 32, TH = 8;            // output pixels per CTA tile
constexpr int HW = TW + 4, HH = TH + 4;   // its input halo
constexpr int CONV_THREADS = 256;

// Position of 16-byte chunk c of pixel column x in a row of nc chunks.
template <int NC>
__device__ __forceinline__ int swz(int c, int x) {
    if constexpr (NC == 4) return c ^ ((x >> 1) & 3);
    else if constexpr (NC == 2) return c ^ ((x >> 2) & 1);
    else return c;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_addr(p)));
}

__device__ __forceinline__ void ldsm_x2(uint32_t (&r)[2], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0, %1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(smem_addr(p)));
}

__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_addr(p)));
}

__device__ __forceinline__ void ldsm_x2_t(uint32_t (&r)[2], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0, %1}, [%2];"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(smem_addr(p)));
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// 16-byte asynchronous global -> shared copy; src_bytes 0 writes zeros (the source is not read).
__device__ __forceinline__ void cp16(void* dst, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}

__device__ __forceinline__ void cp_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Stages the 36 x 12 input halo of the tile whose first output pixel is (x0, y0) of sample b, zeros outside.
template <int C>
__device__ __forceinline__ void stage_halo(__nv_bfloat16* in_s, const __nv_bfloat16* in, int b, int x0, int y0, int H,
                                           int W) {
    constexpr int NC = C / 8;
    for (int i = threadIdx.x; i < HH * HW * NC; i += blockDim.x) {
        const int c = i % NC, px = (i / NC) % HW, py = i / (NC * HW);
        const int gx = x0 + px - 2, gy = y0 + py - 2;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (gx >= 0 && gx < W && gy >= 0 && gy < H)
            v = *reinterpret_cast<const uint4*>(in + (((int64_t)b * H + gy) * W + gx) * C + c * 8);
        *reinterpret_cast<uint4*>(in_s + (py * HW + px) * C + swz<NC>(c, px) * 8) = v;
    }
}

}  // namespace

// Rows per warp of the row-blocked convolutions (tile height 4 R).
#ifndef CONV3_ROWS
#define CONV3_ROWS 4
#endif
#ifndef CONV_ROWS_MINB
#define CONV_ROWS_MINB 2
#endif
constexpr int conv_rows(int cout) { return cout == 8 ? CONV3_ROWS : 4; }

size_t conv_smem(int cin, int cout, bool rows) {
    const int hh = rows ? 4 * conv_rows(cout) + 4 : HH;
    return (size_t)cout * (conv_k(cin) + 8) * 2 + (size_t)hh * HW * cin * 2 + (rows ? 16 : 0);
}

size_t wgrad_smem(int cin, int cout) {
    const int cop = cout < 16 ? 16 : cout;
    return (size_t)HH * HW * cin * 2 + (size_t)TH * TW * cop * 2;
}

template <int CIN, int COUT, int MODE>
__global__ void __launch_bounds__(CONV_THREADS) k_conv(ConvArgs a) {
    constexpr int NC = CIN / 8;
    constexpr int K = conv_k(CIN), KP = K + 8;   // weight row, padded so the 8 rows of an ldmatrix miss each other
    constexpr int NT = COUT / 8;
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* w_s = reinterpret_cast<__nv_bfloat16*>(smem);   // [COUT][KP]
    __nv_bfloat16* in_s = w_s + COUT * KP;                          // [HH][HW][CIN]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < COUT * (K / 8); i += blockDim.x) {
        const int co = i / (K / 8), c = i % (K / 8);
        *reinterpret_cast<uint4*>(w_s + co * KP + c * 8) = *reinterpret_cast<const uint4*>(a.w + (int64_t)co * K + c * 8);
    }
    const int H = a.H, W = a.W;
    const int tx_n = (W + TW - 1) / TW, ty_n = (H + TH - 1) / TH;
    const int total = a.B * tx_n * ty_n;
    for (int tile = blockIdx.x; tile < total; tile += gridDim.x) {
        const int b = tile / (tx_n * ty_n), r = tile % (tx_n * ty_n);
        const int x0 = (r % tx_n) * TW, y0 = (r / tx_n) * TH;
        __syncthreads();   // the weights are in; the previous tile's halo is read
        stage_halo<CIN>(in_s, a.in, b, x0, y0, H, W);
        __syncthreads();
        float acc[2][NT][4];
#pragma unroll
        for (int m = 0; m < 2; m++)
#pragma unroll
            for (int n = 0; n < NT; n++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[m][n][q] = 0.0f;
        // one k step: A fragments of the two pixel tiles at (tap, chunk), B fragments from weight column kk
        auto kstep = [&](const __nv_bfloat16* arow0, const __nv_bfloat16* arow1, int kk) {
            uint32_t af[2][4];
            ldsm_x4(af[0], arow0);
            ldsm_x4(af[1], arow1);
            if constexpr (NT == 1) {
                uint32_t bf[2];
                ldsm_x2(bf, w_s + (lane & 7) * KP + kk + ((lane >> 3) & 1) * 8);
                mma_bf16(acc[0][0], af[0], bf[0], bf[1]);
                mma_bf16(acc[1][0], af[1], bf[0], bf[1]);
            } else {
#pragma unroll
                for (int np = 0; np < NT / 2; np++) {
                    uint32_t bf[4];
                    ldsm_x4(bf, w_s + (np * 16 + ((lane >> 4) << 3) + (lane & 7)) * KP + kk + ((lane >> 3) & 1) * 8);
#pragma unroll
                    for (int m = 0; m < 2; m++) {
                        mma_bf16(acc[m][2 * np], af[m], bf[0], bf[1]);
                        mma_bf16(acc[m][2 * np + 1], af[m], bf[2], bf[3]);
                    }
                }
            }
        };
        const int row = lane & 15, khalf = lane >> 4;
        if constexpr (CIN == 8) {
            // a k step is two taps of 8 channels: lanes 0-15 address tap 2s, lanes 16-31 tap 2s+1 (tap 25 has zero
            // weights; its rows point at tap 24)
#pragma unroll 1
            for (int s = 0; s < 13; s++) {
                const int tap = min(2 * s + khalf, 24), ky = tap / 5, kx = tap % 5;
                const int py = warp + ky;
                kstep(in_s + (py * HW + row + kx) * 8, in_s + (py * HW + 16 + row + kx) * 8, s * 16);
            }
        } else {
#pragma unroll 1
            for (int tap = 0; tap < CNN_TAPS; tap++) {
                const int ky = tap / 5, kx = tap % 5, py = warp + ky;
#pragma unroll
                for (int kc = 0; kc < CIN / 16; kc++) {
                    const int c = kc * 2 + khalf;
                    const int p0 = row + kx, p1 = 16 + row + kx;
                    kstep(in_s + (py * HW + p0) * CIN + swz<NC>(c, p0) * 8, in_s + (py * HW + p1) * CIN + swz<NC>(c, p1) * 8,
                          tap * CIN + kc * 16);
                }
            }
        }
        // epilogue: fragment element q of tile (m, n) is pixel 16 m + lane/4 (+8 for q >= 2), channel 8 n + 2 (lane%4) + q%2
        const int py = y0 + warp;
        if (py < H) {
#pragma unroll
            for (int m = 0; m < 2; m++) {
#pragma unroll
                for (int half = 0; half < 2; half++) {
                    const int px = x0 + 16 * m + (lane >> 2) + half * 8;
                    if (px >= W) continue;
                    const int64_t pix = ((int64_t)b * H + py) * W + px;
#pragma unroll
                    for (int n = 0; n < NT; n++) {
                        const int co = n * 8 + 2 * (lane & 3);
                        float v0 = acc[m][n][2 * half], v1 = acc[m][n][2 * half + 1];
                        if constexpr (MODE != CONV_GRAD_MASK) {
                            if (a.bias) {
                                if (co < a.bias_n) v0 += a.bias[co];
                                if (co + 1 < a.bias_n) v1 += a.bias[co + 1];
                            }
                        }
                        if constexpr (MODE == CONV_RELU) {
                            *reinterpret_cast<__nv_bfloat162*>(a.out_b + pix * COUT + co) =
                                __floats2bfloat162_rn(fmaxf(v0, 0.0f), fmaxf(v1, 0.0f));
                        } else if constexpr (MODE == CONV_LINEAR) {
                            *reinterpret_cast<float2*>(a.out_f + pix * COUT + co) = make_float2(v0, v1);
                        } else {
                            const __nv_bfloat162 mk = *reinterpret_cast<const __nv_bfloat162*>(a.mask + pix * COUT + co);
                            if (!(__bfloat162float(mk.x) > 0.0f)) v0 = 0.0f;
                            if (!(__bfloat162float(mk.y) > 0.0f)) v1 = 0.0f;
                            *reinterpret_cast<__nv_bfloat162*>(a.out_b + pix * COUT + co) = __floats2bfloat162_rn(v0, v1);
                        }
                    }
                }
            }
        }
    }
}

// Row-blocked convolution for 32 input channels. A CTA owns a 32 x 4R output tile (input halo 36 x (4R+4),
// staged by cp.async with zero fill); warp w computes pixel columns 16 (w & 1) .. +15 of output rows
// R (w >> 1) .. +R-1. For each (kx, 16-channel half) the warp loads the A fragments of its R + 4 input rows once
// and issues, for each ky, the MMAs of the R output rows that read them: an A fragment feeds up to five output
// rows and a B fragment (one tap's weights) R rows, against one row each in k_conv.
template <int CIN, int COUT, int MODE, int R>
__global__ void __launch_bounds__(CONV_THREADS, CONV_ROWS_MINB) k_conv_rows(ConvArgs a) {
    constexpr int NC = CIN / 8;
    constexpr int K = conv_k(CIN), KP = K + 8;
    constexpr int NT = COUT / 8;
    constexpr int RH = 4 * R, HR = RH + 4;   // tile height, halo rows
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* w_s = reinterpret_cast<__nv_bfloat16*>(smem);   // [COUT][KP]
    __nv_bfloat16* in_s = w_s + COUT * KP;                          // [HR][HW][CIN]
    __nv_bfloat16* zrow = in_s + HR * HW * CIN;                      // 8 zeros: the A rows of the missing sixth tap
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < COUT * (K / 8); i += blockDim.x) {
        const int co = i / (K / 8), c = i % (K / 8);
        *reinterpret_cast<uint4*>(w_s + co * KP + c * 8) = *reinterpret_cast<const uint4*>(a.w + (int64_t)co * K + c * 8);
    }
    if (tid == 0) *reinterpret_cast<uint4*>(zrow) = make_uint4(0, 0, 0, 0);
    const int H = a.H, W = a.W;
    const int tx_n = (W + TW - 1) / TW, ty_n = (H + RH - 1) / RH;
    const int total = a.B * tx_n * ty_n;
    const int mt = warp & 1, rb = warp >> 1;
    const int row = lane & 15, khalf = lane >> 4;
    for (int tile = blockIdx.x; tile < total; tile += gridDim.x) {
        const int b = tile / (tx_n * ty_n), r0 = tile % (tx_n * ty_n);
        const int x0 = (r0 % tx_n) * TW, y0 = (r0 / tx_n) * RH;
        __syncthreads();   // the previous tile's halo is read
        for (int i = tid; i < HR * HW * NC; i += blockDim.x) {
            const int c = i % NC, px = (i / NC) % HW, py = i / (NC * HW);
            const int gx = x0 + px - 2, gy = y0 + py - 2;
            const bool in = gx >= 0 && gx < W && gy >= 0 && gy < H;
            cp16(in_s + (py * HW + px) * CIN + swz<NC>(c, px) * 8,
                 in ? a.in + (((int64_t)b * H + gy) * W + gx) * CIN + c * 8 : a.in, in ? 16u : 0u);
        }
        cp_wait_all();
        __syncthreads();
        float acc[R][NT][4];
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
            for (int n = 0; n < NT; n++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[r][n][q] = 0.0f;
        // B fragments of the (kk0, kk1) weight columns (k 0-7 from kk0, 8-15 from kk1) into R rows' MMAs
        auto mma_rows = [&](const uint32_t (&af)[R + 4][4], int ky, int kk0, int kk1) {
            const int kk = ((lane >> 3) & 1) ? kk1 : kk0;
            if constexpr (NT == 1) {
                uint32_t bf[2];
                ldsm_x2(bf, w_s + (lane & 7) * KP + kk);
#pragma unroll
                for (int r = 0; r < R; r++) mma_bf16(acc[r][0], af[r + ky], bf[0], bf[1]);
            } else {
#pragma unroll
                for (int np = 0; np < NT / 2; np++) {
                    uint32_t bf[4];
                    ldsm_x4(bf, w_s + (np * 16 + ((lane >> 4) << 3) + (lane & 7)) * KP + kk);
#pragma unroll
                    for (int r = 0; r < R; r++) {
                        mma_bf16(acc[r][2 * np], af[r + ky], bf[0], bf[1]);
                        mma_bf16(acc[r][2 * np + 1], af[r + ky], bf[2], bf[3]);
                    }
                }
            }
        };
        if constexpr (CIN == 8) {
            // a k step is the taps (ky, 2p) and (ky, 2p + 1), p = 0..2: lanes 0-15 address the first tap's pixels,
            // lanes 16-31 the second's; the sixth tap (kx = 5) reads the zero row against the zero weight column
#pragma unroll 1
            for (int p = 0; p < 3; p++) {
                const int kx = 2 * p + khalf;
                uint32_t af[R + 4][4];
#pragma unroll
                for (int ir = 0; ir < R + 4; ir++)
                    ldsm_x4(af[ir], kx <= 4 ? in_s + ((rb * R + ir) * HW + 16 * mt + row + kx) * CIN : zrow);
#pragma unroll
                for (int ky = 0; ky < 5; ky++) {
                    const int kk0 = (ky * 5 + 2 * p) * CIN;
                    mma_rows(af, ky, kk0, p < 2 ? kk0 + CIN : 25 * CIN);
                }
            }
        } else {
#pragma unroll 1
        for (int kx = 0; kx < 5; kx++) {
#pragma unroll
            for (int kc = 0; kc < CIN / 16; kc++) {
                const int c = kc * 2 + khalf, p = 16 * mt + row + kx;
                const __nv_bfloat16* abase = in_s + (rb * R * HW + p) * CIN + swz<NC>(c, p) * 8;
                uint32_t af[R + 4][4];
#pragma unroll
                for (int ir = 0; ir < R + 4; ir++) ldsm_x4(af[ir], abase + ir * HW * CIN);
#pragma unroll
                for (int ky = 0; ky < 5; ky++) {
                    const int kk = (ky * 5 + kx) * CIN + kc * 16;
                    mma_rows(af, ky, kk, kk + 8);
                }
            }
        }
        }
        // epilogue: fragment element q of (row r, n tile) is pixel 16 mt + lane/4 (+8 for q >= 2), channel
        // 8 n + 2 (lane%4) + q%2
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int py = y0 + rb * R + r;
            if (py >= H) continue;
#pragma unroll
            for (int half = 0; half < 2; half++) {
                const int px = x0 + 16 * mt + (lane >> 2) + half * 8;
                if (px >= W) continue;
                const int64_t pix = ((int64_t)b * H + py) * W + px;
#pragma unroll
                for (int n = 0; n < NT; n++) {
                    const int co = n * 8 + 2 * (lane & 3);
                    float v0 = acc[r][n][2 * half], v1 = acc[r][n][2 * half + 1];
                    if constexpr (MODE != CONV_GRAD_MASK) {
                        if (a.bias) {
                            if (co < a.bias_n) v0 += a.bias[co];
                            if (co + 1 < a.bias_n) v1 += a.bias[co + 1];
                        }
                    }
                    if constexpr (MODE == CONV_RELU) {
                        *reinterpret_cast<__nv_bfloat162*>(a.out_b + pix * COUT + co) =
                            __floats2bfloat162_rn(fmaxf(v0, 0.0f), fmaxf(v1, 0.0f));
                    } else if constexpr (MODE == CONV_LINEAR) {
                        *reinterpret_cast<float2*>(a.out_f + pix * COUT + co) = make_float2(v0, v1);
                    } else {
                        const __nv_bfloat162 mk = *reinterpret_cast<const __nv_bfloat162*>(a.mask + pix * COUT + co);
                        if (!(__bfloat162float(mk.x) > 0.0f)) v0 = 0.0f;
                        if (!(__bfloat162float(mk.y) > 0.0f)) v1 = 0.0f;
                        *reinterpret_cast<__nv_bfloat162*>(a.out_b + pix * COUT + co) = __floats2bfloat162_rn(v0, v1);
                    }
                }
            }
        }
    }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(CONV_THREADS, 1) k_conv_wgrad(WgradArgs a) {
    constexpr int NCI = CIN / 8;
    constexpr int COP = COUT < 16 ? 16 : COUT, NCO = COP / 8;   // output channels as staged (zero padded to 16)
    constexpr int MT = COP / 16;
    constexpr int UNITS = CNN_TAPS * MT;                        // (tap, m tile)
    constexpr int UPW = (UNITS + 7) / 8;
    constexpr int NT = CIN / 8;
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* in_s = reinterpret_cast<__nv_bfloat16*>(smem);   // [HH][HW][CIN]
    __nv_bfloat16* dy_s = in_s + HH * HW * CIN;                     // [TH][TW][COP]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int H = a.H, W = a.W;
    const int tx_n = (W + TW - 1) / TW, ty_n = (H + TH - 1) / TH;
    const int total = a.B * tx_n * ty_n;
    float acc[UPW][NT][4];
#pragma unroll
    for (int u = 0; u < UPW; u++)
#pragma unroll
        for (int n = 0; n < NT; n++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[u][n][q] = 0.0f;
    float dbacc = 0.0f;
    for (int tile = blockIdx.x; tile < total; tile += gridDim.x) {
        const int b = tile / (tx_n * ty_n), r = tile % (tx_n * ty_n);
        const int x0 = (r % tx_n) * TW, y0 = (r / tx_n) * TH;
        __syncthreads();
        stage_halo<CIN>(in_s, a.in, b, x0, y0, H, W);
        for (int i = tid; i < TH * TW * NCO; i += blockDim.x) {
            const int c = i % NCO, px = (i / NCO) % TW, py = i / (NCO * TW);
            const int gx = x0 + px, gy = y0 + py;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (c * 8 < COUT && gx < W && gy < H)
                v = *reinterpret_cast<const uint4*>(a.dy + (((int64_t)b * H + gy) * W + gx) * COUT + c * 8);
            *reinterpret_cast<uint4*>(dy_s + (py * TW + px) * COP + swz<NCO>(c, px) * 8) = v;
        }
        __syncthreads();
        if (lane < COUT) {   // the bias gradient: warp w sums pixels w, w+8, ...
            const int c = lane >> 3, e = lane & 7;
            for (int p = warp; p < TH * TW; p += 8) {
                const int px = p % TW;
                dbacc += __bfloat162float(dy_s[p * COP + swz<NCO>(c, px) * 8 + e]);
            }
        }
#pragma unroll 1
        for (int ks = 0; ks < TH * TW / 16; ks++) {
            const int py = ks >> 1, px0 = (ks & 1) * 16;
            // A (output channels x 16 pixels) from dy, transposed: lane -> matrix j = lane/8: pixel (j/2)*8 + lane%8,
            // channel chunk 2 m + j%2
            uint32_t af[MT][4];
#pragma unroll
            for (int m = 0; m < MT; m++) {
                const int j = lane >> 3, px = px0 + (j >> 1) * 8 + (lane & 7);
                ldsm_x4_t(af[m], dy_s + (py * TW + px) * COP + swz<NCO>(m * 2 + (j & 1), px) * 8);
            }
#pragma unroll
            for (int u = 0; u < UPW; u++) {
                const int unit = warp + 8 * u;
                if (unit >= UNITS) break;
                const int tap = unit / MT, m = unit % MT;
                const int ky = tap / 5, kx = tap % 5, hy = py + ky;
                // B (16 pixels x input channels) from the halo, transposed: lane -> matrix j: pixel (j%2)*8 + lane%8,
                // channel chunk 2 np + j/2
                if constexpr (NT == 1) {
                    uint32_t bf[2];
                    const int hx = px0 + ((lane >> 3) & 1) * 8 + (lane & 7) + kx;
                    ldsm_x2_t(bf, in_s + (hy * HW + hx) * CIN);
                    mma_bf16(acc[u][0], af[m], bf[0], bf[1]);
                } else {
#pragma unroll
                    for (int np = 0; np < NT / 2; np++) {
                        uint32_t bf[4];
                        const int j = lane >> 3, hx = px0 + (j & 1) * 8 + (lane & 7) + kx;
                        ldsm_x4_t(bf, in_s + (hy * HW + hx) * CIN + swz<NCI>(np * 2 + (j >> 1), hx) * 8);
                        mma_bf16(acc[u][2 * np], af[m], bf[0], bf[1]);
                        mma_bf16(acc[u][2 * np + 1], af[m], bf[2], bf[3]);
                    }
                }
            }
        }
    }
    // into the fp32 gradient: fragment element q of (unit, n) is output channel 16 m + lane/4 (+8 for q >= 2),
    // input channel 8 n + 2 (lane%4) + q%2
#pragma unroll
    for (int u = 0; u < UPW; u++) {
        const int unit = warp + 8 * u;
        if (unit >= UNITS) break;
        const int tap = unit / MT, m = unit % MT;
#pragma unroll
        for (int n = 0; n < NT; n++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int co = m * 16 + (lane >> 2) + (q >= 2 ? 8 : 0);
                const int ci = n * 8 + 2 * (lane & 3) + (q & 1);
                if (co < a.cout_real && ci < a.cin_real && acc[u][n][q] != 0.0f)
                    atomicAdd(&a.dw[((int64_t)co * CNN_TAPS + tap) * a.cin_real + ci], acc[u][n][q]);
            }
    }
    if (lane < a.cout_real && dbacc != 0.0f) atomicAdd(&a.db[lane], dbacc);
}

// Launches of the instantiations the network uses (the templates stay in this translation unit).
const void* conv_kernel(int cin, int cout, int mode, bool rows) {
    if (rows) {
        if (cin == 8 && cout == 32 && mode == CONV_RELU) return (const void*)k_conv_rows<8, 32, CONV_RELU, 4>;
        if (cin == 32 && cout == 32 && mode == CONV_RELU) return (const void*)k_conv_rows<32, 32, CONV_RELU, 4>;
        if (cin == 32 && cout == 8 && mode == CONV_LINEAR) return (const void*)k_conv_rows<32, 8, CONV_LINEAR, CONV3_ROWS>;
        if (cin == 8 && cout == 32 && mode == CONV_GRAD_MASK) return (const void*)k_conv_rows<8, 32, CONV_GRAD_MASK, 4>;
        if (cin == 32 && cout == 32 && mode == CONV_GRAD_MASK) return (const void*)k_conv_rows<32, 32, CONV_GRAD_MASK, 4>;
        return nullptr;
    }
    if (cin == 8 && cout == 32 && mode == CONV_RELU) return (const void*)k_conv<8, 32, CONV_RELU>;
    if (cin == 32 && cout == 32 && mode == CONV_RELU) return (const void*)k_conv<32, 32, CONV_RELU>;
    if (cin == 32 && cout == 8 && mode == CONV_LINEAR) return (const void*)k_conv<32, 8, CONV_LINEAR>;
    if (cin == 8 && cout == 32 && mode == CONV_GRAD_MASK) return (const void*)k_conv<8, 32, CONV_GRAD_MASK>;
    if (cin == 32 && cout == 32 && mode == CONV_GRAD_MASK) return (const void*)k_conv<32, 32, CONV_GRAD_MASK>;
    return nullptr;
}

const void* wgrad_kernel(int cin, int cout) {
    if (cin == 8 && cout == 32) return (const void*)k_conv_wgrad<8, 32>;
    if (cin == 32 && cout == 32) return (const void*)k_conv_wgrad<32, 32>;
    if (cin == 32 && cout == 8) return (const void*)k_conv_wgrad<32, 8>;
    return nullptr;
}

cudaError_t launch_conv(int cin, int cout, int mode, bool rows, int grid, const ConvArgs& a, cudaStream_t s) {
    const void* k = conv_kernel(cin, cout, mode, rows);
    if (!k) return cudaErrorInvalidValue;
    void* args[] = {const_cast<ConvArgs*>(&a)};
    return cudaLaunchKernel(k, dim3(grid), dim3(CONV_THREADS), args, conv_smem(cin, cout, rows), s);
}

cudaError_t launch_wgrad(int cin, int cout, int grid, const WgradArgs& a, cudaStream_t s) {
    const void* k = wgrad_kernel(cin, cout);
    if (!k) return cudaErrorInvalidValue;
    void* args[] = {const_cast<WgradArgs*>(&a)};
    return cudaLaunchKernel(k, dim3(grid), dim3(CONV_THREADS), args, wgrad_smem(cin, cout), s);
}

}  // namespace vf
