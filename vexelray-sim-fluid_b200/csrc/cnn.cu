// cnn.cu -- the flux-correction network's handle: samples, forward, loss, backward, Adam, and the
// correction of a coarse shallow-water state (vf_cnn_*).
//
// The correction: the network maps the coarse state (h, hu, hv) to six fields per cell, G_e (the east face) and
// G_n (the north face) for each of the three conserved quantities; the state changes by their divergence,
//   U(i,j) -= s_flux * (G_e(i,j) - G_e(i-1,j) + G_n(i,j) - G_n(i,j-1)),
// with the faces on the domain's walls held at zero, so every correction moves mass and momentum between
// neighbours and the totals are conserved exactly as the plain step conserves them (ShallowWater.kernel's
// flux form, ShallowWater.java:206-235).
//
// Training sample: the coarse state S at t, the plain coarse solver's state P after an interval from S, and the
// fine solver's state after the same interval restricted to the coarse grid, T. The loss is the mean over
// cells, components and samples of ((P - s_flux Div G(S) - T) / s_res)^2 / 2.
#include <algorithm>
#include <cmath>
#include <vector>

#include "cnn.cuh"
#include "profiler.cuh"

using namespace vf;

namespace {

using bf16 = __nv_bfloat16;

constexpr int EW_THREADS = 256;

// Features of one sample: (h - 1) * 4, hu * 4, hv * 4, then zeros, as bf16 [cells][8].
__global__ void k_features(const float* __restrict__ s, bf16* __restrict__ x0, int64_t cells) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= cells) return;
    __align__(16) bf16 v[8];
    v[0] = __float2bfloat16_rn((s[p] - 1.0f) * CNN_SCALE_H);
    v[1] = __float2bfloat16_rn(s[cells + p] * CNN_SCALE_Q);
    v[2] = __float2bfloat16_rn(s[2 * cells + p] * CNN_SCALE_Q);
#pragma unroll
    for (int c = 3; c < 8; c++) v[c] = __float2bfloat16_rn(0.0f);
    *reinterpret_cast<uint4*>(x0 + p * 8) = *reinterpret_cast<const uint4*>(v);
}

// The divergence of the six face fields at cell (i, j) for component c, walls' faces zero.
__device__ __forceinline__ float flux_div(const float* __restrict__ y3, int i, int j, int nx, int ny, int c) {
    const int64_t p = (int64_t)j * nx + i;
    const float ge = i < nx - 1 ? y3[p * 8 + c] : 0.0f;
    const float gw = i > 0 ? y3[(p - 1) * 8 + c] : 0.0f;
    const float gn = j < ny - 1 ? y3[p * 8 + 3 + c] : 0.0f;
    const float gs = j > 0 ? y3[(p - nx) * 8 + 3 + c] : 0.0f;
    return (ge - gw) + (gn - gs);
}

// r = P - s_flux Div G - T per cell and component of one sample; sum of (r / s_res)^2 into *loss.
__global__ void k_residual(const float* __restrict__ plain, const float* __restrict__ target, const float* __restrict__ y3,
                           float* __restrict__ r, int nx, int ny, float s_flux, float inv_res, double* loss) {
    const int64_t cells = (int64_t)nx * ny;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float acc = 0.0f;
    if (p < cells) {
        const int i = (int)(p % nx), j = (int)(p / nx);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float v = plain[c * cells + p] - s_flux * (y3 ? flux_div(y3, i, j, nx, ny, c) : 0.0f) - target[c * cells + p];
            r[c * cells + p] = v;
            acc += (v * inv_res) * (v * inv_res);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc != 0.0f) atomicAdd(loss, (double)acc);
}

// The loss's gradient at the network's output, times the number of terms of the mean: for the east face of
// (i, j), (s_flux / s_res^2) (r(i+1, j) - r(i, j)) per component (zero on the east wall), the north face likewise.
__global__ void k_flux_grad(const float* __restrict__ r, bf16* __restrict__ dy3, int nx, int ny, float k) {
    const int64_t cells = (int64_t)nx * ny;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= cells) return;
    const int i = (int)(p % nx), j = (int)(p / nx);
    __align__(16) bf16 v[8];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float rc = r[c * cells + p];
        v[c] = __float2bfloat16_rn(i < nx - 1 ? k * (r[c * cells + p + 1] - rc) : 0.0f);
        v[3 + c] = __float2bfloat16_rn(j < ny - 1 ? k * (r[c * cells + p + nx] - rc) : 0.0f);
    }
    v[6] = v[7] = __float2bfloat16_rn(0.0f);
    *reinterpret_cast<uint4*>(dy3 + p * 8) = *reinterpret_cast<const uint4*>(v);
}

// The correction of a state in place: U -= s_flux Div G, depth kept >= 0.
__global__ void k_apply_flux(float* __restrict__ h, float* __restrict__ hu, float* __restrict__ hv,
                             const float* __restrict__ y3, int nx, int ny, float s_flux) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)nx * ny) return;
    const int i = (int)(p % nx), j = (int)(p / nx);
    const float dh = flux_div(y3, i, j, nx, ny, 0), du = flux_div(y3, i, j, nx, ny, 1), dv = flux_div(y3, i, j, nx, ny, 2);
    h[p] = fmaxf(h[p] - s_flux * dh, 0.0f);
    hu[p] -= s_flux * du;
    hv[p] -= s_flux * dv;
}

// Adam (Kingma & Ba) on the fp32 master parameters; g = grad * scale.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ grad, float* __restrict__ m, float* __restrict__ v,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2, float scale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = grad[i] * scale;
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

struct Packed {
    bf16 *w1, *w2, *w3, *t2, *t3;
};

// The bf16 weight matrices from the master parameters: forward [cout][k] and backward (transposed, taps
// mirrored) for layers 2 and 3.
__global__ void k_pack(const float* __restrict__ P, Packed o) {
    const int K1 = conv_k(8), K2 = conv_k(32);
    const int n1 = CNN_HID * K1, n2 = CNN_HID * K2, n3 = CNN_OUT * K2, nt3 = CNN_HID * K1, nt2 = CNN_HID * K2;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n1 + n2 + n3 + nt3 + nt2; e += gridDim.x * blockDim.x) {
        int k = e;
        if (k < n1) {   // w1 [32][26 x 8]
            const int co = k / K1, tap = (k % K1) / 8, ci = k % 8;
            o.w1[k] = __float2bfloat16_rn(tap < CNN_TAPS && ci < CNN_FEATURES ? P[P_W1 + (co * CNN_TAPS + tap) * CNN_FEATURES + ci] : 0.0f);
            continue;
        }
        k -= n1;
        if (k < n2) {   // w2 [32][25 x 32]
            const int co = k / K2, tap = (k % K2) / 32, ci = k % 32;
            o.w2[k] = __float2bfloat16_rn(P[P_W2 + (co * CNN_TAPS + tap) * CNN_HID + ci]);
            continue;
        }
        k -= n2;
        if (k < n3) {   // w3 [8][25 x 32], rows 6, 7 zero
            const int co = k / K2, tap = (k % K2) / 32, ci = k % 32;
            o.w3[k] = __float2bfloat16_rn(co < CNN_FLUXES ? P[P_W3 + (co * CNN_TAPS + tap) * CNN_HID + ci] : 0.0f);
            continue;
        }
        k -= n3;
        if (k < nt3) {   // layer 3 backward: [32 = its input channel][26 x 8 = mirrored tap, its output channel]
            const int ci = k / K1, t = (k % K1) / 8, co = k % 8;
            o.t3[k] = __float2bfloat16_rn(t < CNN_TAPS && co < CNN_FLUXES
                                              ? P[P_W3 + (co * CNN_TAPS + (CNN_TAPS - 1 - t)) * CNN_HID + ci] : 0.0f);
            continue;
        }
        k -= nt3;
        {   // layer 2 backward: [32][25 x 32]
            const int ci = k / K2, t = (k % K2) / 32, co = k % 32;
            o.t2[k] = __float2bfloat16_rn(P[P_W2 + (co * CNN_TAPS + (CNN_TAPS - 1 - t)) * CNN_HID + ci]);
        }
    }
}

}  // namespace

struct vf_cnn {
    int nx, ny, batch, cap;
    int64_t cells;
    float s_flux, s_res;
    cudaStream_t stream = nullptr;
    DeviceBuffer params, grads, adam_m, adam_v;
    DeviceBuffer w1, w2, w3, t2, t3;
    DeviceBuffer x0, a1, a2, y3, dy3, dy2, dy1, resid, loss;
    DeviceBuffer samples;   // cap x {state, plain, target} x 3 fields x cells floats
    DeviceBuffer state;     // the state a prediction reads, 3 planes
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    int64_t adam_steps = 0;
    bool predicted = false;   // y3 holds a prediction not yet applied
    int path = 0;             // the convolutions: 0 tcgen05, 1 mma.sync row-blocked, 2 mma.sync one row per warp
    int grid_conv[2][5] = {{0}}, grid_wgrad[3] = {0};
    DeviceBuffer status;
    Profiler prof;
};

namespace {

float* sample(vf_cnn* h, int slot, int kind) {
    return h->samples.as<float>() + ((int64_t)slot * 3 + kind) * 3 * h->cells;
}

int32_t pack(vf_cnn* h) {
    Packed o{h->w1.as<bf16>(), h->w2.as<bf16>(), h->w3.as<bf16>(), h->t2.as<bf16>(), h->t3.as<bf16>()};
    VF_LAUNCH(h->prof, "k_pack", h->stream, k_pack, sm_count() * 2, 256, 0, h->params.as<float>(), o);
    return VF_OK;
}

int conv_index(int cin, int cout, int mode) {
    return mode == CONV_RELU ? (cin == 8 ? 0 : 1) : mode == CONV_LINEAR ? 2 : (cin == 8 ? 3 : 4);
}

int32_t conv(vf_cnn* h, const char* name, int cin, int cout, int mode, const bf16* in, const bf16* w,
             const float* bias, int bias_n, bf16* out_b, float* out_f, const bf16* mask, int nb) {
    ConvArgs a{in, w, bias, bias_n, out_b, out_f, mask, h->ny, h->nx, nb};
    h->prof.begin(name, h->stream);
    const int k = conv_index(cin, cout, mode);
    cudaError_t e = h->path == 0   ? launch_conv_tc(cin, cout, mode, a, h->status.as<uint32_t>(), h->stream)
                    : h->path == 2            ? launch_conv(cin, cout, mode, false, h->grid_conv[1][k], a, h->stream)
                                              : launch_conv(cin, cout, mode, true, h->grid_conv[0][k], a, h->stream);
    h->prof.end(h->stream);
    VF_TRY_CUDA(e);
    return VF_OK;
}

int32_t cnn_status(vf_cnn* h) {
    uint32_t st = 0;
    VF_TRY_CUDA(cudaMemcpyAsync(&st, h->status.ptr, 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    if (st) {
        VF_TRY_CUDA(cudaMemsetAsync(h->status.ptr, 0, 4, h->stream));
        set_error("a network kernel flagged device status 0x%x", st);
        return (st & ST_TIMEOUT) ? VF_ETIMEOUT : VF_EDEVICE;
    }
    return VF_OK;
}

int32_t wgrad(vf_cnn* h, const char* name, int cin, int cout, int grid, const bf16* in, const bf16* dy, float* dw,
              float* db, int cin_real, int cout_real, int nb) {
    WgradArgs a{in, dy, dw, db, cin_real, cout_real, h->ny, h->nx, nb};
    h->prof.begin(name, h->stream);
    cudaError_t e = launch_wgrad(cin, cout, grid, a, h->stream);
    h->prof.end(h->stream);
    VF_TRY_CUDA(e);
    return VF_OK;
}

// Forward over nb states laid out as 3 planes each at states[b] (device).
int32_t forward(vf_cnn* h, const float* const* states, int nb) {
    const int64_t cells = h->cells;
    for (int b = 0; b < nb; b++)
        VF_LAUNCH(h->prof, "k_features", h->stream, k_features, div_up(cells, EW_THREADS), EW_THREADS, 0, states[b],
                  h->x0.as<bf16>() + b * cells * 8, cells);
    const float* P = h->params.as<float>();
    int32_t rc;
    if ((rc = conv(h, "k_conv1", 8, 32, CONV_RELU, h->x0.as<bf16>(), h->w1.as<bf16>(), P + P_B1,
                   CNN_HID, h->a1.as<bf16>(), nullptr, nullptr, nb)) ||
        (rc = conv(h, "k_conv2", 32, 32, CONV_RELU, h->a1.as<bf16>(), h->w2.as<bf16>(), P + P_B2,
                   CNN_HID, h->a2.as<bf16>(), nullptr, nullptr, nb)) ||
        (rc = conv(h, "k_conv3", 32, 8, CONV_LINEAR, h->a2.as<bf16>(), h->w3.as<bf16>(), P + P_B3,
                   CNN_FLUXES, nullptr, h->y3.as<float>(), nullptr, nb)))
        return rc;
    return VF_OK;
}

// Forward, loss and backward over the sample slots; gradients (times the number of loss terms) in h->grads.
int32_t forward_backward(vf_cnn* h, const int32_t* slots, int nb, double* loss_out, bool backward) {
    VF_REQUIRE(nb >= 1 && nb <= h->batch, VF_EINVAL, "1 to %d samples per step, got %d", h->batch, nb);
    std::vector<const float*> st((size_t)nb);
    for (int b = 0; b < nb; b++) {
        VF_REQUIRE(slots[b] >= 0 && slots[b] < h->cap, VF_EINVAL, "no sample slot %d", slots[b]);
        st[b] = sample(h, slots[b], 0);
    }
    int32_t rc = forward(h, st.data(), nb);
    if (rc) return rc;
    const int64_t cells = h->cells;
    VF_TRY_CUDA(cudaMemsetAsync(h->loss.ptr, 0, 8, h->stream));
    for (int b = 0; b < nb; b++)
        VF_LAUNCH(h->prof, "k_residual", h->stream, k_residual, div_up(cells, EW_THREADS), EW_THREADS, 0,
                  sample(h, slots[b], 1), sample(h, slots[b], 2), h->y3.as<float>() + b * cells * 8,
                  h->resid.as<float>() + b * 3 * cells, h->nx, h->ny, h->s_flux, 1.0f / h->s_res, h->loss.as<double>());
    double sum = 0;
    VF_TRY_CUDA(cudaMemcpyAsync(&sum, h->loss.ptr, 8, cudaMemcpyDeviceToHost, h->stream));
    if (backward) {
        const float k = h->s_flux / (h->s_res * h->s_res);
        for (int b = 0; b < nb; b++)
            VF_LAUNCH(h->prof, "k_flux_grad", h->stream, k_flux_grad, div_up(cells, EW_THREADS), EW_THREADS, 0,
                      h->resid.as<float>() + b * 3 * cells, h->dy3.as<bf16>() + b * cells * 8, h->nx, h->ny, k);
        float* G = h->grads.as<float>();
        VF_TRY_CUDA(cudaMemsetAsync(G, 0, h->grads.bytes, h->stream));
        if ((rc = wgrad(h, "k_wgrad3", 32, 8, h->grid_wgrad[2], h->a2.as<bf16>(), h->dy3.as<bf16>(), G + P_W3,
                        G + P_B3, CNN_HID, CNN_FLUXES, nb)) ||
            (rc = conv(h, "k_dgrad3", 8, 32, CONV_GRAD_MASK, h->dy3.as<bf16>(), h->t3.as<bf16>(),
                       nullptr, 0, h->dy2.as<bf16>(), nullptr, h->a2.as<bf16>(), nb)) ||
            (rc = wgrad(h, "k_wgrad2", 32, 32, h->grid_wgrad[1], h->a1.as<bf16>(), h->dy2.as<bf16>(), G + P_W2,
                        G + P_B2, CNN_HID, CNN_HID, nb)) ||
            (rc = conv(h, "k_dgrad2", 32, 32, CONV_GRAD_MASK, h->dy2.as<bf16>(), h->t2.as<bf16>(),
                       nullptr, 0, h->dy1.as<bf16>(), nullptr, h->a1.as<bf16>(), nb)) ||
            (rc = wgrad(h, "k_wgrad1", 8, 32, h->grid_wgrad[0], h->x0.as<bf16>(), h->dy1.as<bf16>(), G + P_W1,
                        G + P_B1, CNN_FEATURES, CNN_HID, nb)))
            return rc;
    }
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    if (loss_out) *loss_out = sum / (2.0 * 3.0 * (double)cells * nb);
    return cnn_status(h);
}

}  // namespace

extern "C" {

int64_t vf_cnn_param_count(void) { return CNN_PARAMS; }

int32_t vf_cnn_create(int32_t nx, int32_t ny, int32_t batch, int32_t samples, float s_flux, float s_res, vf_cnn** out) {
    VF_REQUIRE(out, VF_EINVAL, "out is null");
    *out = nullptr;
    VF_REQUIRE(nx >= 1 && ny >= 1 && (int64_t)nx * ny <= (1ll << 28), VF_EINVAL, "grid %d x %d", nx, ny);
    VF_REQUIRE(batch >= 1 && samples >= 1, VF_EINVAL, "batch and samples >= 1, got %d, %d", batch, samples);
    VF_REQUIRE(s_flux > 0 && s_res > 0, VF_EINVAL, "flux and residual scales > 0, got %g, %g", s_flux, s_res);
    int32_t rc = require_device();
    if (rc) return rc;
    vf_cnn* h = new vf_cnn();
    h->nx = nx;
    h->ny = ny;
    h->batch = batch;
    h->cap = samples;
    h->cells = (int64_t)nx * ny;
    h->s_flux = s_flux;
    h->s_res = s_res;
    auto fail = [&](int32_t code) {
        vf_cnn_destroy(h);
        return code;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("cudaStreamCreate failed");
        return fail(VF_ECUDA);
    }
    const size_t bc = (size_t)batch * h->cells;
    const size_t pb = (size_t)CNN_PARAMS * 4;
    if ((rc = h->params.alloc(pb)) || (rc = h->grads.alloc(pb)) || (rc = h->adam_m.alloc(pb)) ||
        (rc = h->adam_v.alloc(pb)) || (rc = h->w1.alloc((size_t)CNN_HID * conv_k(8) * 2)) ||
        (rc = h->w2.alloc((size_t)CNN_HID * conv_k(32) * 2)) || (rc = h->w3.alloc((size_t)CNN_OUT * conv_k(32) * 2)) ||
        (rc = h->t2.alloc((size_t)CNN_HID * conv_k(32) * 2)) || (rc = h->t3.alloc((size_t)CNN_HID * conv_k(8) * 2)) ||
        (rc = h->x0.alloc(bc * 8 * 2)) || (rc = h->a1.alloc(bc * 32 * 2)) || (rc = h->a2.alloc(bc * 32 * 2)) ||
        (rc = h->y3.alloc(bc * 8 * 4)) || (rc = h->dy3.alloc(bc * 8 * 2)) || (rc = h->dy2.alloc(bc * 32 * 2)) ||
        (rc = h->dy1.alloc(bc * 32 * 2)) || (rc = h->resid.alloc(bc * 3 * 4)) || (rc = h->loss.alloc(16)) ||
        (rc = h->samples.alloc((size_t)samples * 9 * h->cells * 4)) || (rc = h->state.alloc((size_t)3 * h->cells * 4)) ||
        (rc = h->status.alloc(16)))
        return fail(rc);
    if (cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming) != cudaSuccess) {
        set_error("cudaEventCreate failed");
        return fail(VF_ECUDA);
    }
    const int modes[5][3] = {{8, 32, CONV_RELU}, {32, 32, CONV_RELU}, {32, 8, CONV_LINEAR}, {8, 32, CONV_GRAD_MASK},
                             {32, 32, CONV_GRAD_MASK}};
    const int wg[3][2] = {{8, 32}, {32, 32}, {32, 8}};
    for (int k = 0; k < 13; k++) {
        const bool is_conv = k < 10;
        const int c = k % 5;
        const bool rows = k < 5;
        const void* fn = is_conv ? conv_kernel(modes[c][0], modes[c][1], modes[c][2], rows)
                                 : wgrad_kernel(wg[k - 10][0], wg[k - 10][1]);
        const size_t smem = is_conv ? conv_smem(modes[c][0], modes[c][1], rows) : wgrad_smem(wg[k - 10][0], wg[k - 10][1]);
        int per = 0;
        if (!fn || cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, 256, smem) != cudaSuccess) {
            set_error("cannot give a convolution kernel %zu bytes of shared memory", smem);
            return fail(VF_ECUDA);
        }
        (is_conv ? h->grid_conv[rows ? 0 : 1][c] : h->grid_wgrad[k - 10]) = std::max(per, 1) * sm_count();
    }
    for (int k = 0; k < 5; k++) {
        const void* fn = conv_tc_kernel(modes[k][0], modes[k][1], modes[k][2]);
        const size_t smem = conv_tc_smem(modes[k][0], modes[k][1]);
        if (!fn || cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
            set_error("cannot give a tensor-core convolution %zu bytes of shared memory", smem);
            return fail(VF_ECUDA);
        }
    }
    for (DeviceBuffer* b : {&h->params, &h->grads, &h->adam_m, &h->adam_v, &h->samples, &h->status})
        if (cudaMemsetAsync(b->ptr, 0, b->bytes, h->stream) != cudaSuccess) return fail(VF_ECUDA);
    if (pack(h) || cudaStreamSynchronize(h->stream) != cudaSuccess) {
        set_error("initialising the network failed");
        return fail(VF_ECUDA);
    }
    *out = h;
    return VF_OK;
}

int32_t vf_cnn_params(vf_cnn* h, float* host, int64_t n, int32_t write) {
    VF_REQUIRE(h && host, VF_EINVAL, "null argument");
    VF_REQUIRE(n == CNN_PARAMS, VF_EINVAL, "the network has %d parameters, got %lld", CNN_PARAMS, (long long)n);
    if (write) {
        VF_TRY_CUDA(cudaMemcpyAsync(h->params.ptr, host, (size_t)n * 4, cudaMemcpyHostToDevice, h->stream));
        VF_TRY_CUDA(cudaMemsetAsync(h->adam_m.ptr, 0, h->adam_m.bytes, h->stream));
        VF_TRY_CUDA(cudaMemsetAsync(h->adam_v.ptr, 0, h->adam_v.bytes, h->stream));
        h->adam_steps = 0;
        int32_t rc = pack(h);
        if (rc) return rc;
    } else {
        VF_TRY_CUDA(cudaMemcpyAsync(host, h->params.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost, h->stream));
    }
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

int32_t vf_cnn_put(vf_cnn* h, int32_t slot, int32_t kind, const float* hcell, const float* hu, const float* hv,
                   int32_t from_host) {
    VF_REQUIRE(h && hcell && hu && hv, VF_EINVAL, "null argument");
    VF_REQUIRE(slot >= 0 && slot < h->cap && kind >= 0 && kind < 3, VF_EINVAL, "slot %d of %d, kind %d of 3", slot,
               h->cap, kind);
    const float* src[3] = {hcell, hu, hv};
    for (int f = 0; f < 3; f++)
        VF_TRY_CUDA(cudaMemcpyAsync(sample(h, slot, kind) + f * h->cells, src[f], (size_t)h->cells * 4,
                                    from_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

int32_t vf_cnn_loss(vf_cnn* h, const int32_t* slots, int32_t n, double* loss, double* loss_plain) {
    VF_REQUIRE(h && slots, VF_EINVAL, "null argument");
    int32_t rc = forward_backward(h, slots, n, loss, false);
    if (rc || !loss_plain) return rc;
    // the same loss with no correction (G = 0)
    const int64_t cells = h->cells;
    VF_TRY_CUDA(cudaMemsetAsync(h->loss.ptr, 0, 8, h->stream));
    for (int b = 0; b < n; b++)
        VF_LAUNCH(h->prof, "k_residual", h->stream, k_residual, div_up(cells, EW_THREADS), EW_THREADS, 0,
                  sample(h, slots[b], 1), sample(h, slots[b], 2), (const float*)nullptr, h->resid.as<float>(), h->nx,
                  h->ny, h->s_flux, 1.0f / h->s_res, h->loss.as<double>());
    double sum = 0;
    VF_TRY_CUDA(cudaMemcpyAsync(&sum, h->loss.ptr, 8, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    *loss_plain = sum / (2.0 * 3.0 * (double)cells * n);
    return VF_OK;
}

int32_t vf_cnn_gradients(vf_cnn* h, const int32_t* slots, int32_t n, float* grads, double* loss) {
    VF_REQUIRE(h && slots && grads, VF_EINVAL, "null argument");
    int32_t rc = forward_backward(h, slots, n, loss, true);
    if (rc) return rc;
    std::vector<float> g((size_t)CNN_PARAMS);
    VF_TRY_CUDA(cudaMemcpyAsync(g.data(), h->grads.ptr, g.size() * 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    const double scale = 1.0 / (3.0 * (double)h->cells * n);
    for (int k = 0; k < CNN_PARAMS; k++) grads[k] = (float)(g[k] * scale);
    return VF_OK;
}

int32_t vf_cnn_train(vf_cnn* h, const int32_t* slots, int32_t n, float lr, double* loss) {
    VF_REQUIRE(h && slots, VF_EINVAL, "null argument");
    VF_REQUIRE(lr > 0, VF_EINVAL, "a learning rate > 0, got %g", lr);
    int32_t rc = forward_backward(h, slots, n, loss, true);
    if (rc) return rc;
    h->adam_steps++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - (float)std::pow(0.9, (double)h->adam_steps);
    const float c2 = 1.0f - (float)std::pow(0.999, (double)h->adam_steps);
    const float scale = (float)(1.0 / (3.0 * (double)h->cells * n));
    VF_LAUNCH(h->prof, "k_adam", h->stream, k_adam, div_up(CNN_PARAMS, 256), 256, 0, h->params.as<float>(),
              h->grads.as<float>(), h->adam_m.as<float>(), h->adam_v.as<float>(), CNN_PARAMS, lr, b1, b2, 1e-8f, c1, c2,
              scale);
    if ((rc = pack(h))) return rc;
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

namespace {

// Orders the network's stream after `stream`'s work so far (no host wait).
int32_t follow(vf_cnn* h, cudaStream_t stream) {
    if (!stream) return VF_OK;
    VF_TRY_CUDA(cudaEventRecord(h->ev_in, stream));
    VF_TRY_CUDA(cudaStreamWaitEvent(h->stream, h->ev_in, 0));
    return VF_OK;
}

// Orders `stream` after the network's work so far; without a stream, waits on the host.
int32_t handback(vf_cnn* h, cudaStream_t stream) {
    if (!stream) {
        VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
        return VF_OK;
    }
    VF_TRY_CUDA(cudaEventRecord(h->ev_out, h->stream));
    VF_TRY_CUDA(cudaStreamWaitEvent(stream, h->ev_out, 0));
    return VF_OK;
}

}  // namespace

int32_t vf_cnn_predict(vf_cnn* h, const float* hcell, const float* hu, const float* hv, void* stream) {
    VF_REQUIRE(h && hcell && hu && hv, VF_EINVAL, "null argument");
    int32_t rc = follow(h, (cudaStream_t)stream);
    if (rc) return rc;
    float* s = h->state.as<float>();   // the state copied into one contiguous 3-plane block for the features
    for (int f = 0; f < 3; f++)
        VF_TRY_CUDA(cudaMemcpyAsync(s + f * h->cells, f == 0 ? hcell : f == 1 ? hu : hv, (size_t)h->cells * 4,
                                    cudaMemcpyDeviceToDevice, h->stream));
    const float* st[1] = {s};
    if ((rc = forward(h, st, 1))) return rc;
    h->predicted = true;
    return handback(h, (cudaStream_t)stream);
}

int32_t vf_cnn_apply(vf_cnn* h, float* hcell, float* hu, float* hv, void* stream) {
    VF_REQUIRE(h && hcell && hu && hv, VF_EINVAL, "null argument");
    VF_REQUIRE(h->predicted, VF_ESTATE, "no prediction to apply");
    int32_t rc = follow(h, (cudaStream_t)stream);
    if (rc) return rc;
    VF_LAUNCH(h->prof, "k_apply_flux", h->stream, k_apply_flux, div_up(h->cells, EW_THREADS), EW_THREADS, 0, hcell, hu,
              hv, h->y3.as<float>(), h->nx, h->ny, h->s_flux);
    h->predicted = false;
    return handback(h, (cudaStream_t)stream);
}

int32_t vf_cnn_correct(vf_cnn* h, float* hcell, float* hu, float* hv, void* stream) {
    int32_t rc = vf_cnn_predict(h, hcell, hu, hv, stream);
    return rc ? rc : vf_cnn_apply(h, hcell, hu, hv, stream);
}

int32_t vf_cnn_fluxes(vf_cnn* h, int32_t slot, float* out) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    VF_REQUIRE(slot >= 0 && slot < h->cap, VF_EINVAL, "no sample slot %d", slot);
    const float* st[1] = {sample(h, slot, 0)};
    int32_t rc = forward(h, st, 1);
    if (rc) return rc;
    VF_TRY_CUDA(cudaMemcpyAsync(out, h->y3.ptr, (size_t)h->cells * 8 * 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return cnn_status(h);
}

void* vf_cnn_stream(vf_cnn* h) { return h ? (void*)h->stream : nullptr; }

int32_t vf_cnn_set_path(vf_cnn* h, int32_t path) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    VF_REQUIRE(path >= 0 && path <= 2, VF_EINVAL,
               "path 0 (tcgen05), 1 (mma.sync, row-blocked) or 2 (mma.sync, one row per warp), got %d", path);
    h->path = path;
    return VF_OK;
}

int32_t vf_cnn_status(vf_cnn* h) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    return cnn_status(h);
}

int32_t vf_cnn_profile(vf_cnn* h, int32_t enable) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    h->prof.collect();
    h->prof.on = enable != 0;
    if (enable) h->prof.reset();
    return VF_OK;
}

int32_t vf_cnn_profile_read(vf_cnn* h, int32_t index, char* name, size_t cap, double* total_ms, int64_t* launches) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    return h->prof.read(index, name, cap, total_ms, launches);
}

int64_t vf_cnn_launches(const vf_cnn* h) { return h ? h->prof.launches : 0; }

void vf_cnn_destroy(vf_cnn* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (DeviceBuffer* b : {&h->params, &h->grads, &h->adam_m, &h->adam_v, &h->w1, &h->w2, &h->w3, &h->t2, &h->t3, &h->x0,
                            &h->a1, &h->a2, &h->y3, &h->dy3, &h->dy2, &h->dy1, &h->resid, &h->loss, &h->samples,
                            &h->state, &h->status})
        b->release();
    if (h->ev_in) cudaEventDestroy(h->ev_in);
    if (h->ev_out) cudaEventDestroy(h->ev_out);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // extern "C"
