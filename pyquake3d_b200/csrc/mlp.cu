// Training and inference of the Newton-seeding MLP (5 -> 64 -> 64 -> 1, tanh, FP32).
// No counterpart in the reference.  Samples come from the V-mode stepper's own
// Newton solves (vmode.cu logs 5 features + the logit of the solution); the
// stepper evaluates the trained network in its stage kernel.
//
// Parameter layout (4609 floats): W1[64][5], b1[64], W2[64][64], b2[64], W3[64], b3.
// Loss: 0.5 * mean((y - t)^2) over a batch.  One step of training:
//   k_mlp_fwd    per sample: H1, H2, y                      (B x 64, B x 64, B)
//   k_mlp_bwd    per sample: d3 = (y - t)/B, D2, D1           (B, B x 64, B x 64)
//   k_mlp_wgrad  per parameter: sum over the batch (fixed order, deterministic)
//   k_adam       Adam update of every parameter
#include "pq3d_common.cuh"
#include <math.h>

namespace {
constexpr int H = 64, NIN = 5;
constexpr int OFF_W1 = 0, OFF_B1 = 320, OFF_W2 = 384, OFF_B2 = 4480, OFF_W3 = 4544, OFF_B3 = 4608, NP = 4609;

__global__ void k_mlp_fwd(const float *__restrict__ P, const float *__restrict__ X, int xstride, int B,
                          float *__restrict__ H1, float *__restrict__ H2, float *__restrict__ Y)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    float x[NIN];
#pragma unroll
    for (int i = 0; i < NIN; ++i) x[i] = X[(int64_t)b * xstride + i];
    float h1[H];
#pragma unroll 8
    for (int j = 0; j < H; ++j) {
        float s = P[OFF_B1 + j];
#pragma unroll
        for (int i = 0; i < NIN; ++i) s += P[OFF_W1 + NIN * j + i] * x[i];
        h1[j] = tanhf(s);
        if (H1) H1[(int64_t)j * B + b] = h1[j];
    }
    float y = P[OFF_B3];
    for (int j = 0; j < H; ++j) {
        float s = P[OFF_B2 + j];
#pragma unroll 16
        for (int i = 0; i < H; ++i) s += P[OFF_W2 + H * j + i] * h1[i];
        const float t = tanhf(s);
        if (H2) H2[(int64_t)j * B + b] = t;
        y += P[OFF_W3 + j] * t;
    }
    Y[b] = y;
}

__global__ void k_mlp_bwd(const float *__restrict__ P, const float *__restrict__ T, int tstride, int B,
                          const float *__restrict__ H1, const float *__restrict__ H2, const float *__restrict__ Y,
                          float *__restrict__ D3, float *__restrict__ D2, float *__restrict__ D1,
                          float *__restrict__ loss)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const float r = Y[b] - T[(int64_t)b * tstride];
    const float d3 = r / (float)B;
    D3[b] = d3;
    float d2[H];
#pragma unroll 8
    for (int j = 0; j < H; ++j) {
        const float h = H2[(int64_t)j * B + b];
        d2[j] = d3 * P[OFF_W3 + j] * (1.0f - h * h);
        D2[(int64_t)j * B + b] = d2[j];
    }
    for (int i = 0; i < H; ++i) {
        float s = 0.0f;
#pragma unroll 16
        for (int j = 0; j < H; ++j) s += P[OFF_W2 + H * j + i] * d2[j];
        const float h = H1[(int64_t)i * B + b];
        D1[(int64_t)i * B + b] = s * (1.0f - h * h);
    }
    if (loss) atomicAdd(loss, 0.5f * r * r / (float)B);
}

// Gradient of parameter p: a sum over the batch in a fixed order (one warp per parameter).
__global__ void k_mlp_wgrad(const float *__restrict__ X, int xstride, int B, const float *__restrict__ H1,
                            const float *__restrict__ H2, const float *__restrict__ D3,
                            const float *__restrict__ D2, const float *__restrict__ D1, float *__restrict__ G)
{
    const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p >= NP) return;
    float s = 0.0f;
    if (p < OFF_B1) {            // W1[j][i]
        const int j = p / NIN, i = p % NIN;
        for (int b = lane; b < B; b += 32) s += D1[(int64_t)j * B + b] * X[(int64_t)b * xstride + i];
    } else if (p < OFF_W2) {     // b1[j]
        const int j = p - OFF_B1;
        for (int b = lane; b < B; b += 32) s += D1[(int64_t)j * B + b];
    } else if (p < OFF_B2) {     // W2[j][i]
        const int q = p - OFF_W2, j = q / H, i = q % H;
        for (int b = lane; b < B; b += 32) s += D2[(int64_t)j * B + b] * H1[(int64_t)i * B + b];
    } else if (p < OFF_W3) {     // b2[j]
        const int j = p - OFF_B2;
        for (int b = lane; b < B; b += 32) s += D2[(int64_t)j * B + b];
    } else if (p < OFF_B3) {     // W3[j]
        const int j = p - OFF_W3;
        for (int b = lane; b < B; b += 32) s += D3[b] * H2[(int64_t)j * B + b];
    } else {                     // b3
        for (int b = lane; b < B; b += 32) s += D3[b];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) G[p] = s;
}

__global__ void k_adam(float *__restrict__ P, const float *__restrict__ G, float *__restrict__ M,
                       float *__restrict__ V, float lr, float b1, float b2, float eps, int step)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NP) return;
    const float g = G[p];
    const float m = b1 * M[p] + (1.0f - b1) * g;
    const float v = b2 * V[p] + (1.0f - b2) * g * g;
    M[p] = m;
    V[p] = v;
    const float mh = m / (1.0f - powf(b1, (float)step));
    const float vh = v / (1.0f - powf(b2, (float)step));
    P[p] -= lr * mh / (sqrtf(vh) + eps);
}
}  // namespace

PQ3D_EXPORT int pq3d_mlp_param_count(void) { return NP; }

// Scratch for a batch of B samples: 5 * 64 * B + 2 * B floats.
PQ3D_EXPORT int64_t pq3d_mlp_scratch_floats(int B) { return (int64_t)4 * H * B + 2 * (int64_t)B; }

// y = MLP(X) for B samples (X rows of xstride floats, the first 5 used).
PQ3D_EXPORT int pq3d_mlp_forward(const float *d_P, const float *d_X, int xstride, int B, float *d_Y,
                                 cudaStream_t stream)
{
    if (!d_P || !d_X || !d_Y || B < 0 || xstride < NIN) return PQ3D_ERR_ARG;
    if (B == 0) return PQ3D_OK;
    k_mlp_fwd<<<(B + 127) / 128, 128, 0, stream>>>(d_P, d_X, xstride, B, nullptr, nullptr, d_Y);
    return pq3d_launch_status();
}

// Gradient of 0.5 mean((MLP(X) - T)^2) into d_G (4609 floats); loss added to *d_loss if non-null.
PQ3D_EXPORT int pq3d_mlp_grad(const float *d_P, const float *d_X, int xstride, const float *d_T, int tstride, int B,
                              float *d_scratch, float *d_G, float *d_loss, cudaStream_t stream)
{
    if (!d_P || !d_X || !d_T || !d_scratch || !d_G || B <= 0 || xstride < NIN) return PQ3D_ERR_ARG;
    float *H1 = d_scratch, *H2 = H1 + (int64_t)H * B, *D2 = H2 + (int64_t)H * B, *D1 = D2 + (int64_t)H * B;
    float *Y = D1 + (int64_t)H * B, *D3 = Y + B;
    const int g = (B + 127) / 128;
    k_mlp_fwd<<<g, 128, 0, stream>>>(d_P, d_X, xstride, B, H1, H2, Y);
    k_mlp_bwd<<<g, 128, 0, stream>>>(d_P, d_T, tstride, B, H1, H2, Y, D3, D2, D1, d_loss);
    k_mlp_wgrad<<<(NP * 32 + 255) / 256, 256, 0, stream>>>(d_X, xstride, B, H1, H2, D3, D2, D1, d_G);
    return pq3d_launch_status();
}

// One Adam step (gradient of the batch, then the update); step counts from 1.
PQ3D_EXPORT int pq3d_mlp_train_step(float *d_P, float *d_M, float *d_V, const float *d_X, int xstride,
                                    const float *d_T, int tstride, int B, float *d_scratch, float *d_G,
                                    float lr, float beta1, float beta2, float eps, int step, float *d_loss,
                                    cudaStream_t stream)
{
    if (!d_M || !d_V || step < 1) return PQ3D_ERR_ARG;
    int rc = pq3d_mlp_grad(d_P, d_X, xstride, d_T, tstride, B, d_scratch, d_G, d_loss, stream);
    if (rc != PQ3D_OK) return rc;
    k_adam<<<(NP + 255) / 256, 256, 0, stream>>>(d_P, d_G, d_M, d_V, lr, beta1, beta2, eps, step);
    return pq3d_launch_status();
}
