// Learned selector support: matrix features and a small FP32 MLP
// (inputs F -> H -> H -> outputs O, ReLU) with hand-written forward,
// backward and Adam kernels.  The network predicts the log run time of each
// (ordering, accumulator) configuration of the tiled SpGEMM from cheap matrix
// features; the selector picks the argmin.
//
// Training runs one CTA per step over a minibatch (B <= TSG_MLP_MAX_B rows):
// weights, activations and gradients of the whole network fit in shared
// memory, so forward, backward (masked mean squared error) and the Adam
// update are one launch.  All arithmetic is FP32.
#include <math.h>
#include <stdlib.h>

#include "tsg_internal.h"

#define TSG_MLP_MAX_F 32
#define TSG_MLP_MAX_H 64
#define TSG_MLP_MAX_O 32
#define TSG_MLP_MAX_B 64
#define MLP_THREADS 256

struct tsg_mlp
{
    tsg_context *ctx;
    int F, H, O;
    int nparam;
    float *w;  // parameters: W1[F][H] b1[H] W2[H][H] b2[H] W3[H][O] b3[O]
    float *m1; // Adam first moments
    float *m2; // Adam second moments
    float *g;  // last gradients
    float *loss;
    long long steps;
};

struct MlpDims
{
    int F, H, O, B;
    int oW1, ob1, oW2, ob2, oW3, ob3;
};

static MlpDims dims(const tsg_mlp *m, int B)
{
    MlpDims d;
    d.F = m->F;
    d.H = m->H;
    d.O = m->O;
    d.B = B;
    d.oW1 = 0;
    d.ob1 = d.oW1 + m->F * m->H;
    d.oW2 = d.ob1 + m->H;
    d.ob2 = d.oW2 + m->H * m->H;
    d.oW3 = d.ob2 + m->H;
    d.ob3 = d.oW3 + m->H * m->O;
    return d;
}

// y[b][j] = act(sum_i x[b][i] * W[i][j] + bias[j])
__device__ void dense_fwd(const float *x, int B, int nin, const float *W, const float *bias, int nout, float *y,
                          bool relu)
{
    for (int idx = threadIdx.x; idx < B * nout; idx += blockDim.x)
    {
        const int b = idx / nout, j = idx % nout;
        float s = bias[j];
        for (int i = 0; i < nin; i++)
            s = fmaf(x[b * nin + i], W[i * nout + j], s);
        y[idx] = relu ? fmaxf(s, 0.f) : s;
    }
}

// one step: forward, masked MSE, backward; writes gradients into g and the
// loss into *loss; with lr > 0 also applies Adam (bias-corrected) to w.
__global__ void __launch_bounds__(MLP_THREADS)
    k_mlp_step(MlpDims d, int nparam, float *w, float *m1, float *m2, float *g, const float *__restrict__ X,
               const float *__restrict__ T, const float *__restrict__ M, float lr, float beta1, float beta2, float eps,
               long long step, float *loss)
{
    extern __shared__ float sh[];
    const int F = d.F, H = d.H, O = d.O, B = d.B;
    float *x = sh;                 // B*F
    float *h1 = x + B * F;         // B*H
    float *h2 = h1 + B * H;        // B*H
    float *y = h2 + B * H;         // B*O (then dY)
    float *d2 = y + B * O;         // B*H (dH2 then dH1)
    float *d1 = d2 + B * H;        // B*H
    __shared__ float s_red[MLP_THREADS];
    for (int i = threadIdx.x; i < B * F; i += blockDim.x)
        x[i] = X[i];
    __syncthreads();
    dense_fwd(x, B, F, w + d.oW1, w + d.ob1, H, h1, true);
    __syncthreads();
    dense_fwd(h1, B, H, w + d.oW2, w + d.ob2, H, h2, true);
    __syncthreads();
    dense_fwd(h2, B, H, w + d.oW3, w + d.ob3, O, y, false);
    __syncthreads();
    // masked MSE: L = sum M (y - t)^2 / sum M ; dY = 2 M (y - t) / sum M
    float msum = 0.f, lsum = 0.f;
    for (int i = threadIdx.x; i < B * O; i += blockDim.x)
    {
        const float mk = M ? M[i] : 1.f;
        const float r = y[i] - T[i];
        msum += mk;
        lsum += mk * r * r;
    }
    s_red[threadIdx.x] = msum;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1)
    {
        if (threadIdx.x < s)
            s_red[threadIdx.x] += s_red[threadIdx.x + s];
        __syncthreads();
    }
    const float denom = fmaxf(s_red[0], 1.f);
    __syncthreads();
    s_red[threadIdx.x] = lsum;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1)
    {
        if (threadIdx.x < s)
            s_red[threadIdx.x] += s_red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *loss = s_red[0] / denom;
    __syncthreads();
    for (int i = threadIdx.x; i < B * O; i += blockDim.x)
    {
        const float mk = M ? M[i] : 1.f;
        y[i] = 2.f * mk * (y[i] - T[i]) / denom;
    }
    __syncthreads();
    // layer 3 grads: dW3 = h2^T dY, db3 = sum dY
    for (int idx = threadIdx.x; idx < H * O; idx += blockDim.x)
    {
        const int i = idx / O, j = idx % O;
        float s = 0.f;
        for (int b = 0; b < B; b++)
            s = fmaf(h2[b * H + i], y[b * O + j], s);
        g[d.oW3 + idx] = s;
    }
    for (int j = threadIdx.x; j < O; j += blockDim.x)
    {
        float s = 0.f;
        for (int b = 0; b < B; b++)
            s += y[b * O + j];
        g[d.ob3 + j] = s;
    }
    // dH2 = (dY W3^T) * [h2 > 0]
    for (int idx = threadIdx.x; idx < B * H; idx += blockDim.x)
    {
        const int b = idx / H, i = idx % H;
        float s = 0.f;
        for (int j = 0; j < O; j++)
            s = fmaf(y[b * O + j], w[d.oW3 + i * O + j], s);
        d2[idx] = h2[idx] > 0.f ? s : 0.f;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < H * H; idx += blockDim.x)
    {
        const int i = idx / H, j = idx % H;
        float s = 0.f;
        for (int b = 0; b < B; b++)
            s = fmaf(h1[b * H + i], d2[b * H + j], s);
        g[d.oW2 + idx] = s;
    }
    for (int j = threadIdx.x; j < H; j += blockDim.x)
    {
        float s = 0.f;
        for (int b = 0; b < B; b++)
            s += d2[b * H + j];
        g[d.ob2 + j] = s;
    }
    for (int idx = threadIdx.x; idx < B * H; idx += blockDim.x)
    {
        const int b = idx / H, i = idx % H;
        float s = 0.f;
        for (int j = 0; j < H; j++)
            s = fmaf(d2[b * H + j], w[d.oW2 + i * H + j], s);
        d1[idx] = h1[idx] > 0.f ? s : 0.f;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < F * H; idx += blockDim.x)
    {
        const int i = idx / H, j = idx % H;
        float s = 0.f;
        for (int b = 0; b < B; b++)
            s = fmaf(x[b * F + i], d1[b * H + j], s);
        g[d.oW1 + idx] = s;
    }
    for (int j = threadIdx.x; j < H; j += blockDim.x)
    {
        float s = 0.f;
        for (int b = 0; b < B; b++)
            s += d1[b * H + j];
        g[d.ob1 + j] = s;
    }
    __syncthreads();
    if (lr > 0.f)
    {
        const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
        for (int i = threadIdx.x; i < nparam; i += blockDim.x)
        {
            const float gi = g[i];
            const float a = m1[i] = beta1 * m1[i] + (1.f - beta1) * gi;
            const float v = m2[i] = beta2 * m2[i] + (1.f - beta2) * gi * gi;
            w[i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
        }
    }
}

__global__ void __launch_bounds__(MLP_THREADS)
    k_mlp_forward(MlpDims d, const float *__restrict__ w, const float *__restrict__ X, float *__restrict__ Y)
{
    extern __shared__ float sh[];
    const int F = d.F, H = d.H, O = d.O, B = d.B;
    float *x = sh, *h1 = x + B * F, *h2 = h1 + B * H, *y = h2 + B * H;
    for (int i = threadIdx.x; i < B * F; i += blockDim.x)
        x[i] = X[(long long)blockIdx.x * B * F + i];
    __syncthreads();
    dense_fwd(x, B, F, w + d.oW1, w + d.ob1, H, h1, true);
    __syncthreads();
    dense_fwd(h1, B, H, w + d.oW2, w + d.ob2, H, h2, true);
    __syncthreads();
    dense_fwd(h2, B, H, w + d.oW3, w + d.ob3, O, y, false);
    __syncthreads();
    for (int i = threadIdx.x; i < B * O; i += blockDim.x)
        Y[(long long)blockIdx.x * B * O + i] = y[i];
}

// counter-based normal samples for He initialisation (Box-Muller on
// SplitMix64 uniforms)
static unsigned long long mix64(unsigned long long x)
{
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

static double uniform01(unsigned long long seed, unsigned long long i)
{
    return ((mix64(seed * 2654435761ULL + i) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

extern "C" int tsg_mlp_create(tsg_context *ctx, int F, int H, int O, unsigned long long seed, tsg_mlp **out)
{
    if (!ctx || !out || F < 1 || F > TSG_MLP_MAX_F || H < 1 || H > TSG_MLP_MAX_H || O < 1 || O > TSG_MLP_MAX_O)
        return tsg_set_error(TSG_ERR_INVALID, "MLP sizes must be F<=%d, H<=%d, O<=%d", TSG_MLP_MAX_F, TSG_MLP_MAX_H,
                             TSG_MLP_MAX_O);
    tsg_mlp *m = (tsg_mlp *)calloc(1, sizeof(tsg_mlp));
    m->ctx = ctx;
    m->F = F;
    m->H = H;
    m->O = O;
    m->nparam = F * H + H + H * H + H + H * O + O;
    float *hw = (float *)calloc((size_t)m->nparam, sizeof(float));
    MlpDims d = dims(m, 1);
    auto he = [&](int off, int nin, int count) {
        const double sd = sqrt(2.0 / nin);
        for (int i = 0; i < count; i++)
        {
            const double u1 = uniform01(seed, (unsigned long long)(off + i) * 2);
            const double u2 = uniform01(seed, (unsigned long long)(off + i) * 2 + 1);
            hw[off + i] = (float)(sd * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
        }
    };
    he(d.oW1, F, F * H);
    he(d.oW2, H, H * H);
    he(d.oW3, H, H * O);
    int st = tsg_alloc(ctx, &m->w, (size_t)m->nparam);
    if (st == TSG_OK)
        st = tsg_alloc(ctx, &m->m1, (size_t)m->nparam);
    if (st == TSG_OK)
        st = tsg_alloc(ctx, &m->m2, (size_t)m->nparam);
    if (st == TSG_OK)
        st = tsg_alloc(ctx, &m->g, (size_t)m->nparam);
    if (st == TSG_OK)
        st = tsg_alloc(ctx, &m->loss, 1);
    if (st != TSG_OK)
    {
        free(hw);
        free(m);
        return st;
    }
    cudaMemcpyAsync(m->w, hw, sizeof(float) * m->nparam, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemsetAsync(m->m1, 0, sizeof(float) * m->nparam, ctx->stream);
    cudaMemsetAsync(m->m2, 0, sizeof(float) * m->nparam, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    free(hw);
    *out = m;
    return TSG_OK;
}

extern "C" int tsg_mlp_destroy(tsg_mlp *m)
{
    if (!m)
        return TSG_OK;
    tsg_context *ctx = m->ctx;
    tsg_release(ctx, m->w);
    tsg_release(ctx, m->m1);
    tsg_release(ctx, m->m2);
    tsg_release(ctx, m->g);
    tsg_release(ctx, m->loss);
    cudaStreamSynchronize(ctx->stream);
    free(m);
    return TSG_OK;
}

extern "C" int tsg_mlp_num_params(const tsg_mlp *m) { return m ? m->nparam : 0; }

static size_t step_smem(const MlpDims &d)
{
    return sizeof(float) * ((size_t)d.B * d.F + 4 * (size_t)d.B * d.H + (size_t)d.B * d.O);
}

// One training step on device minibatch X[B][F], targets T[B][O], optional
// mask M[B][O] (1 = target present).  lr <= 0 computes gradients only.
extern "C" int tsg_mlp_train_step(tsg_mlp *m, int B, const float *d_X, const float *d_T, const float *d_M, float lr,
                                  float *loss)
{
    if (!m || B < 1 || B > TSG_MLP_MAX_B)
        return tsg_set_error(TSG_ERR_INVALID, "minibatch must have 1..%d rows", TSG_MLP_MAX_B);
    tsg_context *ctx = m->ctx;
    MlpDims d = dims(m, B);
    const size_t smem = step_smem(d);
    TSG_CUDA(cudaFuncSetAttribute(k_mlp_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (lr > 0.f)
        m->steps++;
    k_mlp_step<<<1, MLP_THREADS, smem, ctx->stream>>>(d, m->nparam, m->w, m->m1, m->m2, m->g, d_X, d_T, d_M, lr, 0.9f,
                                                      0.999f, 1e-8f, m->steps > 0 ? m->steps : 1, m->loss);
    TSG_LAUNCH_CHECK();
    if (loss)
    {
        TSG_CUDA(cudaMemcpyAsync(ctx->h_pinned, m->loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        TSG_CUDA(cudaStreamSynchronize(ctx->stream));
        *loss = *(float *)ctx->h_pinned;
    }
    return TSG_OK;
}

// Y[n][O] = network(X[n][F]) for any n (chunks of TSG_MLP_MAX_B rows).
extern "C" int tsg_mlp_forward(tsg_mlp *m, int n, const float *d_X, float *d_Y)
{
    if (!m || n < 0)
        return tsg_set_error(TSG_ERR_INVALID, "bad argument");
    tsg_context *ctx = m->ctx;
    for (int s = 0; s < n; s += TSG_MLP_MAX_B)
    {
        const int B = n - s < TSG_MLP_MAX_B ? n - s : TSG_MLP_MAX_B;
        MlpDims d = dims(m, B);
        const size_t smem = sizeof(float) * ((size_t)B * d.F + 2 * (size_t)B * d.H + (size_t)B * d.O);
        TSG_CUDA(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_mlp_forward<<<1, MLP_THREADS, smem, ctx->stream>>>(d, m->w, d_X + (size_t)s * d.F, d_Y + (size_t)s * d.O);
        TSG_LAUNCH_CHECK();
    }
    return TSG_OK;
}

// host copies of parameters / last gradients (nparam floats)
extern "C" int tsg_mlp_get(tsg_mlp *m, int which, float *host)
{
    if (!m || !host)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    const float *src = which == 0 ? m->w : m->g;
    TSG_CUDA(cudaMemcpyAsync(host, src, sizeof(float) * m->nparam, cudaMemcpyDeviceToHost, m->ctx->stream));
    TSG_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return TSG_OK;
}

extern "C" int tsg_mlp_set(tsg_mlp *m, const float *host)
{
    if (!m || !host)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    TSG_CUDA(cudaMemcpyAsync(m->w, host, sizeof(float) * m->nparam, cudaMemcpyHostToDevice, m->ctx->stream));
    TSG_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return TSG_OK;
}

// ---------------------------------------------------------------------------
// matrix features (device CSR): per-row statistics reduced on the device
// ---------------------------------------------------------------------------


// out[0] sum len, [1] sum len^2, [2] max len, [3] sum |i-j|, [4] max |i-j|,
// [5] empty rows, [6..17] row-length histogram (0,1,2-3,4-7,...,>=1024),
// [18] entries within |i-j| < 16
__global__ void k_row_feats(int m, const int *__restrict__ rowptr, const int *__restrict__ col,
                            unsigned long long *__restrict__ acc)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= m)
        return;
    const int r = (int)w, s = rowptr[r], e = rowptr[r + 1];
    unsigned long long dsum = 0, near = 0;
    unsigned dmax = 0;
    for (int p = s + lane; p < e; p += 32)
    {
        const int dd = abs(col[p] - r);
        dsum += (unsigned long long)dd;
        dmax = max(dmax, (unsigned)dd);
        near += dd < 16 ? 1 : 0;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1)
    {
        dsum += __shfl_xor_sync(0xffffffffu, dsum, d);
        near += __shfl_xor_sync(0xffffffffu, near, d);
        dmax = max(dmax, __shfl_xor_sync(0xffffffffu, dmax, d));
    }
    if (lane == 0)
    {
        const unsigned long long len = (unsigned long long)(e - s);
        atomicAdd(&acc[0], len);
        atomicAdd(&acc[1], len * len);
        atomicMax(&acc[2], len);
        atomicAdd(&acc[3], dsum);
        atomicMax(&acc[4], (unsigned long long)dmax);
        if (len == 0)
            atomicAdd(&acc[5], 1ULL);
        int bucket = 0;
        unsigned long long l = len;
        while (l > 0 && bucket < 11)
        {
            l >>= 1;
            bucket++;
        }
        atomicAdd(&acc[6 + bucket], 1ULL);
        atomicAdd(&acc[18], near);
    }
}

extern "C" int tsg_row_features(tsg_context *ctx, int m, const int *d_rowptr, const int *d_col,
                                unsigned long long *h_out /* TSG_NFEAT_RAW */)
{
    if (!ctx || !h_out)
        return tsg_set_error(TSG_ERR_INVALID, "null argument");
    unsigned long long *d;
    TSG_TRY(tsg_alloc(ctx, &d, TSG_NFEAT_RAW));
    TSG_CUDA(cudaMemsetAsync(d, 0, TSG_NFEAT_RAW * sizeof(unsigned long long), ctx->stream));
    if (m > 0)
    {
        k_row_feats<<<tsg_blocks((long long)m * 32, 256), 256, 0, ctx->stream>>>(m, d_rowptr, d_col, d);
        TSG_LAUNCH_CHECK();
    }
    TSG_CUDA(cudaMemcpyAsync(h_out, d, TSG_NFEAT_RAW * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             ctx->stream));
    TSG_CUDA(cudaStreamSynchronize(ctx->stream));
    tsg_release(ctx, d);
    return TSG_OK;
}
