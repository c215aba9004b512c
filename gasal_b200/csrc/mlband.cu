/*
 * mlband.cu -- learned band width for ksw extension: pair features and a
 * small MLP (forward, backward, Adam) written as plain CUDA kernels.
 *
 * No reference counterpart: GASAL2's ksw kernel always fills the whole
 * trimmed matrix.  The band a pair gets only decides how much of the matrix
 * the banded kernel computes; the band certificate (ksw_wc.cu) decides
 * whether that result is the exact one, and pairs that fail it are
 * recomputed without a band.  So nothing here can change a result.
 *
 * Features (BAND_FEATS floats per pair):
 *   [0] qlen/1024  [1] tlen/1024  [2] (tlen-qlen)/128
 *   [3..66] histogram of the diagonal offsets (target position - query
 *           position) of the query's 11-mers found in the target, 64 bins
 *           (32 per sign, |d| < 8 one bin each, then 4 bins per doubling
 *           from the two bits after the leading one), divided by the number
 *           of query 11-mers.
 *   [67] 0 (padding)
 * One 128-thread block per pair: the target's 11-mers go into a
 * 4096-slot shared-memory table (slot = hash, value = max over writers of
 * (kmer+1) << 32 | position, so the table is deterministic), then each query
 * 11-mer looks its slot up.
 *
 * MLP: 67 -> 64 (ReLU) -> 64 (ReLU) -> 1, 8,577 parameters, kept in FP32 for
 * training and in BF16 for inference, FP32 accumulation everywhere.  One warp
 * evaluates one pair (two hidden units per lane).  The network is far too
 * small for tensor cores to matter: 4M pairs cost about 34 GFLOP.
 */
#include <cuda_bf16.h>
#include <cstdint>
#include <cuda_runtime.h>

#include "mlband.h"

namespace gb {

namespace {

constexpr int KMER = 11;
constexpr int TAB = 4096;
constexpr unsigned FULL = 0xFFFFFFFFu;

/* 4-bit code -> 2-bit base (A C G T), 4 for anything else */
__device__ __forceinline__ uint32_t base2(uint32_t c)
{
    return c == 1u ? 0u : c == 3u ? 1u : c == 7u ? 2u : c == 4u ? 3u : 4u;
}

__device__ __forceinline__ uint32_t code_at(const uint32_t *w, int p) { return (w[p >> 3] >> (28 - 4 * (p & 7))) & 15u; }

__device__ __forceinline__ uint32_t khash(uint32_t k) { return (k * 2654435761u) >> (32 - 12); }

/* |d| < 8: one bin each; then four bins per doubling (the two bits after
 * the leading one), up to bin 31; negative offsets use bins 32..63 */
__device__ __forceinline__ int diag_bin(int d)
{
    const int a = d < 0 ? -d : d;
    int b;
    if (a < 8) {
        b = a;
    } else {
        const int e = 31 - __clz(a);
        b = min(31, 8 + 4 * (e - 3) + ((a >> (e - 2)) & 3));
    }
    return d < 0 ? 32 + b : b;
}

__global__ void __launch_bounds__(128) band_feature_kernel(const uint32_t *pq, const uint32_t *pt,
                                                           const uint32_t *q_off, const uint32_t *t_off,
                                                           const uint32_t *q_len, const uint32_t *t_len, int n,
                                                           float *feat)
{
    __shared__ unsigned long long tab[TAB];
    __shared__ int hist[64];
    for (int pid = blockIdx.x; pid < n; pid += gridDim.x) {
        for (int s = threadIdx.x; s < TAB; s += blockDim.x) tab[s] = 0ull;
        if (threadIdx.x < 64) hist[threadIdx.x] = 0;
        __syncthreads();
        const int qlen = (int)q_len[pid], tlen = (int)t_len[pid];
        const uint32_t *q = pq + (q_off[pid] >> 3), *t = pt + (t_off[pid] >> 3);
        /* target 11-mers: each thread rolls a contiguous run of positions */
        const int nt = tlen - KMER + 1;
        if (nt > 0) {
            const int per = (nt + blockDim.x - 1) / blockDim.x;
            const int p0 = threadIdx.x * per, p1 = min(p0 + per, nt);
            uint32_t k = 0;
            int valid = 0; /* consecutive valid bases ending at the current position */
            for (int p = p0; p < p1 + KMER - 1 && p0 < p1; p++) {
                const uint32_t b = base2(code_at(t, p));
                valid = b < 4u ? valid + 1 : 0;
                k = ((k << 2) | (b & 3u)) & ((1u << (2 * KMER)) - 1u);
                const int start = p - KMER + 1;
                if (start >= p0 && valid >= KMER)
                    atomicMax(&tab[khash(k)], ((unsigned long long)(k + 1u) << 32) | (unsigned)start);
            }
        }
        __syncthreads();
        const int nq = qlen - KMER + 1;
        if (nq > 0) {
            const int per = (nq + blockDim.x - 1) / blockDim.x;
            const int p0 = threadIdx.x * per, p1 = min(p0 + per, nq);
            uint32_t k = 0;
            int valid = 0;
            for (int p = p0; p < p1 + KMER - 1 && p0 < p1; p++) {
                const uint32_t b = base2(code_at(q, p));
                valid = b < 4u ? valid + 1 : 0;
                k = ((k << 2) | (b & 3u)) & ((1u << (2 * KMER)) - 1u);
                const int start = p - KMER + 1;
                if (start >= p0 && valid >= KMER) {
                    const unsigned long long v = tab[khash(k)];
                    if ((uint32_t)(v >> 32) == k + 1u) atomicAdd(&hist[diag_bin((int)(uint32_t)v - start)], 1);
                }
            }
        }
        __syncthreads();
        float *f = feat + (size_t)pid * BAND_FEATS_PAD;
        const float inv = nq > 0 ? 1.0f / (float)nq : 0.0f;
        if (threadIdx.x < 64) f[3 + threadIdx.x] = (float)hist[threadIdx.x] * inv;
        if (threadIdx.x == 64) f[0] = (float)qlen * (1.0f / 1024.0f);
        if (threadIdx.x == 65) f[1] = (float)tlen * (1.0f / 1024.0f);
        if (threadIdx.x == 66) f[2] = (float)(tlen - qlen) * (1.0f / 128.0f);
        if (threadIdx.x == 67) f[67] = 0.0f;
        __syncthreads();
    }
}

/* ----------------------------------------------------------------------- */
/* MLP.  Parameter vector layout (FP32, MLP_PARAMS floats):
 *   W1[64][67], b1[64], W2[64][64], b2[64], W3[64], b3  */
constexpr int IN = BAND_FEATS, H = 64;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * IN, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
              OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + H;
static_assert(OFF_B3 + 1 == MLP_PARAMS, "parameter layout");
/* shared-memory copy: W2 rows padded to 65 floats so that lanes reading
 * (or accumulating) W2[lane][i] hit distinct banks (W1's 67 already do) */
constexpr int H2P = H + 1;
constexpr int S_W1 = 0, S_B1 = S_W1 + H * IN, S_W2 = S_B1 + H, S_B2 = S_W2 + H * H2P, S_W3 = S_B2 + H,
              S_B3 = S_W3 + H, S_TOTAL = S_B3 + 1;
__device__ __forceinline__ int s_index(int g)
{
    if (g < OFF_W2 || g >= OFF_B2) return g < OFF_W2 ? g : g - OFF_B2 + S_B2;
    const int r = g - OFF_W2;
    return S_W2 + (r / H) * H2P + (r % H);
}

template <class T> __device__ __forceinline__ float ld(const T *p, int i);
template <> __device__ __forceinline__ float ld<float>(const float *p, int i) { return p[i]; }
template <> __device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16 *p, int i)
{
    return __bfloat162float(p[i]);
}

/* One warp, one pair: lane l owns hidden units l and l+32 of both layers.
 * x, h1 and h2 go through shared memory (per warp). */
struct Acts {
    float x[IN + 1], h1[H], h2[H];
};

template <class T>
__device__ __forceinline__ float mlp_fwd_warp(const float *sp, const float *xin, Acts &A, int lane)
{
    for (int i = lane; i < IN; i += 32) A.x[i] = xin[i];
    __syncwarp();
    float a0 = sp[S_B1 + lane], a1 = sp[S_B1 + lane + 32];
    for (int i = 0; i < IN; i++) {
        const float xi = A.x[i];
        a0 = fmaf(sp[S_W1 + lane * IN + i], xi, a0);
        a1 = fmaf(sp[S_W1 + (lane + 32) * IN + i], xi, a1);
    }
    A.h1[lane] = fmaxf(a0, 0.f), A.h1[lane + 32] = fmaxf(a1, 0.f);
    __syncwarp();
    float c0 = sp[S_B2 + lane], c1 = sp[S_B2 + lane + 32];
    for (int i = 0; i < H; i++) {
        const float hi = A.h1[i];
        c0 = fmaf(sp[S_W2 + lane * H2P + i], hi, c0);
        c1 = fmaf(sp[S_W2 + (lane + 32) * H2P + i], hi, c1);
    }
    c0 = fmaxf(c0, 0.f), c1 = fmaxf(c1, 0.f);
    A.h2[lane] = c0, A.h2[lane + 32] = c1;
    float y = sp[S_W3 + lane] * c0 + sp[S_W3 + lane + 32] * c1;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) y += __shfl_xor_sync(FULL, y, d);
    __syncwarp();
    return y + sp[S_B3];
}

/* parameters -> shared memory as FP32 (padded layout) */
template <class T> __device__ void stage_params(float *sp, const T *w)
{
    for (int i = threadIdx.x; i < MLP_PARAMS; i += blockDim.x) sp[s_index(i)] = ld<T>(w, i);
    __syncthreads();
}

__global__ void __launch_bounds__(256) mlp_forward_kernel(const __nv_bfloat16 *w, const float *feat, int n,
                                                          float *out)
{
    extern __shared__ float mlp_smem[];
    float *sp = mlp_smem;
    Acts *acts = reinterpret_cast<Acts *>(sp + S_TOTAL + 3);
    stage_params(sp, w);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    for (int pid = blockIdx.x * warps + warp; pid < n; pid += gridDim.x * warps) {
        const float y = mlp_fwd_warp<__nv_bfloat16>(sp, feat + (size_t)pid * BAND_FEATS_PAD, acts[warp], lane);
        if (lane == 0) out[pid] = y;
    }
}

/* Pinball (quantile tau) loss on y - label: d loss / d y = -tau when the
 * label is above the prediction, 1 - tau otherwise.  Gradients of the whole
 * batch are summed into grad (MLP_PARAMS floats, zeroed by the caller),
 * divided by n; the loss sum goes to loss[0]. */
__global__ void __launch_bounds__(256) mlp_grad_kernel(const float *w, const float *feat, const float *label, int n,
                                                       float tau, float *grad, float *loss)
{
    extern __shared__ float mlp_smem[];
    float *sp = mlp_smem;
    float *sg = sp + S_TOTAL;
    Acts *acts = reinterpret_cast<Acts *>(sg + S_TOTAL + 3);
    stage_params(sp, w);
    for (int i = threadIdx.x; i < S_TOTAL; i += blockDim.x) sg[i] = 0.f;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    const float inv_n = 1.0f / (float)n;
    float lsum = 0.f;
    for (int pid = blockIdx.x * warps + warp; pid < n; pid += gridDim.x * warps) {
        Acts &A = acts[warp];
        const float y = mlp_fwd_warp<float>(sp, feat + (size_t)pid * BAND_FEATS_PAD, A, lane);
        const float r = label[pid] - y;
        lsum += r > 0.f ? tau * r : (tau - 1.f) * r;
        const float dy = (r > 0.f ? -tau : 1.f - tau) * inv_n;
        /* layer 3 */
        const float h2a = A.h2[lane], h2b = A.h2[lane + 32];
        atomicAdd(&sg[S_W3 + lane], dy * h2a);
        atomicAdd(&sg[S_W3 + lane + 32], dy * h2b);
        if (lane == 0) atomicAdd(&sg[S_B3], dy);
        const float d2a = h2a > 0.f ? dy * sp[S_W3 + lane] : 0.f;
        const float d2b = h2b > 0.f ? dy * sp[S_W3 + lane + 32] : 0.f;
        /* layer 2: dW2[u][i] = d2[u] * h1[i]; d1[i] = sum_u W2[u][i] d2[u] */
        atomicAdd(&sg[S_B2 + lane], d2a);
        atomicAdd(&sg[S_B2 + lane + 32], d2b);
        for (int i = 0; i < H; i++) {
            const float hi = A.h1[i];
            if (hi != 0.f) {
                atomicAdd(&sg[S_W2 + lane * H2P + i], d2a * hi);
                atomicAdd(&sg[S_W2 + (lane + 32) * H2P + i], d2b * hi);
            }
        }
        float d1a = 0.f, d1b = 0.f;
        for (int u = 0; u < H; u++) {
            const float du = __shfl_sync(FULL, u < 32 ? d2a : d2b, u & 31);
            d1a = fmaf(sp[S_W2 + u * H2P + lane], du, d1a);
            d1b = fmaf(sp[S_W2 + u * H2P + lane + 32], du, d1b);
        }
        d1a = A.h1[lane] > 0.f ? d1a : 0.f;
        d1b = A.h1[lane + 32] > 0.f ? d1b : 0.f;
        /* layer 1 */
        atomicAdd(&sg[S_B1 + lane], d1a);
        atomicAdd(&sg[S_B1 + lane + 32], d1b);
        for (int i = 0; i < IN; i++) {
            const float xi = A.x[i];
            if (xi != 0.f) {
                atomicAdd(&sg[S_W1 + lane * IN + i], d1a * xi);
                atomicAdd(&sg[S_W1 + (lane + 32) * IN + i], d1b * xi);
            }
        }
        __syncwarp();
    }
    if (lane == 0) atomicAdd(loss, lsum);
    __syncthreads();
    for (int i = threadIdx.x; i < MLP_PARAMS; i += blockDim.x) atomicAdd(&grad[i], sg[s_index(i)]);
}

/* Adam with bias correction; refreshes the BF16 inference copy. */
__global__ void mlp_adam_kernel(float *w, float *m, float *v, const float *g, __nv_bfloat16 *wb, float lr,
                                float b1, float b2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MLP_PARAMS) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi, v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16(wi);
}

__global__ void to_bf16_kernel(const float *w, __nv_bfloat16 *wb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < MLP_PARAMS) wb[i] = __float2bfloat16(w[i]);
}

/* predicted log2 half-width -> band: rounded up to a multiple of 8, clamped
 * to [bmin, bmax]; -1 (no band) when it would cover the whole matrix */
__global__ void band_from_pred_kernel(const float *pred, const uint32_t *q_len, const uint32_t *t_len, int n, int bmin,
                                      int bmax, int32_t *band)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float y = fminf(fmaxf(pred[i], 0.f), 20.f);
    int w = (int)ceilf(exp2f(y));
    w = max(bmin, min(bmax, w));
    /* a banded row spans at most 2w + 1 columns from a tile start up to 7
     * columns left of it; the warp kernel runs it as one 64- or 128-column
     * tile, or 256-column tiles: widen w to the widest band of the same tile
     * cost (more results kept, no more work) */
    const int span = 2 * w + 8;
    w = span <= 64 ? 28 : span <= 128 ? 60 : 128 * ((span + 255) / 256) - 4;
    w = min(bmax, w);
    const int cover = (int)max(q_len[i], t_len[i]);
    band[i] = w >= cover ? -1 : w;
}

/* band_ok[p] = 1 for every pair, then 0 for the pairs in retry[0..*nretry) */
__global__ void band_ok_kernel(uint8_t *ok, int n, const uint32_t *retry, const uint32_t *nretry)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) ok[i] = 1;
}
__global__ void band_fail_kernel(uint8_t *ok, int n, const uint32_t *retry, const uint32_t *nretry)
{
    const uint32_t c = min(*nretry, (uint32_t)n);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) ok[retry[i]] = 0;
}

int sm_count()
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

} // namespace

cudaError_t launch_band_features(const uint32_t *pq, const uint32_t *pt, const uint32_t *q_off, const uint32_t *t_off,
                                 const uint32_t *q_len, const uint32_t *t_len, int n, float *feat, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    const int blocks = n < sm_count() * 8 ? n : sm_count() * 8;
    band_feature_kernel<<<blocks, 128, 0, s>>>(pq, pt, q_off, t_off, q_len, t_len, n, feat);
    return cudaGetLastError();
}

static size_t fwd_smem(int warps) { return (S_TOTAL + 3) * sizeof(float) + warps * sizeof(Acts); }
static size_t grad_smem(int warps) { return 2 * (S_TOTAL + 3) * sizeof(float) + warps * sizeof(Acts); }

cudaError_t launch_mlp_forward(const __nv_bfloat16 *w, const float *feat, int n, float *out, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    const size_t sm = fwd_smem(8);
    cudaError_t e = cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    int blocks = (n + 7) / 8;
    if (blocks > sm_count() * 4) blocks = sm_count() * 4;
    mlp_forward_kernel<<<blocks, 256, sm, s>>>(w, feat, n, out);
    return cudaGetLastError();
}

cudaError_t launch_mlp_grad(const float *w, const float *feat, const float *label, int n, float tau, float *grad,
                            float *loss, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    const size_t sm = grad_smem(8);
    cudaError_t e = cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(grad, 0, MLP_PARAMS * sizeof(float), s);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(loss, 0, sizeof(float), s);
    if (e != cudaSuccess) return e;
    int blocks = (n + 7) / 8;
    if (blocks > sm_count() * 2) blocks = sm_count() * 2;
    mlp_grad_kernel<<<blocks, 256, sm, s>>>(w, feat, label, n, tau, grad, loss);
    return cudaGetLastError();
}

cudaError_t launch_mlp_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *wb, float lr, int step,
                            cudaStream_t s)
{
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.f, c2 = 1.f;
    for (int i = 0; i < step; i++) c1 *= b1, c2 *= b2;
    c1 = 1.f - c1, c2 = 1.f - c2;
    mlp_adam_kernel<<<(MLP_PARAMS + 255) / 256, 256, 0, s>>>(w, m, v, g, wb, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError();
}

cudaError_t launch_band_from_pred(const float *pred, const uint32_t *q_len, const uint32_t *t_len, int n, int bmin,
                                  int bmax, int32_t *band, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    band_from_pred_kernel<<<(n + 255) / 256, 256, 0, s>>>(pred, q_len, t_len, n, bmin, bmax, band);
    return cudaGetLastError();
}

cudaError_t launch_band_ok(uint8_t *ok, int n, const uint32_t *retry, const uint32_t *nretry, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    band_ok_kernel<<<(n + 255) / 256, 256, 0, s>>>(ok, n, retry, nretry);
    band_fail_kernel<<<sm_count() * 4, 256, 0, s>>>(ok, n, retry, nretry);
    return cudaGetLastError();
}

cudaError_t launch_to_bf16(const float *w, __nv_bfloat16 *wb, cudaStream_t s)
{
    to_bf16_kernel<<<(MLP_PARAMS + 255) / 256, 256, 0, s>>>(w, wb);
    return cudaGetLastError();
}

} // namespace gb
