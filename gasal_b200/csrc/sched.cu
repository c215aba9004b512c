/*
 * sched.cu -- length-binned visiting order for the one-pair-per-thread DP.
 *
 * A warp runs until its slowest lane finishes, so pairs of unequal length in
 * one warp waste lanes (uniform 150-300 bp targets leave a warp ~76% busy).
 * A counting sort groups pairs with the same (query words, target words) --
 * identical forward DP work -- and lists the biggest classes first so the
 * grid's tail holds the short pairs.  The start passes, run after the
 * forward pass, are ordered the same way by (reverse-region words, forward
 * score): how far a start pass runs follows the score it has to reach.  Three stream-ordered kernels: class
 * histogram, exclusive scan over classes, scatter.  Both counting kernels
 * aggregate per warp (one atomic per distinct class in a warp).  The order
 * inside a class is not deterministic; results are written per pair, so
 * output is.
 */
#include "gb_internal.h"

namespace gb {

constexpr int ORDER_BITS = 7;
constexpr int ORDER_BINS = 1 << (2 * ORDER_BITS); /* 128 x 128 classes */
static_assert((1u << ORDER_BITS) - 1 == ORDER_CAP_WORDS, "class cap of the length order");

__device__ __forceinline__ uint32_t work_bin(uint32_t qlen, uint32_t tlen)
{
    const uint32_t cap = (1u << ORDER_BITS) - 1;
    const uint32_t qw = (qlen + 7) >> 3, tw = (tlen + 7) >> 3;
    /* queries of cap+ words form the order's prefix (bins 0..cap): sorted by
     * the DP size qw * tw in classes of 4096 words^2, largest first, so the
     * launches that pull them from a work counter start the longest ones
     * first */
    if (qw >= cap) return cap - min((uint32_t)(((uint64_t)qw * tw) >> 12), cap);
    const uint32_t tr = min(tw, cap);
    /* descending work -> ascending bin */
    return (uint32_t)(ORDER_BINS - 1) - ((qw << ORDER_BITS) | tr);
}

/* start passes: (reverse-region query words, forward score / 2), descending */
__device__ __forceinline__ uint32_t start_bin(uint32_t qlen, int32_t q_end, int32_t score)
{
    const uint32_t cap = (1u << ORDER_BITS) - 1;
    const uint32_t qwords = (qlen + 7) >> 3;
    const uint32_t rr = q_end >= 0 ? min(((uint32_t)q_end >> 3) + 1, qwords) : 0u;
    const uint32_t sb = score > 0 ? min((uint32_t)score >> 1, cap) : 0u;
    return (uint32_t)(ORDER_BINS - 1) - ((min(rr, cap) << ORDER_BITS) | sb);
}

/* the pair's class: by lengths, or (start order) by reverse region and score.
 * The key is evaluated twice (histogram, scatter) and must not change in
 * between: pairs of q_cut+ bases belong to the warp-cooperative kernel,
 * which may still be writing their outputs on another stream, so they take
 * the last class without reading them. */
struct BinOf {
    const uint32_t *q_len, *t_len;
    const int32_t *q_end, *score;
    uint32_t q_cut;
    __device__ __forceinline__ uint32_t operator()(int i) const
    {
        if (!score) return work_bin(q_len[i], t_len[i]);
        const uint32_t ql = q_len[i];
        if (q_cut && ql >= q_cut) return (uint32_t)(ORDER_BINS - 1);
        return start_bin(ql, q_end[i], score[i]);
    }
};

__global__ void __launch_bounds__(256) order_hist_kernel(BinOf key, int n, uint32_t *hist)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const uint32_t bin = live ? key(i) : 0xFFFFFFFFu;
    const unsigned same = __match_any_sync(0xFFFFFFFFu, bin);
    const int leader = __ffs(same) - 1;
    if (live && (int)(threadIdx.x & 31) == leader) atomicAdd(&hist[bin], (uint32_t)__popc(same));
}

/* one block of 1024 threads: exclusive scan of ORDER_BINS counts in place */
__global__ void __launch_bounds__(1024) order_scan_kernel(uint32_t *hist)
{
    constexpr int PER = ORDER_BINS / 1024;
    __shared__ uint32_t part[1024];
    uint32_t v[PER], s = 0;
    const int base = threadIdx.x * PER;
#pragma unroll
    for (int k = 0; k < PER; k++) {
        v[k] = hist[base + k];
        s += v[k];
    }
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const uint32_t add = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0u;
        __syncthreads();
        part[threadIdx.x] += add;
        __syncthreads();
    }
    uint32_t run = part[threadIdx.x] - s;
#pragma unroll
    for (int k = 0; k < PER; k++) {
        hist[base + k] = run;
        run += v[k];
    }
}

__global__ void __launch_bounds__(256) order_scatter_kernel(BinOf key, int n, uint32_t *offs, uint32_t *order)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const uint32_t bin = live ? key(i) : 0xFFFFFFFFu;
    const unsigned same = __match_any_sync(0xFFFFFFFFu, bin);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(same) - 1;
    uint32_t base = 0;
    if (live && lane == leader) base = atomicAdd(&offs[bin], (uint32_t)__popc(same));
    base = __shfl_sync(same, base, leader);
    if (live) order[base + __popc(same & ((1u << lane) - 1u))] = (uint32_t)i;
}

int order_bins() { return ORDER_BINS; }

static cudaError_t order_by(BinOf key, int n, uint32_t *bins, uint32_t *order, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(bins, 0, ORDER_BINS * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    const int blocks = (n + 255) / 256;
    order_hist_kernel<<<blocks, 256, 0, s>>>(key, n, bins);
    order_scan_kernel<<<1, 1024, 0, s>>>(bins);
    order_scatter_kernel<<<blocks, 256, 0, s>>>(key, n, bins, order);
    return cudaGetLastError();
}

cudaError_t launch_order(const uint32_t *q_len, const uint32_t *t_len, int n, uint32_t *bins, uint32_t *order,
                         cudaStream_t s)
{
    return order_by(BinOf{q_len, t_len, nullptr, nullptr, 0u}, n, bins, order, s);
}

cudaError_t launch_start_order(const uint32_t *q_len, const int32_t *q_end, const int32_t *score, int n,
                               uint32_t q_cut, uint32_t *bins, uint32_t *order, cudaStream_t s)
{
    return order_by(BinOf{q_len, nullptr, q_end, score, q_cut}, n, bins, order, s);
}

} // namespace gb
