/*
 * dp_kernels.cu -- Gotoh dynamic programming for GASAL2's alignment modes on
 * sm_100a, one pair per thread.
 *
 * Replaces reference src/kernels/local_kernel_template.h (LOCAL),
 * src/kernels/global.h (GLOBAL), src/kernels/semiglobal_kernel_template.h
 * (SEMI_GLOBAL, all 16 head/tail variants), src/kernels/banded.h:10-139
 * (BANDED) and src/kernels/ksw_kernel_template.h (KSW).
 *
 * Results are bit-identical to the reference because the sweep order is the
 * reference's: bands of 8 target rows, each band swept query column by query
 * column, each column top to bottom.  "First maximum" positions and the
 * second-best rule (largest value below the running maximum when its cell is
 * swept) depend on that order.  Per band the 8 rows' diagonal (D), horizontal
 * gap (F) and, for semi-global, previous-column H live in registers; H and E
 * cross band boundaries through a row buffer of one 32-bit word per query
 * column holding both as int16 -- the reference stores them as short2 there,
 * so the truncation is part of the result.
 *
 * Instruction choices for the cell update (integer ALU is the bound):
 *   H = __vimax3_s32_relu(M, F, E)     one DPX op for max(M, F, E, 0)
 *   F = __viaddmax_s32(F, -ext, M-OE)  one DPX op for max(F-ext, M-OE)
 * The row buffer sits in shared memory laid out [column][thread] (bank-
 * conflict free), or for very long queries in a global scratch laid out
 * [column][thread] across the grid (coalesced).
 */
#include "dp_core.cuh"

namespace gb {

/* ============================ kernel ==================================== */
template <int ALGO, int START, bool SECOND, class SC>
__device__ __forceinline__ void run_pair(const DpArgs &a, const uint32_t *q, int qregs, int qlen, const uint32_t *t,
                                         int tregs, int tlen, int i, RowBuf rb, uint4 *tb, SC scr, Res &r)
{
    if (START == START_ONLY_) { /* the forward outputs are already in place */
        if (ALGO == LOCAL_) {
            r.score = a.score[i], r.q_end = a.q_end[i], r.t_end = a.t_end[i];
            local_start(q, qregs, t, tregs, a.sc, rb, scr, r);
        } else if (ALGO == SEMI_GLOBAL_) {
            semi_start(q, qregs, qlen, t, tregs, tlen, a.sc, a.head, a.tail, a.mql, rb, scr, a.score[i], a.t_end[i],
                       a.q_end[i], r);
        }
        return;
    }
    if (ALGO == LOCAL_) {
        local_fwd<SECOND, START == WITH_TB_>(q, qregs, t, tregs, a.sc, rb, tb, scr, r);
        if (START == WITH_START_) local_start(q, qregs, t, tregs, a.sc, rb, scr, r);
    } else if (ALGO == GLOBAL_) {
        if (START == WITH_TB_) global_fwd<true>(q, qregs, qlen, t, tregs, tlen, a.sc, rb, tb, scr, r);
        else global_fwd2(q, qregs, qlen, t, tregs, tlen, a.sc, rb, scr, r);
    } else if (ALGO == SEMI_GLOBAL_) {
        if (START == WITH_TB_ && tb) /* target-tail SEMI_GLOBAL with a traceback (an extension) */
            semi_global<SECOND, false, SC, true>(q, qregs, qlen, t, tregs, tlen, a.sc, a.head, a.tail, a.mql, rb, scr,
                                                 r, tb);
        else
            semi_global<SECOND, START == WITH_START_>(q, qregs, qlen, t, tregs, tlen, a.sc, a.head, a.tail, a.mql,
                                                     rb, scr, r);
    } else if (ALGO == BANDED_) {
        banded(q, qregs, t, tregs, a.k_band >> 3, a.sc, rb, scr, r);
        if (START == WITH_START_) banded_start(q, qregs, t, tregs, a.k_band >> 3, a.sc, rb, scr, r);
    }
}

template <int ALGO, int START, bool SECOND>
__device__ __forceinline__ void dp_one(const DpArgs &a, uint32_t w, RowBuf rb, const uint2 *stab, bool fast_scores,
                                       uint32_t row_cols)
{
    const int i = a.order ? (int)a.order[w] : (int)w;
    const int qlen = (int)a.q_len[i], tlen = (int)a.t_len[i];
    /* a pair outside this launch's length tier belongs to the other launch */
    if ((uint32_t)qlen < a.q_min || (a.q_max && (uint32_t)qlen > a.q_max)) return;
    /* rows that would not fit the row buffer are never written (the engine
     * sizes buffers for every pair it routes here; this only guards memory) */
    const uint32_t need = ALGO == KSW_ ? 2u * ((uint32_t)qlen + 2u) : (((uint32_t)qlen + 7u) & ~7u);
    if (need > row_cols) return;
    Res r = {0, 0, 0, 0, 0, 0, 0, 0};
    if (ALGO == KSW_) {
        /* empty sequences included: the reference returns h0 for them */
        ksw(a.pq + (a.q_off[i] >> 3), qlen, a.pt + (a.t_off[i] >> 3), tlen, a.seed ? a.seed[i] : 0u, a.zdrop, a.sc,
            rb, r);
    } else if (qlen > 0 && tlen > 0) {
        const uint32_t *q = a.pq + (a.q_off[i] >> 3);
        const uint32_t *t = a.pt + (a.t_off[i] >> 3);
        const int qregs = (qlen + 7) >> 3, tregs = (tlen + 7) >> 3;
        uint4 *tb = nullptr;
        if (START == WITH_TB_ && (ALGO == LOCAL_ || ALGO == GLOBAL_ || ALGO == SEMI_GLOBAL_)) {
            tb = a.tb + a.tb_off[i];
            /* two zero tile rows past the matrix: the GLOBAL traceback
             * starts one past the last cell */
            uint4 *z = tb + (size_t)tregs * 2 * qregs;
            for (int k = 0; k < 4 * qregs; k++) z[k] = make_uint4(0, 0, 0, 0);
        }
        if (fast_scores && plain_words(q, qregs) && plain_words(t, tregs)) {
            ScFast sf;
            sf.tab = stab;
            run_pair<ALGO, START, SECOND>(a, q, qregs, qlen, t, tregs, tlen, i, rb, tb, sf, r);
        } else {
            ScCmp scmp{};
            run_pair<ALGO, START, SECOND>(a, q, qregs, qlen, t, tregs, tlen, i, rb, tb, scmp, r);
        }
    }
    if (START == START_ONLY_) {
        if (a.q_start) a.q_start[i] = r.q_start;
        if (a.t_start) a.t_start[i] = r.t_start;
        return;
    }
    if (a.score) a.score[i] = r.score;
    if (ALGO == KSW_ && a.max_off) a.max_off[i] = r.score2;
    if (ALGO != GLOBAL_) {
        if (a.q_end) a.q_end[i] = r.q_end;
        if (a.t_end) a.t_end[i] = r.t_end;
        if ((ALGO == LOCAL_ || ALGO == SEMI_GLOBAL_ || ALGO == BANDED_) && START == WITH_START_) {
            if (a.q_start) a.q_start[i] = r.q_start;
            if (a.t_start) a.t_start[i] = r.t_start;
        }
        if (SECOND && (ALGO == LOCAL_ || ALGO == SEMI_GLOBAL_)) {
            if (a.score2) a.score2[i] = r.score2;
            if (a.q_end2) a.q_end2[i] = r.q_end2;
            if (a.t_end2) a.t_end2[i] = r.t_end2;
        }
    }
}

/* One pair per thread.  With a.queue set the launch is persistent: each warp
 * takes the next 32 entries of the (length-binned) visiting order from a
 * device counter until the batch is exhausted, so warps that drew short pairs
 * come back for more instead of idling; without it, a grid-stride loop. */
template <int ALGO, int START, bool SECOND, bool SMEM>
__global__ void __launch_bounds__(128) dp_kernel(DpArgs a)
{
    extern __shared__ uint32_t smem[];
    __shared__ uint2 stab[16];
    build_score_table(stab, a.sc, ALGO != GLOBAL_);
    __syncthreads();
    const bool fast_scores = a.sc.match >= -128 && a.sc.match <= 127 && a.sc.mismatch >= -127 && a.sc.mismatch <= 128;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nthr = gridDim.x * blockDim.x;
    RowBuf rb;
    uint32_t row_cols;
    if (SMEM) {
        rb.base = smem + threadIdx.x;
        rb.stride = blockDim.x;
        row_cols = (uint32_t)a.smem_cols;
    } else {
        rb.base = a.scratch + gtid;
        rb.stride = nthr;
        row_cols = a.scratch_cols;
    }
    const uint32_t n = a.n_dev ? min(*a.n_dev, (uint32_t)a.n) : (uint32_t)a.n;
    if (a.queue) {
        const int lane = threadIdx.x & 31;
        for (;;) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(a.queue, 32u);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base >= n) break;
            const uint32_t w = base + lane;
            if (w < n) dp_one<ALGO, START, SECOND>(a, w, rb, stab, fast_scores, row_cols);
        }
    } else {
        for (uint32_t w = gtid; w < n; w += nthr) dp_one<ALGO, START, SECOND>(a, w, rb, stab, fast_scores, row_cols);
    }
}

/* Grid of the scratch (global row buffer) variant: at most what the GPU holds
 * resident, each thread looping over pairs. */
int dp_scratch_blocks(int n, int block)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int need = (n + block - 1) / block;
    const int cap = sms * (2048 / block);
    return need < cap ? need : cap;
}

template <int ALGO, int START, bool SECOND>
static cudaError_t launch_one(const DpArgs &a, int block, cudaStream_t s)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (a.smem_cols > 0) {
        const size_t smem = (size_t)a.smem_cols * block * sizeof(uint32_t);
        auto k = dp_kernel<ALGO, START, SECOND, true>;
        cudaError_t e = allow_dyn_smem(k);
        if (e != cudaSuccess) return e;
        int blocks = (a.n + block - 1) / block;
        if (a.queue) {
            int per_sm = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block, smem);
            if (e != cudaSuccess) return e;
            if (per_sm < 1) per_sm = 1;
            if (blocks > per_sm * sms) blocks = per_sm * sms;
        }
        k<<<blocks, block, smem, s>>>(a);
    } else {
        /* scratch holds scratch_cols columns for every thread of the grid */
        dp_kernel<ALGO, START, SECOND, false><<<dp_scratch_blocks(a.n, block), block, 0, s>>>(a);
    }
    return cudaGetLastError();
}

/* Global-scratch variant on an explicit grid (blocks x block threads must
 * all fit in a.scratch at a.scratch_cols columns each). */
template <int ALGO, int START, bool SECOND>
static cudaError_t launch_scratch_grid(const DpArgs &a, int block, int blocks, cudaStream_t s)
{
    dp_kernel<ALGO, START, SECOND, false><<<blocks, block, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_dp_scratch_grid(int algo, int start, bool second, const DpArgs &a, int block, int blocks,
                                   cudaStream_t s)
{
    if (a.n <= 0) return cudaSuccess;
#define GB_SG(A, S, B) launch_scratch_grid<A, S, B>(a, block, blocks, s)
    switch (algo) {
    case LOCAL_:
        if (start == START_ONLY_) return GB_SG(LOCAL_, START_ONLY_, false);
        if (start == WITH_START_) return second ? GB_SG(LOCAL_, WITH_START_, true) : GB_SG(LOCAL_, WITH_START_, false);
        if (start == WITH_TB_) return second ? GB_SG(LOCAL_, WITH_TB_, true) : GB_SG(LOCAL_, WITH_TB_, false);
        return second ? GB_SG(LOCAL_, WITHOUT_START_, true) : GB_SG(LOCAL_, WITHOUT_START_, false);
    case GLOBAL_:
        if (start == WITH_TB_) return GB_SG(GLOBAL_, WITH_TB_, false);
        return GB_SG(GLOBAL_, WITHOUT_START_, false);
    case SEMI_GLOBAL_:
        if (start == START_ONLY_) return GB_SG(SEMI_GLOBAL_, START_ONLY_, false);
        if (start == WITH_TB_) return second ? GB_SG(SEMI_GLOBAL_, WITH_TB_, true) : GB_SG(SEMI_GLOBAL_, WITH_TB_, false);
        if (start == WITH_START_)
            return second ? GB_SG(SEMI_GLOBAL_, WITH_START_, true) : GB_SG(SEMI_GLOBAL_, WITH_START_, false);
        return second ? GB_SG(SEMI_GLOBAL_, WITHOUT_START_, true) : GB_SG(SEMI_GLOBAL_, WITHOUT_START_, false);
    case BANDED_:
        if (start == WITH_START_) return GB_SG(BANDED_, WITH_START_, false);
        return GB_SG(BANDED_, WITHOUT_START_, false);
    case KSW_:
        return GB_SG(KSW_, WITHOUT_START_, false);
    default:
        return cudaErrorInvalidValue;
    }
#undef GB_SG
}

cudaError_t launch_dp(int algo, int start, bool second, const DpArgs &a, int block, int max_q8, cudaStream_t s)
{
    (void)max_q8;
    if (a.n <= 0) return cudaSuccess;
    switch (algo) {
    case LOCAL_:
        if (start == START_ONLY_) return launch_one<LOCAL_, START_ONLY_, false>(a, block, s);
        if (start == WITH_START_)
            return second ? launch_one<LOCAL_, WITH_START_, true>(a, block, s) : launch_one<LOCAL_, WITH_START_, false>(a, block, s);
        if (start == WITH_TB_)
            return second ? launch_one<LOCAL_, WITH_TB_, true>(a, block, s) : launch_one<LOCAL_, WITH_TB_, false>(a, block, s);
        return second ? launch_one<LOCAL_, WITHOUT_START_, true>(a, block, s) : launch_one<LOCAL_, WITHOUT_START_, false>(a, block, s);
    case GLOBAL_:
        if (start == WITH_TB_) return launch_one<GLOBAL_, WITH_TB_, false>(a, block, s);
        return launch_one<GLOBAL_, WITHOUT_START_, false>(a, block, s);
    case SEMI_GLOBAL_:
        if (start == START_ONLY_) return launch_one<SEMI_GLOBAL_, START_ONLY_, false>(a, block, s);
        if (start == WITH_TB_)
            return second ? launch_one<SEMI_GLOBAL_, WITH_TB_, true>(a, block, s) : launch_one<SEMI_GLOBAL_, WITH_TB_, false>(a, block, s);
        if (start == WITH_START_)
            return second ? launch_one<SEMI_GLOBAL_, WITH_START_, true>(a, block, s) : launch_one<SEMI_GLOBAL_, WITH_START_, false>(a, block, s);
        return second ? launch_one<SEMI_GLOBAL_, WITHOUT_START_, true>(a, block, s) : launch_one<SEMI_GLOBAL_, WITHOUT_START_, false>(a, block, s);
    case BANDED_:
        if (start == WITH_START_) return launch_one<BANDED_, WITH_START_, false>(a, block, s);
        return launch_one<BANDED_, WITHOUT_START_, false>(a, block, s);
    case KSW_:
        return launch_one<KSW_, WITHOUT_START_, false>(a, block, s);
    default:
        return cudaErrorInvalidValue;
    }
}

} // namespace gb
