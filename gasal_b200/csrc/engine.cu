/*
 * engine.cu -- stream-ordered batch execution (device half of
 * reference src/gasal_align.cu:180-264).
 *
 * Planning is host-side and O(n): the longest query decides where the row
 * buffers live (shared memory when a block's buffers fit, else a global
 * scratch sized for the resident grid), and WITH_TB batches are split into
 * chunks whose traceback tiles fit the tile budget -- the reference sizes one
 * max_q x max_t matrix per pair, which does not fit HBM for long uneven
 * batches.  Every chunk runs the DP kernel and then the traceback kernel on
 * the same stream, reusing one tile buffer.
 */
#include "engine.h"
#include "mlband.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

namespace gb {

cudaError_t allow_dyn_smem_fn(const void *fn)
{
    static std::mutex mu;
    static std::vector<std::pair<const void *, int>> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    for (const auto &d : done)
        if (d.first == fn && d.second == dev) return cudaSuccess;
    int optin = 0;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, fn);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    if (e != cudaSuccess) return e;
    done.emplace_back(fn, dev);
    return cudaSuccess;
}

Settings &settings()
{
    static Settings s = [] {
        Settings v;
        if (const char *e = getenv("GASAL_B200_TB_BUDGET_MB")) v.tb_budget_bytes = (size_t)atoll(e) << 20;
        if (const char *e = getenv("GASAL_B200_BLOCK")) v.block = atoi(e);
        if (const char *e = getenv("GASAL_B200_MIN_ORDER_PAIRS")) v.min_order_pairs = atoi(e);
        if (const char *e = getenv("GASAL_B200_WC_MIN_QREGS")) v.wc_min_qregs = atoi(e);
        if (const char *e = getenv("GASAL_B200_WC_BIG_GROUP")) v.wc_big_group = atoi(e);
        if (const char *e = getenv("GASAL_B200_KSW_GROUPS")) v.ksw_groups = atoi(e);
        return v;
    }();
    return s;
}

/* ---- optional per-kernel timing ---- */
namespace {
struct Mark {
    int kind;
    cudaEvent_t a, b;
};
struct Timing {
    std::mutex mu;
    bool on = false;
    std::vector<Mark> pending;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t open[K_KINDS] = {};
    double ms[K_KINDS] = {};
    int64_t n[K_KINDS] = {};
};
Timing &timing()
{
    static Timing t;
    return t;
}
cudaEvent_t take_event(Timing &t)
{
    if (!t.pool.empty()) {
        cudaEvent_t e = t.pool.back();
        t.pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}
} // namespace

void timing_enable(bool on)
{
    Timing &t = timing();
    std::lock_guard<std::mutex> lk(t.mu);
    t.on = on;
    for (int k = 0; k < K_KINDS; k++) t.ms[k] = 0, t.n[k] = 0;
}

void timing_mark(int kind, bool start, cudaStream_t s)
{
    Timing &t = timing();
    std::lock_guard<std::mutex> lk(t.mu);
    if (!t.on) return;
    cudaEvent_t e = take_event(t);
    cudaEventRecord(e, s);
    if (start) {
        t.open[kind] = e;
    } else {
        t.pending.push_back({kind, t.open[kind], e});
        t.open[kind] = nullptr;
    }
}

int timing_read(double ms[K_KINDS], int64_t launches[K_KINDS])
{
    Timing &t = timing();
    std::lock_guard<std::mutex> lk(t.mu);
    for (Mark &m : t.pending) {
        if (cudaEventSynchronize(m.b) != cudaSuccess) return GB_ERR_CUDA;
        float x = 0;
        cudaEventElapsedTime(&x, m.a, m.b);
        t.ms[m.kind] += x;
        t.n[m.kind] += 1;
        t.pool.push_back(m.a);
        t.pool.push_back(m.b);
    }
    t.pending.clear();
    for (int k = 0; k < K_KINDS; k++) ms[k] = t.ms[k], launches[k] = t.n[k];
    return GB_OK;
}

Workspace::~Workspace()
{
    /* device memory is released by the owner (release_workspace) while its
     * context is current; nothing to do at static destruction time */
}

void release_workspace(Workspace &w)
{
    if (w.tb) cudaFree(w.tb);
    if (w.d_tb_off) cudaFree(w.d_tb_off);
    if (w.h_tb_off) cudaFreeHost(w.h_tb_off);
    if (w.scratch) cudaFree(w.scratch);
    if (w.tb_off_free) cudaEventDestroy(w.tb_off_free);
    if (w.order) cudaFree(w.order);
    if (w.order2) cudaFree(w.order2);
    if (w.wc_rows) cudaFree(w.wc_rows);
    if (w.wc_defer) cudaFree(w.wc_defer);
    if (w.aux) cudaStreamDestroy(w.aux);
    if (w.queue) cudaFree(w.queue);
    if (w.fork) cudaEventDestroy(w.fork);
    if (w.join) cudaEventDestroy(w.join);
    if (w.bins) cudaFree(w.bins);
    if (w.fb) cudaFree(w.fb);
    if (w.retry) cudaFree(w.retry);
    if (w.feat) cudaFree(w.feat);
    if (w.pred) cudaFree(w.pred);
    if (w.bandw) cudaFree(w.bandw);
    const int dev = w.device;
    w = Workspace();
    w.device = dev;
}

/* Every device allocation of the engine's workspaces and of the storage API's
 * regrowth goes through here.  GASAL_B200_FAIL_ALLOC_AFTER=k (read once) makes
 * the allocation after the first k fail once, as an out-of-memory would, so
 * the callers' GB_ERR_ALLOC paths can be exercised without exhausting a GPU;
 * later allocations are served normally. */
cudaError_t dev_malloc(void **p, size_t bytes)
{
    static std::mutex mu;
    static long countdown = [] {
        const char *e = getenv("GASAL_B200_FAIL_ALLOC_AFTER");
        return e ? atol(e) : -1L;
    }();
    {
        std::lock_guard<std::mutex> lk(mu);
        if (countdown == 0) {
            countdown = -1;
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
        if (countdown > 0) countdown--;
    }
    return cudaMalloc(p, bytes);
}

static int grow(void **p, size_t *cap, size_t need, size_t elem)
{
    if (*cap >= need) return GB_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    size_t want = need + need / 4 + 1024;
    if (dev_malloc(p, want * elem) != cudaSuccess) {
        cudaGetLastError();
        if (dev_malloc(p, need * elem) != cudaSuccess) {
            cudaGetLastError();
            *p = nullptr;
            return GB_ERR_ALLOC;
        }
        want = need;
    }
    *cap = want;
    return GB_OK;
}

#define GB_CUDA(call)                                                                                  \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            fprintf(stderr, "[GASAL-B200 CUDA ERROR] %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
                    __LINE__);                                                                         \
            return GB_ERR_CUDA;                                                                        \
        }                                                                                              \
    } while (0)

/* ---------------------------------------------------------------------- */
/* Planning: every host-side decision and every allocation of a batch, so
 * that enqueue_batch() issues stream operations only (and can be captured
 * into a CUDA graph). */

static int ensure_order_buffers(Workspace &ws, size_t n)
{
    if (grow((void **)&ws.order, &ws.order_cap, n, 4) != GB_OK) return GB_ERR_ALLOC;
    if (!ws.bins && dev_malloc((void **)&ws.bins, (size_t)order_bins() * 4) != cudaSuccess) {
        cudaGetLastError();
        return GB_ERR_ALLOC;
    }
    return GB_OK;
}

int plan_batch(const RunCfg &cfg, const DevBatch &b, const DevOut &o, Workspace &ws, Plan &p, cudaStream_t s)
{
    if (b.n <= 0) return GB_ERR_ARG;
    const Settings &st = settings();
    p = Plan();
    p.block = st.block;

    /* split: long LOCAL/GLOBAL (and target-tail SEMI_GLOBAL) pairs go warp-cooperative */
    bool wc_algo = cfg.algo == LOCAL_ || cfg.algo == GLOBAL_ || (cfg.algo == SEMI_GLOBAL_ && cfg.tail == TARGET_);
    /* target-tail SEMI_GLOBAL WITH_TB (the extension) runs one pair per thread */
    const bool semi_tb = cfg.algo == SEMI_GLOBAL_ && cfg.start == WITH_TB_ && cfg.tail == TARGET_;
    if (semi_tb) wc_algo = false;
    if (wc_algo && cfg.start != WITHOUT_START_ && cfg.sc.match > 0) {
        /* start passes and tracebacks of pairs whose scores can leave the
         * 16-bit row buffer (match * min(qlen, tlen) >= 2^15) stay on the
         * one-pair-per-thread kernel: the warp-cooperative start sweep's stop
         * test does not follow the reference once values wrap */
        uint32_t longest = 0;
        for (int i = 0; i < b.n; i++) longest = std::max(longest, std::min(b.h_q_len[i], b.h_t_len[i]));
        if ((uint64_t)cfg.sc.match * longest >= (1u << 15)) wc_algo = false;
    }
    uint32_t max_q_short = 0, max_q_long = 0, max_t_long = 0, max_q_big = 0, max_t_big = 0;
    int nlong = 0, nbig = 0;
    const uint32_t big_q = ORDER_CAP_WORDS * 8 - 7;
    /* a pair needs at least as many query words as its lane group (the
     * group's ring reader must trail its writer) */
    const int min_words = std::max(st.wc_min_qregs, st.wc_group > 0 ? st.wc_group : 8);
    p.wc_min_q = (uint32_t)min_words * 8 - 7;
    for (int i = 0; i < b.n; i++) {
        const uint32_t ql = b.h_q_len[i];
        if (wc_algo && ql >= p.wc_min_q) {
            nlong++;
            if (ql >= big_q) {
                nbig++;
                max_q_big = std::max(max_q_big, ql);
                max_t_big = std::max(max_t_big, b.h_t_len[i]);
            } else {
                max_q_long = std::max(max_q_long, ql);
                max_t_long = std::max(max_t_long, b.h_t_len[i]);
            }
        } else {
            max_q_short = std::max(max_q_short, ql);
        }
    }
    /* lane group of the warp kernel: forced, or the narrowest that keeps its
     * occupancy (each group holds a ring of q8 words and band maxima, or for
     * SEMI_GLOBAL the last-column H of every row, in shared memory) */
    {
        const int wstart = (cfg.algo == SEMI_GLOBAL_ && cfg.start == WITH_TB_) ? WITHOUT_START_ : cfg.start;
        const bool wsecond = cfg.second && (cfg.algo == LOCAL_ || cfg.algo == SEMI_GLOBAL_);
        const int max_group = min_words >= 32 ? 32 : min_words >= 16 ? 16 : 8;
        auto shape_for = [&](int n, uint32_t mq, uint32_t mt, int mg) {
            const int mq8 = (int)((mq + 7) & ~7u), mt8 = (int)((mt + 7) & ~7u);
            if (n <= 0 || mq8 > st.wc_max_q8) return WcLaunch{};
            return wc_plan(cfg.algo, wstart, wsecond, n, mq8, mt8, st.wc_group, mg);
        };
        const int nsmall = nlong - nbig;
        if (nlong > 0 && b.n >= st.min_order_pairs) {
            p.wc = shape_for(nsmall, max_q_long, max_t_long, max_group);
            /* the long launch's pairs all have 127+ query words: two-warp groups fit */
            p.wc_big = st.wc_big_group > 0 && st.wc_group == 0
                           ? [&] {
                                 const int mq8 = (int)((max_q_big + 7) & ~7u), mt8 = (int)((max_t_big + 7) & ~7u);
                                 if (nbig <= 0 || mq8 > st.wc_max_q8) return WcLaunch{};
                                 return wc_plan(cfg.algo, wstart, wsecond, nbig, mq8, mt8, st.wc_big_group, 64);
                             }()
                           : shape_for(nbig, max_q_big, max_t_big, 64);
        }
        p.use_wc = nlong > 0 && b.n >= st.min_order_pairs && (nsmall == 0 || p.wc.group > 0) &&
                   (nbig == 0 || p.wc_big.group > 0);
        if (p.use_wc) {
            /* the two launches run one after the other on one stream: one
             * last-column scratch serves both */
            const size_t rows = std::max(wc_scratch_words(cfg.algo, p.wc, (int)((max_t_long + 7) & ~7u)),
                                         wc_scratch_words(cfg.algo, p.wc_big, (int)((max_t_big + 7) & ~7u)));
            if (rows > 0 && grow((void **)&ws.wc_rows, &ws.wc_rows_cap, rows, 4) != GB_OK) return GB_ERR_ALLOC;
            if (grow((void **)&ws.wc_defer, &ws.wc_defer_cap, (size_t)nlong, 4) != GB_OK) return GB_ERR_ALLOC;
        }
    }
    if (!p.use_wc) {
        max_q_short = std::max({max_q_short, max_q_long, max_q_big});
        nlong = 0, nbig = 0;
    }
    p.mq8 = (int)((max_q_long + 7) & ~7u), p.mt8 = (int)((max_t_long + 7) & ~7u);
    p.mq8_big = (int)((max_q_big + 7) & ~7u), p.mt8_big = (int)((max_t_big + 7) & ~7u);

    /* row buffer placement (one-thread kernel) */
    const uint32_t max_q = max_q_short;
    const int cols = cfg.algo == KSW_ ? 2 * ((int)max_q + 2) : (int)((max_q + 7) & ~7u);
    const size_t smem_limit = 160u << 10;
    DpArgs &a = p.a;
    a = DpArgs{};
    a.pq = b.pq, a.pt = b.pt, a.q_off = b.q_off, a.t_off = b.t_off, a.q_len = b.q_len, a.t_len = b.t_len;
    a.seed = b.seed, a.order = nullptr, a.n = b.n;
    a.score = o.score, a.q_end = o.q_end, a.t_end = o.t_end, a.q_start = o.q_start, a.t_start = o.t_start;
    a.score2 = o.score2, a.q_end2 = o.q_end2, a.t_end2 = o.t_end2;
    a.max_off = cfg.algo == KSW_ ? o.max_off : nullptr;
    a.sc = cfg.sc, a.head = cfg.head, a.tail = cfg.tail, a.k_band = cfg.k_band, a.zdrop = cfg.zdrop, a.mql = cfg.mql;
    if (!ws.queue && dev_malloc((void **)&ws.queue, 128) != cudaSuccess) {
        cudaGetLastError();
        return GB_ERR_ALLOC;
    }
    a.queue = st.persistent ? ws.queue : nullptr;
    /* ksw: warp per pair; the one-thread kernel only takes what that hands
     * back (queries beyond 2046 bases, huge seed scores) */
    if (cfg.algo == KSW_ && st.ksw_wc && ksw_wc_scores_ok(cfg.sc)) {
        ksw_wc_classes(b.h_q_len, b.n, p.ksw_slots);
        p.ksw_short = st.ksw_groups ? ksw_grp_short(b.h_q_len, b.n) : 0;
        if (grow((void **)&ws.fb, &ws.fb_cap, (size_t)b.n, 4) != GB_OK) return GB_ERR_ALLOC;
        p.band = cfg.band_w != nullptr || cfg.band_model != nullptr;
        if (p.band) {
            if (grow((void **)&ws.retry, &ws.retry_cap, (size_t)b.n, 4) != GB_OK) return GB_ERR_ALLOC;
            if (cfg.band_model) {
                if (grow((void **)&ws.feat, &ws.feat_cap, (size_t)b.n * BAND_FEATS_PAD, 4) != GB_OK)
                    return GB_ERR_ALLOC;
                size_t cap = ws.pred_cap;
                if (grow((void **)&ws.pred, &cap, (size_t)b.n, 4) != GB_OK) return GB_ERR_ALLOC;
                if (grow((void **)&ws.bandw, &ws.pred_cap, (size_t)b.n, 4) != GB_OK) return GB_ERR_ALLOC;
            }
        }
    }
    auto cols_of = [&](uint32_t q) {
        return cfg.algo == KSW_ ? 2 * ((int)q + 2) : (int)((q + 7) & ~7u);
    };
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if ((size_t)std::max(cols, 8) * p.block * 4 <= smem_limit) {
        a.smem_cols = std::max(cols, 8);
    } else {
        /* the longest query does not leave room for shared-memory rows: split
         * the one-thread pairs into a shared-memory tier and a long tier with
         * global rows on a small grid (a long pair needs many cells per
         * thread, not many threads) */
        const int fit_cols = (int)(smem_limit / (4 * (size_t)p.block));
        const uint32_t q_fit = cfg.algo == KSW_ ? (uint32_t)std::max(fit_cols / 2 - 2, 0) : (uint32_t)(fit_cols & ~7);
        uint32_t max_s = 0, max_l = 0;
        int n_s = 0, n_l = 0;
        if (p.ksw_slots[0] == 0) {
            for (int i = 0; i < b.n; i++) {
                const uint32_t ql = b.h_q_len[i];
                if (p.use_wc && ql >= p.wc_min_q) continue;
                if (ql <= q_fit) n_s++, max_s = std::max(max_s, ql);
                else n_l++, max_l = std::max(max_l, ql);
            }
        }
        if (n_s > 0 && n_l > 0) {
            p.tier2 = true;
            p.tier_q = q_fit;
            a.smem_cols = std::max(cols_of(max_s), 8);
            a.q_max = q_fit;
            p.tier2_cols = cols_of(max_l);
            p.tier2_blocks = std::min(dp_scratch_blocks(n_l, p.block), 4 * sms);
            const size_t threads = (size_t)p.tier2_blocks * p.block;
            if (grow((void **)&ws.scratch, &ws.scratch_cap, threads * p.tier2_cols, 4) != GB_OK) return GB_ERR_ALLOC;
        } else {
            a.smem_cols = 0;
            int blocks = dp_scratch_blocks(b.n, p.block);
            if (p.ksw_slots[0] > 0) {
                blocks = std::min(blocks, 2 * sms);
                p.fb_blocks = blocks;
            }
            const size_t threads = (size_t)blocks * p.block;
            if (grow((void **)&ws.scratch, &ws.scratch_cap, threads * cols, 4) != GB_OK) return GB_ERR_ALLOC;
            a.scratch = ws.scratch;
            a.scratch_cols = (uint32_t)cols;
        }
    }
    if (p.use_wc && !ws.aux) {
        /* the warp-cooperative kernels run on the auxiliary stream: with the
         * launch stream's priority, so a caller's prioritised batch keeps it */
        int prio = 0;
        if (s && cudaStreamGetPriority(s, &prio) != cudaSuccess) {
            cudaGetLastError();
            prio = 0;
        }
        if (cudaStreamCreateWithPriority(&ws.aux, cudaStreamNonBlocking, prio) != cudaSuccess ||
            cudaEventCreateWithFlags(&ws.fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ws.join, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return GB_ERR_CUDA;
        }
    }

    p.tb = cfg.start == WITH_TB_ && (cfg.algo == LOCAL_ || cfg.algo == GLOBAL_ || semi_tb);
    /* SEMI_GLOBAL WITH_TB with another tail returns the reference's outputs: the forward pass alone */
    p.start = (cfg.algo == SEMI_GLOBAL_ && cfg.start == WITH_TB_ && !semi_tb) ? WITHOUT_START_ : cfg.start;
    p.second = cfg.second && (cfg.algo == LOCAL_ || cfg.algo == SEMI_GLOBAL_);
    p.split_start = st.split_start && p.start == WITH_START_ && (cfg.algo == LOCAL_ || cfg.algo == SEMI_GLOBAL_) &&
                    b.n >= st.min_order_pairs && o.score && o.q_end && o.t_end;
    if (p.split_start) {
        if (grow((void **)&ws.order2, &ws.order2_cap, (size_t)b.n, 4) != GB_OK) return GB_ERR_ALLOC;
        if (!ws.bins && dev_malloc((void **)&ws.bins, (size_t)order_bins() * 4) != cudaSuccess) {
            cudaGetLastError();
            return GB_ERR_ALLOC;
        }
    }

    if (!p.tb) {
        p.cut = {0, b.n};
        p.nlong = {nlong};
        p.nbig = {nbig};
        p.order_on = p.use_wc || b.n >= st.min_order_pairs;
        if (p.order_on && ensure_order_buffers(ws, (size_t)b.n) != GB_OK) return GB_ERR_ALLOC;
        return GB_OK;
    }

    /* traceback: chunk pairs so the tiles fit the budget */
    if (ws.tb_off_free && cudaEventSynchronize(ws.tb_off_free) != cudaSuccess) return GB_ERR_CUDA;
    if (ws.tb_off_cap < (size_t)b.n) {
        if (ws.h_tb_off) cudaFreeHost(ws.h_tb_off);
        if (ws.d_tb_off) cudaFree(ws.d_tb_off);
        ws.h_tb_off = nullptr, ws.d_tb_off = nullptr, ws.tb_off_cap = 0;
        const size_t want = (size_t)b.n + b.n / 4 + 1024;
        if (cudaMallocHost((void **)&ws.h_tb_off, want * 8) != cudaSuccess ||
            dev_malloc((void **)&ws.d_tb_off, want * 8) != cudaSuccess) {
            cudaGetLastError();
            return GB_ERR_ALLOC;
        }
        ws.tb_off_cap = want;
    }
    if (!ws.tb_off_free && cudaEventCreateWithFlags(&ws.tb_off_free, cudaEventDisableTiming) != cudaSuccess)
        return GB_ERR_CUDA;
    /* tile budget: the setting, but at most half of the device memory that is
     * free or already held as this stream's tiles (fewer, longer chunks on a
     * large device; room left for other streams) */
    uint64_t budget_bytes = st.tb_budget_bytes;
    {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            const uint64_t avail = ((uint64_t)free_b + (uint64_t)ws.tb_cap * 16) / 2;
            budget_bytes = std::min<uint64_t>(budget_bytes, std::max<uint64_t>(avail, (uint64_t)1 << 30));
        } else {
            cudaGetLastError();
        }
    }
    const uint64_t budget = std::max<uint64_t>(budget_bytes / 16, 1);
    p.cut = {0};
    uint64_t run = 0, chunk_max = 0;
    for (int i = 0; i < b.n; i++) {
        const uint64_t t = tb_tiles(b.h_q_len[i], b.h_t_len[i]);
        if (run > 0 && run + t > budget) {
            chunk_max = std::max(chunk_max, run);
            p.cut.push_back(i);
            run = 0;
        }
        ws.h_tb_off[i] = run;
        run += t;
    }
    chunk_max = std::max(chunk_max, run);
    p.cut.push_back(b.n);
    if (grow((void **)&ws.tb, &ws.tb_cap, chunk_max, sizeof(uint4)) != GB_OK) return GB_ERR_ALLOC;
    size_t max_chunk = 0;
    for (size_t c = 0; c + 1 < p.cut.size(); c++) {
        const int p0 = p.cut[c], p1 = p.cut[c + 1];
        int nl = 0, nb = 0;
        if (p.use_wc)
            for (int i = p0; i < p1; i++) {
                nl += b.h_q_len[i] >= p.wc_min_q ? 1 : 0;
                nb += b.h_q_len[i] >= big_q ? 1 : 0;
            }
        p.nlong.push_back(nl);
        p.nbig.push_back(nb);
        max_chunk = std::max(max_chunk, (size_t)(p1 - p0));
    }
    p.order_on = p.use_wc || b.n >= st.min_order_pairs;
    if (p.order_on && ensure_order_buffers(ws, max_chunk) != GB_OK) return GB_ERR_ALLOC;
    return GB_OK;
}

/* The one-thread launch(es) for DpArgs a: with two length tiers, the short
 * tier from a (shared-memory rows) and the long tier from a's copy with
 * global rows on a small grid.  queue words 0 and 1 are their counters. */
/* `upper` (0: none) bounds the query lengths of the long tier: the start
 * pass launch visits every pair and must skip the warp-cooperative ones. */
static int launch_tiers(int algo, int start, bool second, const Plan &p, DpArgs a, Workspace &ws, cudaStream_t s,
                        uint32_t upper = 0)
{
    if (a.queue) GB_CUDA(cudaMemsetAsync(a.queue, 0, 8, s));
    timing_mark(K_DP, true, s);
    GB_CUDA(launch_dp(algo, start, second, a, p.block, 0, s));
    if (p.tier2) {
        DpArgs l = a;
        l.smem_cols = 0;
        l.scratch = ws.scratch;
        l.scratch_cols = (uint32_t)p.tier2_cols;
        l.q_min = p.tier_q + 1;
        l.q_max = upper;
        l.queue = a.queue ? a.queue + 1 : nullptr;
        GB_CUDA(launch_dp_scratch_grid(algo, start, second, l, p.block, p.tier2_blocks, s));
    }
    timing_mark(K_DP, false, s);
    return GB_OK;
}

/* With split_start the forward pass runs first; then the start passes of the
 * same pairs, visited by (reverse-region words, forward score) so the lanes
 * of a warp stop at similar bands (a start pass runs until it reaches the
 * forward score).  Pairs the warp-cooperative kernel owns are skipped by
 * their length. */
static int launch_one_thread(int algo, int start, bool second, const Plan &p, DpArgs a, Workspace &ws,
                             cudaStream_t s)
{
    if (!(p.split_start && start == WITH_START_)) return launch_tiers(algo, start, second, p, a, ws, s);
    int rc = launch_tiers(algo, WITHOUT_START_, second, p, a, ws, s);
    if (rc != GB_OK) return rc;
    timing_mark(K_ORDER, true, s);
    /* the warp-cooperative pairs' outputs may still be in flight on the
     * auxiliary stream: the order must not read them */
    const uint32_t cut = p.use_wc ? (uint32_t)p.wc_min_q : 0u;
    GB_CUDA(launch_start_order(p.a.q_len, p.a.q_end, p.a.score, p.a.n, cut, ws.bins, ws.order2, s));
    timing_mark(K_ORDER, false, s);
    DpArgs st = p.a;
    st.order = ws.order2;
    const uint32_t upper = cut ? cut - 1 : 0;
    if (upper && (st.q_max == 0 || st.q_max > upper)) st.q_max = upper;
    return launch_tiers(algo, START_ONLY_, false, p, st, ws, s, upper);
}

/* DP over pairs [0, a.n) visited in `order` (nullptr: identity): the first
 * nlong entries of order on the warp-cooperative kernel (auxiliary stream;
 * the leading nbig of them, ORDER_CAP_WORDS+ query words, as a launch of
 * their own,
 * forked from and joined back into s), the rest on the one-thread kernel. */
static int launch_dp_split(int algo, int start, bool second, const Plan &p, DpArgs a, const uint32_t *order,
                           int nlong, int nbig, Workspace &ws, cudaStream_t s)
{
    if (nlong > 0 && order) {
        GB_CUDA(cudaEventRecord(ws.fork, s));
        GB_CUDA(cudaStreamWaitEvent(ws.aux, ws.fork, 0));
        timing_mark(K_DP, true, ws.aux);
        /* queue words 12 and 13: the two launches' counts of pairs left to
         * compare scoring; 16-17 and 18-19: their work counters */
        if (nbig > 0)
            GB_CUDA(launch_dp_wc(algo, start, second, a, order, nbig, p.mq8_big, p.mt8_big, p.wc_big, ws.wc_rows,
                                 ws.wc_defer, ws.queue + 12, ws.queue + 16, ws.aux));
        if (nlong > nbig)
            GB_CUDA(launch_dp_wc(algo, start, second, a, order + nbig, nlong - nbig, p.mq8, p.mt8, p.wc, ws.wc_rows,
                                 ws.wc_defer, ws.queue + 13, ws.queue + 18, ws.aux));
        timing_mark(K_DP, false, ws.aux);
        GB_CUDA(cudaEventRecord(ws.join, ws.aux));
        DpArgs rest = a;
        rest.order = order + nlong;
        rest.n = a.n - nlong;
        if (rest.n > 0) {
            const int rc = launch_one_thread(algo, start, second, p, rest, ws, s);
            if (rc != GB_OK) return rc;
        }
        GB_CUDA(cudaStreamWaitEvent(s, ws.join, 0));
        return GB_OK;
    }
    a.order = order;
    return launch_one_thread(algo, start, second, p, a, ws, s);
}

/* ksw: every pair (in `order`, or 0..n-1) to the warp-per-pair kernel --
 * banded first when a band is given, the certificate's refusals again
 * without one -- then the pairs it handed back to the one-thread kernel,
 * whose counts it reads on the device.  queue words: [0..1] one-thread work
 * counters, [2] handed-back count, [3] refused count, [4..5] computed cells
 * (u64), [6..7] warp work counters of the two length classes, [8..9] the
 * same for the recomputation pass, [10] and [11] the lane-group launches'
 * counters of the two passes. */
static int launch_ksw_split(const RunCfg &cfg, const DevBatch &b, const Plan &p, const uint32_t *order, int n,
                            Workspace &ws, cudaStream_t s)
{
    GB_CUDA(cudaMemsetAsync(ws.queue, 0, 64, s));
    unsigned long long *cells = reinterpret_cast<unsigned long long *>(ws.queue + 4);
    timing_mark(K_DP, true, s);
    if (p.band) {
        const int32_t *bw = cfg.band_w;
        if (!bw) {
            GB_CUDA(launch_band_features(b.pq, b.pt, b.q_off, b.t_off, b.q_len, b.t_len, n, ws.feat, s));
            GB_CUDA(launch_mlp_forward(static_cast<const __nv_bfloat16 *>(cfg.band_model), ws.feat, n, ws.pred, s));
            GB_CUDA(launch_band_from_pred(ws.pred, b.q_len, b.t_len, n, cfg.band_min, cfg.band_max, ws.bandw, s));
            bw = ws.bandw;
        }
        GB_CUDA(launch_ksw_band(p.a, order, n, p.ksw_slots, bw, ws.fb, ws.queue + 2, ws.retry, ws.queue + 3, cells,
                                ws.queue + 6, s));
        if (cfg.band_ok) GB_CUDA(launch_band_ok(cfg.band_ok, n, ws.retry, ws.queue + 3, s));
        DpArgs ra = p.a;
        ra.n_dev = ws.queue + 3;
        GB_CUDA(launch_ksw_wc(ra, ws.retry, n, p.ksw_slots, ws.fb, ws.queue + 2, ws.queue + 8, cells, s,
                              p.ksw_short > 0 ? -1 : -2, ws.queue + 11));
    } else {
        /* a length order lists the short pairs last */
        const int split = p.ksw_short <= 0 ? -2 : (order ? n - p.ksw_short : -1);
        GB_CUDA(launch_ksw_wc(p.a, order, n, p.ksw_slots, ws.fb, ws.queue + 2, ws.queue + 6, cells, s, split,
                              ws.queue + 10));
    }
    timing_mark(K_DP, false, s);
    DpArgs fa = p.a;
    fa.order = ws.fb;
    fa.n = n;
    fa.n_dev = ws.queue + 2;
    fa.queue = ws.queue;
    timing_mark(K_DP, true, s);
    if (fa.smem_cols > 0) GB_CUDA(launch_dp(KSW_, WITHOUT_START_, false, fa, p.block, 0, s));
    else GB_CUDA(launch_dp_scratch_grid(KSW_, WITHOUT_START_, false, fa, p.block, p.fb_blocks, s));
    timing_mark(K_DP, false, s);
    return GB_OK;
}

static int enqueue_order(const uint32_t *q_len, const uint32_t *t_len, int n, Workspace &ws, cudaStream_t s)
{
    timing_mark(K_ORDER, true, s);
    const cudaError_t e = launch_order(q_len, t_len, n, ws.bins, ws.order, s);
    timing_mark(K_ORDER, false, s);
    return e == cudaSuccess ? GB_OK : GB_ERR_CUDA;
}

static int enqueue_align(const RunCfg &cfg, const DevBatch &b, const DevOut &o, Workspace &ws, const Plan &p,
                         cudaStream_t s);

int enqueue_batch(const RunCfg &cfg, const DevBatch &b, const DevOut &o, Workspace &ws, const Plan &p,
                  cudaStream_t s)
{
    /* pack and reverse/complement */
    if (!cfg.is_packed) {
        timing_mark(K_PACK, true, s);
        GB_CUDA(launch_pack(b.q, b.q_bytes, b.pq, s));
        timing_mark(K_PACK, false, s);
        timing_mark(K_PACK, true, s);
        GB_CUDA(launch_pack(b.t, b.t_bytes, b.pt, s));
        timing_mark(K_PACK, false, s);
    }
    if (cfg.reverse_complement) {
        timing_mark(K_RC, true, s);
        GB_CUDA(launch_revcomp(b.pq, b.pt, b.q_off, b.t_off, b.q_len, b.t_len, b.q_op, b.t_op, b.n,
                               cfg.ref_reverse, s));
        timing_mark(K_RC, false, s);
    }
    timing_mark(K_SPAN, true, s);
    const int rc = enqueue_align(cfg, b, o, ws, p, s);
    timing_mark(K_SPAN, false, s);
    return rc;
}

/* ordering, DP and traceback of a packed batch */
static int enqueue_align(const RunCfg &cfg, const DevBatch &b, const DevOut &o, Workspace &ws, const Plan &p,
                         cudaStream_t s)
{
    if (!p.tb) {
        const uint32_t *ord = nullptr;
        if (p.order_on) {
            const int rc = enqueue_order(b.q_len, b.t_len, b.n, ws, s);
            if (rc != GB_OK) return rc;
            ord = ws.order;
        }
        if (p.ksw_slots[0] > 0) return launch_ksw_split(cfg, b, p, ord, b.n, ws, s);
        return launch_dp_split(cfg.algo, p.start, p.second, p, p.a, ord, ord ? p.nlong[0] : 0, ord ? p.nbig[0] : 0,
                               ws, s);
    }
    GB_CUDA(cudaMemcpyAsync(ws.d_tb_off, ws.h_tb_off, (size_t)b.n * 8, cudaMemcpyHostToDevice, s));
    for (size_t c = 0; c + 1 < p.cut.size(); c++) {
        const int p0 = p.cut[c], p1 = p.cut[c + 1];
        DpArgs ca = p.a;
        ca.n = p1 - p0;
        ca.q_off = b.q_off + p0, ca.t_off = b.t_off + p0, ca.q_len = b.q_len + p0, ca.t_len = b.t_len + p0;
        auto sh = [p0](int32_t *x) { return x ? x + p0 : x; };
        ca.score = sh(o.score), ca.q_end = sh(o.q_end), ca.t_end = sh(o.t_end);
        ca.q_start = sh(o.q_start), ca.t_start = sh(o.t_start);
        ca.score2 = sh(o.score2), ca.q_end2 = sh(o.q_end2), ca.t_end2 = sh(o.t_end2);
        ca.tb = ws.tb, ca.tb_off = ws.d_tb_off + p0;
        const uint32_t *ord = nullptr;
        if (p.order_on) {
            const int rc = enqueue_order(ca.q_len, ca.t_len, ca.n, ws, s);
            if (rc != GB_OK) return rc;
            ord = ws.order;
        }
        const int rc = launch_dp_split(cfg.algo, p.start, p.second, p, ca, ord, ord ? p.nlong[c] : 0,
                                       ord ? p.nbig[c] : 0, ws, s);
        if (rc != GB_OK) return rc;
        TbArgs t{};
        t.tb = ws.tb, t.tb_off = ws.d_tb_off + p0;
        t.q_off = ca.q_off, t.q_len = ca.q_len, t.t_len = ca.t_len;
        t.score = ca.score, t.q_end = ca.q_end, t.t_end = ca.t_end;
        t.q_start = ca.q_start, t.t_start = ca.t_start;
        t.cigar = o.cigar, t.cigar_bytes = b.q_bytes;
        t.n_cigar = o.n_cigar ? o.n_cigar + p0 : nullptr;
        t.n = ca.n, t.algo = cfg.algo, t.sc = cfg.sc, t.head = cfg.head;
        timing_mark(K_TB, true, s);
        GB_CUDA(launch_traceback(t, s));
        timing_mark(K_TB, false, s);
    }
    return GB_OK;
}

int run_batch(const RunCfg &cfg, const DevBatch &b, const DevOut &o, Workspace &ws, cudaStream_t s)
{
    Plan p;
    int rc = plan_batch(cfg, b, o, ws, p, s);
    if (rc != GB_OK) return rc;
    rc = enqueue_batch(cfg, b, o, ws, p, s);
    if (rc == GB_OK && p.tb) GB_CUDA(cudaEventRecord(ws.tb_off_free, s));
    return rc;
}

bool timing_on()
{
    Timing &t = timing();
    std::lock_guard<std::mutex> lk(t.mu);
    return t.on;
}

} // namespace gb
