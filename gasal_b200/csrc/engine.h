/*
 * engine.h -- the batch engine behind both the GASAL2 C++ API and the C ABI.
 *
 * One call of run_batch() is the device half of reference
 * gasal_aln_async (src/gasal_align.cu:180-264): pack -> reverse/complement ->
 * alignment kernel -> traceback, all stream-ordered on one CUDA stream,
 * reading inputs already in device memory.  Planning (row-buffer placement,
 * traceback chunking) uses the host copy of the lengths.
 */
#ifndef GB_ENGINE_H
#define GB_ENGINE_H

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include <vector>

#include "gb_internal.h"
#include "gasal_b200_capi.h"

namespace gb {

struct RunCfg {
    int algo, start, second, head, tail, k_band, zdrop;
    Scores sc;
    int ref_reverse; /* reference-identical reversal (default 1) */
    int mql;         /* reference MAX_QUERY_LEN for the semi-global last-row scan */
    int is_packed;   /* inputs are already 4-bit words */
    int reverse_complement;
    /* ksw band (warp kernel only): an explicit per-pair half-width array, or
     * an MLP (BF16 parameters) that predicts it from pair features */
    const int32_t *band_w = nullptr;
    const void *band_model = nullptr;
    int band_min = 16, band_max = 1024;
    uint8_t *band_ok = nullptr; /* optional: 1 where the banded result was kept */
};

struct DevBatch {
    int32_t n;
    uint32_t q_bytes, t_bytes;
    const uint8_t *q, *t;       /* ASCII (or packed words when is_packed) */
    uint32_t *pq, *pt;          /* packed word outputs (may equal q/t when is_packed) */
    const uint32_t *q_off, *t_off, *q_len, *t_len;
    const uint8_t *q_op, *t_op;
    const uint32_t *seed;
    const uint32_t *h_q_len, *h_t_len; /* host copies, for planning */
};

struct DevOut {
    int32_t *score, *q_end, *t_end, *q_start, *t_start, *score2, *q_end2, *t_end2;
    uint8_t *cigar;             /* device buffer of q_bytes (the query batch) */
    uint32_t *n_cigar;
    int32_t *max_off;           /* ksw: largest diagonal offset of a rise of the maximum (optional) */
};

/* Device scratch owned by one stream (grown on demand, never shrunk). */
struct Workspace {
    int device = -1;
    uint4 *tb = nullptr;
    size_t tb_cap = 0;          /* uint4 units */
    uint64_t *d_tb_off = nullptr, *h_tb_off = nullptr;
    size_t tb_off_cap = 0;
    uint32_t *scratch = nullptr;
    size_t scratch_cap = 0;     /* uint32 units */
    cudaEvent_t tb_off_free = nullptr;
    uint32_t *order = nullptr;   /* length-binned visiting order */
    size_t order_cap = 0;
    int32_t *wc_rows = nullptr;  /* warp-cooperative SEMI_GLOBAL last-column rows */
    size_t wc_rows_cap = 0;
    uint32_t *wc_defer = nullptr; /* pairs the table-scoring warp-cooperative launch leaves to compare scoring */
    size_t wc_defer_cap = 0;
    uint32_t *order2 = nullptr;  /* visiting order of the separate start passes */
    size_t order2_cap = 0;
    uint32_t *bins = nullptr;    /* order_bins() class counters */
    cudaStream_t aux = nullptr;  /* second stream for the warp-cooperative kernel */
    uint32_t *queue = nullptr;   /* work counter of the persistent one-thread launch */
    cudaEvent_t fork = nullptr, join = nullptr;
    uint32_t *fb = nullptr;      /* pairs the warp ksw kernel hands back */
    size_t fb_cap = 0;
    uint32_t *retry = nullptr;   /* pairs whose banded result the certificate refused */
    size_t retry_cap = 0;
    float *feat = nullptr;       /* band features, BAND_FEATS_PAD per pair */
    size_t feat_cap = 0;         /* floats */
    float *pred = nullptr;       /* predicted log2 band */
    int32_t *bandw = nullptr;    /* per-pair band */
    size_t pred_cap = 0;
    ~Workspace();
};

/* Frees every buffer, stream and event of a workspace (no work of it may be
 * in flight) and leaves it empty, ready to grow again. */
void release_workspace(Workspace &w);
/* the buffers gb_align_dev_mixed keeps per (device, stream) (mixed.cu) */
void mix_release_all();
/* the band entry points' per-stream workspaces (band_api.cu) */
void band_release_all();

/* The decisions and allocations for one batch (plan_batch), so that
 * enqueue_batch issues stream operations only -- capturable into a graph. */
struct Plan {
    bool tb = false, second = false, use_wc = false, order_on = false;
    int start = 0, block = 64, mq8 = 0, mt8 = 0;
    uint32_t wc_min_q = 0;
    WcLaunch wc;                 /* shape of the warp-cooperative launch */
    /* warp-cooperative pairs of ORDER_CAP_WORDS+ query words (the order's
     * prefix) run as a launch of their own with their own shape and buffer
     * sizes, so their long rings leave the shorter pairs' groups alone */
    WcLaunch wc_big;
    int mq8_big = 0, mt8_big = 0;
    int ksw_slots[2] = {0, 0}; /* [0] > 0: ksw runs warp-per-pair; eh columns per warp of the two length classes */
    int ksw_short = 0;         /* unbanded ksw pairs of at most 31 query words, run on lane groups (0: none) */
    bool tier2 = false;     /* one-thread pairs split: short ones with shared-memory rows (a), long ones
                               with global rows on a small grid (tier2_* overrides of a) */
    uint32_t tier_q = 0;    /* queries up to tier_q: shared-memory tier */
    int tier2_cols = 0, tier2_blocks = 0;
    bool band = false;      /* ksw through the banded kernel + certificate */
    bool split_start = false; /* one-thread start passes as a second launch (order2) */
    int fb_blocks = 0;      /* grid of the one-thread ksw launch for handed-back pairs (scratch rows) */
    DpArgs a{};
    std::vector<int> cut;   /* pair ranges [cut[c], cut[c+1]) run one after another */
    std::vector<int> nlong; /* per range: pairs on the warp-cooperative kernel */
    std::vector<int> nbig;  /* per range: of those, the leading ORDER_CAP_WORDS+ word ones */
};

/* status codes of gasal_b200_capi.h */
/* s: the stream the batch will run on (its priority is given to the
 * workspace's auxiliary stream when that is created) */
int plan_batch(const RunCfg &cfg, const DevBatch &b, const DevOut &o, Workspace &ws, Plan &p,
               cudaStream_t s = nullptr);
int enqueue_batch(const RunCfg &cfg, const DevBatch &b, const DevOut &o, Workspace &ws, const Plan &p,
                  cudaStream_t s);
int run_batch(const RunCfg &cfg, const DevBatch &b, const DevOut &o, Workspace &ws, cudaStream_t s);

/* Traceback tiles of one pair, in uint4 units (two spare tile rows). */
inline uint64_t tb_tiles(uint32_t qlen, uint32_t tlen)
{
    const uint64_t qr = (qlen + 7) >> 3, tr = (tlen + 7) >> 3;
    return (tr + 2) * 2 * qr;
}

/* Process-wide settings (set through the C ABI). */
struct Settings {
    Scores sc = {1, 4, 6, 1, 7};
    int ref_reverse = 1;
    int mql = 2048;
    size_t tb_budget_bytes = (size_t)96 << 30; /* traceback tiles per stream (at most half the free memory) */
    int block = 32;             /* one-pair-per-thread block: 32 packs the most row buffers per SM */
    int min_order_pairs = 2048; /* batches at least this large visit pairs length-binned */
    int wc_min_qregs = 32;      /* pairs with at least this many query words go warp-cooperative */
    int wc_max_q8 = 12000;      /* ... while the batch's longest query fits the warp's ring */
    int graphs = 1;             /* gasal_aln_async runs each batch as a CUDA graph */
    int ksw_wc = 1;             /* ksw pairs run warp-per-pair (ksw_wc.cu) */
    int split_start = 1;        /* one-thread LOCAL/SEMI_GLOBAL start passes run as their own launch,
                                   pairs re-ordered by forward score */
    int wc_group = 0;           /* lanes per pair in the warp-cooperative kernels: 32, 16 or 8, or 0 to pick
                                   per launch from the kernel's occupancy */
    int persistent = 1;         /* one-thread launches pull pairs from a device counter; 0: one thread per
                                   pair on a grid over the batch */
    const void *band_model = nullptr; /* installed band MLP (BF16 parameters on the device) */
    int band_min = 16, band_max = 1024;
    int wc_big_group = 0;       /* lane group of the 127+ word launch: 0 = automatic (64 when it fits), 32 or 64 */
    int ksw_groups = 1;         /* unbanded ksw pairs of at most 31 query words run 4 to a warp (lane groups) */
};
Settings &settings();

/* cudaMalloc with an optional injected failure (GASAL_B200_FAIL_ALLOC_AFTER). */
cudaError_t dev_malloc(void **p, size_t bytes);

/* Optional per-kernel CUDA-event timing (off by default).  Kinds: */
/* K_SPAN is not a kernel: one mark per batch on the launch stream, from the
 * first alignment-phase operation (ordering or DP) to the last (DP joined back
 * from the auxiliary stream, traceback included) -- the phase's wall clock. */
enum KernelKind { K_PACK = 0, K_RC = 1, K_DP = 2, K_TB = 3, K_ORDER = 4, K_SPAN = 5, K_KINDS = 6 };
void timing_enable(bool on);
void timing_mark(int kind, bool start, cudaStream_t s);
int timing_read(double ms[K_KINDS], int64_t launches[K_KINDS]);
bool timing_on();
int probe_int_peak(double *iadd, double *imnmx, double *dpx);
int probe_dpx16x2_peak(double *halfword_tops);

} // namespace gb

#endif
