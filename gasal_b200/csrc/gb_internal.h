/*
 * gb_internal.h -- kernel-side interface of the B200 GASAL2-compatible engine.
 *
 * Device data layout (one batch, all in HBM):
 *   packed query / target words  uint32, 8 bases per word, 4-bit codes, first
 *                                base in bits 31..28; word offset of pair i is
 *                                byte_offset[i] >> 3 (GASAL2's layout)
 *   per-pair lengths, offsets    uint32 [n]
 *   row-buffer scratch           one uint32 per query column per active
 *                                thread: H in the low, E in the high 16 bits
 *                                (int16 each, as the reference's short2)
 *   traceback tiles              uint4 per 8 target rows x 4 query columns,
 *                                a 4-bit direction code per cell; pair i owns
 *                                (tregs+2) x 2*qregs tiles from tb_off[i]
 */
#ifndef GB_INTERNAL_H
#define GB_INTERNAL_H

#include <cstdint>
#include <cuda_runtime.h>

namespace gb {

enum Algo { GLOBAL_ = 1, SEMI_GLOBAL_ = 2, LOCAL_ = 3, BANDED_ = 5, KSW_ = 6 };
enum Start { WITHOUT_START_ = 0, WITH_START_ = 1, WITH_TB_ = 2,
             START_ONLY_ = 3 /* engine-internal: the start pass alone, from the forward outputs */ };
enum Src { NONE_ = 0, QUERY_ = 1, TARGET_ = 2, BOTH_ = 3 };

struct Scores {
    int32_t match, mismatch, o, e, oe;
};

/* Everything a DP launch reads and writes.  Passed by value (kernel
 * parameter space). */
struct DpArgs {
    const uint32_t *pq, *pt;            /* packed words */
    const uint32_t *q_off, *t_off;      /* byte offsets */
    const uint32_t *q_len, *t_len;
    const uint32_t *seed;               /* ksw h0 */
    const uint32_t *order;              /* pair visiting order, or null */
    int32_t n;
    int32_t *score, *q_end, *t_end, *q_start, *t_start;
    int32_t *score2, *q_end2, *t_end2;
    uint4 *tb;                          /* traceback tiles */
    const uint64_t *tb_off;             /* per pair, in uint4 units */
    uint32_t *scratch;                  /* global row buffers (when not in shared memory) */
    uint32_t scratch_cols;              /* columns per thread in scratch */
    Scores sc;
    int32_t head, tail, k_band, zdrop, mql;
    int32_t smem_cols;                  /* columns per thread held in shared memory (0 = use scratch) */
    uint32_t *queue;                    /* work counter of the persistent launch (zeroed), or null */
    const uint32_t *n_dev;              /* if set, the number of pairs is read here on the device
                                           (n is then an upper bound, used to size the grid) */
    uint32_t q_min, q_max;              /* one-thread kernel: only pairs with q_min <= qlen <= q_max
                                           (q_max 0: no upper limit) */
    int32_t *lastcol;                   /* warp-cooperative SEMI_GLOBAL: last-column H of every row,
                                           one slot of scratch_cols words per lane group of the grid */
    int32_t *max_off;                   /* unbanded ksw: largest |column - row| of the cells where the
                                           running maximum rose (ksw_extend2's max_off), or null */
    uint32_t *defer, *ndefer;           /* warp-cooperative table-scoring launch: pairs it leaves to the
                                           compare-scoring launch, and their count */
};

/* Shape of one warp-cooperative launch: lanes per pair (0: it cannot run),
 * warps per block, grid, dynamic shared memory, resident warps per SM. */
struct WcLaunch {
    int group = 0, warps = 4, blocks = 0, resident_warps = 0;
    size_t smem = 0;
};

struct TbArgs {
    const uint4 *tb;
    const uint64_t *tb_off;
    const uint32_t *q_off, *q_len, *t_len;
    const int32_t *score, *q_end, *t_end;
    int32_t *q_start, *t_start;
    uint8_t *cigar;                     /* = the device query batch, as in GASAL2 */
    uint32_t cigar_bytes;
    uint32_t *n_cigar;
    int32_t n;
    int32_t algo;
    Scores sc;
    int32_t head;                       /* SEMI_GLOBAL: which leading bases are free */
};

/* ---- launchers (stream-ordered, no allocation) ---- */
cudaError_t launch_pack(const uint8_t *ascii, uint32_t nbytes, uint32_t *words, cudaStream_t s);
cudaError_t launch_revcomp(uint32_t *pq, uint32_t *pt, const uint32_t *q_off, const uint32_t *t_off,
                           const uint32_t *q_len, const uint32_t *t_len, const uint8_t *q_op,
                           const uint8_t *t_op, int32_t n, int ref_reverse, cudaStream_t s);
cudaError_t launch_dp(int algo, int start, bool second, const DpArgs &a, int block, int max_q8,
                      cudaStream_t s);
cudaError_t launch_traceback(const TbArgs &a, cudaStream_t s);

/* Lets a kernel use the most dynamic shared memory the device gives a block
 * (set once per kernel and device).  Kernels launched with different sizes
 * -- the length classes of one batch, other storages, occupancy queries --
 * then never depend on which size an earlier call set: a launch captured in
 * a CUDA graph and replayed later (or profiled node by node) finds the
 * attribute still covering it. */
cudaError_t allow_dyn_smem_fn(const void *fn);
template <class K> inline cudaError_t allow_dyn_smem(K *k) { return allow_dyn_smem_fn((const void *)k); }

/* forward CIGAR text of every pair (cigar_text.cu) */
cudaError_t launch_cigar_text(const uint8_t *cigar, const uint32_t *q_off, const uint32_t *n_cigar, int n,
                              char *text, int stride, int32_t *text_len, cudaStream_t s);

/* the length order's classes stop at this many query (and target) words:
 * pairs of at least ORDER_CAP_WORDS query words form the order's prefix */
constexpr uint32_t ORDER_CAP_WORDS = 127;

/* length-binned visiting order (sched.cu): bins = order_bins() words of
 * scratch, order = n words */
int order_bins();
cudaError_t launch_order(const uint32_t *q_len, const uint32_t *t_len, int n, uint32_t *bins, uint32_t *order,
                         cudaStream_t s);
/* order for the start passes: by query words of the reverse region and the
 * forward score (a proxy for how far the start pass runs), most work first.
 * Pairs of q_cut+ bases (0: none) go last without their outputs being read. */
cudaError_t launch_start_order(const uint32_t *q_len, const int32_t *q_end, const int32_t *score, int n,
                               uint32_t q_cut, uint32_t *bins, uint32_t *order, cudaStream_t s);

/* warp-cooperative DP (dp_wc.cu) for the pairs listed in `list`: LOCAL,
 * GLOBAL and target-tail SEMI_GLOBAL, each pair on `l.group` lanes (32, 16
 * or 8; queries of at least that many words); `rows`: SEMI_GLOBAL's
 * last-column scratch of wc_scratch_words(...) words.  With `defer` (nlist
 * words) and `ndefer` (one word) the pairs run on the kernels that score with
 * the prmt table, and the few they cannot (codes outside A/C/G/T/N, scores
 * beyond a byte) on the compare-scoring kernels after them. */
cudaError_t launch_dp_wc(int algo, int start, bool second, const DpArgs &a, const uint32_t *list, int nlist,
                         int max_q8, int max_t8, const WcLaunch &l, int32_t *rows, uint32_t *defer, uint32_t *ndefer,
                         uint32_t *wq, cudaStream_t s);
/* dynamic shared memory of one warp-cooperative block */
size_t wc_smem_bytes(int algo, int group, int warps, int max_q8, int max_t8);
/* launch shape for nlist pairs: the forced group, or (forced_group 0) the
 * narrowest group up to max_group that keeps 3/4 of the 32-lane kernel's
 * resident warps; per group the warps per block with the most resident
 * warps.  group 0: no shape fits. */
WcLaunch wc_plan(int algo, int start, bool second, int nlist, int max_q8, int max_t8, int forced_group,
                 int max_group);
/* global scratch words a launch of that shape needs */
size_t wc_scratch_words(int algo, const WcLaunch &l, int max_t8);

/* the global-scratch DP variant on a caller-chosen grid */
cudaError_t launch_dp_scratch_grid(int algo, int start, bool second, const DpArgs &a, int block, int blocks,
                                   cudaStream_t s);

/* warp-per-pair ksw extension (ksw_wc.cu) for the pairs listed in `list`
 * (null: pairs 0..nlist-1; a.n_dev, if set, caps the count on the device).
 * One launch per length class (wq[0], wq[1]: zeroed work counters); pairs
 * it cannot take (query above 8190 bases, seed + match*qlen >= 2^15) are
 * appended to fb, counted in *fbn, for the one-pair-per-thread kernel.
 * Needs gap_extend >= 0, gap_open + gap_extend >= 0 and every score below
 * 4096 in magnitude (ksw_wc_scores_ok). */
bool ksw_wc_scores_ok(const Scores &sc);
/* Shared-memory slots of the (up to two) length classes of warp launches for
 * these query lengths: class 0 takes queries up to 2046 bases, class 1 up to
 * 8190 (0 = no such pairs). */
void ksw_wc_classes(const uint32_t *h_q_len, int n, int slots[2]);
/* split: -2 no lane-group launch; -1 a lane-group launch over the whole list
 * for queries of at most 248 bases (31 words), the class launches skipping
 * them; >= 0 the list is length-ordered and its short pairs are exactly
 * list[split, nlist): lane groups take those, the class launches the prefix.
 * gq: the lane-group launch's zeroed work counter. */
cudaError_t launch_ksw_wc(const DpArgs &a, const uint32_t *list, int nlist, const int slots[2], uint32_t *fb,
                          uint32_t *fbn, uint32_t *wq, unsigned long long *cells, cudaStream_t s, int split = -2,
                          uint32_t *gq = nullptr);
/* pairs with at most 31 query words (the lane-group launch's) */
int ksw_grp_short(const uint32_t *h_q_len, int n);
/* The same with a band: pair p is computed within half-width band_w[p]
 * (negative: unbanded) and kept only if the band certificate proves it equal
 * to the unbanded result; otherwise nothing is written and p goes to retry
 * (count *nretry).  cells (optional) accumulates the computed cells. */
cudaError_t launch_ksw_band(const DpArgs &a, const uint32_t *list, int nlist, const int slots[2],
                            const int32_t *band_w, uint32_t *fb, uint32_t *fbn, uint32_t *retry, uint32_t *nretry,
                            unsigned long long *cells, uint32_t *wq, cudaStream_t s);

int dp_scratch_blocks(int n, int block);

} // namespace gb

#endif
