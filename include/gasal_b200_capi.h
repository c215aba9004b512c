/*
 * gasal_b200_capi.h -- plain C ABI of the B200 GASAL2-compatible library.
 *
 * GASAL2's own interface is C++ (reference src/ctors.h:5-15,
 * src/host_batch.h:9-17, src/interfaces.h:9-14, src/gasal_align.h:114-120) and
 * is reproduced with the same signatures in gasal_header.h.  This header is the
 * extern "C" face of the same library: every entry point takes plain pointers
 * and sizes, so FFI callers (ctypes, cgo, JNI, N-API) can bind it without a C++
 * compiler.  Each declaration names the reference interface it stands in for.
 *
 * All functions return 0 on success and a negative gb_status value on error;
 * none of them terminates the process (the C++ API keeps the reference's
 * print-and-exit behaviour).
 */
#ifndef GASAL_B200_CAPI_H
#define GASAL_B200_CAPI_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
enum gb_status {
    GB_OK = 0,
    GB_ERR_ARG = -1,       /* bad size, NULL pointer, unsupported option */
    GB_ERR_CUDA = -2,      /* a CUDA runtime call failed */
    GB_ERR_NOT_READY = -3, /* work still in flight */
    GB_ERR_NO_WORK = -4,   /* nothing was launched on this stream */
    GB_ERR_ALLOC = -5,     /* device or pinned allocation failed */
    GB_ERR_LIMIT = -6      /* a size is beyond a documented limit */
};

/* ---- per-launch options: the fields of GASAL2's Parameters that the
 *      alignment path reads (reference src/args_parser.h:37-53) ------------- */
typedef struct {
    int32_t algo;         /* enum algo_type: GLOBAL, SEMI_GLOBAL, LOCAL, BANDED, KSW */
    int32_t start_pos;    /* enum comp_start: WITHOUT_START, WITH_START, WITH_TB */
    int32_t second_best;  /* enum Bool */
    int32_t head;         /* enum data_source: semi-global skipped head */
    int32_t tail;         /* enum data_source: semi-global skipped tail */
    int32_t k_band;       /* banded: band width in bases (tiles = k_band >> 3) */
    int32_t reverse_complement; /* apply per-sequence ops (isReverseComplement) */
    int32_t zdrop;        /* ksw z-drop; 0 = off, as the reference hard-codes.  Honoured by every C entry
                             point (gasal_c_aln_async takes it from gasal_c_params_set); the
                             C++ gasal_aln_async keeps the reference's 0 */
    int32_t match;        /* gasal_subst_scores (reference src/gasal.h:160-165) */
    int32_t mismatch;
    int32_t gap_open;
    int32_t gap_extend;
} gb_params_t;

/* ---- one batch of pairs, laid out exactly as GASAL2 stages it: ASCII bases,
 *      each sequence starting at its byte offset and N-padded to a multiple of
 *      8 (reference src/host_batch.cpp:100-146). --------------------------- */
typedef struct {
    int32_t n;                 /* number of pairs */
    uint32_t q_bytes;          /* total query bytes (multiple of 8) */
    uint32_t t_bytes;          /* total target bytes (multiple of 8) */
    const uint8_t *q;          /* query bytes  [q_bytes] */
    const uint8_t *t;          /* target bytes [t_bytes] */
    const uint32_t *q_off;     /* byte offset of each query  [n] */
    const uint32_t *t_off;     /* byte offset of each target [n] */
    const uint32_t *q_len;     /* unpadded query length  [n] */
    const uint32_t *t_len;     /* unpadded target length [n] */
    const uint8_t *q_op;       /* enum operation_on_seq per query, or NULL */
    const uint8_t *t_op;       /* per target, or NULL */
    const uint32_t *seed;      /* ksw seed score h0 per pair, or NULL */
} gb_batch_t;

/* ---- results, structure of arrays (reference gasal_res_t, src/gasal.h:86-95).
 *      Any pointer may be NULL when the caller does not want that array. ---- */
typedef struct {
    int32_t *score;
    int32_t *q_end;
    int32_t *t_end;
    int32_t *q_start;
    int32_t *t_start;
    int32_t *score2;    /* second best (host_res_second) */
    int32_t *q_end2;
    int32_t *t_end2;
    uint8_t *cigar;     /* [q_bytes]: run-length CIGAR bytes at each query offset */
    uint32_t *n_cigar;  /* [n] */
    uint32_t *packed_q; /* [q_bytes/8] optional dump of packed words after pack+rc */
    uint32_t *packed_t; /* [t_bytes/8] */
} gb_out_t;

/* ---- device-resident batch (kernel-level entry point) ------------------- */
typedef struct {
    int32_t n;
    uint32_t q_bytes, t_bytes;
    const uint8_t *q, *t;          /* device: ASCII batches */
    uint32_t *pq, *pt;             /* device: packed words out [q_bytes/8], [t_bytes/8] */
    const uint32_t *q_off, *t_off; /* device */
    const uint32_t *q_len, *t_len; /* device */
    const uint8_t *q_op, *t_op;    /* device or NULL */
    const uint32_t *seed;          /* device or NULL */
    const uint32_t *h_q_len, *h_t_len; /* host copies of the lengths (launch planning) */
} gb_dev_batch_t;

typedef struct {
    int32_t *score, *q_end, *t_end, *q_start, *t_start, *score2, *q_end2, *t_end2; /* device or NULL */
    uint8_t *cigar;     /* device [q_bytes] (may be the ASCII query batch, as GASAL2 does) */
    uint32_t *n_cigar;  /* device [n] */
} gb_dev_out_t;

/* ---- host-side arrays of one stream storage, for callers that cannot read
 *      gasal_gpu_storage_t directly (the C++ API exposes them as members) --- */
typedef struct {
    uint32_t *host_query_batch_offsets, *host_target_batch_offsets;
    uint32_t *host_query_batch_lens, *host_target_batch_lens;
    uint8_t *host_query_op, *host_target_op;
    uint32_t *host_seed_scores;
    int32_t *aln_score, *query_batch_end, *target_batch_end, *query_batch_start, *target_batch_start;
    uint8_t *cigar;
    uint32_t *n_cigar_ops;
    int32_t *aln_score2, *query_batch_end2, *target_batch_end2;
    void *stream;                  /* cudaStream_t of the storage */
    uint32_t host_max_n_alns, host_max_query_batch_bytes, host_max_target_batch_bytes;
} gb_storage_view_t;

/* ==== entry points ======================================================== */
/* Each gasal_c_* function is the C-linkage twin of the GASAL2 C++ function
 * named in its comment, with the same meaning; where the reference prints and
 * exits, these return a gb_status instead. */

/* Parameters object (reference src/args_parser.h:24-68): opaque handle. */
void *gasal_c_params_new(void);
int gasal_c_params_set(void *params, const gb_params_t *p);
void gasal_c_params_free(void *params);

/* gasal_copy_subst_scores, reference src/gasal_align.cu:329 (scores are
 * process-wide).  Takes match, mismatch, gap_open, gap_extend. */
int gasal_c_copy_subst_scores(int32_t match, int32_t mismatch, int32_t gap_open, int32_t gap_extend);

/* gasal_init_gpu_storage_v / gasal_init_streams / gasal_destroy_streams /
 * gasal_destroy_gpu_storage_v, reference src/ctors.h:5-15.  The storage
 * vector is returned as an opaque handle; gasal_c_storage() gives element i. */
void *gasal_c_init_gpu_storage_v(int n_streams);
int gasal_c_init_streams(void *storage_v, int max_query_len, int max_target_len, int max_n_alns, void *params);
int gasal_c_destroy_streams(void *storage_v, void *params);
int gasal_c_destroy_gpu_storage_v(void *storage_v);
void *gasal_c_storage(void *storage_v, int i);
int gasal_c_storage_view(void *storage, gb_storage_view_t *view);

/* gasal_host_batch_fill / _add / _reset, reference src/host_batch.h:9-17.
 * src: 1 = QUERY, 2 = TARGET.  Returns the next free byte index. */
uint32_t gasal_c_host_batch_fill(void *storage, uint32_t idx, const char *data, uint32_t size, int src);
uint32_t gasal_c_host_batch_add(void *storage, uint32_t idx, const char *data, uint32_t size, int src);
int gasal_c_host_batch_reset(void *storage);
/* Extension: gasal_host_batch_fill with the copy split over `threads` host
 * threads (0 = every hardware thread); same page, padding and return value. */
uint32_t gasal_c_host_batch_fill_mt(void *storage, uint32_t idx, const char *data, uint32_t size, int src,
                                    int threads);

/* gasal_op_fill / gasal_host_alns_resize / gasal_set_device, reference
 * src/interfaces.h:9-14. */
int gasal_c_op_fill(void *storage, const uint8_t *ops, uint32_t n, int src);
int gasal_c_host_alns_resize(void *storage, int new_max_alns, void *params);
int gasal_c_set_device(int gpu);

/* gasal_aln_async / gasal_is_aln_async_done, reference
 * src/gasal_align.h:116-120.  aln_async returns a gb_status; is_done returns
 * 0 (done), -1 (running), -2 (nothing launched) or GB_ERR_CUDA. */
int gasal_c_aln_async(void *storage, uint32_t query_batch_bytes, uint32_t target_batch_bytes, uint32_t n_alns,
                      void *params);
int gasal_c_is_aln_async_done(void *storage);

/* One-shot convenience over the calls above: copies the batch from host
 * memory, aligns, and fills every non-NULL output array (synchronous).  No
 * reference counterpart; it is the sequence test_prog.cpp:264-437 performs. */
int gb_align(const gb_params_t *p, const gb_batch_t *b, gb_out_t *o);

/* Kernel-level entry point: pack -> reverse/complement -> alignment ->
 * traceback on inputs already in device memory, queued on `stream`
 * (a cudaStream_t, NULL = legacy default stream).  Uses a workspace per
 * (device, stream) that the library grows on demand; calls on one stream must
 * come from one host thread at a time.  The device half of gasal_aln_async
 * (src/gasal_align.cu:180-264).  n == 0 returns GB_OK and launches nothing. */
int gb_align_dev(const gb_params_t *p, const gb_dev_batch_t *b, const gb_dev_out_t *o, void *stream);

/* The two preparation kernels alone, on device buffers, queued on `stream`:
 * gb_pack_dev packs nbytes (a multiple of 8) of N-padded ASCII bases into
 * nbytes / 8 words of 4-bit codes (reference gasal_pack_kernel,
 * src/kernels/pack_rc_seqs.h:13-53); gb_revcomp_dev applies each sequence's
 * operation_on_seq (q_op / t_op may be NULL) to the packed words in place
 * (reference gasal_reversecomplement_kernel, src/kernels/pack_rc_seqs.h:
 * 56-212; gb_set_reference_reverse selects the reversal form).  Both are the
 * first steps of gb_align_dev. */
int gb_pack_dev(const uint8_t *ascii, uint32_t nbytes, uint32_t *packed, void *stream);
int gb_revcomp_dev(uint32_t *pq, uint32_t *pt, const uint32_t *q_off, const uint32_t *t_off, const uint32_t *q_len,
                   const uint32_t *t_len, const uint8_t *q_op, const uint8_t *t_op, int32_t n, void *stream);

/* Allocation-free variant of gb_align_dev, for callers that cannot call
 * cudaMalloc (inside stream capture, under a device-memory arena, or as a
 * plugin that must not allocate).  No counterpart in the reference.  The
 * caller passes every buffer (including pq/pt); the DP row buffers live in a
 * 32 MiB static device array that each GPU loading the library holds until
 * exit.  Rejects WITH_TB (GB_ERR_ARG) and batches whose longest query leaves
 * the array room for fewer than 32 threads (GB_ERR_LIMIT).  Calls share the
 * array, so calls that overlap on the GPU race.  The first call in a device's
 * context (again after a cudaDeviceReset) resolves the array's address and
 * should precede any stream capture.  n == 0 returns GB_OK and launches
 * nothing, as gb_align_dev does. */
int gb_align_dev_noalloc(const gb_params_t *p, const gb_dev_batch_t *b, const gb_dev_out_t *o, void *stream);

/* Frees the device and pinned buffers that gb_align_dev, gb_align_dev_mixed,
 * gb_autotune and the band entry points keep per (device, stream) between
 * calls (traceback tiles, row buffers, orders, streams, events), after waiting
 * for the current device to finish its work.  The next call grows them again.
 * Storages keep theirs until gasal_destroy_streams.  No reference
 * counterpart: GASAL2 allocates per storage only. */
int gb_release_workspaces(void);

/* Per-pair mixed-algorithm dispatch (an extension: GASAL2 takes one algorithm
 * per launch, Parameters::algo, reference src/gasal_align.cu:249 and
 * src/gasal_align.h:89-107).  Pair i of the device batch is aligned under
 * kinds[h_kind[i]] (h_kind: host array of b->n bytes, each < n_kinds <=
 * GB_MIXED_MAX_KINDS), with the same results gb_align_dev gives that pair
 * under those options.  The batch is packed once; each kind then runs on its
 * own stream, forked from `stream` and joined back before the call's last
 * operation, so the kinds overlap.  Result arrays a pair's kind does not
 * produce keep their values; CIGAR bytes land at each pair's query offset.
 * KSW kinds need b->seed.  n == 0 returns GB_OK and launches nothing.  Calls
 * on one stream must come from one host thread at a time. */
#define GB_MIXED_MAX_KINDS 8
int gb_align_dev_mixed(const gb_params_t *kinds, int n_kinds, const uint8_t *h_kind, const gb_dev_batch_t *b,
                       const gb_dev_out_t *o, void *stream);
/* The argument check of gb_align_dev_mixed alone (no CUDA call): GB_OK, with
 * the pairs of each kind in counts[0..n_kinds) when counts is not NULL, or
 * GB_ERR_ARG (kind index out of range, too many kinds, unknown algorithm, a
 * KSW kind with pairs but has_seed 0). */
int gb_mixed_check(const gb_params_t *kinds, int n_kinds, const uint8_t *h_kind, int32_t n, int has_seed,
                   uint32_t *counts);

/* Forward CIGAR text on the device (no counterpart in the reference
 * library; its test program decodes on the host, test_prog/test_prog.cpp:
 * 382-428).  Input: the traceback's run-length bytes (count << 2 | op, last
 * operation first) at each pair's query offset -- gb_dev_out_t::cigar /
 * n_cigar, or GASAL2's device CIGAR buffer -- all device pointers.  Pair i's
 * text (neighbouring runs of one operation merged, each run as its count and
 * M / X / D / I, NUL-terminated) goes to text + i * stride; text_len[i] is its
 * length, or -1 when it needs more than stride - 1 characters (the slot then
 * holds ""); a pair without operations gets "".  Asynchronous on `stream`. */
int gb_cigar_text(const uint8_t *cigar, const uint32_t *q_off, const uint32_t *n_cigar, int n, char *text, int stride,
                  int32_t *text_len, void *stream);

/* Library settings.
 * reference_reverse: 1 (default) reverses sequences exactly as the
 *   reference's sm_100a build does; 0 reverses the real bases only.
 * reference_max_query_len: the reference build's MAX_QUERY_LEN, which bounds
 *   the semi-global last-row scan (default 2048).
 * tb_budget_mb: device memory for traceback tiles per stream (default 98304,
 *   and never more than half of the device memory free when a batch is
 *   planned); larger WITH_TB batches run in chunks. */
int gb_set_reference_reverse(int on);
int gb_set_reference_max_query_len(int mql);
int gb_set_tb_budget_mb(int64_t mb);
const char *gb_version(void);

/* CUDA graphs for gasal_aln_async / gasal_c_aln_async (no reference
 * counterpart; on by default).  Each storage keeps one executable graph of
 * its whole batch (host->device copies, kernels, device->host copies): a batch
 * with the same sizes, options, buffers and plan relaunches it as is, any
 * other batch is captured and the graph updated in place.  Graphs are skipped
 * while gb_kernel_timing is on.  gb_graph_stats() fills counts[4]: batches
 * that relaunched a graph, that updated it, that instantiated a new one, and
 * whose capture was refused (those ran without a graph). */
int gb_set_graphs(int on);
int gb_graph_stats(int64_t *counts);

/* Launch tuning (no reference counterpart).  block: threads per block of the
 * one-pair-per-thread DP kernel (32, 64 or 128); wc_min_qregs: pairs
 * whose query has at least this many 8-base words run warp-cooperative
 * (LOCAL/GLOBAL/target-tail SEMI_GLOBAL; at least 8, and never fewer than
 * wc_group, which that kernel needs); min_order_pairs: batches with at least this many pairs are
 * visited length-binned.  Results never depend on these. */
typedef struct {
    int32_t block;
    int32_t wc_min_qregs;
    int32_t min_order_pairs;
    int32_t ksw_warp;      /* 1: ksw pairs run one warp per pair (default); 0: one thread per pair */
    int32_t split_start;   /* 1: LOCAL / SEMI_GLOBAL start passes run as their own launch, pairs re-ordered
                              by forward score (default); 0: in the forward launch */
    int32_t persistent;    /* 1: one-pair-per-thread launches are persistent, warps pulling pairs from a
                              device counter (default); 0: one thread per pair on a grid over the batch.
                              With min_order_pairs above the batch size, ksw_warp 0 and split_start 0
                              this is the plain full-DP form: every pair one per thread, in input order */
    int32_t wc_group;      /* lanes per pair in the warp-cooperative kernels: 64 (two warps per pair),
                              32, 16 or 8 (a warp sweeps 32/wc_group pairs side by side), or 0 (default):
                              per launch the narrowest group that keeps 3/4 of the 32-lane kernel's
                              resident warps, and two-warp groups for the launch of 127+ word queries.
                              Pairs go warp-cooperative from max(wc_min_qregs, wc_group) query words */
} gb_tuning_t;
int gb_set_tuning(const gb_tuning_t *t);
int gb_get_tuning(gb_tuning_t *t);

/* Autotuner (no reference counterpart): runs gb_align_dev on the caller's
 * batch under each candidate tuning (block 32/64/128; for LOCAL, GLOBAL and
 * target-tail SEMI_GLOBAL also warp-cooperative thresholds 16/32/48/64 words
 * x lane groups automatic/8/16/32, thresholds below the group skipped), `reps` timed runs each
 * after a warm-up run, timed with CUDA events on `stream`; installs and
 * returns the fastest (best_ms: its mean milliseconds per run; may be NULL).
 * The outputs hold the batch's results afterwards.  Synchronizes `stream`;
 * not for use during stream capture. */
int gb_autotune(const gb_params_t *p, const gb_dev_batch_t *b, const gb_dev_out_t *o, void *stream, int reps,
                gb_tuning_t *best, double *best_ms);
/* Text of the last CUDA failure the calling thread met in gb_autotune ("" if none). */
const char *gb_last_error(void);

/* Instrumentation (no reference counterpart).  gb_kernel_timing(1) resets
 * and starts recording a CUDA event pair around every kernel the library
 * launches; gb_kernel_timing_read() waits for them and returns, per kind
 * (0 pack, 1 reverse/complement, 2 alignment DP, 3 traceback, 4 length-binned
 * ordering = 3 kernels per mark, 5 the alignment phase's wall clock on the
 * launch stream: ordering through DP -- auxiliary-stream kernels joined back --
 * and traceback, one mark per batch), the summed milliseconds and the number
 * of marks, in arrays of 6.  gb_probe_int_peak() times the
 * integer instructions the DP is bound by on the current GPU (tera-ops/s). */
/* ---- Learned ksw band (no reference counterpart) ----
 * A small MLP (67 pair features -> 64 -> 64 -> 1, ReLU, BF16 inference,
 * FP32 training) predicts a log2 band half-width per ksw pair.  The banded
 * warp kernel keeps a pair's result only when its certificate proves it equal
 * to the unbanded one; the rest are recomputed without a band, so results
 * never depend on the model.  Features (gb_band_features): n x
 * gb_band_feature_stride() device floats: qlen/1024, tlen/1024,
 * (tlen-qlen)/128, then a 64-bin histogram of the diagonal offsets of shared
 * 11-mers.  Parameters: gb_band_param_count() floats, layout W1[64][67],
 * b1[64], W2[64][64], b2[64], W3[64], b3. */
typedef struct gb_band_model gb_band_model_t;
typedef struct {
    int64_t pairs;        /* pairs in the batch */
    int64_t accepted;     /* banded results the certificate kept */
    int64_t retried;      /* refused, recomputed without a band */
    int64_t handed_back;  /* outside the warp kernel's range, one-thread kernel */
    int64_t cells;        /* computed cells, banded attempts and recomputations included */
} gb_band_stats_t;
int gb_band_param_count(void);
int gb_band_feature_stride(void);
gb_band_model_t *gb_band_model_new(uint64_t seed);
void gb_band_model_free(gb_band_model_t *m);
/* copy parameters out (out) and/or in (in); either may be NULL */
int gb_band_model_params(gb_band_model_t *m, float *out, const float *in);
/* packs b->q/b->t (when given) into b->pq/b->pt, then writes the features */
int gb_band_features(const gb_dev_batch_t *b, float *feat, void *stream);
int gb_band_predict(gb_band_model_t *m, const float *feat, int n, float *out, void *stream);
/* gradient of the mean pinball loss (quantile tau) of prediction vs label
 * into grad (gb_band_param_count() device floats), summed loss into *loss
 * (one device float) */
int gb_band_grad(gb_band_model_t *m, const float *feat, const float *label, int n, float tau, float *grad, float *loss,
                 void *stream);
/* one Adam step on a batch; loss (host, may be NULL; syncs) = mean loss */
int gb_band_train_step(gb_band_model_t *m, const float *feat, const float *label, int n, float tau, float lr,
                       void *stream, float *loss);
/* install (or with NULL remove) the model for every ksw call; predicted
 * widths are clamped to [band_min, band_max] */
int gb_set_band_model(gb_band_model_t *m, int band_min, int band_max);
/* Unbanded ksw with max_off (device int32 per pair): the largest
 * |column - row| over the cells where the running maximum rose, as
 * ksw_extend2 tracks it -- the diagonal reach the alignment needed, from
 * which band labels are made. */
int gb_ksw_align_max_off(const gb_params_t *p, const gb_dev_batch_t *b, const gb_dev_out_t *o, int32_t *max_off,
                         void *stream);
/* ksw with a band: band_w (device int32 per pair, negative = none) or, when
 * NULL, the installed model's prediction.  band_ok (device, optional): 1 where
 * the banded result was kept.  stats (optional) syncs the stream. */
int gb_ksw_band_align(const gb_params_t *p, const gb_dev_batch_t *b, const gb_dev_out_t *o, const int32_t *band_w,
                      uint8_t *band_ok, void *stream, gb_band_stats_t *stats);

int gb_kernel_timing(int on);
int gb_kernel_timing_read(double *ms, int64_t *launches);
int gb_probe_int_peak(double *iadd_tops, double *imnmx_tops, double *dpx_tops);
/* The int16x2 form of the add-then-max (__viaddmax_s16x2) timed the same way,
 * in halfword results per second (two per instruction), tera. */
int gb_probe_dpx16x2_peak(double *halfword_tops);

#ifdef __cplusplus
}
#endif

#endif /* GASAL_B200_CAPI_H */
