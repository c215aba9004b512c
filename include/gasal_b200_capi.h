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
    int32_t zdrop;        /* ksw z-drop; 0 = off, as the reference hard-codes */
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

#ifdef __cplusplus
}
#endif

#endif /* GASAL_B200_CAPI_H */
