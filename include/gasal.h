/*
 * gasal.h -- public types of the B200 GASAL2-compatible alignment library.
 *
 * Drop-in replacement for GASAL2's src/gasal.h.  Every enum value, struct
 * member, member order and type below is part of the binary interface that
 * existing GASAL2 callers (bwa-gasal2, test_prog, ...) compile against, so the
 * layouts are kept identical to the reference:
 *   enums          reference src/gasal.h:37-72
 *   host_batch_t   reference src/gasal.h:75-83
 *   gasal_res_t    reference src/gasal.h:86-95
 *   storage        reference src/gasal.h:98-150
 *   storage vector reference src/gasal.h:153-156
 *   scores         reference src/gasal.h:160-165
 * The reference hard-codes an absolute path to a CUDA 10.1 runtime header; this
 * header includes <cuda_runtime.h> from the toolkit search path instead.
 */
#ifndef GASAL_B200_GASAL_H
#define GASAL_B200_GASAL_H

#include <stdlib.h>
#include <stdint.h>
#include <stdio.h>
#include <cuda_runtime.h>

#ifndef HOST_MALLOC_SAFETY_FACTOR
#define HOST_MALLOC_SAFETY_FACTOR 5
#endif

/* Compile-time N code and query limit keep their GASAL2 meaning for callers
 * that build with -DN_CODE=... / -DMAX_QUERY_LEN=...; the library itself takes
 * both as run-time values (see gasal_b200_capi.h). */
#ifndef N_CODE
#define N_CODE 0x4E
#endif
#ifndef MAX_QUERY_LEN
#define MAX_QUERY_LEN 1024
#endif

/* Same contract as the reference macro: needs a `cudaError_t err` in scope,
 * prints the failing call and terminates the process. */
#define CHECKCUDAERROR(error)                                                        \
    do {                                                                             \
        err = (error);                                                               \
        if (cudaSuccess != err) {                                                    \
            fprintf(stderr, "[GASAL CUDA ERROR:] %s(CUDA error no.=%d). Line no. %d " \
                            "in file %s\n",                                          \
                    cudaGetErrorString(err), err, __LINE__, __FILE__);               \
            exit(EXIT_FAILURE);                                                      \
        }                                                                            \
    } while (0)

static inline int CudaCheckKernelLaunch(void)
{
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/* Which positions an alignment reports. */
enum comp_start {
    WITHOUT_START,
    WITH_START,
    WITH_TB
};

/* Integer-valued boolean (used as a template tag in the reference). */
enum Bool {
    FALSE,
    TRUE
};

/* Which sequence of a pair a call refers to; also the semi-global
 * "skip head / skip tail" selector. */
enum data_source {
    NONE,
    QUERY,
    TARGET,
    BOTH
};

enum algo_type {
    UNKNOWN,
    GLOBAL,
    SEMI_GLOBAL,
    LOCAL,
    MICROLOCAL,
    BANDED,
    KSW
};

/* Per-sequence transformation applied on the GPU before alignment:
 * bit 0 = reverse, bit 1 = complement. */
enum operation_on_seq {
    FORWARD_NATURAL,
    REVERSE_NATURAL,
    FORWARD_COMPLEMENT,
    REVERSE_COMPLEMENT,
};

/* One page of the chained, pinned host staging buffer. */
struct host_batch {
    uint8_t *data;
    uint32_t page_size;
    uint32_t data_size;
    uint32_t offset;
    int is_locked;
    struct host_batch *next;
};
typedef struct host_batch host_batch_t;

/* Structure-of-arrays alignment results (host or device instance). */
struct gasal_res {
    int32_t *aln_score;
    int32_t *query_batch_end;
    int32_t *target_batch_end;
    int32_t *query_batch_start;
    int32_t *target_batch_start;
    uint8_t *cigar;
    uint32_t *n_cigar_ops;
};
typedef struct gasal_res gasal_res_t;

/* Everything one stream of work owns. */
typedef struct {
    uint8_t *unpacked_query_batch;
    uint8_t *unpacked_target_batch;
    uint32_t *packed_query_batch;
    uint32_t *packed_target_batch;
    uint32_t *query_batch_offsets;
    uint32_t *target_batch_offsets;
    uint32_t *query_batch_lens;
    uint32_t *target_batch_lens;

    uint32_t *host_seed_scores;
    uint32_t *seed_scores;

    host_batch_t *extensible_host_unpacked_query_batch;
    host_batch_t *extensible_host_unpacked_target_batch;

    uint8_t *host_query_op;
    uint8_t *host_target_op;
    uint8_t *query_op;
    uint8_t *target_op;

    uint32_t *host_query_batch_offsets;
    uint32_t *host_target_batch_offsets;
    uint32_t *host_query_batch_lens;
    uint32_t *host_target_batch_lens;

    gasal_res_t *host_res;   /* host struct, host arrays */
    gasal_res_t *device_cpy; /* host struct, device arrays */
    gasal_res_t *device_res; /* device struct, device arrays */

    gasal_res_t *host_res_second;
    gasal_res_t *device_res_second;
    gasal_res_t *device_cpy_second;

    uint32_t gpu_max_query_batch_bytes;
    uint32_t gpu_max_target_batch_bytes;

    uint32_t host_max_query_batch_bytes;
    uint32_t host_max_target_batch_bytes;

    uint32_t gpu_max_n_alns;
    uint32_t host_max_n_alns;
    uint32_t current_n_alns;

    uint64_t packed_tb_matrix_size;
    uint4 *packed_tb_matrices;

    cudaStream_t str;
    int is_free;
    int id;
} gasal_gpu_storage_t;

typedef struct {
    int n;
    gasal_gpu_storage_t *a;
} gasal_gpu_storage_v;

typedef struct {
    int32_t match;
    int32_t mismatch;
    int32_t gap_open;
    int32_t gap_extend;
} gasal_subst_scores;

#endif /* GASAL_B200_GASAL_H */
