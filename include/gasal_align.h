/*
 * gasal_align.h -- launch and completion of one alignment batch (drop-in).
 * Replaces reference src/gasal_align.h:114-120.
 */
#ifndef GASAL_B200_GASAL_ALIGN_H
#define GASAL_B200_GASAL_ALIGN_H

#include "gasal.h"
class Parameters;

/* Scores shared by every stream of the process (src/gasal_align.cu:329-339). */
void gasal_copy_subst_scores(gasal_subst_scores *subst);

/* Queues copy-in, pack, reverse/complement, alignment, traceback and copy-out
 * of one batch on gpu_storage->str and returns without waiting
 * (src/gasal_align.cu:29-307). */
void gasal_aln_async(gasal_gpu_storage_t *gpu_storage, const uint32_t actual_query_batch_bytes,
                     const uint32_t actual_target_batch_bytes, const uint32_t actual_n_alns, Parameters *params);

/* 0 when the batch finished (host batches reset, results readable), -1 while
 * it runs, -2 when nothing was launched (src/gasal_align.cu:310-326). */
int gasal_is_aln_async_done(gasal_gpu_storage_t *gpu_storage);

#endif
