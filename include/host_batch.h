/*
 * host_batch.h -- chained pinned host staging pages (drop-in).
 * Replaces reference src/host_batch.h:9-17.
 */
#ifndef GASAL_B200_HOST_BATCH_H
#define GASAL_B200_HOST_BATCH_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "gasal.h"

host_batch_t *gasal_host_batch_new(uint32_t batch_bytes, uint32_t offset);
void gasal_host_batch_destroy(host_batch_t *res);
host_batch_t *gasal_host_batch_getlast(host_batch_t *arg);
void gasal_host_batch_reset(gasal_gpu_storage_t *gpu_storage);
/* Appends a sequence at byte index idx, N-pads it to a multiple of 8 and
 * returns the next free index (src/host_batch.cpp:79-153). */
uint32_t gasal_host_batch_fill(gasal_gpu_storage_t *gpu_storage, uint32_t idx, const char *data, uint32_t size,
                               data_source SRC);
/* Appends without padding (src/host_batch.cpp:156-223). */
uint32_t gasal_host_batch_add(gasal_gpu_storage_t *gpu_storage, uint32_t idx, const char *data, uint32_t size,
                              data_source SRC);
uint32_t gasal_host_batch_addbase(gasal_gpu_storage_t *gpu_storage, uint32_t idx, const char base,
                                  data_source SRC);
/* Extension (no reference counterpart): gasal_host_batch_fill with the copy
 * split over `threads` host threads (0 = all), for a whole padded batch staged
 * as one block. */
uint32_t gasal_host_batch_fill_mt(gasal_gpu_storage_t *gpu_storage, uint32_t idx, const char *data, uint32_t size,
                                  data_source SRC, int threads);
void gasal_host_batch_print(host_batch_t *res);
void gasal_host_batch_printall(host_batch_t *res);

#endif
