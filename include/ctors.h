/*
 * ctors.h -- stream storage construction and teardown (drop-in).
 * Replaces reference src/ctors.h:5-15.
 */
#ifndef GASAL_B200_CTORS_H
#define GASAL_B200_CTORS_H

#include "gasal.h"
class Parameters;

gasal_gpu_storage_v gasal_init_gpu_storage_v(int n_streams);
void gasal_init_streams(gasal_gpu_storage_v *gpu_storage_vec, int max_query_len, int max_target_len,
                        int max_n_alns, Parameters *params);
void gasal_gpu_mem_alloc(gasal_gpu_storage_t *gpu_storage, int gpu_max_query_batch_bytes,
                         int gpu_max_target_batch_bytes, int gpu_max_n_alns, Parameters *params);
void gasal_gpu_mem_free(gasal_gpu_storage_t *gpu_storage, Parameters *params);
void gasal_destroy_streams(gasal_gpu_storage_v *gpu_storage_vec, Parameters *params);
void gasal_destroy_gpu_storage_v(gasal_gpu_storage_v *gpu_storage_vec);

#endif
