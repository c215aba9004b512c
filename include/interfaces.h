/*
 * interfaces.h -- per-alignment host arrays and device selection (drop-in).
 * Replaces reference src/interfaces.h:9-14.
 */
#ifndef GASAL_B200_INTERFACES_H
#define GASAL_B200_INTERFACES_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "gasal.h"
class Parameters;

void gasal_host_alns_resize(gasal_gpu_storage_t *gpu_storage, int new_max_alns, Parameters *params);
void gasal_op_fill(gasal_gpu_storage_t *gpu_storage_t, uint8_t *data, uint32_t nbr_seqs_in_stream, data_source SRC);
void gasal_set_device(int gpu_select = 0, bool isPrintingProp = true);

#endif
