/*
 * res.h -- result array allocation (drop-in).  Replaces reference
 * src/res.h:4-9; which arrays exist follows src/res.cpp:8-70 (NULL start/end
 * arrays for GLOBAL, start arrays only for WITH_START / WITH_TB, n_cigar_ops
 * only for WITH_TB).
 */
#ifndef GASAL_B200_RES_H
#define GASAL_B200_RES_H

#include "gasal.h"
class Parameters;

gasal_res_t *gasal_res_new_host(uint32_t max_n_alns, Parameters *params);
gasal_res_t *gasal_res_new_device(gasal_res_t *device_cpy);
gasal_res_t *gasal_res_new_device_cpy(uint32_t max_n_alns, Parameters *params);
void gasal_res_destroy_host(gasal_res_t *res);
void gasal_res_destroy_device(gasal_res_t *device_res, gasal_res_t *device_cpy);

#endif
