/*
 * gasal_header.h -- the single include for GASAL2 callers (drop-in for
 * reference src/gasal_header.h).  Link with -lgasal_b200 -lcudart.
 */
#ifndef GASAL_B200_GASAL_HEADER_H
#define GASAL_B200_GASAL_HEADER_H

#include "gasal.h"
#include "args_parser.h"
#include "gasal_align.h"
#include "host_batch.h"
#include "ctors.h"
#include "interfaces.h"

#endif
