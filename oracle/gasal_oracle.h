/*
 * gasal_oracle.h -- scalar C restatement of GASAL2's alignment path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against and the timed CPU baseline; the product never links it.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks every function here
 * against the reference GASAL2 library compiled for sm_100a and run on a
 * B200 (the .npz fixtures in tests/golden, made by tests/golden/make_golden.py), and against
 * the reference kernel headers compiled for the host.
 *
 * Every reference quirk is reproduced by default.  The quirk switches below
 * (bits of `compat`) turn individual ones off, for experiments only; with any
 * of them off the results no longer match the reference.
 */
#ifndef GASAL_ORACLE_H
#define GASAL_ORACLE_H

#include "../include/gasal_b200_capi.h"

#ifdef __cplusplus
extern "C" {
#endif

enum oracle_compat {
    /* K2: reverse a sequence the way the sm_100a build of
     * src/kernels/pack_rc_seqs.h:259-316 does (undefined 32-bit shifts; see
     * oracle_revcomp); off = reverse only the real bases. */
    ORC_RC_REF_REVERSE = 1 << 0,
    /* H and E crossing an 8-row tile boundary are stored as int16
     * (short2 row buffers, e.g. local_kernel_template.h:102,112,152-154). */
    ORC_INT16_ROWS = 1 << 1,
    /* local start pass records target row gidx+(m-1) while gidx counts down
     * (local_kernel_template.h:41,468,476). */
    ORC_LOCAL_START_ROW = 1 << 2,
    /* ksw: "m == 0" and z-drop leave only the current 8-row target tile
     * (ksw_kernel_template.h:89-185); off = stop the extension. */
    ORC_KSW_TILE_BREAK = 1 << 3,
    ORC_ALL = 0x0F
};

/* Runs one batch.  `compat` = ORC_ALL for reference behaviour; `threads` = 0
 * uses every OpenMP thread.  `mql` is the reference's compile-time
 * MAX_QUERY_LEN, which bounds the semi-global last-row scan
 * (semiglobal_kernel_template.h:187,364); pass 0 for 2048. */
int oracle_align_ex(const gb_params_t *p, const gb_batch_t *b, gb_out_t *o, int threads, int compat, int mql);
int oracle_align(const gb_params_t *p, const gb_batch_t *b, gb_out_t *o, int threads, int compat);

/* The two preprocessing kernels on their own (for unit tests). */
void oracle_pack(const uint8_t *ascii, uint32_t nbytes, uint32_t *words);
void oracle_revcomp(uint32_t *words, uint32_t word_off, uint32_t len, int op, int compat);

/* Forward CIGAR text of every pair from the run-length bytes the traceback
 * wrote (count << 2 | op, last operation first, at each pair's query offset),
 * as the reference's test program prints it (test_prog/test_prog.cpp:382-428):
 * bytes read from last to first, neighbouring runs of one operation merged,
 * each run printed as its count and M / X / D / I.  Pair i's text goes to
 * text + i * stride, NUL-terminated; text_len[i] = its length, or -1 when
 * it needs more than stride - 1 characters.  A pair without operations gets
 * "" (the reference's loop would read the byte before the pair's slot). */
void oracle_cigar_text(const uint8_t *cigar, const uint32_t *q_off, const uint32_t *n_cigar, int n, char *text,
                       int stride, int32_t *text_len);

#ifdef __cplusplus
}
#endif

#endif
