/*
 * ref_gpu_driver.cpp -- drives the UNMODIFIED reference GASAL2 library (built
 * for sm_100a from the reference sources by oracle/Makefile) through its own
 * public C++ API, for one batch described by the plain C structs of
 * gasal_b200_capi.h.
 *
 * TEST INFRASTRUCTURE ONLY (oracle "A"): produces reference outputs on the GPU
 * box for golden fixtures and for the reference-GPU timing beside the bench.
 * Never linked into the product.
 *
 * The call sequence is the one the reference's example driver uses
 * (test_prog/test_prog.cpp:202-437): gasal_copy_subst_scores ->
 * gasal_init_gpu_storage_v -> gasal_init_streams -> gasal_host_batch_fill per
 * sequence -> gasal_op_fill -> gasal_aln_async -> poll gasal_is_aln_async_done
 * -> read host_res / host_res_second -> gasal_destroy_streams.
 */
#include "gasal_header.h"   /* reference src/gasal_header.h */
#include "../include/gasal_b200_capi.h"

#include <chrono>
#include <cstring>
#include <vector>

static uint32_t round8(uint32_t x) { return (x + 7u) & ~7u; }

extern "C" int ref_gpu_align(const gb_params_t *p, const gb_batch_t *b, gb_out_t *o,
                             int repeats, double *ms_per_call)
{
    if (!p || !b || !o || b->n <= 0) return GB_ERR_ARG;
    cudaError_t err;
    const int n = b->n;

    gasal_subst_scores sc;
    sc.match = p->match;
    sc.mismatch = p->mismatch;
    sc.gap_open = p->gap_open;
    sc.gap_extend = p->gap_extend;
    gasal_copy_subst_scores(&sc);

    Parameters *params = new Parameters(0, NULL);
    params->algo = (algo_type)p->algo;
    params->start_pos = (comp_start)p->start_pos;
    params->secondBest = (Bool)p->second_best;
    params->semiglobal_skipping_head = (data_source)p->head;
    params->semiglobal_skipping_tail = (data_source)p->tail;
    params->k_band = p->k_band;
    params->isReverseComplement = p->reverse_complement != 0;
    params->isPacked = false;
    params->sa = p->match;
    params->sb = p->mismatch;
    params->gapo = p->gap_open;
    params->gape = p->gap_extend;

    uint32_t max_q = 8, max_t = 8;
    for (int i = 0; i < n; i++) {
        if (round8(b->q_len[i]) > max_q) max_q = round8(b->q_len[i]);
        if (round8(b->t_len[i]) > max_t) max_t = round8(b->t_len[i]);
    }
    /* Two spare pairs of slack: the reference's traceback kernel may write a
     * CIGAR longer than the padded query past the last pair's slot. */
    const int max_n = n + 2;

    /* The reference's GLOBAL traceback starts one past the last cell
     * (src/kernels/get_tb.h:21-23,50-57), which for lengths that are multiples
     * of 8 addresses a traceback tile row beyond the pair's matrix; 16 spare
     * target rows keep that read inside the allocation. */
    const uint32_t alloc_t = p->start_pos == WITH_TB ? max_t + 16 : max_t;

    gasal_gpu_storage_v v = gasal_init_gpu_storage_v(1);
    gasal_init_streams(&v, (int)max_q, (int)alloc_t, max_n, params);
    gasal_gpu_storage_t *st = &v.a[0];
    /* Tiles the kernels never write read as zero, i.e. as on a fresh
     * allocation, so results that depend on them are reproducible. */
    if (st->packed_tb_matrices)
        CHECKCUDAERROR(cudaMemset(st->packed_tb_matrices, 0, st->packed_tb_matrix_size * sizeof(uint4)));
    /* The reference allocates result structs with malloc and leaves the cigar /
     * n_cigar_ops members unset unless WITH_TB (src/res.cpp:8-66,106-140), yet
     * its destructors free them when non-NULL (src/res.cpp:150-177,
     * src/ctors.cpp:165).  Clear them here so teardown frees only what exists. */
    gasal_res_t *rs[4] = {st->host_res, st->device_cpy, st->host_res_second, st->device_cpy_second};
    for (int k = 0; k < 4; k++) {
        if (!rs[k]) continue;
        const bool host_side = (k == 0 || k == 2);
        if (!(k == 0 && p->start_pos == WITH_TB)) rs[k]->cigar = NULL;
        if (!(host_side && p->start_pos == WITH_TB)) rs[k]->n_cigar_ops = NULL;
    }

    double total_ms = 0.0;
    if (repeats < 1) repeats = 1;
    for (int rep = 0; rep < repeats; rep++) {
        uint32_t qi = 0, ti = 0;
        for (int i = 0; i < n; i++) {
            st->host_query_batch_offsets[i] = qi;
            st->host_target_batch_offsets[i] = ti;
            qi = gasal_host_batch_fill(st, qi, (const char *)(b->q + b->q_off[i]), b->q_len[i], QUERY);
            ti = gasal_host_batch_fill(st, ti, (const char *)(b->t + b->t_off[i]), b->t_len[i], TARGET);
            st->host_query_batch_lens[i] = b->q_len[i];
            st->host_target_batch_lens[i] = b->t_len[i];
        }
        std::vector<uint8_t> zeros(n, 0);
        gasal_op_fill(st, b->q_op ? (uint8_t *)b->q_op : zeros.data(), n, QUERY);
        gasal_op_fill(st, b->t_op ? (uint8_t *)b->t_op : zeros.data(), n, TARGET);
        if (p->algo == KSW) {
            for (int i = 0; i < n; i++) st->host_seed_scores[i] = b->seed ? b->seed[i] : 0u;
        }
        st->current_n_alns = n;

        auto t0 = std::chrono::steady_clock::now();
        gasal_aln_async(st, qi, ti, n, params);
        int rc;
        while ((rc = gasal_is_aln_async_done(st)) != 0) {
            if (rc == -2) break;
        }
        auto t1 = std::chrono::steady_clock::now();
        total_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();

        if (rep == repeats - 1) {
            gasal_res_t *r = st->host_res;
            if (o->score && r->aln_score) memcpy(o->score, r->aln_score, n * 4);
            if (o->q_end && r->query_batch_end) memcpy(o->q_end, r->query_batch_end, n * 4);
            if (o->t_end && r->target_batch_end) memcpy(o->t_end, r->target_batch_end, n * 4);
            if (p->start_pos != WITHOUT_START) {
                if (o->q_start && r->query_batch_start) memcpy(o->q_start, r->query_batch_start, n * 4);
                if (o->t_start && r->target_batch_start) memcpy(o->t_start, r->target_batch_start, n * 4);
            }
            if (p->start_pos == WITH_TB) {
                if (o->cigar && r->cigar) memcpy(o->cigar, r->cigar, qi);
                if (o->n_cigar && r->n_cigar_ops) memcpy(o->n_cigar, r->n_cigar_ops, n * 4);
            }
            if (p->second_best && st->host_res_second) {
                gasal_res_t *r2 = st->host_res_second;
                if (o->score2 && r2->aln_score) memcpy(o->score2, r2->aln_score, n * 4);
                if (o->q_end2 && r2->query_batch_end) memcpy(o->q_end2, r2->query_batch_end, n * 4);
                if (o->t_end2 && r2->target_batch_end) memcpy(o->t_end2, r2->target_batch_end, n * 4);
            }
            if (o->packed_q) CHECKCUDAERROR(cudaMemcpy(o->packed_q, st->packed_query_batch, (qi / 8) * 4, cudaMemcpyDeviceToHost));
            if (o->packed_t) CHECKCUDAERROR(cudaMemcpy(o->packed_t, st->packed_target_batch, (ti / 8) * 4, cudaMemcpyDeviceToHost));
        }
    }
    if (ms_per_call) *ms_per_call = total_ms / repeats;

    gasal_destroy_streams(&v, params);
    gasal_destroy_gpu_storage_v(&v);
    delete params;
    return GB_OK;
}
