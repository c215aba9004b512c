/*
 * ref_host.cpp -- the reference GASAL2 kernels (src/gasal_kernels.h, included
 * in place from the reference tree) run on host cores.
 *
 * TEST INFRASTRUCTURE ONLY.  It replays the launch sequence of the
 * reference's gasal_aln_async (src/gasal_align.cu:180-264): pack kernel with
 * the same grid and tasks-per-thread, optional reverse-complement kernel, the
 * alignment kernel chosen as in src/gasal_align.h:89-107, then the traceback
 * kernel for LOCAL/GLOBAL WITH_TB.  Pairs are spread over OpenMP threads.
 * Used to cross-check the scalar oracle without a GPU and as the bench's
 * reference CPU arm.
 */
#include "ref_host_shim.h"
#include "gasal_kernels.h" /* reference src/gasal_kernels.h */
#include "../include/gasal_b200_capi.h"

#include <cstring>
#include <cmath>
#include <algorithm>
#include <vector>
#include <omp.h>

thread_local gb_dim3 gb_thread_idx, gb_block_idx;
gb_dim3 gb_block_dim, gb_grid_dim;

namespace {

template <typename F>
void launch_per_pair(int n, int nthreads, F kern)
{
    gb_block_dim = {1u, 1u, 1u};
    gb_grid_dim = {(unsigned)n, 1u, 1u};
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
    for (int tid = 0; tid < n; tid++) {
        gb_block_idx = {(unsigned)tid, 0u, 0u};
        gb_thread_idx = {0u, 0u, 0u};
        kern();
    }
}

template <typename S, typename B, typename H, typename T>
void run_semi(uint32_t *pq, uint32_t *pt, uint32_t *ql, uint32_t *tl, uint32_t *qo, uint32_t *to,
              gasal_res_t *r, gasal_res_t *r2, uint4 *tb, int n, int nt)
{
    launch_per_pair(n, nt, [&] {
        gasal_semi_global_kernel<Int2Type<SEMI_GLOBAL>, S, B, H, T>(pq, pt, ql, tl, qo, to, r, r2, tb, n);
    });
}

template <typename S, typename B, typename H>
void semi_tail(int tail, uint32_t *pq, uint32_t *pt, uint32_t *ql, uint32_t *tl, uint32_t *qo, uint32_t *to,
               gasal_res_t *r, gasal_res_t *r2, uint4 *tb, int n, int nt)
{
    switch (tail) {
    case NONE: run_semi<S, B, H, Int2Type<NONE>>(pq, pt, ql, tl, qo, to, r, r2, tb, n, nt); break;
    case QUERY: run_semi<S, B, H, Int2Type<QUERY>>(pq, pt, ql, tl, qo, to, r, r2, tb, n, nt); break;
    case TARGET: run_semi<S, B, H, Int2Type<TARGET>>(pq, pt, ql, tl, qo, to, r, r2, tb, n, nt); break;
    default: run_semi<S, B, H, Int2Type<BOTH>>(pq, pt, ql, tl, qo, to, r, r2, tb, n, nt); break;
    }
}

template <typename S, typename B>
void semi_head(int head, int tail, uint32_t *pq, uint32_t *pt, uint32_t *ql, uint32_t *tl, uint32_t *qo,
               uint32_t *to, gasal_res_t *r, gasal_res_t *r2, uint4 *tb, int n, int nt)
{
    switch (head) {
    case NONE: semi_tail<S, B, Int2Type<NONE>>(tail, pq, pt, ql, tl, qo, to, r, r2, tb, n, nt); break;
    case QUERY: semi_tail<S, B, Int2Type<QUERY>>(tail, pq, pt, ql, tl, qo, to, r, r2, tb, n, nt); break;
    case TARGET: semi_tail<S, B, Int2Type<TARGET>>(tail, pq, pt, ql, tl, qo, to, r, r2, tb, n, nt); break;
    default: semi_tail<S, B, Int2Type<BOTH>>(tail, pq, pt, ql, tl, qo, to, r, r2, tb, n, nt); break;
    }
}

template <typename B>
void semi_start(int start, int head, int tail, uint32_t *pq, uint32_t *pt, uint32_t *ql, uint32_t *tl,
                uint32_t *qo, uint32_t *to, gasal_res_t *r, gasal_res_t *r2, uint4 *tb, int n, int nt)
{
    switch (start) {
    case WITH_START: semi_head<Int2Type<WITH_START>, B>(head, tail, pq, pt, ql, tl, qo, to, r, r2, tb, n, nt); break;
    case WITH_TB: semi_head<Int2Type<WITH_TB>, B>(head, tail, pq, pt, ql, tl, qo, to, r, r2, tb, n, nt); break;
    default: semi_head<Int2Type<WITHOUT_START>, B>(head, tail, pq, pt, ql, tl, qo, to, r, r2, tb, n, nt); break;
    }
}

template <typename S, typename B>
void run_local(uint32_t *pq, uint32_t *pt, uint32_t *ql, uint32_t *tl, uint32_t *qo, uint32_t *to,
               gasal_res_t *r, gasal_res_t *r2, uint4 *tb, int n, int nt)
{
    launch_per_pair(n, nt, [&] {
        gasal_local_kernel<Int2Type<LOCAL>, S, B>(pq, pt, ql, tl, qo, to, r, r2, tb, n);
    });
}

} // namespace

extern "C" int ref_host_align(const gb_params_t *p, const gb_batch_t *b, gb_out_t *o, int nthreads)
{
    if (!p || !b || !o || b->n <= 0 || (b->q_bytes & 7) || (b->t_bytes & 7)) return GB_ERR_ARG;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    const int n = b->n;

    _cudaGapO = p->gap_open;
    _cudaGapExtend = p->gap_extend;
    _cudaGapOE = p->gap_open + p->gap_extend;
    _cudaMatchScore = p->match;
    _cudaMismatchScore = p->mismatch;

    std::vector<uint32_t> uq((b->q_bytes + 3) / 4 + 2, 0), ut((b->t_bytes + 3) / 4 + 2, 0);
    memcpy(uq.data(), b->q, b->q_bytes);
    memcpy(ut.data(), b->t, b->t_bytes);
    std::vector<uint32_t> pq(b->q_bytes / 8 + 2, 0), pt(b->t_bytes / 8 + 2, 0);
    std::vector<uint32_t> ql(b->q_len, b->q_len + n), tl(b->t_len, b->t_len + n);
    std::vector<uint32_t> qo(b->q_off, b->q_off + n), to(b->t_off, b->t_off + n);
    std::vector<uint8_t> qop(n, 0), top(n, 0);
    if (b->q_op) memcpy(qop.data(), b->q_op, n);
    if (b->t_op) memcpy(top.data(), b->t_op, n);
    std::vector<uint32_t> seed(n, 0);
    if (b->seed) memcpy(seed.data(), b->seed, n * 4);
    /* the traceback kernel writes CIGAR bytes over the unpacked query batch */
    std::vector<uint8_t> cigar_buf(b->q_bytes + 4096, 0);
    memcpy(cigar_buf.data(), b->q, b->q_bytes);

    /* pack: same grid and per-thread task count as src/gasal_align.cu:180-194 */
    {
        const uint32_t BLOCKDIM = 128, NB = (n + BLOCKDIM - 1) / BLOCKDIM;
        int qtpt = (int)ceil((double)b->q_bytes / (8 * BLOCKDIM * NB));
        int ttpt = (int)ceil((double)b->t_bytes / (8 * BLOCKDIM * NB));
        gb_block_dim = {BLOCKDIM, 1u, 1u};
        gb_grid_dim = {NB, 1u, 1u};
        const int total = (int)(NB * BLOCKDIM);
#pragma omp parallel for schedule(static) num_threads(nthreads)
        for (int g = 0; g < total; g++) {
            gb_block_idx = {(unsigned)(g / BLOCKDIM), 0u, 0u};
            gb_thread_idx = {(unsigned)(g % BLOCKDIM), 0u, 0u};
            gasal_pack_kernel(uq.data(), ut.data(), pq.data(), pt.data(), qtpt, ttpt, b->q_bytes / 4, b->t_bytes / 4);
        }
    }
    if (p->reverse_complement) {
        launch_per_pair(n, nthreads, [&] {
            gasal_reversecomplement_kernel(pq.data(), pt.data(), ql.data(), tl.data(), qo.data(), to.data(),
                                           qop.data(), top.data(), n);
        });
    }
    if (o->packed_q) memcpy(o->packed_q, pq.data(), (b->q_bytes / 8) * 4);
    if (o->packed_t) memcpy(o->packed_t, pt.data(), (b->t_bytes / 8) * 4);

    std::vector<int32_t> sc(n, 0), qe(n, 0), te(n, 0), qs(n, 0), ts(n, 0);
    std::vector<int32_t> sc2(n, 0), qe2(n, 0), te2(n, 0), qs2(n, 0), ts2(n, 0);
    gasal_res_t res = {sc.data(), qe.data(), te.data(), qs.data(), ts.data(), NULL, NULL};
    gasal_res_t res2 = {sc2.data(), qe2.data(), te2.data(), qs2.data(), ts2.data(), NULL, NULL};

    const uint32_t maxq8 = (uint32_t)(*std::max_element(ql.begin(), ql.end()) + 7) & ~7u;
    /* 16 spare target rows, as the GPU driver allocates (the GLOBAL traceback
     * reads one tile row past the matrix when a length is a multiple of 8) */
    const uint32_t maxt8 = ((uint32_t)(*std::max_element(tl.begin(), tl.end()) + 7) & ~7u) + 16;
    /* The reference allocates its tile buffer once, at gasal_init_streams
     * (src/ctors.cpp:60-66), not per batch: keep one buffer across calls and
     * grow it.  GLOBAL traceback reads a tile row past the matrix, which a
     * fresh device allocation holds as zeros, so those tiles are cleared. */
    static std::vector<uint4> tb_keep;
    uint4 *tbp = NULL;
    if (p->start_pos == WITH_TB && (p->algo == LOCAL || p->algo == GLOBAL)) {
        const size_t tiles = (size_t)ceil((double)((uint64_t)maxq8 * maxt8) / 32.0) * (size_t)n;
        if (tb_keep.size() < tiles) tb_keep.resize(tiles);
        if (p->algo == GLOBAL) std::fill(tb_keep.begin(), tb_keep.begin() + tiles, make_uint4(0, 0, 0, 0));
        tbp = tb_keep.data();
    }
    uint32_t *PQ = pq.data(), *PT = pt.data(), *QL = ql.data(), *TL = tl.data(), *QO = qo.data(), *TO = to.data();
    const bool sb = p->second_best != 0;

    switch (p->algo) {
    case LOCAL:
        if (p->start_pos == WITH_START) {
            if (sb) run_local<Int2Type<WITH_START>, Int2Type<TRUE>>(PQ, PT, QL, TL, QO, TO, &res, &res2, tbp, n, nthreads);
            else run_local<Int2Type<WITH_START>, Int2Type<FALSE>>(PQ, PT, QL, TL, QO, TO, &res, &res2, tbp, n, nthreads);
        } else if (p->start_pos == WITH_TB) {
            if (sb) run_local<Int2Type<WITH_TB>, Int2Type<TRUE>>(PQ, PT, QL, TL, QO, TO, &res, &res2, tbp, n, nthreads);
            else run_local<Int2Type<WITH_TB>, Int2Type<FALSE>>(PQ, PT, QL, TL, QO, TO, &res, &res2, tbp, n, nthreads);
            launch_per_pair(n, nthreads, [&] {
                gasal_get_tb<Int2Type<LOCAL>>(cigar_buf.data(), QL, TL, QO, tbp, &res, n);
            });
        } else {
            if (sb) run_local<Int2Type<WITHOUT_START>, Int2Type<TRUE>>(PQ, PT, QL, TL, QO, TO, &res, &res2, tbp, n, nthreads);
            else run_local<Int2Type<WITHOUT_START>, Int2Type<FALSE>>(PQ, PT, QL, TL, QO, TO, &res, &res2, tbp, n, nthreads);
        }
        break;
    case GLOBAL:
        if (p->start_pos == WITH_TB) {
            launch_per_pair(n, nthreads, [&] {
                gasal_global_kernel<Int2Type<WITH_TB>>(PQ, PT, QL, TL, QO, TO, &res, tbp, n);
            });
            launch_per_pair(n, nthreads, [&] {
                gasal_get_tb<Int2Type<GLOBAL>>(cigar_buf.data(), QL, TL, QO, tbp, &res, n);
            });
        } else if (p->start_pos == WITH_START) {
            launch_per_pair(n, nthreads, [&] {
                gasal_global_kernel<Int2Type<WITH_START>>(PQ, PT, QL, TL, QO, TO, &res, tbp, n);
            });
        } else {
            launch_per_pair(n, nthreads, [&] {
                gasal_global_kernel<Int2Type<WITHOUT_START>>(PQ, PT, QL, TL, QO, TO, &res, tbp, n);
            });
        }
        break;
    case SEMI_GLOBAL:
        if (sb) semi_start<Int2Type<TRUE>>(p->start_pos, p->head, p->tail, PQ, PT, QL, TL, QO, TO, &res, &res2, tbp, n, nthreads);
        else semi_start<Int2Type<FALSE>>(p->start_pos, p->head, p->tail, PQ, PT, QL, TL, QO, TO, &res, &res2, tbp, n, nthreads);
        break;
    case BANDED:
        launch_per_pair(n, nthreads, [&] {
            gasal_banded_tiled_kernel(PQ, PT, QL, TL, QO, TO, &res, n, p->k_band >> 3);
        });
        break;
    case KSW: {
        uint32_t *SD = seed.data();
        if (sb) launch_per_pair(n, nthreads, [&] { gasal_ksw_kernel<Int2Type<TRUE>>(PQ, PT, QL, TL, QO, TO, SD, &res, &res2, n); });
        else launch_per_pair(n, nthreads, [&] { gasal_ksw_kernel<Int2Type<FALSE>>(PQ, PT, QL, TL, QO, TO, SD, &res, &res2, n); });
        break;
    }
    default:
        return GB_ERR_ARG;
    }

    if (o->score) memcpy(o->score, sc.data(), n * 4);
    if (p->algo != GLOBAL) {
        if (o->q_end) memcpy(o->q_end, qe.data(), n * 4);
        if (o->t_end) memcpy(o->t_end, te.data(), n * 4);
        if (p->start_pos != WITHOUT_START) {
            if (o->q_start) memcpy(o->q_start, qs.data(), n * 4);
            if (o->t_start) memcpy(o->t_start, ts.data(), n * 4);
        }
    }
    if (p->start_pos == WITH_TB) {
        if (o->cigar) memcpy(o->cigar, cigar_buf.data(), b->q_bytes);
        if (o->n_cigar) memcpy(o->n_cigar, ql.data(), n * 4);
    }
    if (sb) {
        if (o->score2) memcpy(o->score2, sc2.data(), n * 4);
        if (o->q_end2) memcpy(o->q_end2, qe2.data(), n * 4);
        if (o->t_end2) memcpy(o->t_end2, te2.data(), n * 4);
    }
    return GB_OK;
}
