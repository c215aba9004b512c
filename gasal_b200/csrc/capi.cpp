/*
 * capi.cpp -- extern "C" face of the library (declared in
 * include/gasal_b200_capi.h).  Thin: every gasal_c_* call forwards to the C++
 * API implementation with errors returned instead of terminating.
 */
#include "gasal_header.h"
#include "res.h"
#include "gasal_b200_capi.h"
#include "engine.h"

#include <cstdio>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace gbapi {
int aln_async(gasal_gpu_storage_t *s, uint32_t qbytes, uint32_t tbytes, uint32_t n, Parameters *params, bool fatal,
              int zdrop);
int is_done(gasal_gpu_storage_t *s, bool fatal);
void graph_stats(int64_t out[4]);
}

static Parameters *P(void *p) { return static_cast<Parameters *>(p); }
static gasal_gpu_storage_t *S(void *s) { return static_cast<gasal_gpu_storage_t *>(s); }

/* The ksw z-drop of each C parameter object (GASAL2's Parameters has no such
 * member; its kernel hard-codes 0). */
static std::mutex g_zdrop_mu;
static std::unordered_map<const void *, int> g_zdrop;
static int zdrop_of(const void *params)
{
    std::lock_guard<std::mutex> lk(g_zdrop_mu);
    auto it = g_zdrop.find(params);
    return it == g_zdrop.end() ? 0 : it->second;
}

extern "C" {

void *gasal_c_params_new(void) { return new Parameters(0, nullptr); }

int gasal_c_params_set(void *params, const gb_params_t *p)
{
    if (!params || !p) return GB_ERR_ARG;
    Parameters *q = P(params);
    q->algo = (algo_type)p->algo;
    q->start_pos = (comp_start)p->start_pos;
    q->secondBest = p->second_best ? TRUE : FALSE;
    q->semiglobal_skipping_head = (data_source)p->head;
    q->semiglobal_skipping_tail = (data_source)p->tail;
    q->k_band = p->k_band;
    q->isReverseComplement = p->reverse_complement != 0;
    q->sa = p->match, q->sb = p->mismatch, q->gapo = p->gap_open, q->gape = p->gap_extend;
    std::lock_guard<std::mutex> lk(g_zdrop_mu);
    g_zdrop[params] = p->zdrop > 0 ? p->zdrop : 0;
    return GB_OK;
}

void gasal_c_params_free(void *params)
{
    {
        std::lock_guard<std::mutex> lk(g_zdrop_mu);
        g_zdrop.erase(params);
    }
    delete P(params);
}

int gasal_c_copy_subst_scores(int32_t match, int32_t mismatch, int32_t gap_open, int32_t gap_extend)
{
    gasal_subst_scores s = {match, mismatch, gap_open, gap_extend};
    gasal_copy_subst_scores(&s);
    return GB_OK;
}

void *gasal_c_init_gpu_storage_v(int n_streams)
{
    if (n_streams <= 0) return nullptr;
    gasal_gpu_storage_v *v = new gasal_gpu_storage_v;
    *v = gasal_init_gpu_storage_v(n_streams);
    return v;
}

int gasal_c_init_streams(void *storage_v, int max_query_len, int max_target_len, int max_n_alns, void *params)
{
    if (!storage_v || !params || max_query_len <= 0 || max_target_len <= 0 || max_n_alns <= 0) return GB_ERR_ARG;
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
        cudaGetLastError();
        return GB_ERR_CUDA;
    }
    gasal_init_streams(static_cast<gasal_gpu_storage_v *>(storage_v), max_query_len, max_target_len, max_n_alns,
                       P(params));
    return GB_OK;
}

int gasal_c_destroy_streams(void *storage_v, void *params)
{
    if (!storage_v) return GB_ERR_ARG;
    gasal_destroy_streams(static_cast<gasal_gpu_storage_v *>(storage_v), P(params));
    return GB_OK;
}

int gasal_c_destroy_gpu_storage_v(void *storage_v)
{
    if (!storage_v) return GB_ERR_ARG;
    gasal_gpu_storage_v *v = static_cast<gasal_gpu_storage_v *>(storage_v);
    gasal_destroy_gpu_storage_v(v);
    delete v;
    return GB_OK;
}

void *gasal_c_storage(void *storage_v, int i)
{
    gasal_gpu_storage_v *v = static_cast<gasal_gpu_storage_v *>(storage_v);
    if (!v || i < 0 || i >= v->n) return nullptr;
    return &v->a[i];
}

int gasal_c_storage_view(void *storage, gb_storage_view_t *w)
{
    if (!storage || !w) return GB_ERR_ARG;
    gasal_gpu_storage_t *s = S(storage);
    memset(w, 0, sizeof(*w));
    w->host_query_batch_offsets = s->host_query_batch_offsets;
    w->host_target_batch_offsets = s->host_target_batch_offsets;
    w->host_query_batch_lens = s->host_query_batch_lens;
    w->host_target_batch_lens = s->host_target_batch_lens;
    w->host_query_op = s->host_query_op;
    w->host_target_op = s->host_target_op;
    w->host_seed_scores = s->host_seed_scores;
    if (s->host_res) {
        w->aln_score = s->host_res->aln_score;
        w->query_batch_end = s->host_res->query_batch_end;
        w->target_batch_end = s->host_res->target_batch_end;
        w->query_batch_start = s->host_res->query_batch_start;
        w->target_batch_start = s->host_res->target_batch_start;
        w->cigar = s->host_res->cigar;
        w->n_cigar_ops = s->host_res->n_cigar_ops;
    }
    if (s->host_res_second) {
        w->aln_score2 = s->host_res_second->aln_score;
        w->query_batch_end2 = s->host_res_second->query_batch_end;
        w->target_batch_end2 = s->host_res_second->target_batch_end;
    }
    w->stream = (void *)s->str;
    w->host_max_n_alns = s->host_max_n_alns;
    w->host_max_query_batch_bytes = s->host_max_query_batch_bytes;
    w->host_max_target_batch_bytes = s->host_max_target_batch_bytes;
    return GB_OK;
}

uint32_t gasal_c_host_batch_fill(void *storage, uint32_t idx, const char *data, uint32_t size, int src)
{
    return gasal_host_batch_fill(S(storage), idx, data, size, (data_source)src);
}

uint32_t gasal_c_host_batch_fill_mt(void *storage, uint32_t idx, const char *data, uint32_t size, int src,
                                    int threads)
{
    return gasal_host_batch_fill_mt(S(storage), idx, data, size, (data_source)src, threads);
}

uint32_t gasal_c_host_batch_add(void *storage, uint32_t idx, const char *data, uint32_t size, int src)
{
    return gasal_host_batch_add(S(storage), idx, data, size, (data_source)src);
}

int gasal_c_host_batch_reset(void *storage)
{
    if (!storage) return GB_ERR_ARG;
    gasal_host_batch_reset(S(storage));
    return GB_OK;
}

int gasal_c_op_fill(void *storage, const uint8_t *ops, uint32_t n, int src)
{
    if (!storage || !ops || (src != QUERY && src != TARGET) || n > S(storage)->host_max_n_alns) return GB_ERR_ARG;
    gasal_op_fill(S(storage), const_cast<uint8_t *>(ops), n, (data_source)src);
    return GB_OK;
}

int gasal_c_host_alns_resize(void *storage, int new_max_alns, void *params)
{
    if (!storage || !params || new_max_alns < (int)S(storage)->host_max_n_alns) return GB_ERR_ARG;
    gasal_host_alns_resize(S(storage), new_max_alns, P(params));
    return GB_OK;
}

int gasal_c_set_device(int gpu)
{
    return cudaSetDevice(gpu) == cudaSuccess ? GB_OK : GB_ERR_CUDA;
}

int gasal_c_aln_async(void *storage, uint32_t qb, uint32_t tb, uint32_t n, void *params)
{
    if (!storage || !params) return GB_ERR_ARG;
    return gbapi::aln_async(S(storage), qb, tb, n, P(params), false, zdrop_of(params));
}

int gasal_c_is_aln_async_done(void *storage)
{
    if (!storage) return GB_ERR_ARG;
    return gbapi::is_done(S(storage), false);
}

int gb_align(const gb_params_t *p, const gb_batch_t *b, gb_out_t *o)
{
    if (!p || !b || !o || b->n <= 0 || (b->q_bytes & 7) || (b->t_bytes & 7)) return GB_ERR_ARG;
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
        cudaGetLastError();
        return GB_ERR_CUDA;
    }
    const int n = b->n;
    uint32_t max_q = 8, max_t = 8;
    for (int i = 0; i < n; i++) {
        if (b->q_len[i] > max_q) max_q = b->q_len[i];
        if (b->t_len[i] > max_t) max_t = b->t_len[i];
        if ((b->q_off[i] & 7) || (b->t_off[i] & 7) || b->q_off[i] + b->q_len[i] > b->q_bytes ||
            b->t_off[i] + b->t_len[i] > b->t_bytes)
            return GB_ERR_ARG;
    }
    gb::Settings &set = gb::settings();
    const gb::Scores saved = set.sc;
    gasal_c_copy_subst_scores(p->match, p->mismatch, p->gap_open, p->gap_extend);
    Parameters params(0, nullptr);
    gasal_c_params_set(&params, p);
    gasal_gpu_storage_v v = gasal_init_gpu_storage_v(1);
    /* size the host staging for the batch as laid out by the caller */
    const uint32_t per_q = (b->q_bytes + n - 1) / n, per_t = (b->t_bytes + n - 1) / n;
    gasal_init_streams(&v, (int)std::max(per_q, max_q), (int)std::max(per_t, max_t), n, &params);
    gasal_gpu_storage_t *s = &v.a[0];
    /* stage exactly the caller's bytes and offsets */
    uint32_t qi = gasal_host_batch_add(s, 0, (const char *)b->q, b->q_bytes, QUERY);
    uint32_t ti = gasal_host_batch_add(s, 0, (const char *)b->t, b->t_bytes, TARGET);
    s->extensible_host_unpacked_query_batch->data_size = qi;
    s->extensible_host_unpacked_target_batch->data_size = ti;
    memcpy(s->host_query_batch_offsets, b->q_off, n * 4);
    memcpy(s->host_target_batch_offsets, b->t_off, n * 4);
    memcpy(s->host_query_batch_lens, b->q_len, n * 4);
    memcpy(s->host_target_batch_lens, b->t_len, n * 4);
    if (b->q_op) memcpy(s->host_query_op, b->q_op, n);
    if (b->t_op) memcpy(s->host_target_op, b->t_op, n);
    if (p->algo == KSW) {
        for (int i = 0; i < n; i++) s->host_seed_scores[i] = b->seed ? b->seed[i] : 0u;
    }
    s->current_n_alns = n;
    int rc = gbapi::aln_async(s, b->q_bytes, b->t_bytes, n, &params, false, p->zdrop);
    if (rc == GB_OK) {
        cudaError_t e = cudaStreamSynchronize(s->str);
        rc = e == cudaSuccess ? GB_OK : GB_ERR_CUDA;
    }
    if (rc == GB_OK) {
        gasal_res_t *r = s->host_res;
        if (o->score && r->aln_score) memcpy(o->score, r->aln_score, n * 4);
        if (o->q_end && r->query_batch_end) memcpy(o->q_end, r->query_batch_end, n * 4);
        if (o->t_end && r->target_batch_end) memcpy(o->t_end, r->target_batch_end, n * 4);
        const bool has_start = p->start_pos == WITH_START ||
                               (p->start_pos == WITH_TB && (p->algo == LOCAL || (p->algo == SEMI_GLOBAL && p->tail == TARGET)));
        if (has_start && p->algo != GLOBAL && p->algo != KSW && !(p->algo == BANDED && p->start_pos != WITH_START)) {
            if (o->q_start && r->query_batch_start) memcpy(o->q_start, r->query_batch_start, n * 4);
            if (o->t_start && r->target_batch_start) memcpy(o->t_start, r->target_batch_start, n * 4);
        }
        if (p->start_pos == WITH_TB) {
            if (o->cigar && r->cigar) memcpy(o->cigar, r->cigar, b->q_bytes);
            if (o->n_cigar && r->n_cigar_ops) memcpy(o->n_cigar, r->n_cigar_ops, n * 4);
        }
        if (p->second_best && s->host_res_second) {
            gasal_res_t *r2 = s->host_res_second;
            if (o->score2 && r2->aln_score) memcpy(o->score2, r2->aln_score, n * 4);
            if (o->q_end2 && r2->query_batch_end) memcpy(o->q_end2, r2->query_batch_end, n * 4);
            if (o->t_end2 && r2->target_batch_end) memcpy(o->t_end2, r2->target_batch_end, n * 4);
        }
        if (o->packed_q) cudaMemcpy(o->packed_q, s->packed_query_batch, (b->q_bytes / 8) * 4, cudaMemcpyDeviceToHost);
        if (o->packed_t) cudaMemcpy(o->packed_t, s->packed_target_batch, (b->t_bytes / 8) * 4, cudaMemcpyDeviceToHost);
    }
    gasal_host_batch_reset(s);
    gasal_destroy_streams(&v, &params);
    gasal_destroy_gpu_storage_v(&v);
    set.sc = saved;
    return rc;
}

} // extern "C"

namespace {
struct DevWs {
    gb::Workspace ws;
};
std::mutex g_dev_mu;
/* one workspace per (device, stream): work on different streams may overlap */
std::unordered_map<unsigned long long, DevWs *> g_dev_ws;
} // namespace

namespace {
DevWs *dev_ws(void *stream)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lk(g_dev_mu);
    const unsigned long long key = ((unsigned long long)(uintptr_t)stream << 8) ^ (unsigned long long)dev;
    DevWs *&slot = g_dev_ws[key];
    if (!slot) slot = new DevWs();
    return slot;
}

void dev_args(const gb_params_t *p, const gb_dev_batch_t *b, const gb_dev_out_t *o, gb::RunCfg &cfg,
              gb::DevBatch &db, gb::DevOut &dout)
{
    const gb::Settings &set = gb::settings();
    cfg = gb::RunCfg{};
    cfg.algo = p->algo, cfg.start = p->start_pos, cfg.second = p->second_best != 0;
    cfg.head = p->head, cfg.tail = p->tail, cfg.k_band = p->k_band, cfg.zdrop = p->zdrop;
    cfg.sc = {p->match, p->mismatch, p->gap_open, p->gap_extend, p->gap_open + p->gap_extend};
    cfg.ref_reverse = set.ref_reverse, cfg.mql = set.mql, cfg.is_packed = 0;
    cfg.reverse_complement = p->reverse_complement;
    cfg.band_model = set.band_model, cfg.band_min = set.band_min, cfg.band_max = set.band_max;
    db = gb::DevBatch{};
    db.n = b->n, db.q_bytes = b->q_bytes, db.t_bytes = b->t_bytes, db.q = b->q, db.t = b->t;
    db.pq = b->pq, db.pt = b->pt, db.q_off = b->q_off, db.t_off = b->t_off, db.q_len = b->q_len;
    db.t_len = b->t_len, db.q_op = b->q_op, db.t_op = b->t_op, db.seed = b->seed;
    db.h_q_len = b->h_q_len, db.h_t_len = b->h_t_len;
    dout = gb::DevOut{};
    dout.score = o->score, dout.q_end = o->q_end, dout.t_end = o->t_end, dout.q_start = o->q_start;
    dout.t_start = o->t_start, dout.score2 = o->score2, dout.q_end2 = o->q_end2, dout.t_end2 = o->t_end2;
    dout.cigar = o->cigar, dout.n_cigar = o->n_cigar;
}
} // namespace

extern "C" int gb_release_workspaces(void)
{
    if (cudaDeviceSynchronize() != cudaSuccess) return GB_ERR_CUDA;
    {
        std::lock_guard<std::mutex> lk(g_dev_mu);
        for (auto &kv : g_dev_ws) {
            gb::release_workspace(kv.second->ws);
            delete kv.second;
        }
        g_dev_ws.clear();
    }
    gb::mix_release_all();
    gb::band_release_all();
    return cudaGetLastError() == cudaSuccess ? GB_OK : GB_ERR_CUDA;
}

extern "C" int gb_align_dev(const gb_params_t *p, const gb_dev_batch_t *b, const gb_dev_out_t *o, void *stream)
{
    if (!p || !b || !o || b->n < 0) return GB_ERR_ARG;
    if (b->n == 0) return GB_OK; /* an empty batch: nothing to launch */
    if (!b->h_q_len || !b->h_t_len) return GB_ERR_ARG;
    DevWs *w = dev_ws(stream);
    if (!w) return GB_ERR_CUDA;
    gb::RunCfg cfg;
    gb::DevBatch db;
    gb::DevOut dout;
    dev_args(p, b, o, cfg, db, dout);
    return gb::run_batch(cfg, db, dout, w->ws, (cudaStream_t)stream);
}

/* Launch autotuner: times the batch under every candidate setting (CUDA
 * events on `stream`, `reps` runs after one warm-up run each) and keeps the
 * fastest.  Candidates: DP block 32/64/128 x warp-cooperative threshold
 * 16/32/48/64 query words x lane groups automatic/8/16/32 (LOCAL, GLOBAL and
 * target-tail SEMI_GLOBAL; other algorithms keep the
 * current threshold). */
namespace {
thread_local char g_last_error[256] = "";
void set_last_error(const char *where, cudaError_t e)
{
    snprintf(g_last_error, sizeof g_last_error, "%s: %s", where, cudaGetErrorString(e));
}
} // namespace

/* The pack kernel alone (reference gasal_pack_kernel, src/kernels/pack_rc_seqs.h:13-53). */
extern "C" int gb_pack_dev(const uint8_t *ascii, uint32_t nbytes, uint32_t *packed, void *stream)
{
    if ((nbytes & 7) || (nbytes && (!ascii || !packed))) return GB_ERR_ARG;
    return gb::launch_pack(ascii, nbytes, packed, (cudaStream_t)stream) == cudaSuccess ? GB_OK : GB_ERR_CUDA;
}

/* The reverse/complement kernel alone on packed words (reference
 * gasal_reversecomplement_kernel, src/kernels/pack_rc_seqs.h:56-212). */
extern "C" int gb_revcomp_dev(uint32_t *pq, uint32_t *pt, const uint32_t *q_off, const uint32_t *t_off,
                              const uint32_t *q_len, const uint32_t *t_len, const uint8_t *q_op, const uint8_t *t_op,
                              int32_t n, void *stream)
{
    if (n < 0 || (n && (!pq || !pt || !q_off || !t_off || !q_len || !t_len))) return GB_ERR_ARG;
    return gb::launch_revcomp(pq, pt, q_off, t_off, q_len, t_len, q_op, t_op, n, gb::settings().ref_reverse,
                              (cudaStream_t)stream) == cudaSuccess
               ? GB_OK
               : GB_ERR_CUDA;
}

extern "C" const char *gb_last_error(void) { return g_last_error; }

extern "C" int gb_autotune(const gb_params_t *p, const gb_dev_batch_t *b, const gb_dev_out_t *o, void *stream,
                           int reps, gb_tuning_t *best, double *best_ms)
{
    if (!p || !b || !o || b->n <= 0 || !b->h_q_len || !b->h_t_len || reps <= 0 || !best) return GB_ERR_ARG;
    DevWs *w = dev_ws(stream);
    if (!w) return GB_ERR_CUDA;
    gb::RunCfg cfg;
    gb::DevBatch db;
    gb::DevOut dout;
    dev_args(p, b, o, cfg, db, dout);
    gb::Settings &st = gb::settings();
    const gb::Settings saved = st;
    const cudaStream_t s = (cudaStream_t)stream;
    std::vector<int> blocks = {32, 64, 128};
    std::vector<int> wcs = {st.wc_min_qregs};
    std::vector<int> groups = {st.wc_group};
    if (p->algo == LOCAL || p->algo == GLOBAL || (p->algo == SEMI_GLOBAL && p->tail == TARGET)) {
        wcs = {16, 32, 48, 64};
        groups = {0, 8, 16, 32};
    }
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return GB_ERR_CUDA;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return GB_ERR_CUDA;
    }
    int rc = GB_OK;
    float best_t = 0.f;
    gb_tuning_t bt{saved.block, saved.wc_min_qregs, saved.min_order_pairs, saved.ksw_wc, saved.split_start,
                   saved.persistent, saved.wc_group};
    char where[96];
    for (int blk : blocks) {
        for (size_t c = 0; c < wcs.size() * groups.size() && rc == GB_OK; c++) {
            const int wc = wcs[c % wcs.size()], grp = groups[c / wcs.size()];
            if (groups.size() > 1 && wc < grp) continue; /* the threshold is at least the group */
            st.block = blk, st.wc_min_qregs = wc, st.wc_group = grp;
            snprintf(where, sizeof where, "gb_autotune block %d threshold %d group %d", blk, wc, grp);
            rc = gb::run_batch(cfg, db, dout, w->ws, s);
            for (int r = 0; r < reps && rc == GB_OK; r++) {
                if (r == 0 && cudaEventRecord(e0, s) != cudaSuccess) rc = GB_ERR_CUDA;
                if (rc == GB_OK) rc = gb::run_batch(cfg, db, dout, w->ws, s);
            }
            if (rc != GB_OK) set_last_error(where, cudaGetLastError());
            float ms = 0.f;
            cudaError_t ce = cudaSuccess;
            if (rc == GB_OK && ((ce = cudaEventRecord(e1, s)) != cudaSuccess || (ce = cudaEventSynchronize(e1)) != cudaSuccess ||
                                (ce = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess)) {
                rc = GB_ERR_CUDA;
                set_last_error(where, ce);
            }
            if (rc != GB_OK) break;
            if (best_t == 0.f || ms < best_t) best_t = ms, bt.block = blk, bt.wc_min_qregs = wc, bt.wc_group = grp;
        }
        if (rc != GB_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    st = saved;
    if (rc != GB_OK) return rc;
    st.block = bt.block, st.wc_min_qregs = bt.wc_min_qregs, st.wc_group = bt.wc_group;
    *best = bt;
    if (best_ms) *best_ms = best_t / reps;
    return GB_OK;
}

extern "C" int gb_set_reference_reverse(int on)
{
    gb::settings().ref_reverse = on ? 1 : 0;
    return GB_OK;
}

extern "C" int gb_set_reference_max_query_len(int mql)
{
    if (mql <= 0) return GB_ERR_ARG;
    gb::settings().mql = mql;
    return GB_OK;
}

extern "C" int gb_set_tb_budget_mb(int64_t mb)
{
    if (mb <= 0) return GB_ERR_ARG;
    gb::settings().tb_budget_bytes = (size_t)mb << 20;
    return GB_OK;
}

extern "C" int gb_set_graphs(int on)
{
    gb::settings().graphs = on ? 1 : 0;
    return GB_OK;
}

extern "C" int gb_graph_stats(int64_t *counts)
{
    if (!counts) return GB_ERR_ARG;
    gbapi::graph_stats(counts);
    return GB_OK;
}

extern "C" int gb_set_tuning(const gb_tuning_t *t)
{
    if (!t) return GB_ERR_ARG;
    if (t->block != 32 && t->block != 64 && t->block != 128) return GB_ERR_ARG;
    if (t->wc_min_qregs < 8 || t->min_order_pairs < 0) return GB_ERR_ARG;
    if (t->wc_group != 0 && t->wc_group != 8 && t->wc_group != 16 && t->wc_group != 32 && t->wc_group != 64)
        return GB_ERR_ARG;
    gb::Settings &st = gb::settings();
    st.block = t->block, st.wc_min_qregs = t->wc_min_qregs, st.min_order_pairs = t->min_order_pairs;
    st.ksw_wc = t->ksw_warp ? 1 : 0;
    st.split_start = t->split_start ? 1 : 0;
    st.persistent = t->persistent ? 1 : 0;
    st.wc_group = t->wc_group;
    return GB_OK;
}

extern "C" int gb_get_tuning(gb_tuning_t *t)
{
    if (!t) return GB_ERR_ARG;
    const gb::Settings &st = gb::settings();
    t->block = st.block, t->wc_min_qregs = st.wc_min_qregs, t->min_order_pairs = st.min_order_pairs;
    t->ksw_warp = st.ksw_wc;
    t->split_start = st.split_start;
    t->persistent = st.persistent;
    t->wc_group = st.wc_group;
    return GB_OK;
}

extern "C" int gb_cigar_text(const uint8_t *cigar, const uint32_t *q_off, const uint32_t *n_cigar, int n, char *text,
                             int stride, int32_t *text_len, void *stream)
{
    if (n < 0 || stride <= 0 || (n > 0 && (!cigar || !q_off || !n_cigar || !text || !text_len))) return GB_ERR_ARG;
    return gb::launch_cigar_text(cigar, q_off, n_cigar, n, text, stride, text_len, (cudaStream_t)stream) == cudaSuccess
               ? GB_OK
               : GB_ERR_CUDA;
}

extern "C" const char *gb_version(void) { return "gasal-b200 0.1 (sm_100a)"; }

extern "C" int gb_kernel_timing(int on)
{
    gb::timing_enable(on != 0);
    return GB_OK;
}

extern "C" int gb_kernel_timing_read(double *ms, int64_t *launches)
{
    if (!ms || !launches) return GB_ERR_ARG;
    return gb::timing_read(ms, launches);
}

extern "C" int gb_probe_dpx16x2_peak(double *halfword_tops)
{
    if (!halfword_tops) return GB_ERR_ARG;
    return gb::probe_dpx16x2_peak(halfword_tops) == 0 ? GB_OK : GB_ERR_CUDA;
}

extern "C" int gb_probe_int_peak(double *iadd_tops, double *imnmx_tops, double *dpx_tops)
{
    if (!iadd_tops || !imnmx_tops || !dpx_tops) return GB_ERR_ARG;
    return gb::probe_int_peak(iadd_tops, imnmx_tops, dpx_tops) == 0 ? GB_OK : GB_ERR_CUDA;
}
