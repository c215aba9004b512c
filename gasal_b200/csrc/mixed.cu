/*
 * mixed.cu -- per-pair mixed-algorithm dispatch (an extension; GASAL2 picks
 * one algorithm per launch through Parameters::algo, src/gasal_align.cu:249
 * and the kernel switch of src/gasal_align.h:89-107).
 *
 * gb_align_dev_mixed aligns one device batch whose pairs each name one of up
 * to GB_MIXED_MAX_KINDS option sets ("kinds": algorithm, start/traceback,
 * second best, semi-global ends, band, z-drop, scores).  The batch is packed
 * once; then every kind runs the same plan -> order -> specialised kernels ->
 * traceback pipeline as gb_align_dev, over that kind's pairs only, each kind
 * on a stream of its own forked from the caller's stream and joined back, so
 * a kind whose long pairs finish last overlaps the others.
 *
 * No sequence bytes move: a kind's pairs are addressed through gathered copies
 * of their offsets and lengths, which still point into the caller's packed
 * words, so reverse/complement and CIGAR writes land at each pair's own
 * offsets.  Results come back through per-kind result arrays that are
 * gathered from the caller's arrays before the kinds run and scattered back
 * after them: a result array that a pair's kind does not produce keeps the
 * value it had, as it would after gb_align_dev with that kind's options.
 */
#include "engine.h"

#include <mutex>
#include <unordered_map>
#include <vector>

namespace gb {
namespace {

constexpr int MIX_OUTS = 9; /* score .. t_end2, n_cigar */

struct MixArgs {
    const uint32_t *idx; /* pair of each kind-major position */
    int32_t n;
    const uint32_t *q_off, *t_off, *q_len, *t_len, *seed;
    const uint8_t *q_op, *t_op;
    uint32_t *s_q_off, *s_t_off, *s_q_len, *s_t_len, *s_seed;
    uint8_t *s_q_op, *s_t_op;
    int32_t *out[MIX_OUTS], *sub[MIX_OUTS];
};

/* kind-major copies of the per-pair inputs, and of the caller's result values */
__global__ void mix_gather_kernel(MixArgs a)
{
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < a.n; m += gridDim.x * blockDim.x) {
        const uint32_t i = a.idx[m];
        a.s_q_off[m] = a.q_off[i];
        a.s_t_off[m] = a.t_off[i];
        a.s_q_len[m] = a.q_len[i];
        a.s_t_len[m] = a.t_len[i];
        if (a.seed) a.s_seed[m] = a.seed[i];
        if (a.q_op) a.s_q_op[m] = a.q_op[i];
        if (a.t_op) a.s_t_op[m] = a.t_op[i];
#pragma unroll
        for (int k = 0; k < MIX_OUTS; k++)
            if (a.out[k]) a.sub[k][m] = a.out[k][i];
    }
}

__global__ void mix_scatter_kernel(MixArgs a)
{
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < a.n; m += gridDim.x * blockDim.x) {
        const uint32_t i = a.idx[m];
#pragma unroll
        for (int k = 0; k < MIX_OUTS; k++)
            if (a.out[k]) a.out[k][i] = a.sub[k][m];
    }
}

/* Device and pinned buffers of one (device, stream), grown on demand. */
struct MixState {
    Workspace ws[GB_MIXED_MAX_KINDS];
    cudaStream_t ks[GB_MIXED_MAX_KINDS] = {};
    cudaEvent_t fork = nullptr, join[GB_MIXED_MAX_KINDS] = {}, idx_free = nullptr;
    uint32_t *h_idx = nullptr;  /* pinned: the kind-major pair list */
    uint32_t *d = nullptr;      /* idx, q_off, t_off, q_len, t_len, seed, 9 result arrays: 15 words per pair */
    uint8_t *d_ops = nullptr;   /* q_op, t_op */
    size_t cap = 0;
    std::vector<uint32_t> h_ql, h_tl; /* host lengths of the kind-major list (planning) */
    ~MixState()
    {
        for (int k = 0; k < GB_MIXED_MAX_KINDS; k++) {
            if (ks[k]) cudaStreamDestroy(ks[k]);
            if (join[k]) cudaEventDestroy(join[k]);
        }
        if (fork) cudaEventDestroy(fork);
        if (idx_free) cudaEventDestroy(idx_free);
        if (h_idx) cudaFreeHost(h_idx);
        if (d) cudaFree(d);
        if (d_ops) cudaFree(d_ops);
    }
};

std::mutex g_mix_mu;
std::unordered_map<unsigned long long, MixState *> g_mix;

} // namespace

/* every stream's mixed-dispatch buffers and kind workspaces (gb_release_workspaces) */
void mix_release_all()
{
    std::lock_guard<std::mutex> lk(g_mix_mu);
    for (auto &kv : g_mix) {
        MixState *m = kv.second;
        for (auto &w : m->ws) release_workspace(w);
        delete m;
    }
    g_mix.clear();
}

namespace {

MixState *mix_state(cudaStream_t s)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lk(g_mix_mu);
    const unsigned long long key = ((unsigned long long)(uintptr_t)s << 8) ^ (unsigned long long)dev;
    MixState *&m = g_mix[key];
    if (!m) m = new MixState();
    return m;
}

int mix_reserve(MixState &m, size_t n)
{
    if (m.idx_free && cudaEventSynchronize(m.idx_free) != cudaSuccess) return GB_ERR_CUDA;
    if (m.cap >= n) return GB_OK;
    const size_t want = n + n / 4 + 1024;
    if (m.h_idx) cudaFreeHost(m.h_idx);
    if (m.d) cudaFree(m.d);
    if (m.d_ops) cudaFree(m.d_ops);
    m.h_idx = nullptr, m.d = nullptr, m.d_ops = nullptr, m.cap = 0;
    if (cudaMallocHost((void **)&m.h_idx, want * 4) != cudaSuccess ||
        dev_malloc((void **)&m.d, want * 4 * 15) != cudaSuccess ||
        dev_malloc((void **)&m.d_ops, want * 2) != cudaSuccess) {
        cudaGetLastError();
        return GB_ERR_ALLOC;
    }
    m.cap = want;
    return GB_OK;
}

int mix_streams(MixState &m)
{
    if (!m.fork && cudaEventCreateWithFlags(&m.fork, cudaEventDisableTiming) != cudaSuccess) return GB_ERR_CUDA;
    if (!m.idx_free && cudaEventCreateWithFlags(&m.idx_free, cudaEventDisableTiming) != cudaSuccess)
        return GB_ERR_CUDA;
    for (int k = 0; k < GB_MIXED_MAX_KINDS; k++) {
        if (!m.ks[k] && cudaStreamCreateWithFlags(&m.ks[k], cudaStreamNonBlocking) != cudaSuccess) return GB_ERR_CUDA;
        if (!m.join[k] && cudaEventCreateWithFlags(&m.join[k], cudaEventDisableTiming) != cudaSuccess)
            return GB_ERR_CUDA;
    }
    return GB_OK;
}

/* Options of one kind as the engine reads them (gb_align_dev's rules). */
void mix_cfg(const gb_params_t &p, RunCfg &cfg)
{
    const Settings &set = settings();
    cfg = RunCfg{};
    cfg.algo = p.algo, cfg.start = p.start_pos, cfg.second = p.second_best != 0;
    cfg.head = p.head, cfg.tail = p.tail, cfg.k_band = p.k_band, cfg.zdrop = p.zdrop;
    cfg.sc = {p.match, p.mismatch, p.gap_open, p.gap_extend, p.gap_open + p.gap_extend};
    cfg.ref_reverse = set.ref_reverse, cfg.mql = set.mql;
    cfg.is_packed = 1; /* packed once for every kind */
    cfg.reverse_complement = p.reverse_complement;
    cfg.band_model = set.band_model, cfg.band_min = set.band_min, cfg.band_max = set.band_max;
}

} // namespace
} // namespace gb

extern "C" int gb_mixed_check(const gb_params_t *kinds, int n_kinds, const uint8_t *h_kind, int32_t n,
                              int has_seed, uint32_t *counts)
{
    if (!kinds || n_kinds < 1 || n_kinds > GB_MIXED_MAX_KINDS || n < 0 || (n > 0 && !h_kind)) return GB_ERR_ARG;
    uint32_t c[GB_MIXED_MAX_KINDS] = {};
    for (int32_t i = 0; i < n; i++) {
        if (h_kind[i] >= n_kinds) return GB_ERR_ARG;
        c[h_kind[i]]++;
    }
    for (int k = 0; k < n_kinds; k++) {
        const int a = kinds[k].algo;
        if (a != gb::GLOBAL_ && a != gb::SEMI_GLOBAL_ && a != gb::LOCAL_ && a != gb::BANDED_ && a != gb::KSW_)
            return GB_ERR_ARG;
        if (a == gb::KSW_ && c[k] && !has_seed) return GB_ERR_ARG;
    }
    if (counts)
        for (int k = 0; k < n_kinds; k++) counts[k] = c[k];
    return GB_OK;
}

extern "C" int gb_align_dev_mixed(const gb_params_t *kinds, int n_kinds, const uint8_t *h_kind,
                                  const gb_dev_batch_t *b, const gb_dev_out_t *o, void *stream)
{
    using namespace gb;
    if (!b || !o || !b->h_q_len || !b->h_t_len) return GB_ERR_ARG;
    uint32_t counts[GB_MIXED_MAX_KINDS] = {};
    int rc = gb_mixed_check(kinds, n_kinds, h_kind, b->n, b->seed != nullptr, counts);
    if (rc != GB_OK) return rc;
    if (b->n == 0) return GB_OK;
    const cudaStream_t s = (cudaStream_t)stream;
    MixState *mp = mix_state(s);
    if (!mp) return GB_ERR_CUDA;
    MixState &m = *mp;
    if ((rc = mix_streams(m)) != GB_OK) return rc;
    const size_t n = (size_t)b->n;
    if ((rc = mix_reserve(m, n)) != GB_OK) return rc;

    /* kind-major pair list and its host lengths */
    uint32_t base[GB_MIXED_MAX_KINDS + 1] = {};
    for (int k = 0; k < n_kinds; k++) base[k + 1] = base[k] + counts[k];
    uint32_t fill[GB_MIXED_MAX_KINDS];
    for (int k = 0; k < n_kinds; k++) fill[k] = base[k];
    m.h_ql.resize(n), m.h_tl.resize(n);
    for (size_t i = 0; i < n; i++) {
        const uint32_t at = fill[h_kind[i]]++;
        m.h_idx[at] = (uint32_t)i;
        m.h_ql[at] = b->h_q_len[i];
        m.h_tl[at] = b->h_t_len[i];
    }

    /* device views of the kind-major arrays */
    const size_t cap = m.cap;
    uint32_t *d_idx = m.d, *s_q_off = m.d + cap, *s_t_off = m.d + 2 * cap, *s_q_len = m.d + 3 * cap;
    uint32_t *s_t_len = m.d + 4 * cap, *s_seed = m.d + 5 * cap;
    int32_t *sub[MIX_OUTS];
    for (int k = 0; k < MIX_OUTS; k++) sub[k] = (int32_t *)(m.d + (6 + k) * cap);
    uint8_t *s_q_op = m.d_ops, *s_t_op = m.d_ops + cap;
    int32_t *outs[MIX_OUTS] = {o->score, o->q_end, o->t_end, o->q_start, o->t_start,
                               o->score2, o->q_end2, o->t_end2, (int32_t *)o->n_cigar};

    /* pack once and gather on the caller's stream, then plan and enqueue the
     * kinds one by one: a kind's planning may wait for its own buffers from
     * the previous call (a traceback kind's tile offsets), and the kinds
     * already enqueued keep the GPU busy meanwhile */
#define GB_MIX_CUDA(call)                                                                                  \
    do {                                                                                                   \
        if ((call) != cudaSuccess) return GB_ERR_CUDA;                                                     \
    } while (0)
    GB_MIX_CUDA(launch_pack(b->q, b->q_bytes, b->pq, s));
    GB_MIX_CUDA(launch_pack(b->t, b->t_bytes, b->pt, s));
    GB_MIX_CUDA(cudaMemcpyAsync(d_idx, m.h_idx, n * 4, cudaMemcpyHostToDevice, s));
    GB_MIX_CUDA(cudaEventRecord(m.idx_free, s));
    MixArgs a{};
    a.idx = d_idx, a.n = (int32_t)n;
    a.q_off = b->q_off, a.t_off = b->t_off, a.q_len = b->q_len, a.t_len = b->t_len, a.seed = b->seed;
    a.q_op = b->q_op, a.t_op = b->t_op;
    a.s_q_off = s_q_off, a.s_t_off = s_t_off, a.s_q_len = s_q_len, a.s_t_len = s_t_len, a.s_seed = s_seed;
    a.s_q_op = s_q_op, a.s_t_op = s_t_op;
    for (int k = 0; k < MIX_OUTS; k++) a.out[k] = outs[k], a.sub[k] = sub[k];
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)sms * 8);
    mix_gather_kernel<<<blocks, 256, 0, s>>>(a);
    GB_MIX_CUDA(cudaGetLastError());
    GB_MIX_CUDA(cudaEventRecord(m.fork, s));
    for (int k = 0; k < n_kinds; k++) {
        if (!counts[k]) continue;
        RunCfg cfg;
        mix_cfg(kinds[k], cfg);
        const uint32_t b0 = base[k];
        DevBatch x{};
        x.n = (int32_t)counts[k], x.q_bytes = b->q_bytes, x.t_bytes = b->t_bytes;
        x.q = b->q, x.t = b->t, x.pq = b->pq, x.pt = b->pt;
        x.q_off = s_q_off + b0, x.t_off = s_t_off + b0, x.q_len = s_q_len + b0, x.t_len = s_t_len + b0;
        x.seed = b->seed ? s_seed + b0 : nullptr;
        x.q_op = b->q_op ? s_q_op + b0 : nullptr;
        x.t_op = b->t_op ? s_t_op + b0 : nullptr;
        x.h_q_len = m.h_ql.data() + b0, x.h_t_len = m.h_tl.data() + b0;
        DevOut y{};
        auto sh = [&](int j) { return outs[j] ? sub[j] + b0 : nullptr; };
        y.score = sh(0), y.q_end = sh(1), y.t_end = sh(2), y.q_start = sh(3), y.t_start = sh(4);
        y.score2 = sh(5), y.q_end2 = sh(6), y.t_end2 = sh(7);
        y.n_cigar = o->n_cigar ? (uint32_t *)sub[8] + b0 : nullptr;
        y.cigar = o->cigar;
        Plan plan;
        if ((rc = plan_batch(cfg, x, y, m.ws[k], plan, m.ks[k])) != GB_OK) return rc;
        GB_MIX_CUDA(cudaStreamWaitEvent(m.ks[k], m.fork, 0));
        if ((rc = enqueue_batch(cfg, x, y, m.ws[k], plan, m.ks[k])) != GB_OK) return rc;
        if (plan.tb) GB_MIX_CUDA(cudaEventRecord(m.ws[k].tb_off_free, m.ks[k]));
        GB_MIX_CUDA(cudaEventRecord(m.join[k], m.ks[k]));
        GB_MIX_CUDA(cudaStreamWaitEvent(s, m.join[k], 0));
    }
    mix_scatter_kernel<<<blocks, 256, 0, s>>>(a);
    GB_MIX_CUDA(cudaGetLastError());
#undef GB_MIX_CUDA
    return GB_OK;
}
