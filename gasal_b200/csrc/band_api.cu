/*
 * band_api.cu -- C entry points of the learned ksw band (no reference
 * counterpart): the band model (MLP parameters, Adam state), pair features,
 * prediction, gradients, a training step, and banded alignment with its
 * certificate and exact fallback.
 */
#include "gasal_header.h"
#include "gasal_b200_capi.h"
#include "engine.h"
#include "mlband.h"

#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <unordered_map>
#include <vector>

struct gb_band_model {
    float *w = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *loss = nullptr;
    __nv_bfloat16 *wb = nullptr;
    int step = 0;
    int device = 0;
};

namespace {
constexpr int IN = gb::BAND_FEATS, H = gb::MLP_HIDDEN;

/* He-uniform initialisation on the host; biases zero except the output's */
std::vector<float> init_params(uint64_t seed)
{
    std::vector<float> p(gb::MLP_PARAMS, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int rows, int cols) {
        const float a = std::sqrt(6.f / (float)cols);
        std::uniform_real_distribution<float> u(-a, a);
        for (int i = 0; i < rows * cols; i++) p[off + i] = u(rng);
    };
    int off = 0;
    fill(off, H, IN), off += H * IN + H;
    fill(off, H, H), off += H * H + H;
    fill(off, 1, H), off += H;
    p[off] = 6.f; /* start near a 64-column band */
    return p;
}

struct DevWs {
    gb::Workspace ws;
};
std::mutex g_mu;
std::unordered_map<unsigned long long, DevWs *> g_ws;
DevWs *band_ws(void *stream)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    const unsigned long long key = ((unsigned long long)(uintptr_t)stream << 8) ^ (unsigned long long)dev;
    DevWs *&slot = g_ws[key];
    if (!slot) slot = new DevWs();
    return slot;
}
} // namespace

namespace gb {
/* the band entry points' per-stream workspaces (gb_release_workspaces) */
void band_release_all()
{
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto &kv : g_ws) {
        release_workspace(kv.second->ws);
        delete kv.second;
    }
    g_ws.clear();
}
} // namespace gb

extern "C" {

int gb_band_param_count(void) { return gb::MLP_PARAMS; }
int gb_band_feature_stride(void) { return gb::BAND_FEATS_PAD; }

gb_band_model_t *gb_band_model_new(uint64_t seed)
{
    gb_band_model_t *m = new gb_band_model_t();
    cudaGetDevice(&m->device);
    const size_t nb = (size_t)gb::MLP_PARAMS * sizeof(float);
    if (cudaMalloc((void **)&m->w, nb) != cudaSuccess || cudaMalloc((void **)&m->m, nb) != cudaSuccess ||
        cudaMalloc((void **)&m->v, nb) != cudaSuccess || cudaMalloc((void **)&m->grad, nb) != cudaSuccess ||
        cudaMalloc((void **)&m->loss, sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&m->wb, (size_t)gb::MLP_PARAMS * sizeof(__nv_bfloat16)) != cudaSuccess) {
        cudaGetLastError();
        gb_band_model_free(m);
        return nullptr;
    }
    const std::vector<float> p = init_params(seed);
    if (cudaMemcpy(m->w, p.data(), nb, cudaMemcpyHostToDevice) != cudaSuccess || cudaMemset(m->m, 0, nb) != cudaSuccess ||
        cudaMemset(m->v, 0, nb) != cudaSuccess || gb::launch_to_bf16(m->w, m->wb, 0) != cudaSuccess ||
        cudaDeviceSynchronize() != cudaSuccess) {
        cudaGetLastError();
        gb_band_model_free(m);
        return nullptr;
    }
    return m;
}

void gb_band_model_free(gb_band_model_t *m)
{
    if (!m) return;
    if (gb::settings().band_model == m->wb) gb::settings().band_model = nullptr;
    cudaFree(m->w), cudaFree(m->m), cudaFree(m->v), cudaFree(m->grad), cudaFree(m->loss), cudaFree(m->wb);
    delete m;
}

int gb_band_model_params(gb_band_model_t *m, float *out, const float *in)
{
    if (!m) return GB_ERR_ARG;
    const size_t nb = (size_t)gb::MLP_PARAMS * sizeof(float);
    if (out && cudaMemcpy(out, m->w, nb, cudaMemcpyDeviceToHost) != cudaSuccess) return GB_ERR_CUDA;
    if (in) {
        if (cudaMemcpy(m->w, in, nb, cudaMemcpyHostToDevice) != cudaSuccess) return GB_ERR_CUDA;
        if (gb::launch_to_bf16(m->w, m->wb, 0) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
            return GB_ERR_CUDA;
    }
    return GB_OK;
}

int gb_band_features(const gb_dev_batch_t *b, float *feat, void *stream)
{
    if (!b || !feat || b->n <= 0 || !b->pq || !b->pt) return GB_ERR_ARG;
    const cudaStream_t s = (cudaStream_t)stream;
    if (b->q && gb::launch_pack(b->q, b->q_bytes, b->pq, s) != cudaSuccess) return GB_ERR_CUDA;
    if (b->t && gb::launch_pack(b->t, b->t_bytes, b->pt, s) != cudaSuccess) return GB_ERR_CUDA;
    return gb::launch_band_features(b->pq, b->pt, b->q_off, b->t_off, b->q_len, b->t_len, b->n, feat, s) == cudaSuccess
               ? GB_OK
               : GB_ERR_CUDA;
}

int gb_band_predict(gb_band_model_t *m, const float *feat, int n, float *out, void *stream)
{
    if (!m || !feat || !out || n <= 0) return GB_ERR_ARG;
    return gb::launch_mlp_forward(m->wb, feat, n, out, (cudaStream_t)stream) == cudaSuccess ? GB_OK : GB_ERR_CUDA;
}

int gb_band_grad(gb_band_model_t *m, const float *feat, const float *label, int n, float tau, float *grad, float *loss,
                 void *stream)
{
    if (!m || !feat || !label || !grad || !loss || n <= 0) return GB_ERR_ARG;
    return gb::launch_mlp_grad(m->w, feat, label, n, tau, grad, loss, (cudaStream_t)stream) == cudaSuccess
               ? GB_OK
               : GB_ERR_CUDA;
}

int gb_band_train_step(gb_band_model_t *m, const float *feat, const float *label, int n, float tau, float lr,
                       void *stream, float *loss)
{
    if (!m || !feat || !label || n <= 0) return GB_ERR_ARG;
    const cudaStream_t s = (cudaStream_t)stream;
    if (gb::launch_mlp_grad(m->w, feat, label, n, tau, m->grad, m->loss, s) != cudaSuccess) return GB_ERR_CUDA;
    m->step++;
    if (gb::launch_mlp_adam(m->w, m->m, m->v, m->grad, m->wb, lr, m->step, s) != cudaSuccess) return GB_ERR_CUDA;
    if (loss) {
        if (cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return GB_ERR_CUDA;
        *loss /= (float)n;
    }
    return GB_OK;
}

int gb_set_band_model(gb_band_model_t *m, int band_min, int band_max)
{
    gb::Settings &st = gb::settings();
    if (!m) {
        st.band_model = nullptr;
        return GB_OK;
    }
    if (band_min < 0 || band_max < band_min) return GB_ERR_ARG;
    st.band_model = m->wb, st.band_min = band_min, st.band_max = band_max;
    return GB_OK;
}

int gb_ksw_band_align(const gb_params_t *p, const gb_dev_batch_t *b, const gb_dev_out_t *o, const int32_t *band_w,
                      uint8_t *band_ok, void *stream, gb_band_stats_t *stats)
{
    if (!p || !b || !o || b->n <= 0 || !b->h_q_len || !b->h_t_len || p->algo != KSW) return GB_ERR_ARG;
    const gb::Settings &set = gb::settings();
    if (!band_w && !set.band_model) return GB_ERR_ARG;
    if (!gb::ksw_wc_scores_ok(gb::Scores{p->match, p->mismatch, p->gap_open, p->gap_extend, p->gap_open + p->gap_extend}) ||
        !set.ksw_wc)
        return GB_ERR_ARG;
    DevWs *w = band_ws(stream);
    if (!w) return GB_ERR_CUDA;
    gb::RunCfg cfg{};
    cfg.algo = p->algo, cfg.start = p->start_pos, cfg.second = 0, cfg.head = p->head, cfg.tail = p->tail;
    cfg.k_band = p->k_band, cfg.zdrop = p->zdrop;
    cfg.sc = {p->match, p->mismatch, p->gap_open, p->gap_extend, p->gap_open + p->gap_extend};
    cfg.ref_reverse = set.ref_reverse, cfg.mql = set.mql, cfg.is_packed = 0;
    cfg.reverse_complement = p->reverse_complement;
    cfg.band_w = band_w;
    cfg.band_model = band_w ? nullptr : set.band_model;
    cfg.band_min = set.band_min, cfg.band_max = set.band_max;
    cfg.band_ok = band_ok;
    gb::DevBatch db{};
    db.n = b->n, db.q_bytes = b->q_bytes, db.t_bytes = b->t_bytes, db.q = b->q, db.t = b->t;
    db.pq = b->pq, db.pt = b->pt, db.q_off = b->q_off, db.t_off = b->t_off, db.q_len = b->q_len;
    db.t_len = b->t_len, db.q_op = b->q_op, db.t_op = b->t_op, db.seed = b->seed;
    db.h_q_len = b->h_q_len, db.h_t_len = b->h_t_len;
    gb::DevOut dout{};
    dout.score = o->score, dout.q_end = o->q_end, dout.t_end = o->t_end;
    const int rc = gb::run_batch(cfg, db, dout, w->ws, (cudaStream_t)stream);
    if (rc != GB_OK || !stats) return rc;
    uint32_t q[8];
    if (cudaMemcpyAsync(q, w->ws.queue, sizeof q, cudaMemcpyDeviceToHost, (cudaStream_t)stream) != cudaSuccess ||
        cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
        return GB_ERR_CUDA;
    unsigned long long cells;
    std::memcpy(&cells, q + 4, sizeof cells);
    stats->pairs = b->n;
    stats->retried = q[3];
    stats->handed_back = q[2];
    stats->accepted = (int64_t)b->n - q[3] - q[2];
    stats->cells = (int64_t)cells;
    return GB_OK;
}

/* Unbanded ksw (the plain computation every banded result must equal) with
 * one more output per pair: max_off, the largest |column - row| over the cells
 * where the running maximum rose (ksw_extend2's max_off), the diagonal reach
 * the alignment needed -- the band labels' source. */
int gb_ksw_align_max_off(const gb_params_t *p, const gb_dev_batch_t *b, const gb_dev_out_t *o, int32_t *max_off,
                         void *stream)
{
    if (!p || !b || !o || !max_off || b->n <= 0 || !b->h_q_len || !b->h_t_len || p->algo != KSW) return GB_ERR_ARG;
    DevWs *w = band_ws(stream);
    if (!w) return GB_ERR_CUDA;
    const gb::Settings &set = gb::settings();
    gb::RunCfg cfg{};
    cfg.algo = p->algo, cfg.start = p->start_pos, cfg.second = 0, cfg.head = p->head, cfg.tail = p->tail;
    cfg.k_band = p->k_band, cfg.zdrop = p->zdrop;
    cfg.sc = {p->match, p->mismatch, p->gap_open, p->gap_extend, p->gap_open + p->gap_extend};
    cfg.ref_reverse = set.ref_reverse, cfg.mql = set.mql, cfg.is_packed = 0;
    cfg.reverse_complement = p->reverse_complement;
    cfg.band_w = nullptr, cfg.band_model = nullptr; /* unbanded, whatever model is installed */
    gb::DevBatch db{};
    db.n = b->n, db.q_bytes = b->q_bytes, db.t_bytes = b->t_bytes, db.q = b->q, db.t = b->t;
    db.pq = b->pq, db.pt = b->pt, db.q_off = b->q_off, db.t_off = b->t_off, db.q_len = b->q_len;
    db.t_len = b->t_len, db.q_op = b->q_op, db.t_op = b->t_op, db.seed = b->seed;
    db.h_q_len = b->h_q_len, db.h_t_len = b->h_t_len;
    gb::DevOut dout{};
    dout.score = o->score, dout.q_end = o->q_end, dout.t_end = o->t_end;
    dout.max_off = max_off;
    return gb::run_batch(cfg, db, dout, w->ws, (cudaStream_t)stream);
}

} // extern "C"
