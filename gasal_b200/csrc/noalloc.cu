/*
 * noalloc.cu -- an alignment entry point that allocates no memory.
 *
 * Some callers cannot call cudaMalloc: code running inside a CUDA stream
 * capture that must not add allocation nodes, processes whose device memory
 * is owned by a pool or arena they must not bypass, and plugins loaded into a
 * host application that forbids device allocations from third-party code.
 * gb_align_dev_noalloc serves them.  The caller passes every input and output
 * buffer; the only scratch the DP kernel needs -- one 32-bit row-buffer word
 * per query column per thread -- lives in the file-scope device array below,
 * which every GPU that loads this library holds until the process exits.
 *
 * Limit: NOALLOC_SCRATCH_WORDS words (32 MiB).  A launch uses
 * (threads x columns) words, columns = longest padded query (2 x (query+2)
 * for ksw); the grid is shrunk to fit, and a batch whose longest query needs
 * more than the array can give 32 threads is rejected with GB_ERR_LIMIT.
 * Traceback (WITH_TB) needs tile storage and is rejected with GB_ERR_ARG.
 *
 * The array is shared by every call and keeps the last call's contents; the
 * kernel writes each pair's row buffer before reading it, so nothing needs
 * clearing between calls.  Calls whose work overlaps on the GPU (two streams,
 * or two host threads) race on the array: serialise them.
 *
 * The first call in a device's context resolves the array's device address
 * with cudaGetSymbolAddress while that device is current (again after a
 * cudaDeviceReset, which gives the device a new context); make that first call
 * before any stream capture.  An empty batch (n == 0) returns GB_OK and
 * launches nothing.
 */
#include "engine.h"

#include <cuda.h>
#include <mutex>
#include <unordered_map>

namespace gb {

constexpr size_t NOALLOC_SCRATCH_WORDS = (size_t)8 << 20;

static __device__ __align__(256) uint32_t g_noalloc_scratch[NOALLOC_SCRATCH_WORDS];

namespace {

/* The array's device address belongs to the context the library's module
 * was loaded into: a cudaDeviceReset (or any teardown of the primary context)
 * loads the module again, possibly at another address.  The cache is
 * therefore keyed on the driver's context id, which is unique for the life of
 * the process, and an address is never reused across contexts. */
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

std::mutex g_addr_mu;
std::unordered_map<unsigned long long, uint32_t *> g_addr;

bool current_context_id(unsigned long long *id)
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
        cudaGetLastError();
    });
    CUcontext ctx = nullptr;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

/* Device address of g_noalloc_scratch in the current device's context (the
 * host-side symbol is only a stand-in; kernels must be given this address).
 * Resolved with cudaGetSymbolAddress once per context; when the context id
 * cannot be read the address is resolved on every call. */
int scratch_address(uint32_t **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return GB_ERR_CUDA;
    }
    unsigned long long id = 0;
    bool keyed = current_context_id(&id);
    if (keyed) {
        std::lock_guard<std::mutex> lk(g_addr_mu);
        auto it = g_addr.find(id);
        if (it != g_addr.end()) {
            *out = it->second;
            return GB_OK;
        }
    }
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
        cudaGetLastError();
        return GB_ERR_CUDA;
    }
    if (!keyed) keyed = current_context_id(&id); /* the lookup above made the context current */
    if (keyed) {
        std::lock_guard<std::mutex> lk(g_addr_mu);
        g_addr[id] = static_cast<uint32_t *>(p);
    }
    *out = static_cast<uint32_t *>(p);
    return GB_OK;
}
} // namespace

} // namespace gb

extern "C" int gb_align_dev_noalloc(const gb_params_t *p, const gb_dev_batch_t *b, const gb_dev_out_t *o,
                                    void *stream)
{
    using namespace gb;
    if (!p || !b || !o || b->n < 0) return GB_ERR_ARG;
    if (b->n == 0) return GB_OK; /* an empty batch: nothing to launch */
    if (!b->h_q_len || !b->h_t_len || !b->pq || !b->pt) return GB_ERR_ARG;
    if (p->algo != LOCAL_ && p->algo != GLOBAL_ && p->algo != SEMI_GLOBAL_ && p->algo != BANDED_ && p->algo != KSW_)
        return GB_ERR_ARG;
    if (p->start_pos == WITH_TB_ && (p->algo == LOCAL_ || p->algo == GLOBAL_)) return GB_ERR_ARG;
    uint32_t *scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc != GB_OK) return rc;

    uint32_t max_q = 0;
    for (int i = 0; i < b->n; i++) max_q = max_q > b->h_q_len[i] ? max_q : b->h_q_len[i];
    const size_t cols = p->algo == KSW_ ? 2 * ((size_t)max_q + 2) : (size_t)((max_q + 7) & ~7u);
    if (cols == 0) return GB_ERR_ARG;
    const int block = 64;
    const size_t fit_threads = NOALLOC_SCRATCH_WORDS / cols;
    if (fit_threads < 32) return GB_ERR_LIMIT;
    int blocks = (int)((fit_threads / block) > 0 ? (fit_threads / block) : 0);
    const int need = (b->n + block - 1) / block;
    const int resident = dp_scratch_blocks(b->n, block);
    if (blocks > need) blocks = need;
    if (blocks > resident) blocks = resident;
    int use_block = block;
    if (blocks == 0) { /* fewer than 64 threads fit: one block of 32 */
        use_block = 32;
        blocks = 1;
    }

    cudaStream_t s = (cudaStream_t)stream;
    if (launch_pack(b->q, b->q_bytes, b->pq, s) != cudaSuccess) return GB_ERR_CUDA;
    if (launch_pack(b->t, b->t_bytes, b->pt, s) != cudaSuccess) return GB_ERR_CUDA;
    if (p->reverse_complement &&
        launch_revcomp(b->pq, b->pt, b->q_off, b->t_off, b->q_len, b->t_len, b->q_op, b->t_op, b->n,
                       settings().ref_reverse, s) != cudaSuccess)
        return GB_ERR_CUDA;

    DpArgs a{};
    a.pq = b->pq, a.pt = b->pt, a.q_off = b->q_off, a.t_off = b->t_off, a.q_len = b->q_len, a.t_len = b->t_len;
    a.seed = b->seed, a.order = nullptr, a.n = b->n;
    a.score = o->score, a.q_end = o->q_end, a.t_end = o->t_end, a.q_start = o->q_start, a.t_start = o->t_start;
    a.score2 = o->score2, a.q_end2 = o->q_end2, a.t_end2 = o->t_end2;
    a.sc = {p->match, p->mismatch, p->gap_open, p->gap_extend, p->gap_open + p->gap_extend};
    a.head = p->head, a.tail = p->tail, a.k_band = p->k_band, a.zdrop = p->zdrop, a.mql = settings().mql;
    a.smem_cols = 0;
    a.scratch = scratch;
    a.scratch_cols = (uint32_t)cols;
    const int start = (p->algo == SEMI_GLOBAL_ && p->start_pos == WITH_TB_) ? WITHOUT_START_ : p->start_pos;
    const bool second = p->second_best && (p->algo == LOCAL_ || p->algo == SEMI_GLOBAL_);
    if (launch_dp_scratch_grid(p->algo, start, second, a, use_block, blocks, s) != cudaSuccess) return GB_ERR_CUDA;
    return GB_OK;
}
