/*
 * api_host.cpp -- GASAL2's C++ API, re-implemented for the B200 engine.
 *
 * Same functions, signatures, buffer ownership and observable behaviour as the
 * reference (src/ctors.cpp, src/res.cpp, src/host_batch.cpp,
 * src/interfaces.cpp, src/args_parser.cpp, src/gasal_align.cu:29-339):
 * which result arrays exist, how host pages chain, which warnings print, and
 * that errors print "[GASAL ...]" and terminate the process.  The device work
 * of gasal_aln_async is gb::run_batch.  Per-stream engine state that has no
 * place in gasal_gpu_storage_t (traceback tiles, row-buffer scratch, n_cigar)
 * lives in a side table keyed by the storage address, so the struct layout is
 * the reference's.
 */
#include "gasal_header.h"
#include "res.h"
#include "gasal_b200_capi.h"
#include "engine.h"

#include <cmath>
#include <cstring>
#include <memory>
#include <atomic>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include <unordered_map>

/* ========================= Parameters =================================== */

Parameters::Parameters(int argc_, char **argv_)
{
    sa = 1;
    sb = 4;
    gapo = 6;
    gape = 1;
    start_pos = WITHOUT_START;
    print_out = 0;
    n_threads = 1;
    k_band = 0;
    isPacked = false;
    isReverseComplement = false;
    secondBest = FALSE;
    semiglobal_skipping_head = TARGET;
    semiglobal_skipping_tail = TARGET;
    algo = UNKNOWN;
    query_batch_fasta_filename = "";
    target_batch_fasta_filename = "";
    argc = argc_;
    argv = argv_;
}

Parameters::~Parameters()
{
    query_batch_fasta.close();
    target_batch_fasta.close();
}

/* The CLI members exist so that callers such as the reference's test program
 * link unchanged; the option grammar is the one that program relies on (flags
 * before the two FASTA names, -x taking a head and a tail keyword). */

void Parameters::print()
{
    std::cerr << "[gasal_b200] algo " << algo << ", start " << start_pos << ", scores " << sa << '/' << sb << '/'
              << gapo << '/' << gape << ", second-best " << secondBest << ", semi-global skip " << semiglobal_skipping_head
              << '/' << semiglobal_skipping_tail << ", threads " << n_threads << ", band " << k_band << ", files "
              << query_batch_fasta_filename << ' ' << target_batch_fasta_filename << std::endl;
}

void Parameters::failure(fail_type f)
{
    static const char *const why[] = {"too few arguments", "too many arguments", "unknown or malformed option",
                                      "cannot open an input file", "unknown alignment type"};
    const int k = (int)f;
    std::cerr << "[gasal_b200] " << (k >= 0 && k < 5 ? why[k] : "bad arguments") << "; -h lists the options"
              << std::endl;
    exit(1);
}

void Parameters::help()
{
    std::cerr << "usage: <program> [options] <query.fasta> <target.fasta>\n"
                 "  -y local|global|semi_global|ksw   alignment type\n"
                 "  -a/-b/-q/-r N                     match, mismatch, gap open, gap extend ("
              << sa << '/' << sb << '/' << gapo << '/' << gape
              << ")\n"
                 "  -s | -t                           start positions | traceback\n"
                 "  -x HEAD TAIL                      semi-global skipped ends: NONE QUERY TARGET BOTH\n"
                 "  -k N  -n N  -p  --second-best     band width, threads, print results, second best\n";
}

namespace {

bool skip_keyword(const char *s, data_source *out)
{
    static const struct { const char *name; data_source v; } kw[] = {
        {"NONE", NONE}, {"QUERY", QUERY}, {"TARGET", TARGET}, {"BOTH", BOTH}};
    for (const auto &k : kw)
        if (std::strcmp(s, k.name) == 0) {
            *out = k.v;
            return true;
        }
    return false;
}

} // namespace

void Parameters::parse()
{
    for (int k = 1; k < argc; k++)
        if (!std::strcmp(argv[k], "-h") || !std::strcmp(argv[k], "--help")) {
            help();
            exit(0);
        }
    if (argc < 4) failure(NOT_ENOUGH_ARGS);

    /* integer-valued flags and where they land */
    struct IntFlag { char flag; int32_t Parameters::*field; };
    static const IntFlag ints[] = {{'a', &Parameters::sa},   {'b', &Parameters::sb},
                                   {'q', &Parameters::gapo}, {'r', &Parameters::gape},
                                   {'n', &Parameters::n_threads}, {'k', &Parameters::k_band}};
    const int last_opt = argc - 2; /* the final two words are the FASTA files */
    int k = 1;
    auto value = [&]() -> const char * { return argv[++k]; };
    for (; k < last_opt; k++) {
        const char *w = argv[k];
        if (w[0] != '-') failure(WRONG_ARG);
        if (w[1] == '-') { /* long options: only --second-best means anything */
            if (!std::strcmp(w, "--second-best")) secondBest = TRUE;
            continue;
        }
        if (w[1] == '\0' || w[2] != '\0') failure(WRONG_ARG);
        const char f = w[1];
        bool done = false;
        for (const IntFlag &x : ints)
            if (x.flag == f) {
                this->*(x.field) = std::stoi(value());
                done = true;
            }
        if (done) continue;
        switch (f) {
        case 'y': {
            static const struct { const char *name; algo_type a; } algos[] = {
                {"local", LOCAL}, {"global", GLOBAL}, {"semi_global", SEMI_GLOBAL}, {"ksw", KSW}};
            const char *v = value();
            for (const auto &x : algos)
                if (!std::strcmp(v, x.name)) algo = x.a;
            break;
        }
        case 's': start_pos = WITH_START; break;
        case 't': start_pos = WITH_TB; break;
        case 'p': print_out = 1; break;
        case 'x':
            if (!skip_keyword(value(), &semiglobal_skipping_head)) failure(WRONG_ARG);
            if (!skip_keyword(value(), &semiglobal_skipping_tail)) failure(WRONG_ARG);
            break;
        default: break; /* other single-letter flags are ignored */
        }
    }
    query_batch_fasta_filename = argv[k];
    target_batch_fasta_filename = argv[k + 1];
    fileopen();
}

void Parameters::fileopen()
{
    query_batch_fasta.open(query_batch_fasta_filename, std::ifstream::in);
    if (!query_batch_fasta) failure(WRONG_FILES);
    target_batch_fasta.open(target_batch_fasta_filename);
    if (!target_batch_fasta) failure(WRONG_FILES);
}

/* ========================= helpers ====================================== */

#define GB_FATAL_CUDA(call)                                                                              \
    do {                                                                                                 \
        cudaError_t err_ = (call);                                                                       \
        if (cudaSuccess != err_) {                                                                       \
            fprintf(stderr, "[GASAL CUDA ERROR:] %s(CUDA error no.=%d). Line no. %d in file %s\n",       \
                    cudaGetErrorString(err_), err_, __LINE__, __FILE__);                                 \
            exit(EXIT_FAILURE);                                                                          \
        }                                                                                                \
    } while (0)

namespace {

struct StreamState {
    gb::Workspace ws;
    uint32_t *d_n_cigar = nullptr;
    size_t n_cigar_cap = 0;
    cudaGraphExec_t exec = nullptr; /* the storage's batch graph */
    std::vector<uint8_t> sig;       /* what `exec` was captured for */
};

std::mutex g_mu;
std::unordered_map<const gasal_gpu_storage_t *, std::unique_ptr<StreamState>> g_state;

StreamState &state_of(const gasal_gpu_storage_t *s)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto &p = g_state[s];
    if (!p) p.reset(new StreamState());
    return *p;
}

void release_state(const gasal_gpu_storage_t *s)
{
    std::unique_ptr<StreamState> p;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_state.find(s);
        if (it == g_state.end()) return;
        p = std::move(it->second);
        g_state.erase(it);
    }
    gb::release_workspace(p->ws);
    if (p->d_n_cigar) cudaFree(p->d_n_cigar);
    if (p->exec) cudaGraphExecDestroy(p->exec);
}

/* graph statistics: 0 relaunched, 1 captured and updated in place,
 * 2 captured and instantiated, 3 capture failed (ran without a graph) */
std::atomic<int64_t> g_graph_stats[4];
void graph_stat(int k) { g_graph_stats[k].fetch_add(1, std::memory_order_relaxed); }

template <class T> void put(std::vector<uint8_t> &v, const T &x)
{
    const uint8_t *p = reinterpret_cast<const uint8_t *>(&x);
    v.insert(v.end(), p, p + sizeof(T));
}

/* Everything a captured batch graph depends on except the contents of the
 * buffers it copies: sizes, options, every pointer the copies and kernels
 * take (host pages included), and the engine plan. */
void batch_signature(std::vector<uint8_t> &v, const gasal_gpu_storage_t *s, const StreamState &ss,
                     const Parameters *params, uint32_t n, uint32_t qbytes, uint32_t tbytes, const gb::RunCfg &cfg,
                     const gb::Plan &plan)
{
    v.clear();
    v.reserve(1024);
    int dev = -1;
    cudaGetDevice(&dev);
    put(v, dev), put(v, n), put(v, qbytes), put(v, tbytes);
    put(v, params->algo), put(v, params->start_pos), put(v, params->secondBest), put(v, params->isPacked);
    put(v, params->isReverseComplement), put(v, params->k_band);
    put(v, params->semiglobal_skipping_head), put(v, params->semiglobal_skipping_tail);
    put(v, cfg.sc), put(v, cfg.ref_reverse), put(v, cfg.mql), put(v, cfg.zdrop);
    for (const host_batch_t *p = s->extensible_host_unpacked_query_batch; p; p = p->next)
        put(v, (const void *)p->data), put(v, p->offset), put(v, p->data_size);
    put(v, -1);
    for (const host_batch_t *p = s->extensible_host_unpacked_target_batch; p; p = p->next)
        put(v, (const void *)p->data), put(v, p->offset), put(v, p->data_size);
    put(v, -1);
    const void *ptrs[] = {s->unpacked_query_batch, s->unpacked_target_batch, s->packed_query_batch,
                          s->packed_target_batch, s->query_batch_offsets, s->target_batch_offsets,
                          s->query_batch_lens, s->target_batch_lens, s->query_op, s->target_op, s->seed_scores,
                          s->host_query_batch_lens, s->host_target_batch_lens, s->host_query_batch_offsets,
                          s->host_target_batch_offsets, s->host_query_op, s->host_target_op, s->host_seed_scores,
                          ss.d_n_cigar, ss.ws.tb, ss.ws.d_tb_off, ss.ws.h_tb_off, ss.ws.order, ss.ws.bins,
                          ss.ws.queue, ss.ws.aux, ss.ws.fork, ss.ws.join, ss.ws.fb, ss.ws.retry, ss.ws.wc_defer, ss.ws.feat, ss.ws.order2,
                          ss.ws.pred, ss.ws.bandw, (const void *)s->str};
    for (const void *q : ptrs) put(v, q);
    const gasal_res_t *rs[] = {s->host_res, s->device_cpy, s->host_res_second, s->device_cpy_second};
    for (const gasal_res_t *r : rs) {
        put(v, (const void *)r);
        if (!r) continue;
        put(v, (const void *)r->aln_score), put(v, (const void *)r->query_batch_start);
        put(v, (const void *)r->target_batch_start), put(v, (const void *)r->query_batch_end);
        put(v, (const void *)r->target_batch_end), put(v, (const void *)r->cigar);
        put(v, (const void *)r->n_cigar_ops);
    }
    put(v, plan.tb), put(v, plan.second), put(v, plan.use_wc), put(v, plan.order_on);
    put(v, plan.start), put(v, plan.block), put(v, plan.mq8), put(v, plan.mt8), put(v, plan.wc_min_q);
    put(v, plan.ksw_slots), put(v, plan.fb_blocks), put(v, plan.band), put(v, plan.ksw_short);
    put(v, plan.tier2), put(v, plan.tier_q), put(v, plan.tier2_cols), put(v, plan.tier2_blocks);
    put(v, plan.split_start), put(v, plan.wc), put(v, plan.wc_big), put(v, plan.mq8_big);
    put(v, plan.mt8_big), put(v, (const void *)ss.ws.wc_rows);
    put(v, (const void *)cfg.band_w), put(v, cfg.band_model), put(v, cfg.band_min), put(v, cfg.band_max);
    put(v, (const void *)cfg.band_ok);
    put(v, plan.a);
    for (int c : plan.cut) put(v, c);
    put(v, -1);
    for (int c : plan.nlong) put(v, c);
    put(v, -1);
    for (int c : plan.nbig) put(v, c);
}

/* Captures issue() on stream st into a graph, updates (or instantiates) the
 * storage's executable graph from it, and launches that.  When the capture
 * itself is refused, issue() runs again without a graph. */
template <class F> cudaError_t capture_and_launch(StreamState &ss, F &issue, cudaStream_t st)
{
    cudaError_t ce = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        graph_stat(3);
        return issue();
    }
    const cudaError_t ie = issue();
    cudaGraph_t g = nullptr;
    ce = cudaStreamEndCapture(st, &g);
    if (ie != cudaSuccess || ce != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (ss.exec) cudaGraphExecDestroy(ss.exec);
        ss.exec = nullptr;
        graph_stat(3);
        if (ie != cudaSuccess) return ie; /* a failure of the operations themselves */
        return issue();
    }
    bool updated = false;
    if (ss.exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(ss.exec, g, &info) == cudaSuccess) {
            updated = true;
        } else {
            cudaGetLastError();
            cudaGraphExecDestroy(ss.exec);
            ss.exec = nullptr;
        }
    }
    if (!ss.exec) {
        ce = cudaGraphInstantiate(&ss.exec, g, 0);
        if (ce != cudaSuccess) {
            ss.exec = nullptr;
            cudaGraphDestroy(g);
            return ce;
        }
    }
    cudaGraphDestroy(g);
    graph_stat(updated ? 1 : 2);
    return cudaGraphLaunch(ss.exec, st);
}

uint32_t round8(uint32_t x) { return (x + 7u) & ~7u; }

} // namespace

/* ========================= host batches ================================= */
/* Pinned pages chained into a list; src/host_batch.cpp:11-244. */

host_batch_t *gasal_host_batch_new(uint32_t batch_bytes, uint32_t offset)
{
    host_batch_t *res = (host_batch_t *)calloc(1, sizeof(host_batch_t));
    GB_FATAL_CUDA(cudaHostAlloc(&(res->data), batch_bytes * sizeof(uint8_t), cudaHostAllocDefault));
    res->page_size = batch_bytes;
    res->data_size = 0;
    res->is_locked = 0;
    res->offset = offset;
    res->next = NULL;
    return res;
}

void gasal_host_batch_destroy(host_batch_t *res)
{
    if (res == NULL) {
        fprintf(stderr, "[GASAL ERROR] Trying to free a NULL pointer\n");
        exit(1);
    }
    while (res != NULL) {
        host_batch_t *next = res->next;
        if (res->data != NULL) GB_FATAL_CUDA(cudaFreeHost(res->data));
        free(res);
        res = next;
    }
}

host_batch_t *gasal_host_batch_getlast(host_batch_t *arg)
{
    while (arg->next != NULL) arg = arg->next;
    return arg;
}

void gasal_host_batch_reset(gasal_gpu_storage_t *gpu_storage)
{
    host_batch_t *heads[2] = {gpu_storage->extensible_host_unpacked_query_batch,
                              gpu_storage->extensible_host_unpacked_target_batch};
    for (host_batch_t *p : heads) {
        for (; p != NULL; p = p->next) {
            p->data_size = 0;
            p->offset = 0;
            p->is_locked = 0;
        }
    }
}

namespace {

/* One side's page chain and the storage's running total of its host bytes. */
struct PageChain {
    host_batch_t *head;
    uint32_t *total;
    const char *side;
};

PageChain chain_of(gasal_gpu_storage_t *s, data_source src)
{
    if (src == QUERY) return {s->extensible_host_unpacked_query_batch, &s->host_max_query_batch_bytes, "query"};
    return {s->extensible_host_unpacked_target_batch, &s->host_max_target_batch_bytes, "target"};
}

uint32_t page_room(const host_batch_t *p) { return p->page_size - p->data_size; }

} // namespace

namespace {

/* The page a fill of `need` bytes writes to: the chain's open page (the first
 * one not yet locked).  When that page lacks room, it is locked and the write
 * moves to its successor -- re-based to start where the locked page's data
 * ends -- or, past the last page, to a new page of twice the size (which also
 * grows the storage's host byte total).  The move happens once per call;
 * nullptr when the page reached still lacks room. */
host_batch_t *fill_page(const PageChain &ch, uint32_t need)
{
    host_batch_t *pg = ch.head;
    while (pg->is_locked) pg = pg->next;
    if (page_room(pg) < need) {
        const uint32_t data_end = pg->offset + pg->data_size;
        if (pg->next == NULL) {
            const uint32_t grown = pg->page_size * 2;
            fprintf(stderr,
                    "[GASAL WARNING:] %s pages: %u bytes needed, %u free on the last page; chaining a new page of %u "
                    "bytes (host total %u). Size the storage for the batch to avoid this.\n",
                    ch.side, need, page_room(pg), grown, *ch.total + grown);
            pg->next = gasal_host_batch_new(grown, data_end);
            *ch.total += grown;
        } else {
            pg->next->offset = data_end;
        }
        pg->is_locked = 1;
        pg = pg->next;
    }
    return page_room(pg) < need ? nullptr : pg;
}

/* memcpy split into `threads` contiguous slices of at least 1 MiB, one
 * std::thread each (the calling thread takes the first) */
void copy_parallel(uint8_t *dst, const char *src, size_t n, int threads)
{
    const size_t min_slice = (size_t)1 << 20;
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    size_t parts = std::min<size_t>((size_t)threads, std::max<size_t>(1, n / min_slice));
    if (parts <= 1) {
        memcpy(dst, src, n);
        return;
    }
    const size_t slice = (n + parts - 1) / parts;
    std::vector<std::thread> pool;
    pool.reserve(parts - 1);
    for (size_t k = 1; k < parts; k++) {
        const size_t lo = k * slice, hi = std::min(n, lo + slice);
        if (lo < hi) pool.emplace_back([=] { memcpy(dst + lo, src + lo, hi - lo); });
    }
    memcpy(dst, src, std::min(n, slice));
    for (auto &t : pool) t.join();
}

} // namespace

/* Appends one sequence, N-padded to a multiple of 8, to the chain's open page
 * (fill_page).  Returns the byte index after the written sequence, or `idx`
 * unchanged when even the page moved to lacks room. */
uint32_t gasal_host_batch_fill(gasal_gpu_storage_t *gpu_storage, uint32_t idx, const char *data, uint32_t size,
                               data_source SRC)
{
    const uint32_t need = round8(size);
    host_batch_t *pg = fill_page(chain_of(gpu_storage, SRC), need);
    if (!pg) return idx;
    uint8_t *dst = pg->data + (idx - pg->offset);
    memcpy(dst, data, size);
    memset(dst + size, N_CODE, need - size);
    pg->data_size += need;
    return idx + need;
}

/* gasal_host_batch_fill with the copy split over `threads` host threads (0:
 * every hardware thread): the same page, padding and return value.  Meant
 * for a whole batch staged as one block (sequences already padded to 8 at
 * ascending offsets), where one thread's memcpy bandwidth would otherwise
 * bound the host side of a multi-gigabyte step. */
uint32_t gasal_host_batch_fill_mt(gasal_gpu_storage_t *gpu_storage, uint32_t idx, const char *data, uint32_t size,
                                  data_source SRC, int threads)
{
    const uint32_t need = round8(size);
    host_batch_t *pg = fill_page(chain_of(gpu_storage, SRC), need);
    if (!pg) return idx;
    uint8_t *dst = pg->data + (idx - pg->offset);
    copy_parallel(dst, data, size, threads);
    memset(dst + size, N_CODE, need - size);
    pg->data_size += need;
    return idx + need;
}

uint32_t gasal_host_batch_addbase(gasal_gpu_storage_t *gpu_storage, uint32_t idx, const char base, data_source SRC)
{
    return gasal_host_batch_add(gpu_storage, idx, &base, 1, SRC);
}

/* Writes raw bytes (no padding) at batch index idx into the page that covers
 * [idx, idx + size): walking from the head, the first page with no successor
 * or whose successor starts at or after idx + size.  When the storage's host
 * byte total is below idx + size, the total doubles (until it holds `size`)
 * and a new page of the new total, starting at idx, is hung after the page the
 * walk stands on (in place of any successor). */
uint32_t gasal_host_batch_add(gasal_gpu_storage_t *gpu_storage, uint32_t idx, const char *data, uint32_t size,
                              data_source SRC)
{
    const PageChain ch = chain_of(gpu_storage, SRC);
    const uint32_t stop = idx + size;
    host_batch_t *pg = ch.head;
    while (*ch.total < stop || (pg->next != NULL && pg->next->offset < stop)) {
        if (*ch.total >= stop) {
            pg = pg->next;
            continue;
        }
        const uint32_t before = *ch.total;
        do {
            *ch.total *= 2;
        } while (*ch.total < size);
        fprintf(stderr,
                "[GASAL WARNING:] %s pages: %u bytes at index %u exceed the %u host bytes; chaining a page of %u "
                "bytes. Size the storage for the batch to avoid this.\n",
                ch.side, size, idx, before, *ch.total);
        pg->next = gasal_host_batch_new(*ch.total, idx);
        pg = pg->next;
    }
    memcpy(pg->data + (idx - pg->offset), data, size);
    return stop;
}

void gasal_host_batch_print(host_batch_t *res)
{
    fprintf(stderr, "[GASAL PRINT] Page data: offset=%d, next_offset=%d, data size=%d, page size=%d\n", res->offset,
            (res->next != NULL ? (int)res->next->offset : -1), res->data_size, res->page_size);
}

void gasal_host_batch_printall(host_batch_t *res)
{
    for (; res != NULL; res = res->next) {
        gasal_host_batch_print(res);
        if (res->next != NULL) fprintf(stderr, "+--->");
    }
}

/* ========================= results ====================================== */
/* Which arrays exist: src/res.cpp:8-70 and :106-140. */

gasal_res_t *gasal_res_new_host(uint32_t max_n_alns, Parameters *params)
{
    gasal_res_t *res = (gasal_res_t *)calloc(1, sizeof(gasal_res_t));
    if (res == NULL) {
        fprintf(stderr, "Malloc error on res host ");
        exit(1);
    }
    GB_FATAL_CUDA(cudaHostAlloc(&(res->aln_score), max_n_alns * sizeof(int32_t), cudaHostAllocDefault));
    if (params->algo != GLOBAL) {
        if (params->start_pos == WITH_START || params->start_pos == WITH_TB) {
            GB_FATAL_CUDA(cudaHostAlloc(&(res->query_batch_start), max_n_alns * sizeof(uint32_t), cudaHostAllocDefault));
            GB_FATAL_CUDA(cudaHostAlloc(&(res->target_batch_start), max_n_alns * sizeof(uint32_t), cudaHostAllocDefault));
        }
        GB_FATAL_CUDA(cudaHostAlloc(&(res->query_batch_end), max_n_alns * sizeof(uint32_t), cudaHostAllocDefault));
        GB_FATAL_CUDA(cudaHostAlloc(&(res->target_batch_end), max_n_alns * sizeof(uint32_t), cudaHostAllocDefault));
    }
    if (params->start_pos == WITH_TB)
        GB_FATAL_CUDA(cudaHostAlloc(&(res->n_cigar_ops), max_n_alns * sizeof(uint32_t), cudaHostAllocDefault));
    return res;
}

gasal_res_t *gasal_res_new_device_cpy(uint32_t max_n_alns, Parameters *params)
{
    gasal_res_t *res = (gasal_res_t *)calloc(1, sizeof(gasal_res_t));
    GB_FATAL_CUDA(cudaMalloc(&(res->aln_score), max_n_alns * sizeof(int32_t)));
    if (params->algo != GLOBAL) {
        if (params->start_pos == WITH_START || params->start_pos == WITH_TB) {
            GB_FATAL_CUDA(cudaMalloc(&(res->query_batch_start), max_n_alns * sizeof(uint32_t)));
            GB_FATAL_CUDA(cudaMalloc(&(res->target_batch_start), max_n_alns * sizeof(uint32_t)));
        }
        GB_FATAL_CUDA(cudaMalloc(&(res->query_batch_end), max_n_alns * sizeof(uint32_t)));
        GB_FATAL_CUDA(cudaMalloc(&(res->target_batch_end), max_n_alns * sizeof(uint32_t)));
    }
    return res;
}

gasal_res_t *gasal_res_new_device(gasal_res_t *device_cpy)
{
    gasal_res_t *d_c;
    GB_FATAL_CUDA(cudaMalloc((void **)&d_c, sizeof(gasal_res_t)));
    GB_FATAL_CUDA(cudaMemcpy(d_c, device_cpy, sizeof(gasal_res_t), cudaMemcpyHostToDevice));
    return d_c;
}

void gasal_res_destroy_host(gasal_res_t *res)
{
    if (res == NULL) return;
    if (res->aln_score) GB_FATAL_CUDA(cudaFreeHost(res->aln_score));
    if (res->query_batch_start) GB_FATAL_CUDA(cudaFreeHost(res->query_batch_start));
    if (res->target_batch_start) GB_FATAL_CUDA(cudaFreeHost(res->target_batch_start));
    if (res->query_batch_end) GB_FATAL_CUDA(cudaFreeHost(res->query_batch_end));
    if (res->target_batch_end) GB_FATAL_CUDA(cudaFreeHost(res->target_batch_end));
    if (res->n_cigar_ops) GB_FATAL_CUDA(cudaFreeHost(res->n_cigar_ops));
    if (res->cigar) GB_FATAL_CUDA(cudaFreeHost(res->cigar));
    free(res);
}

void gasal_res_destroy_device(gasal_res_t *device_res, gasal_res_t *device_cpy)
{
    if (device_cpy == NULL || device_res == NULL) return;
    if (device_cpy->aln_score) GB_FATAL_CUDA(cudaFree(device_cpy->aln_score));
    if (device_cpy->query_batch_start) GB_FATAL_CUDA(cudaFree(device_cpy->query_batch_start));
    if (device_cpy->target_batch_start) GB_FATAL_CUDA(cudaFree(device_cpy->target_batch_start));
    if (device_cpy->query_batch_end) GB_FATAL_CUDA(cudaFree(device_cpy->query_batch_end));
    if (device_cpy->target_batch_end) GB_FATAL_CUDA(cudaFree(device_cpy->target_batch_end));
    if (device_cpy->cigar) GB_FATAL_CUDA(cudaFree(device_cpy->cigar));
    GB_FATAL_CUDA(cudaFree(device_res));
    free(device_cpy);
}

/* ========================= streams ====================================== */

gasal_gpu_storage_v gasal_init_gpu_storage_v(int n_streams)
{
    gasal_gpu_storage_v v;
    v.a = (gasal_gpu_storage_t *)calloc(n_streams, sizeof(gasal_gpu_storage_t));
    v.n = n_streams;
    return v;
}

void gasal_init_streams(gasal_gpu_storage_v *vec, int max_query_len, int max_target_len, int max_n_alns,
                        Parameters *params)
{
    const uint32_t q8 = round8((uint32_t)max_query_len), t8 = round8((uint32_t)max_target_len);
    const uint32_t qbytes = (uint32_t)max_n_alns * q8, tbytes = (uint32_t)max_n_alns * t8;
    for (int i = 0; i < vec->n; i++) {
        gasal_gpu_storage_t *s = &vec->a[i];
        s->extensible_host_unpacked_query_batch = gasal_host_batch_new(qbytes, 0);
        s->extensible_host_unpacked_target_batch = gasal_host_batch_new(tbytes, 0);
        GB_FATAL_CUDA(cudaMalloc(&s->unpacked_query_batch, qbytes));
        GB_FATAL_CUDA(cudaMalloc(&s->unpacked_target_batch, tbytes));
        GB_FATAL_CUDA(cudaHostAlloc(&s->host_query_op, max_n_alns, cudaHostAllocDefault));
        GB_FATAL_CUDA(cudaHostAlloc(&s->host_target_op, max_n_alns, cudaHostAllocDefault));
        memset(s->host_query_op, 0, max_n_alns);
        memset(s->host_target_op, 0, max_n_alns);
        GB_FATAL_CUDA(cudaMalloc(&s->query_op, max_n_alns));
        GB_FATAL_CUDA(cudaMalloc(&s->target_op, max_n_alns));
        if (params->isPacked) {
            s->packed_query_batch = (uint32_t *)s->unpacked_query_batch;
            s->packed_target_batch = (uint32_t *)s->unpacked_target_batch;
        } else {
            GB_FATAL_CUDA(cudaMalloc(&s->packed_query_batch, (qbytes / 8) * sizeof(uint32_t)));
            GB_FATAL_CUDA(cudaMalloc(&s->packed_target_batch, (tbytes / 8) * sizeof(uint32_t)));
        }
        if (params->algo == KSW) {
            GB_FATAL_CUDA(cudaHostAlloc(&s->host_seed_scores, max_n_alns * sizeof(uint32_t), cudaHostAllocDefault));
            GB_FATAL_CUDA(cudaMalloc(&s->seed_scores, max_n_alns * sizeof(uint32_t)));
        } else {
            s->host_seed_scores = NULL;
            s->seed_scores = NULL;
        }
        GB_FATAL_CUDA(cudaHostAlloc(&s->host_query_batch_lens, max_n_alns * sizeof(uint32_t), cudaHostAllocDefault));
        GB_FATAL_CUDA(cudaHostAlloc(&s->host_target_batch_lens, max_n_alns * sizeof(uint32_t), cudaHostAllocDefault));
        GB_FATAL_CUDA(cudaHostAlloc(&s->host_query_batch_offsets, max_n_alns * sizeof(uint32_t), cudaHostAllocDefault));
        GB_FATAL_CUDA(cudaHostAlloc(&s->host_target_batch_offsets, max_n_alns * sizeof(uint32_t), cudaHostAllocDefault));
        GB_FATAL_CUDA(cudaMalloc(&s->query_batch_lens, max_n_alns * sizeof(uint32_t)));
        GB_FATAL_CUDA(cudaMalloc(&s->target_batch_lens, max_n_alns * sizeof(uint32_t)));
        GB_FATAL_CUDA(cudaMalloc(&s->query_batch_offsets, max_n_alns * sizeof(uint32_t)));
        GB_FATAL_CUDA(cudaMalloc(&s->target_batch_offsets, max_n_alns * sizeof(uint32_t)));
        s->host_res = gasal_res_new_host(max_n_alns, params);
        if (params->start_pos == WITH_TB)
            GB_FATAL_CUDA(cudaHostAlloc(&s->host_res->cigar, qbytes, cudaHostAllocDefault));
        s->device_cpy = gasal_res_new_device_cpy(max_n_alns, params);
        s->device_res = gasal_res_new_device(s->device_cpy);
        if (params->secondBest) {
            s->host_res_second = gasal_res_new_host(max_n_alns, params);
            s->device_cpy_second = gasal_res_new_device_cpy(max_n_alns, params);
            s->device_res_second = gasal_res_new_device(s->device_cpy_second);
        } else {
            s->host_res_second = NULL;
            s->device_cpy_second = NULL;
            s->device_res_second = NULL;
        }
        /* traceback tiles are sized per batch by the engine (packed_tb_matrices
         * stays NULL; the reference's max_q x max_t x n_alns matrix is not used) */
        s->packed_tb_matrix_size = 0;
        s->packed_tb_matrices = NULL;
        GB_FATAL_CUDA(cudaStreamCreate(&s->str));
        s->is_free = 1;
        s->host_max_query_batch_bytes = qbytes;
        s->host_max_target_batch_bytes = tbytes;
        s->host_max_n_alns = max_n_alns;
        s->gpu_max_query_batch_bytes = qbytes;
        s->gpu_max_target_batch_bytes = tbytes;
        s->gpu_max_n_alns = max_n_alns;
        s->current_n_alns = 0;
        StreamState &ss = state_of(s);
        (void)ss;
    }
}

void gasal_destroy_streams(gasal_gpu_storage_v *vec, Parameters *params)
{
    (void)params;
    for (int i = 0; i < vec->n; i++) {
        gasal_gpu_storage_t *s = &vec->a[i];
        if (s->str) cudaStreamSynchronize(s->str);
        release_state(s);
        if (s->extensible_host_unpacked_query_batch) gasal_host_batch_destroy(s->extensible_host_unpacked_query_batch);
        if (s->extensible_host_unpacked_target_batch) gasal_host_batch_destroy(s->extensible_host_unpacked_target_batch);
        gasal_res_destroy_host(s->host_res);
        gasal_res_destroy_device(s->device_res, s->device_cpy);
        gasal_res_destroy_host(s->host_res_second);
        gasal_res_destroy_device(s->device_res_second, s->device_cpy_second);
        if (s->seed_scores) GB_FATAL_CUDA(cudaFree(s->seed_scores));
        if (s->host_seed_scores) GB_FATAL_CUDA(cudaFreeHost(s->host_seed_scores));
        if (s->query_op) GB_FATAL_CUDA(cudaFree(s->query_op));
        if (s->target_op) GB_FATAL_CUDA(cudaFree(s->target_op));
        if (s->host_query_op) GB_FATAL_CUDA(cudaFreeHost(s->host_query_op));
        if (s->host_target_op) GB_FATAL_CUDA(cudaFreeHost(s->host_target_op));
        if (s->host_query_batch_offsets) GB_FATAL_CUDA(cudaFreeHost(s->host_query_batch_offsets));
        if (s->host_target_batch_offsets) GB_FATAL_CUDA(cudaFreeHost(s->host_target_batch_offsets));
        if (s->host_query_batch_lens) GB_FATAL_CUDA(cudaFreeHost(s->host_query_batch_lens));
        if (s->host_target_batch_lens) GB_FATAL_CUDA(cudaFreeHost(s->host_target_batch_lens));
        if (s->packed_query_batch && (void *)s->packed_query_batch != (void *)s->unpacked_query_batch)
            GB_FATAL_CUDA(cudaFree(s->packed_query_batch));
        if (s->packed_target_batch && (void *)s->packed_target_batch != (void *)s->unpacked_target_batch)
            GB_FATAL_CUDA(cudaFree(s->packed_target_batch));
        if (s->unpacked_query_batch) GB_FATAL_CUDA(cudaFree(s->unpacked_query_batch));
        if (s->unpacked_target_batch) GB_FATAL_CUDA(cudaFree(s->unpacked_target_batch));
        if (s->query_batch_offsets) GB_FATAL_CUDA(cudaFree(s->query_batch_offsets));
        if (s->target_batch_offsets) GB_FATAL_CUDA(cudaFree(s->target_batch_offsets));
        if (s->query_batch_lens) GB_FATAL_CUDA(cudaFree(s->query_batch_lens));
        if (s->target_batch_lens) GB_FATAL_CUDA(cudaFree(s->target_batch_lens));
        if (s->packed_tb_matrices) GB_FATAL_CUDA(cudaFree(s->packed_tb_matrices));
        if (s->str) GB_FATAL_CUDA(cudaStreamDestroy(s->str));
        memset(s, 0, sizeof(*s));
    }
}

void gasal_destroy_gpu_storage_v(gasal_gpu_storage_v *vec)
{
    if (vec->a != NULL) free(vec->a);
    vec->a = NULL;
}

void gasal_gpu_mem_alloc(gasal_gpu_storage_t *s, int gpu_max_query_batch_bytes, int gpu_max_target_batch_bytes,
                         int gpu_max_n_alns, Parameters *params)
{
    GB_FATAL_CUDA(cudaMalloc(&s->unpacked_query_batch, gpu_max_query_batch_bytes));
    GB_FATAL_CUDA(cudaMalloc(&s->unpacked_target_batch, gpu_max_target_batch_bytes));
    GB_FATAL_CUDA(cudaMalloc(&s->packed_query_batch, (gpu_max_query_batch_bytes / 8) * sizeof(uint32_t)));
    GB_FATAL_CUDA(cudaMalloc(&s->packed_target_batch, (gpu_max_target_batch_bytes / 8) * sizeof(uint32_t)));
    GB_FATAL_CUDA(cudaMalloc(&s->query_batch_lens, gpu_max_n_alns * sizeof(uint32_t)));
    GB_FATAL_CUDA(cudaMalloc(&s->target_batch_lens, gpu_max_n_alns * sizeof(uint32_t)));
    GB_FATAL_CUDA(cudaMalloc(&s->query_batch_offsets, gpu_max_n_alns * sizeof(uint32_t)));
    GB_FATAL_CUDA(cudaMalloc(&s->target_batch_offsets, gpu_max_n_alns * sizeof(uint32_t)));
    s->device_cpy = gasal_res_new_device_cpy(gpu_max_n_alns, params);
    s->device_res = gasal_res_new_device(s->device_cpy);
    s->gpu_max_query_batch_bytes = gpu_max_query_batch_bytes;
    s->gpu_max_target_batch_bytes = gpu_max_target_batch_bytes;
    s->gpu_max_n_alns = gpu_max_n_alns;
}

void gasal_gpu_mem_free(gasal_gpu_storage_t *s, Parameters *params)
{
    if (s->unpacked_query_batch) GB_FATAL_CUDA(cudaFree(s->unpacked_query_batch));
    if (s->unpacked_target_batch) GB_FATAL_CUDA(cudaFree(s->unpacked_target_batch));
    if (s->packed_query_batch) GB_FATAL_CUDA(cudaFree(s->packed_query_batch));
    if (s->packed_target_batch) GB_FATAL_CUDA(cudaFree(s->packed_target_batch));
    if (s->query_batch_offsets) GB_FATAL_CUDA(cudaFree(s->query_batch_offsets));
    if (s->target_batch_offsets) GB_FATAL_CUDA(cudaFree(s->target_batch_offsets));
    if (s->query_batch_lens) GB_FATAL_CUDA(cudaFree(s->query_batch_lens));
    if (s->target_batch_lens) GB_FATAL_CUDA(cudaFree(s->target_batch_lens));
    gasal_res_destroy_device(s->device_res, s->device_cpy);
    if (params->secondBest) gasal_res_destroy_device(s->device_res_second, s->device_cpy_second);
}

/* ========================= interfaces =================================== */

template <typename T> static T *host_realloc(T *src, int new_n, int old_n)
{
    if (new_n < old_n) {
        fprintf(stderr, "[GASAL ERROR] cudoHostRealloc: invalid sizes. New size < old size (%d < %d)", new_n, old_n);
        exit(EXIT_FAILURE);
    }
    T *dst = NULL;
    GB_FATAL_CUDA(cudaHostAlloc(&dst, new_n * sizeof(T), cudaHostAllocMapped));
    if (src) {
        memcpy(dst, src, old_n * sizeof(T));
        GB_FATAL_CUDA(cudaFreeHost(src));
    }
    return dst;
}

void gasal_host_alns_resize(gasal_gpu_storage_t *s, int new_max_alns, Parameters *params)
{
    fprintf(stderr, "[GASAL WARNING] Resizing gpu_storage from %d sequences to %d sequences... ", s->host_max_n_alns,
            new_max_alns);
    const int old = (int)s->host_max_n_alns;
    s->host_query_op = host_realloc(s->host_query_op, new_max_alns, old);
    s->host_target_op = host_realloc(s->host_target_op, new_max_alns, old);
    if (params->algo == KSW) s->host_seed_scores = host_realloc(s->host_seed_scores, new_max_alns, old);
    s->host_query_batch_lens = host_realloc(s->host_query_batch_lens, new_max_alns, old);
    s->host_target_batch_lens = host_realloc(s->host_target_batch_lens, new_max_alns, old);
    s->host_query_batch_offsets = host_realloc(s->host_query_batch_offsets, new_max_alns, old);
    s->host_target_batch_offsets = host_realloc(s->host_target_batch_offsets, new_max_alns, old);
    uint8_t *cigar = s->host_res ? s->host_res->cigar : NULL;
    if (s->host_res) s->host_res->cigar = NULL;
    gasal_res_destroy_host(s->host_res);
    s->host_res = gasal_res_new_host(new_max_alns, params);
    s->host_res->cigar = cigar;
    gasal_res_destroy_device(s->device_res, s->device_cpy);
    s->device_cpy = gasal_res_new_device_cpy(new_max_alns, params);
    s->device_res = gasal_res_new_device(s->device_cpy);
    if (params->secondBest) {
        gasal_res_destroy_host(s->host_res_second);
        gasal_res_destroy_device(s->device_res_second, s->device_cpy_second);
        s->host_res_second = gasal_res_new_host(new_max_alns, params);
        s->device_cpy_second = gasal_res_new_device_cpy(new_max_alns, params);
        s->device_res_second = gasal_res_new_device(s->device_cpy_second);
    }
    s->host_max_n_alns = new_max_alns;
    if (s->gpu_max_n_alns > (uint32_t)new_max_alns) s->gpu_max_n_alns = new_max_alns;
    fprintf(stderr, " done. This can harm performance.\n");
}

void gasal_op_fill(gasal_gpu_storage_t *s, uint8_t *data, uint32_t nbr_seqs_in_stream, data_source SRC)
{
    uint8_t *dst = (SRC == QUERY) ? s->host_query_op : s->host_target_op;
    memcpy(dst, data, nbr_seqs_in_stream);
}

void gasal_set_device(int gpu_select, bool isPrintingProp)
{
    if (isPrintingProp) {
        int num_devices = 0;
        cudaGetDeviceCount(&num_devices);
        fprintf(stderr, "Found %d GPUs\n", num_devices);
        if (gpu_select > num_devices - 1) {
            fprintf(stderr, "Error: can't select device %d when only %d devices are selected (range from 0 to %d)\n",
                    gpu_select, num_devices, num_devices - 1);
            exit(EXIT_FAILURE);
        }
        cudaDeviceProp prop;
        for (int d = 0; d < num_devices; d++) {
            cudaGetDeviceProperties(&prop, d);
            fprintf(stderr, "\tGPU %d: %s\n", d, prop.name);
        }
        if (num_devices > 0) {
            cudaGetDeviceProperties(&prop, gpu_select);
            fprintf(stderr, "Selected device %d : %s\n", gpu_select, prop.name);
            cudaSetDevice(gpu_select);
        }
    } else {
        cudaSetDevice(gpu_select);
    }
}

/* ========================= alignment ==================================== */

void gasal_copy_subst_scores(gasal_subst_scores *subst)
{
    gb::Settings &st = gb::settings();
    st.sc.match = subst->match;
    st.sc.mismatch = subst->mismatch;
    st.sc.o = subst->gap_open;
    st.sc.e = subst->gap_extend;
    st.sc.oe = subst->gap_open + subst->gap_extend;
}

namespace gbapi {

/* Error reporting of one call: the C++ API prints and terminates like the
 * reference; the C ABI returns the status. */
struct Errs {
    bool fatal;
    int fail(int code, const char *msg) const
    {
        fprintf(stderr, "%s", msg);
        if (fatal) exit(EXIT_FAILURE);
        return code;
    }
};

static int grow_dev(void **p, uint32_t old_bytes, uint32_t new_bytes)
{
    (void)old_bytes;
    if (*p) cudaFree(*p);
    *p = NULL;
    if (gb::dev_malloc(p, new_bytes) == cudaSuccess) return GB_OK;
    cudaGetLastError();
    return GB_ERR_ALLOC;
}

/* zdrop: the ksw z-drop threshold.  GASAL2's kernel hard-codes 0
 * (src/kernels/ksw_kernel_template.h:62), so gasal_aln_async passes 0; the
 * one-shot C entry point passes its caller's value. */
int aln_async(gasal_gpu_storage_t *s, uint32_t qbytes, uint32_t tbytes, uint32_t n, Parameters *params, bool fatal,
              int zdrop)
{
    Errs E{fatal};
    char msg[512];
    if (n <= 0) return E.fail(GB_ERR_ARG, "[GASAL ERROR:] actual_n_alns <= 0\n");
    if (qbytes <= 0) return E.fail(GB_ERR_ARG, "[GASAL ERROR:] actual_query_batch_bytes <= 0\n");
    if (tbytes <= 0) return E.fail(GB_ERR_ARG, "[GASAL ERROR:] actual_target_batch_bytes <= 0\n");
    if (qbytes % 8) {
        snprintf(msg, sizeof msg, "[GASAL ERROR:] actual_query_batch_bytes=%d is not a multiple of 8\n", qbytes);
        return E.fail(GB_ERR_ARG, msg);
    }
    if (tbytes % 8) {
        snprintf(msg, sizeof msg, "[GASAL ERROR:] actual_target_batch_bytes=%d is not a multiple of 8\n", tbytes);
        return E.fail(GB_ERR_ARG, msg);
    }
    if (qbytes > s->host_max_query_batch_bytes) {
        snprintf(msg, sizeof msg, "[GASAL ERROR:] actual_query_batch_bytes(%d) > host_max_query_batch_bytes(%d)\n",
                 qbytes, s->host_max_query_batch_bytes);
        return E.fail(GB_ERR_ARG, msg);
    }
    if (tbytes > s->host_max_target_batch_bytes) {
        snprintf(msg, sizeof msg, "[GASAL ERROR:] actual_target_batch_bytes(%d) > host_max_target_batch_bytes(%d)\n",
                 tbytes, s->host_max_target_batch_bytes);
        return E.fail(GB_ERR_ARG, msg);
    }
    if (n > s->host_max_n_alns) {
        snprintf(msg, sizeof msg, "[GASAL ERROR:] actual_n_alns(%d) > host_max_n_alns(%d)\n", n, s->host_max_n_alns);
        return E.fail(GB_ERR_ARG, msg);
    }
    if (params->algo != LOCAL && params->algo != GLOBAL && params->algo != SEMI_GLOBAL && params->algo != BANDED &&
        params->algo != KSW)
        return E.fail(GB_ERR_ARG, "[GASAL ERROR:] unsupported algorithm\n");

    /* grow device buffers as the reference does (src/gasal_align.cu:70-145) */
    if (s->gpu_max_query_batch_bytes < qbytes) {
        uint32_t k = 2;
        while (s->gpu_max_query_batch_bytes * k < qbytes) k++;
        fprintf(stderr, "[GASAL WARNING:] actual_query_batch_bytes(%d) > Allocated GPU memory (gpu_max_query_batch_bytes=%d). Therefore, allocating %d bytes on GPU (gpu_max_query_batch_bytes=%d). Performance may be lost if this is repeated many times.\n",
                qbytes, s->gpu_max_query_batch_bytes, s->gpu_max_query_batch_bytes * k, s->gpu_max_query_batch_bytes * k);
        const uint32_t nb = s->gpu_max_query_batch_bytes * k;
        const bool aliased = (void *)s->packed_query_batch == (void *)s->unpacked_query_batch;
        if (grow_dev((void **)&s->unpacked_query_batch, 0, nb) != GB_OK) return E.fail(GB_ERR_ALLOC, "[GASAL ERROR:] allocation failed\n");
        if (aliased) s->packed_query_batch = (uint32_t *)s->unpacked_query_batch;
        else if (grow_dev((void **)&s->packed_query_batch, 0, (nb / 8) * 4) != GB_OK) return E.fail(GB_ERR_ALLOC, "[GASAL ERROR:] allocation failed\n");
        s->gpu_max_query_batch_bytes = nb;
        if (params->start_pos == WITH_TB) {
            if (s->host_res->cigar) cudaFreeHost(s->host_res->cigar);
            if (cudaHostAlloc(&s->host_res->cigar, nb, cudaHostAllocDefault) != cudaSuccess)
                return E.fail(GB_ERR_ALLOC, "[GASAL ERROR:] allocation failed\n");
        }
    }
    if (s->gpu_max_target_batch_bytes < tbytes) {
        uint32_t k = 2;
        while (s->gpu_max_target_batch_bytes * k < tbytes) k++;
        fprintf(stderr, "[GASAL WARNING:] actual_target_batch_bytes(%d) > Allocated GPU memory (gpu_max_target_batch_bytes=%d). Therefore, allocating %d bytes on GPU (gpu_max_target_batch_bytes=%d). Performance may be lost if this is repeated many times.\n",
                tbytes, s->gpu_max_target_batch_bytes, s->gpu_max_target_batch_bytes * k, s->gpu_max_target_batch_bytes * k);
        const uint32_t nb = s->gpu_max_target_batch_bytes * k;
        const bool aliased = (void *)s->packed_target_batch == (void *)s->unpacked_target_batch;
        if (grow_dev((void **)&s->unpacked_target_batch, 0, nb) != GB_OK) return E.fail(GB_ERR_ALLOC, "[GASAL ERROR:] allocation failed\n");
        if (aliased) s->packed_target_batch = (uint32_t *)s->unpacked_target_batch;
        else if (grow_dev((void **)&s->packed_target_batch, 0, (nb / 8) * 4) != GB_OK) return E.fail(GB_ERR_ALLOC, "[GASAL ERROR:] allocation failed\n");
        s->gpu_max_target_batch_bytes = nb;
    }
    if (s->gpu_max_n_alns < n) {
        uint32_t k = 2;
        while (s->gpu_max_n_alns * k < n) k++;
        fprintf(stderr, "[GASAL WARNING:] actual_n_alns(%d) > gpu_max_n_alns(%d). Therefore, allocating memory for %d alignments on  GPU (gpu_max_n_alns=%d). Performance may be lost if this is repeated many times.\n",
                n, s->gpu_max_n_alns, s->gpu_max_n_alns * k, s->gpu_max_n_alns * k);
        const uint32_t nn = s->gpu_max_n_alns * k;
        void **arrs[] = {(void **)&s->query_batch_offsets, (void **)&s->target_batch_offsets,
                         (void **)&s->query_batch_lens, (void **)&s->target_batch_lens};
        for (void **a : arrs)
            if (grow_dev(a, 0, nn * 4) != GB_OK) return E.fail(GB_ERR_ALLOC, "[GASAL ERROR:] allocation failed\n");
        if (grow_dev((void **)&s->query_op, 0, nn) != GB_OK || grow_dev((void **)&s->target_op, 0, nn) != GB_OK)
            return E.fail(GB_ERR_ALLOC, "[GASAL ERROR:] allocation failed\n");
        if (s->seed_scores && grow_dev((void **)&s->seed_scores, 0, nn * 4) != GB_OK)
            return E.fail(GB_ERR_ALLOC, "[GASAL ERROR:] allocation failed\n");
        gasal_res_destroy_device(s->device_res, s->device_cpy);
        s->device_cpy = gasal_res_new_device_cpy(nn, params);
        s->device_res = gasal_res_new_device(s->device_cpy);
        if (params->secondBest) {
            gasal_res_destroy_device(s->device_res_second, s->device_cpy_second);
            s->device_cpy_second = gasal_res_new_device_cpy(nn, params);
            s->device_res_second = gasal_res_new_device(s->device_cpy_second);
        }
        s->gpu_max_n_alns = nn;
    }
    StreamState &ss = state_of(s);
    if (params->start_pos == WITH_TB && ss.n_cigar_cap < s->gpu_max_n_alns) {
        if (ss.d_n_cigar) cudaFree(ss.d_n_cigar);
        ss.d_n_cigar = NULL;
        if (cudaMalloc(&ss.d_n_cigar, (size_t)s->gpu_max_n_alns * 4) != cudaSuccess)
            return E.fail(GB_ERR_ALLOC, "[GASAL ERROR:] allocation failed\n");
        ss.n_cigar_cap = s->gpu_max_n_alns;
    }

    cudaStream_t st = s->str;
    const gb::Settings &set = gb::settings();
    gb::RunCfg cfg{};
    cfg.algo = params->algo, cfg.start = params->start_pos, cfg.second = params->secondBest == TRUE;
    cfg.head = params->semiglobal_skipping_head, cfg.tail = params->semiglobal_skipping_tail;
    cfg.k_band = params->k_band, cfg.zdrop = zdrop, cfg.sc = set.sc;
    cfg.band_model = set.band_model, cfg.band_min = set.band_min, cfg.band_max = set.band_max;
    cfg.ref_reverse = set.ref_reverse, cfg.mql = set.mql, cfg.is_packed = params->isPacked;
    cfg.reverse_complement = params->isReverseComplement;
    gb::DevBatch b{};
    b.n = (int32_t)n, b.q_bytes = qbytes, b.t_bytes = tbytes;
    b.q = s->unpacked_query_batch, b.t = s->unpacked_target_batch;
    b.pq = s->packed_query_batch, b.pt = s->packed_target_batch;
    b.q_off = s->query_batch_offsets, b.t_off = s->target_batch_offsets;
    b.q_len = s->query_batch_lens, b.t_len = s->target_batch_lens;
    b.q_op = s->query_op, b.t_op = s->target_op, b.seed = s->seed_scores;
    b.h_q_len = s->host_query_batch_lens, b.h_t_len = s->host_target_batch_lens;
    gb::DevOut o{};
    o.score = s->device_cpy->aln_score, o.q_end = s->device_cpy->query_batch_end;
    o.t_end = s->device_cpy->target_batch_end, o.q_start = s->device_cpy->query_batch_start;
    o.t_start = s->device_cpy->target_batch_start;
    if (params->secondBest && s->device_cpy_second) {
        o.score2 = s->device_cpy_second->aln_score, o.q_end2 = s->device_cpy_second->query_batch_end;
        o.t_end2 = s->device_cpy_second->target_batch_end;
    }
    o.cigar = s->unpacked_query_batch, o.n_cigar = ss.d_n_cigar;
    if (params->algo == KSW && (s->seed_scores == NULL || s->host_seed_scores == NULL)) {
        if (s->seed_scores == NULL) fprintf(stderr, "seed_scores == NULL\n");
        if (s->host_seed_scores == NULL) fprintf(stderr, "host_seed_scores == NULL\n");
        return E.fail(GB_ERR_ARG, "");
    }

    /* every host decision and allocation of the batch */
    gb::Plan plan;
    int rc = gb::plan_batch(cfg, b, o, ss.ws, plan, s->str);
    if (rc != GB_OK) return E.fail(rc, "[GASAL ERROR:] alignment launch failed\n");

    /* the stream operations of the batch: host pages -> device
     * (src/gasal_align.cu:152-175), the kernels, results -> host
     * (src/gasal_align.cu:266-304) */
    int err_line = 0;
    auto issue = [&]() -> cudaError_t {
        cudaError_t ce = cudaSuccess;
#define GB_Q(call)                                                                                  \
    do {                                                                                            \
        ce = (call);                                                                                \
        if (ce != cudaSuccess) {                                                                    \
            err_line = __LINE__;                                                                    \
            return ce;                                                                              \
        }                                                                                           \
    } while (0)
        for (host_batch_t *p = s->extensible_host_unpacked_query_batch; p; p = p->next)
            if (p->data_size) GB_Q(cudaMemcpyAsync(s->unpacked_query_batch + p->offset, p->data, p->data_size, cudaMemcpyHostToDevice, st));
        for (host_batch_t *p = s->extensible_host_unpacked_target_batch; p; p = p->next)
            if (p->data_size) GB_Q(cudaMemcpyAsync(s->unpacked_target_batch + p->offset, p->data, p->data_size, cudaMemcpyHostToDevice, st));
        GB_Q(cudaMemcpyAsync(s->query_batch_lens, s->host_query_batch_lens, n * 4, cudaMemcpyHostToDevice, st));
        GB_Q(cudaMemcpyAsync(s->target_batch_lens, s->host_target_batch_lens, n * 4, cudaMemcpyHostToDevice, st));
        GB_Q(cudaMemcpyAsync(s->query_batch_offsets, s->host_query_batch_offsets, n * 4, cudaMemcpyHostToDevice, st));
        GB_Q(cudaMemcpyAsync(s->target_batch_offsets, s->host_target_batch_offsets, n * 4, cudaMemcpyHostToDevice, st));
        if (params->algo == KSW)
            GB_Q(cudaMemcpyAsync(s->seed_scores, s->host_seed_scores, n * 4, cudaMemcpyHostToDevice, st));
        if (params->isReverseComplement) {
            GB_Q(cudaMemcpyAsync(s->query_op, s->host_query_op, n, cudaMemcpyHostToDevice, st));
            GB_Q(cudaMemcpyAsync(s->target_op, s->host_target_op, n, cudaMemcpyHostToDevice, st));
        }
        rc = gb::enqueue_batch(cfg, b, o, ss.ws, plan, st);
        if (rc != GB_OK) {
            err_line = __LINE__;
            return cudaErrorUnknown;
        }
        gasal_res_t *h = s->host_res, *d = s->device_cpy;
        if (h->aln_score && d->aln_score) GB_Q(cudaMemcpyAsync(h->aln_score, d->aln_score, n * 4, cudaMemcpyDeviceToHost, st));
        if (h->query_batch_start && d->query_batch_start) GB_Q(cudaMemcpyAsync(h->query_batch_start, d->query_batch_start, n * 4, cudaMemcpyDeviceToHost, st));
        if (h->target_batch_start && d->target_batch_start) GB_Q(cudaMemcpyAsync(h->target_batch_start, d->target_batch_start, n * 4, cudaMemcpyDeviceToHost, st));
        if (h->query_batch_end && d->query_batch_end) GB_Q(cudaMemcpyAsync(h->query_batch_end, d->query_batch_end, n * 4, cudaMemcpyDeviceToHost, st));
        if (h->target_batch_end && d->target_batch_end) GB_Q(cudaMemcpyAsync(h->target_batch_end, d->target_batch_end, n * 4, cudaMemcpyDeviceToHost, st));
        if (params->start_pos == WITH_TB) {
            if (h->cigar) GB_Q(cudaMemcpyAsync(h->cigar, s->unpacked_query_batch, qbytes, cudaMemcpyDeviceToHost, st));
            if (h->n_cigar_ops) GB_Q(cudaMemcpyAsync(h->n_cigar_ops, ss.d_n_cigar, n * 4, cudaMemcpyDeviceToHost, st));
        }
        if (params->secondBest && s->host_res_second && s->device_cpy_second) {
            gasal_res_t *h2 = s->host_res_second, *d2 = s->device_cpy_second;
            if (h2->aln_score && d2->aln_score) GB_Q(cudaMemcpyAsync(h2->aln_score, d2->aln_score, n * 4, cudaMemcpyDeviceToHost, st));
            if (h2->query_batch_end && d2->query_batch_end) GB_Q(cudaMemcpyAsync(h2->query_batch_end, d2->query_batch_end, n * 4, cudaMemcpyDeviceToHost, st));
            if (h2->target_batch_end && d2->target_batch_end) GB_Q(cudaMemcpyAsync(h2->target_batch_end, d2->target_batch_end, n * 4, cudaMemcpyDeviceToHost, st));
        }
#undef GB_Q
        return cudaSuccess;
    };

    cudaError_t ce = cudaSuccess;
    if (set.graphs && !gb::timing_on()) {
        /* One CUDA graph per storage: relaunched as is while the batch has the
         * same signature, else recaptured and updated in place. */
        std::vector<uint8_t> sig;
        batch_signature(sig, s, ss, params, n, qbytes, tbytes, cfg, plan);
        if (ss.exec && sig == ss.sig) {
            ce = cudaGraphLaunch(ss.exec, st);
            if (ce == cudaSuccess) graph_stat(0);
        } else {
            ce = capture_and_launch(ss, issue, st);
            if (ce == cudaSuccess) ss.sig.swap(sig);
            else ss.sig.clear();
        }
        if (ce != cudaSuccess && err_line == 0) err_line = __LINE__;
    } else {
        ce = issue();
    }
    if (ce != cudaSuccess) {
        if (rc != GB_OK) return E.fail(rc, "[GASAL ERROR:] alignment launch failed\n");
        snprintf(msg, sizeof msg, "[GASAL CUDA ERROR:] %s(CUDA error no.=%d). Line no. %d in file %s\n",
                 cudaGetErrorString(ce), ce, err_line, __FILE__);
        return E.fail(GB_ERR_CUDA, msg);
    }
    if (plan.tb && cudaEventRecord(ss.ws.tb_off_free, st) != cudaSuccess)
        return E.fail(GB_ERR_CUDA, "[GASAL CUDA ERROR:] event record failed\n");
    s->is_free = 0;
    return GB_OK;
}

void graph_stats(int64_t out[4])
{
    for (int k = 0; k < 4; k++) out[k] = g_graph_stats[k].load();
}

int is_done(gasal_gpu_storage_t *s, bool fatal)
{
    if (s->is_free == 1) return -2;
    const cudaError_t err = cudaStreamQuery(s->str);
    if (err != cudaSuccess) {
        if (err == cudaErrorNotReady) return -1;
        fprintf(stderr, "[GASAL CUDA ERROR:] %s(CUDA error no.=%d). Line no. %d in file %s\n", cudaGetErrorString(err),
                err, __LINE__, __FILE__);
        if (fatal) exit(EXIT_FAILURE);
        return GB_ERR_CUDA;
    }
    gasal_host_batch_reset(s);
    s->is_free = 1;
    s->current_n_alns = 0;
    return 0;
}

} // namespace gbapi

void gasal_aln_async(gasal_gpu_storage_t *gpu_storage, const uint32_t actual_query_batch_bytes,
                     const uint32_t actual_target_batch_bytes, const uint32_t actual_n_alns, Parameters *params)
{
    gbapi::aln_async(gpu_storage, actual_query_batch_bytes, actual_target_batch_bytes, actual_n_alns, params, true, 0);
}

int gasal_is_aln_async_done(gasal_gpu_storage_t *gpu_storage) { return gbapi::is_done(gpu_storage, true); }
