/*
 * workload_gen.c -- seeded synthetic pair sets for the benchmark workloads.
 *
 * Every pair draws from its own xoshiro256** stream whose state is four
 * splitmix64 outputs of (seed, global pair index), so a pair's bases do not
 * depend on the thread count, on the batch size or on which slice of the
 * workload is generated.  Generation runs twice per pair: the first pass
 * records each pair's lengths (the caller lays the batch out from them), the
 * second writes the bases at the caller's offsets, N-padded to a multiple of 8
 * as GASAL2's host batches are.
 *
 * Workloads (sizes are the caller's):
 *   0  query U[100,150] with 0.1% N; target = 0..20 random flank bases on each
 *      side + query, then 2% substitutions, 0.5% indels of length 1..3
 *   1  query 150; target = 0..75 flank bases each side + query, 3% subs, 1%
 *      indels (1..3), clipped to [150, 300]; half the queries flagged
 *      REVERSE_COMPLEMENT
 *   2  query log-uniform [50, 1000]; target = query with U[1,8]% subs and
 *      U[0.5,3]% indels of length 1..10, drawn per pair
 *   3  query U[250, 2000]; indel rate from {0.5, 2, 5, 10}% (length 1..3)
 *      plus U[1,5]% subs; seed score h0 U[20, 60]
 *   4  query round(250 exp(N(0, 0.8))) clipped to [50, 5000]; 60% short-read
 *      like (U[1,2]% subs, 0.2% indels), 30% long-read like (U[5,12]% errors,
 *      a quarter substitutions, the rest indels of length 1..5), 10% an
 *      unrelated random target of the mutated length; h0 U[20, 60]
 * Indels split evenly between insertions and deletions.  Mutation walks the
 * source once: per position one uniform decides substitute / copy then insert
 * L random bases / delete L bases from here (stopping at the sequence end) /
 * copy.  Targets are never empty (an empty one gets one random base).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define N_BASE 0x4E
#define REVERSE_COMPLEMENT 3

typedef struct {
    uint64_t s[4];
    uint64_t bits; /* buffered random bits for 2-bit base draws */
    int nbits;
} rng_t;

static uint64_t splitmix64(uint64_t *x)
{
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static inline uint64_t next64(rng_t *r)
{
    uint64_t *s = r->s;
    const uint64_t out = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return out;
}

static void rng_seed(rng_t *r, uint64_t seed, uint64_t pair)
{
    uint64_t x = seed ^ (pair * 0xD1B54A32D192ED03ull);
    for (int k = 0; k < 4; k++) r->s[k] = splitmix64(&x);
    r->bits = 0;
    r->nbits = 0;
}

static inline double unif(rng_t *r) { return (double)(next64(r) >> 11) * (1.0 / 9007199254740992.0); }

/* integer uniform on [lo, hi] */
static inline int64_t irange(rng_t *r, int64_t lo, int64_t hi)
{
    const uint64_t span = (uint64_t)(hi - lo + 1);
    return lo + (int64_t)(((unsigned __int128)next64(r) * span) >> 64);
}

static inline double normal(rng_t *r)
{
    double u1 = unif(r);
    const double u2 = unif(r);
    if (u1 < 1e-300) u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

static const uint8_t ACGT[4] = {'A', 'C', 'G', 'T'};

static inline uint8_t rbase(rng_t *r)
{
    if (r->nbits == 0) {
        r->bits = next64(r);
        r->nbits = 64;
    }
    const uint8_t b = ACGT[r->bits & 3u];
    r->bits >>= 2;
    r->nbits -= 2;
    return b;
}

static inline int code_of(uint8_t b)
{
    switch (b) {
    case 'C': return 1;
    case 'G': return 2;
    case 'T': return 3;
    default: return 0;
    }
}

/* growable per-thread sequence buffer */
typedef struct {
    uint8_t *p;
    int64_t n, cap;
} buf_t;

static int buf_reserve(buf_t *b, int64_t need)
{
    if (need <= b->cap) return 1;
    int64_t c = b->cap ? b->cap : 4096;
    while (c < need) c *= 2;
    uint8_t *q = (uint8_t *)realloc(b->p, (size_t)c);
    if (!q) return 0;
    b->p = q;
    b->cap = c;
    return 1;
}

static inline int buf_push(buf_t *b, uint8_t v)
{
    if (b->n == b->cap && !buf_reserve(b, b->n + 1)) return 0;
    b->p[b->n++] = v;
    return 1;
}

/* substitutions / insertions / deletions over src -> dst (see header) */
static int mutate(rng_t *r, const uint8_t *src, int64_t n, double ps, double pi, double pd, int max_indel, buf_t *dst)
{
    dst->n = 0;
    if (!buf_reserve(dst, n + 16)) return 0;
    for (int64_t k = 0; k < n;) {
        const double u = unif(r);
        const uint8_t b = src[k];
        if (u < ps) {
            if (!buf_push(dst, ACGT[(code_of(b) + (int)irange(r, 1, 3)) & 3])) return 0;
            k++;
        } else if (u < ps + pi) {
            if (!buf_push(dst, b)) return 0;
            const int L = (int)irange(r, 1, max_indel);
            for (int x = 0; x < L; x++)
                if (!buf_push(dst, rbase(r))) return 0;
            k++;
        } else if (u < ps + pi + pd) {
            k += irange(r, 1, max_indel);
        } else {
            if (!buf_push(dst, b)) return 0;
            k++;
        }
    }
    return 1;
}

typedef struct {
    buf_t q, src, t;
} scratch_t;

/* One pair of workload w: query in s->q, target in s->t, per-pair attributes
 * into *op / *h0.  Returns 0 on allocation failure. */
static int make_pair(int w, uint64_t seed, uint64_t pair, scratch_t *s, uint8_t *op, uint32_t *h0)
{
    rng_t r;
    rng_seed(&r, seed, pair);
    *op = 0;
    *h0 = 0;
    int64_t ql;
    double ps, pi, pd, n_rate = 0.0;
    int max_indel, flank = -1, kind = 0;
    int64_t tclip_lo = 1, tclip_hi = INT64_MAX;
    switch (w) {
    case 0:
        ql = irange(&r, 100, 150), ps = 0.02, pi = pd = 0.0025, max_indel = 3, n_rate = 0.001, flank = 20;
        break;
    case 1:
        ql = 150, ps = 0.03, pi = pd = 0.005, max_indel = 3, flank = 75, tclip_lo = 150, tclip_hi = 300;
        *op = unif(&r) < 0.5 ? REVERSE_COMPLEMENT : 0;
        break;
    case 2: {
        ql = (int64_t)exp(log(50.0) + unif(&r) * (log(1000.0) - log(50.0)));
        ps = 0.01 + 0.07 * unif(&r);
        const double ind = 0.005 + 0.025 * unif(&r);
        pi = pd = ind / 2, max_indel = 10;
        break;
    }
    case 3: {
        ql = irange(&r, 250, 2000);
        static const double rates[4] = {0.005, 0.02, 0.05, 0.10};
        const double ind = rates[irange(&r, 0, 3)];
        ps = 0.01 + 0.04 * unif(&r);
        pi = pd = ind / 2, max_indel = 3;
        *h0 = (uint32_t)irange(&r, 20, 60);
        break;
    }
    case 4: {
        double x = floor(250.0 * exp(0.8 * normal(&r)) + 0.5);
        ql = (int64_t)(x < 50 ? 50 : (x > 5000 ? 5000 : x));
        const double u = unif(&r);
        kind = u < 0.6 ? 0 : (u < 0.9 ? 1 : 2);
        const double err = kind == 0 ? 0.01 + 0.01 * unif(&r) : 0.05 + 0.07 * unif(&r);
        ps = kind == 0 ? err : 0.25 * err;
        const double ind = kind == 0 ? 0.002 : 0.75 * err;
        pi = pd = ind / 2, max_indel = 5;
        *h0 = (uint32_t)irange(&r, 20, 60);
        break;
    }
    default:
        return 0;
    }
    /* query */
    s->q.n = 0;
    if (!buf_reserve(&s->q, ql)) return 0;
    for (int64_t k = 0; k < ql; k++) s->q.p[k] = rbase(&r);
    s->q.n = ql;
    if (n_rate > 0)
        for (int64_t k = 0; k < ql; k++)
            if (unif(&r) < n_rate) s->q.p[k] = N_BASE;
    /* target source: the query, with random flanks */
    const uint8_t *src = s->q.p;
    int64_t sn = ql;
    if (flank >= 0) {
        const int64_t left = irange(&r, 0, flank), right = irange(&r, 0, flank);
        s->src.n = 0;
        if (!buf_reserve(&s->src, left + ql + right)) return 0;
        for (int64_t k = 0; k < left; k++) s->src.p[k] = rbase(&r);
        memcpy(s->src.p + left, s->q.p, (size_t)ql);
        for (int64_t k = 0; k < right; k++) s->src.p[left + ql + k] = rbase(&r);
        src = s->src.p;
        sn = left + ql + right;
    }
    if (!mutate(&r, src, sn, ps, pi, pd, max_indel, &s->t)) return 0;
    if (kind == 2)
        for (int64_t k = 0; k < s->t.n; k++) s->t.p[k] = rbase(&r);
    if (s->t.n > tclip_hi) s->t.n = tclip_hi;
    while (s->t.n < tclip_lo)
        if (!buf_push(&s->t, rbase(&r))) return 0;
    return 1;
}

static void set_threads(int threads)
{
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

/* Pass 1: lengths and per-pair attributes of pairs idx[0..n) (idx NULL:
 * pairs first .. first + n - 1).  q_op / h0 may be NULL.  Returns 0, or -1 on
 * a bad workload id or allocation failure. */
int gbw_lengths(int w, uint64_t seed, int64_t first, const int64_t *idx, int64_t n, uint32_t *q_len, uint32_t *t_len,
                uint8_t *q_op, uint32_t *h0, int threads)
{
    if (w < 0 || w > 4 || n < 0) return -1;
    set_threads(threads);
    int bad = 0;
#pragma omp parallel reduction(| : bad)
    {
        scratch_t s;
        memset(&s, 0, sizeof(s));
#pragma omp for schedule(dynamic, 1024)
        for (int64_t i = 0; i < n; i++) {
            uint8_t op;
            uint32_t h;
            if (!make_pair(w, seed, (uint64_t)(idx ? idx[i] : first + i), &s, &op, &h)) {
                bad = 1;
                continue;
            }
            q_len[i] = (uint32_t)s.q.n;
            t_len[i] = (uint32_t)s.t.n;
            if (q_op) q_op[i] = op;
            if (h0) h0[i] = h;
        }
        free(s.q.p);
        free(s.src.p);
        free(s.t.p);
    }
    return bad ? -1 : 0;
}

/* Pass 2: bases of the same pairs at byte offsets q_off / t_off of q / t,
 * N-padded to the next multiple of 8.  The lengths are pass 1's. */
int gbw_fill(int w, uint64_t seed, int64_t first, const int64_t *idx, int64_t n, const uint64_t *q_off,
             const uint64_t *t_off, uint8_t *q, uint8_t *t, int threads)
{
    if (w < 0 || w > 4 || n < 0) return -1;
    set_threads(threads);
    int bad = 0;
#pragma omp parallel reduction(| : bad)
    {
        scratch_t s;
        memset(&s, 0, sizeof(s));
#pragma omp for schedule(dynamic, 1024)
        for (int64_t i = 0; i < n; i++) {
            uint8_t op;
            uint32_t h;
            if (!make_pair(w, seed, (uint64_t)(idx ? idx[i] : first + i), &s, &op, &h)) {
                bad = 1;
                continue;
            }
            const int64_t qp = (s.q.n + 7) & ~(int64_t)7, tp = (s.t.n + 7) & ~(int64_t)7;
            memcpy(q + q_off[i], s.q.p, (size_t)s.q.n);
            memset(q + q_off[i] + s.q.n, N_BASE, (size_t)(qp - s.q.n));
            memcpy(t + t_off[i], s.t.p, (size_t)s.t.n);
            memset(t + t_off[i] + s.t.n, N_BASE, (size_t)(tp - s.t.n));
        }
        free(s.q.p);
        free(s.src.p);
        free(s.t.p);
    }
    return bad ? -1 : 0;
}

/* Core count OpenMP would use (for reporting). */
int gbw_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
