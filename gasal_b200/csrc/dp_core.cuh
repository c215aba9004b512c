/*
 * dp_core.cuh -- device code of the per-pair Gotoh sweeps, shared by the
 * one-pair-per-thread kernel (dp_kernels.cu) and the warp-cooperative kernel
 * (dp_wc.cu).  Everything here has internal linkage in each translation unit.
 *
 * The conventions (sweep order, int16 row buffer, scorer policies, per-column
 * first-maximum keys) are described at the top of dp_kernels.cu.
 */
#ifndef GB_DP_CORE_CUH
#define GB_DP_CORE_CUH

#include "gb_internal.h"

namespace gb {
namespace {

constexpr int N_CODE4 = 0xE; /* low nibble of 'N' */
constexpr int NEG16 = -32768;

struct RowBuf {
    uint32_t *base;
    uint32_t stride;
    __device__ __forceinline__ uint32_t ld(int c) const { return base[(size_t)c * stride]; }
    __device__ __forceinline__ void st(int c, uint32_t v) const { base[(size_t)c * stride] = v; }
};

__device__ __forceinline__ int sext16(uint32_t v) { return (int)(int16_t)(v & 0xFFFFu); }
__device__ __forceinline__ int hi16(uint32_t v) { return (int)v >> 16; }
__device__ __forceinline__ uint32_t pack_he(int h, int e) { return (uint32_t)(uint16_t)h | ((uint32_t)e << 16); }

__device__ __forceinline__ int code(uint32_t w, int k) { return (int)((w >> (28 - 4 * k)) & 15u); }

/* a * b + c (low 32 bits) as one integer multiply-add.  The cell loops are
 * bound by the ALU pipe (min/max, permutes, logic); position keys and 16-bit
 * merges written this way issue on the FMA pipe instead. */
__device__ __forceinline__ uint32_t mad_lo_u32(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t d;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}
/* the column key 8*H + r (r = 7 - row in the band) */
__device__ __forceinline__ int key8(int H, int r) { return (int)mad_lo_u32((uint32_t)H, 8u, (uint32_t)r); }

__device__ __forceinline__ uint32_t nib_rev(uint32_t x)
{
    const uint32_t r = __byte_perm(x, 0, 0x0123);
    return ((r >> 4) & 0x0F0F0F0Fu) | ((r << 4) & 0xF0F0F0F0u);
}

/* 8 codes at base positions p..p+7 of a packed run, reversed (position p+7
 * first), positions below 0 read as code 0.  Requires p+7 < len, p >= -7. */
__device__ __forceinline__ uint32_t rev_window(const uint32_t *w, int p)
{
    uint32_t win;
    if (p >= 0) {
        const int sh = (p & 7) << 2;
        const uint32_t w0 = w[p >> 3];
        win = sh ? ((w0 << sh) | (w[(p >> 3) + 1] >> (32 - sh))) : w0;
    } else {
        win = w[0] >> ((-p) << 2);
    }
    return nib_rev(win);
}

/* Per-band substitution rows.  LOCAL scoring: N against anything scores 0;
 * GLOBAL scoring: N is an ordinary base (reference src/gasal_kernels.h:39-56,
 * built without N_PENALTY). */
struct Band {
    int g[8], ma[8], mm[8];
    __device__ __forceinline__ void load(uint32_t gw, const Scores &sc, bool local)
    {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            g[k] = code(gw, k);
            const bool n = local && g[k] == N_CODE4;
            ma[k] = n ? 0 : sc.match;
            mm[k] = n ? 0 : -sc.mismatch;
        }
    }
    __device__ __forceinline__ int s(int k, int r, bool rzero) const
    {
        const int v = (r == g[k]) ? ma[k] : mm[k];
        return rzero ? 0 : v;
    }
};

/* PRMT-based substitution lookup.  Base codes fall into classes A C G T N
 * and "0" (the code the reference's reversal writes); a per-block table in
 * shared memory holds, for every query code, the 8 signed score bytes against
 * the classes.  Per band each row gets a byte selector whose upper three
 * nibbles replicate the selected byte's sign, so one prmt yields the
 * sign-extended score of a cell.  Pairs holding any other code (IUPAC letters
 * etc.) use the compare-based Band instead. */
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

/* code -> class: 1(A)->0 3(C)->1 7(G)->2 4(T)->3 14(N)->4 0->5, others 6 */
constexpr uint64_t CLASS_LUT = (5ull << 0) | (0ull << 4) | (6ull << 8) | (1ull << 12) | (3ull << 16) |
                               (6ull << 20) | (6ull << 24) | (2ull << 28) | (6ull << 32) | (6ull << 36) |
                               (6ull << 40) | (6ull << 44) | (6ull << 48) | (6ull << 52) | (4ull << 56) |
                               (6ull << 60);
constexpr uint32_t PLAIN_CODES = (1u << 0) | (1u << 1) | (1u << 3) | (1u << 4) | (1u << 7) | (1u << 14);

__device__ __forceinline__ uint32_t class_of(uint32_t code) { return (uint32_t)(CLASS_LUT >> (4 * code)) & 15u; }

/* 1 when every code of the words is in PLAIN_CODES */
__device__ __forceinline__ bool plain_words(const uint32_t *w, int n)
{
    uint32_t bad = 0;
    for (int i = 0; i < n; i++) {
        const uint32_t x = w[i];
#pragma unroll
        for (int k = 0; k < 8; k++) bad |= ~(PLAIN_CODES >> ((x >> (4 * k)) & 15u)) & 1u;
    }
    return bad == 0;
}

/* score table: entry r = 8 score bytes of query code r against the classes */
__device__ void build_score_table(uint2 *tab, const Scores &sc, bool local)
{
    const int rep[8] = {1, 3, 7, 4, 14, 0, 2, 2};
    for (int r = threadIdx.x; r < 16; r += blockDim.x) {
        uint32_t lo = 0, hi = 0;
        for (int j = 0; j < 8; j++) {
            const int g = rep[j];
            int v;
            if (local && (r == 14 || g == 14)) v = 0;
            else v = (r == g) ? sc.match : -sc.mismatch;
            if (j >= 6) v = 0;
            const uint32_t byte = (uint32_t)(v & 0xFF);
            if (j < 4) lo |= byte << (8 * j);
            else hi |= byte << (8 * (j - 4));
        }
        tab[r] = make_uint2(lo, hi);
    }
}

struct FastBand {
    uint32_t sel[8];
    __device__ __forceinline__ void load(uint32_t gw)
    {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint32_t c = class_of((gw >> (28 - 4 * k)) & 15u);
            sel[k] = c | ((c | 8u) * 0x1110u);
        }
    }
    __device__ __forceinline__ int s(int k, uint2 t) const { return (int)prmt(t.x, t.y, sel[k]); }
};

struct Res {
    int score, q_end, t_end, q_start, t_start, score2, q_end2, t_end2;
};

/* Direction nibble, reference src/kernels/local_kernel_template.h:45-60 and
 * src/kernels/global.h:14-26. */
__device__ __forceinline__ uint32_t dir_nib(int M, int diag, int H, int F, int E, const Scores &sc)
{
    uint32_t d = (H == M) ? (M >= diag ? 0u : 1u) : (H == F ? 3u : 2u);
    d |= ((M - sc.oe) > (F - sc.e)) ? 0u : 8u;
    d |= ((M - sc.oe) > (E - sc.e)) ? 0u : 4u;
    return d;
}

/* Scorer policies: Fast = prmt table lookup, Cmp = compares (any code). */
struct ScFast {
    FastBand b;
    const uint2 *tab;
    uint2 col;
    __device__ __forceinline__ void band(uint32_t gw, const Scores &, bool) { b.load(gw); }
    __device__ __forceinline__ void column(int rbase) { col = tab[rbase]; }
    __device__ __forceinline__ int s(int k) const { return b.s(k, col); }
};
struct ScCmp {
    Band b;
    bool local;
    int r;
    bool rz;
    __device__ __forceinline__ void band(uint32_t gw, const Scores &sc, bool loc)
    {
        local = loc;
        b.load(gw, sc, loc);
    }
    __device__ __forceinline__ void column(int rbase)
    {
        r = rbase;
        rz = local && rbase == N_CODE4;
    }
    __device__ __forceinline__ int s(int k) const { return b.s(k, r, rz); }
};

/* first maximum of a column in sweep order: key = 8*H + (7-k) */
__device__ __forceinline__ int col_key(const int *key)
{
    int m = __vimax3_s32(key[0], key[1], key[2]);
    m = __vimax3_s32(m, key[3], key[4]);
    m = __vimax3_s32(m, key[5], key[6]);
    return max(m, key[7]);
}

/* =========================== LOCAL ====================================== */
template <bool SECOND, bool TB, class SC>
__device__ void local_fwd(const uint32_t *q, int qregs, const uint32_t *t, int tregs, const Scores &sc,
                          RowBuf rb, uint4 *tb, SC scr, Res &r)
{
    const int q8 = qregs << 3;
    for (int c = 0; c < q8; c++) rb.st(c, 0u);
    int best = 0, brow = 0, bcol = 0;
    int sec = 0, srow = 0, scol = 0, sprev = 0;
    for (int T = 0; T < tregs; T++) {
        scr.band(t[T], sc, true);
        int F[8], D[8];
#pragma unroll
        for (int k = 0; k < 8; k++) F[k] = 0, D[k] = 0;
        for (int j = 0; j < qregs; j++) {
            const uint32_t qw = q[j];
            uint32_t dir[8];
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int c = (j << 3) + b;
                scr.column(code(qw, b));
                const uint32_t v = rb.ld(c);
                const int up0 = sext16(v);
                int e = hi16(v);
                int Hn[8], key[8];
                uint32_t dw = 0;
                /* second best: a cell qualifies when H is below the running
                 * maximum before it (local_kernel_template.h:145-150); run
                 * = that running maximum, chained through the column */
                int run = best, cand[8];
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int M = D[k] + scr.s(k);
                    const int H = __vimax3_s32_relu(M, F[k], e);
                    if (TB) dw |= dir_nib(M, D[k], H, F[k], e, sc) << (28 - 4 * k);
                    const int t0 = M - sc.oe;
                    F[k] = __viaddmax_s32(F[k], -sc.e, t0);
                    e = __viaddmax_s32(e, -sc.e, t0);
                    key[k] = key8(H, 7 - k);
                    if (SECOND) {
                        bool ge;
                        run = __vibmax_s32(H, run, &ge);
                        cand[k] = ge ? -1 : key[k];
                    }
                    Hn[k] = H;
                }
                rb.st(c, pack_he(Hn[7], e));
                D[0] = up0;
#pragma unroll
                for (int k = 1; k < 8; k++) D[k] = Hn[k - 1];
                const int ck = col_key(key);
                if ((ck >> 3) > best) best = ck >> 3, brow = (T << 3) + 7 - (ck & 7), bcol = c;
                if (SECOND) {
                    const int cs = col_key(cand);
                    if (cs >= 0 && (cs >> 3) > sec) sec = cs >> 3, srow = (T << 3) + 7 - (cs & 7);
                    if (sprev < best) scol = c;
                    sprev = max(sec, sprev);
                }
                if (TB) dir[b] = dw;
            }
            if (TB) {
                uint4 *tp = tb + (size_t)T * (2 * qregs) + 2 * j;
                tp[0] = make_uint4(dir[0], dir[1], dir[2], dir[3]);
                tp[1] = make_uint4(dir[4], dir[5], dir[6], dir[7]);
            }
        }
    }
    r.score = best, r.q_end = bcol, r.t_end = brow;
    if (SECOND) r.score2 = sec, r.q_end2 = scol, r.t_end2 = srow;
}

/* Start position: the recurrence run backwards from the words holding the end
 * cell, stopping after the column where the score reaches the forward score
 * (reference src/kernels/local_kernel_template.h:441-509).  The target row is
 * recorded as the reference does, gidx + k with gidx the original row of the
 * band's first reversed row. */
template <class SC>
__device__ void local_start(const uint32_t *q, int qregs, const uint32_t *t, int tregs, const Scores &sc,
                            RowBuf rb, SC scr, Res &r)
{
    const int rend_reg = min((r.q_end >> 3) + 1, qregs);
    const int gend_reg = min((r.t_end >> 3) + 1, tregs);
    const int fwd = r.score;
    const int qn = rend_reg << 3;
    int best = 0, xs = 0, ys = 0;
    for (int c = 0; c < qn; c++) rb.st(c, 0u);
    for (int T = 0; T < gend_reg && best < fwd; T++) {
        const int gidx = (gend_reg << 3) - 1 - (T << 3);
        scr.band(nib_rev(t[gend_reg - 1 - T]), sc, true);
        int F[8], D[8];
#pragma unroll
        for (int k = 0; k < 8; k++) F[k] = 0, D[k] = 0;
        for (int j = 0; j < rend_reg && best < fwd; j++) {
            const uint32_t qw = nib_rev(q[rend_reg - 1 - j]);
#pragma unroll
            for (int b = 0; b < 8; b++) {
                if (best >= fwd) break;
                const int c = (j << 3) + b;
                scr.column(code(qw, b));
                const uint32_t v = rb.ld(c);
                const int up0 = sext16(v);
                int e = hi16(v);
                int Hn[8], key[8];
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int M = D[k] + scr.s(k);
                    const int H = __vimax3_s32_relu(M, F[k], e);
                    const int t0 = M - sc.oe;
                    F[k] = __viaddmax_s32(F[k], -sc.e, t0);
                    e = __viaddmax_s32(e, -sc.e, t0);
                    key[k] = key8(H, 7 - k);
                    Hn[k] = H;
                }
                rb.st(c, pack_he(Hn[7], e));
                D[0] = up0;
#pragma unroll
                for (int k = 1; k < 8; k++) D[k] = Hn[k - 1];
                const int ck = col_key(key);
                if ((ck >> 3) > best) best = ck >> 3, ys = gidx + 7 - (ck & 7), xs = qn - 1 - c;
            }
        }
    }
    r.q_start = xs, r.t_start = ys;
}

/* =========================== GLOBAL ===================================== */
/* Reference src/kernels/global.h:30-303: gaps opened from M, no zero floor;
 * row buffer starts H(-1,c) = 0, -(o+e*c) with E = MINUS_INF; column 0 of row
 * R has diagonal 0 (R = 0) else -(o+e*R) and F = MINUS_INF; score = H at the
 * last real cell. */
template <bool TB, class SC>
__device__ void global_fwd(const uint32_t *q, int qregs, int qlen, const uint32_t *t, int tregs, int tlen,
                           const Scores &sc, RowBuf rb, uint4 *tb, SC scr, Res &r)
{
    const int q8 = qregs << 3;
    rb.st(0, pack_he(0, NEG16));
    for (int c = 1; c < q8; c++) rb.st(c, pack_he(-(sc.o + sc.e * c), NEG16));
    const int last_row = tlen - 1 - ((tregs - 1) << 3);
    int score = 0;
    for (int T = 0; T < tregs; T++) {
        scr.band(t[T], sc, false);
        int F[8], D[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int R = (T << 3) + k;
            F[k] = NEG16;
            D[k] = R == 0 ? 0 : -(sc.o + sc.e * R);
        }
        for (int j = 0; j < qregs; j++) {
            const uint32_t qw = q[j];
            uint32_t dir[8];
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int c = (j << 3) + b;
                scr.column(code(qw, b));
                const uint32_t v = rb.ld(c);
                const int up0 = sext16(v);
                int e = hi16(v);
                int Hn[8];
                uint32_t dw = 0;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int M = D[k] + scr.s(k);
                    const int H = __vimax3_s32(M, F[k], e);
                    if (TB) dw |= dir_nib(M, D[k], H, F[k], e, sc) << (28 - 4 * k);
                    const int t0 = M - sc.oe;
                    F[k] = __viaddmax_s32(F[k], -sc.e, t0);
                    e = __viaddmax_s32(e, -sc.e, t0);
                    Hn[k] = H;
                }
                rb.st(c, pack_he(Hn[7], e));
                D[0] = up0;
#pragma unroll
                for (int k = 1; k < 8; k++) D[k] = Hn[k - 1];
                if (T == tregs - 1 && c == qlen - 1) {
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        if (k == last_row) score = Hn[k];
                }
                if (TB) dir[b] = dw;
            }
            if (TB) {
                uint4 *tp = tb + (size_t)T * (2 * qregs) + 2 * j;
                tp[0] = make_uint4(dir[0], dir[1], dir[2], dir[3]);
                tp[1] = make_uint4(dir[4], dir[5], dir[6], dir[7]);
            }
        }
    }
    r.score = score;
}

/* GLOBAL score without traceback, two 8-row bands per sweep of the query:
 * the same cells, in the same order per band, with the same values as
 * global_fwd.  H and E crossing from the first band to the second are
 * narrowed to int16 exactly as the row buffer narrows them between bands;
 * they just stay in registers, so each column carries 16 rows of
 * independent work (the single-band loop is latency-bound) and the row
 * buffer is read and written once per two bands. */
template <class SC>
__device__ void global_fwd2(const uint32_t *q, int qregs, int qlen, const uint32_t *t, int tregs, int tlen,
                            const Scores &sc, RowBuf rb, SC scr, Res &r)
{
    const int q8 = qregs << 3;
    rb.st(0, pack_he(0, NEG16));
    for (int c = 1; c < q8; c++) rb.st(c, pack_he(-(sc.o + sc.e * c), NEG16));
    const int last_row = tlen - 1 - ((tregs - 1) << 3);
    int score = 0;
    SC scb = scr;
    for (int T = 0; T < tregs; T += 2) {
        const bool two = T + 1 < tregs;
        scr.band(t[T], sc, false);
        if (two) scb.band(t[T + 1], sc, false);
        int F[8], D[8], FB[8], DB[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int R = (T << 3) + k, RB = R + 8;
            F[k] = NEG16, FB[k] = NEG16;
            D[k] = R == 0 ? 0 : -(sc.o + sc.e * R);
            DB[k] = -(sc.o + sc.e * RB);
        }
        const bool last_a = T == tregs - 1, last_b = T + 1 == tregs - 1;
        for (int j = 0; j < qregs; j++) {
            const uint32_t qw = q[j];
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int c = (j << 3) + b;
                const int cq = code(qw, b);
                scr.column(cq);
                const uint32_t v = rb.ld(c);
                const int up0 = sext16(v);
                int e = hi16(v);
                int Hn[8];
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int M = D[k] + scr.s(k);
                    const int H = __vimax3_s32(M, F[k], e);
                    const int t0 = M - sc.oe;
                    F[k] = __viaddmax_s32(F[k], -sc.e, t0);
                    e = __viaddmax_s32(e, -sc.e, t0);
                    Hn[k] = H;
                }
                D[0] = up0;
#pragma unroll
                for (int k = 1; k < 8; k++) D[k] = Hn[k - 1];
                if (last_a && c == qlen - 1) {
#pragma unroll
                    for (int k = 0; k < 8; k++)
                        if (k == last_row) score = Hn[k];
                }
                if (two) {
                    /* the second band sees the first through the int16 row buffer */
                    const int upB = (int)(int16_t)Hn[7];
                    int eB = (int)(int16_t)e;
                    scb.column(cq);
                    int HB[8];
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const int M = DB[k] + scb.s(k);
                        const int H = __vimax3_s32(M, FB[k], eB);
                        const int t0 = M - sc.oe;
                        FB[k] = __viaddmax_s32(FB[k], -sc.e, t0);
                        eB = __viaddmax_s32(eB, -sc.e, t0);
                        HB[k] = H;
                    }
                    rb.st(c, pack_he(HB[7], eB));
                    DB[0] = upB;
#pragma unroll
                    for (int k = 1; k < 8; k++) DB[k] = HB[k - 1];
                    if (last_b && c == qlen - 1) {
#pragma unroll
                        for (int k = 0; k < 8; k++)
                            if (k == last_row) score = HB[k];
                    }
                } else {
                    rb.st(c, pack_he(Hn[7], e));
                }
            }
        }
    }
    r.score = score;
}

/* ========================= SEMI_GLOBAL ================================== */
/* Reference src/kernels/semiglobal_kernel_template.h.  Standard Gotoh (gaps
 * opened from H), N scores 0.  head/tail select the free end gaps. */
struct SemiAcc {
    int best, brow, bcol, sec, srow, scol;
};

__device__ __forceinline__ int semi_init_h(int head, int c, const Scores &sc)
{
    if (head == QUERY_ || head == BOTH_) return 0;
    return c == 0 ? 0 : (int)(int16_t)(-(sc.o + sc.e * c));
}

__device__ void semi_init_rows(int head, int q8, const Scores &sc, RowBuf rb)
{
    const bool zero = (head == QUERY_ || head == BOTH_);
    for (int c = 0; c < q8; c++) rb.st(c, zero ? 0u : pack_he(semi_init_h(head, c, sc), NEG16));
}

/* One sweep over bands T0..tregs-1 of (q, t) as given by the word functions;
 * leaves once acc.best >= stop_at (checked per band and per query word).
 *
 * E opens from H here (semiglobal_kernel_template.h:105-107): E_k =
 * max(E_{k-1} - e, H_{k-1} - (o+e)) with H_{k-1} = max(M, F, E_{k-1}) of the
 * row above, a chain of three dependent operations per row.  When o >= 0,
 * E_{k-1} - (o+e) <= E_{k-1} - e, so E_k = max(E_{k-1} - e, max(M, F)_{k-1} -
 * (o+e)) -- the same value with one operation per row on the chain (OPEN_NN). */
/* Direction nibble of SEMI_GLOBAL cell (r, c) for its traceback (an
 * extension: the reference instantiates semi-global WITH_TB empty,
 * semiglobal_kernel_template.h:227).  Bits 0-1: the source of H (0 diagonal
 * with M >= its diagonal predecessor, 1 diagonal with a drop, 3 F, 2 E; ties
 * in that order); bit 3: F(r,c) extends F(r,c-1) (F(r,c-1) - e >= H(r,c-1) -
 * (o+e)); bit 2: E(r,c) extends E(r-1,c) the same way.  Unlike dir_nib, the
 * gap bits describe the cell's own F and E: gaps open from H here. */
__device__ __forceinline__ uint32_t semi_nib(int M, int diag, int H, int F, int Fin, int Hleft, int Ein, int Hup,
                                             const Scores &sc)
{
    uint32_t d = (H == M) ? (M >= diag ? 0u : 1u) : (H == F ? 3u : 2u);
    d |= (Fin - sc.e >= Hleft - sc.oe) ? 8u : 0u;
    d |= (Ein - sc.e >= Hup - sc.oe) ? 4u : 0u;
    return d;
}

template <bool SECOND, bool OPEN_NN, class SC, class QW, class TW, bool TB = false>
__device__ void semi_sweep(QW qword, int qregs, int qlen, TW tword, int tregs, int tlen, const Scores &sc,
                           int head, int tail, int T0, int stop_at, RowBuf rb, SC &scr, SemiAcc &a,
                           uint4 *tb = nullptr)
{
    const bool free_head_t = (head == TARGET_ || head == BOTH_);
    const bool free_tail_t = (tail == TARGET_ || tail == BOTH_);
    int R = 0;
    for (int T = T0; T < tregs && a.best < stop_at; T++, R += 8) {
        scr.band(tword(T), sc, true);
        int F[8], D[8], Hc[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            F[k] = NEG16;
            if (free_head_t) {
                Hc[k] = 0, D[k] = 0;
            } else {
                Hc[k] = -(sc.o + sc.e * (R + k));
                D[k] = (R + k) == 0 ? 0 : -(sc.o + sc.e * (R + k));
            }
        }
        for (int j = 0; j < qregs && a.best < stop_at; j++) {
            const uint32_t qw = qword(j);
            uint32_t dir[8];
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int c = (j << 3) + b;
                scr.column(code(qw, b));
                const uint32_t v = rb.ld(c);
                const int up0 = sext16(v);
                int e = hi16(v), up = up0;
                int Hn[8];
                if (OPEN_NN) {
                    int x = up0 - sc.oe; /* H of the row above the band, opened */
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        F[k] = __viaddmax_s32(F[k], -sc.e, Hc[k] - sc.oe);
                        const int M = D[k] + scr.s(k);
                        e = __viaddmax_s32(e, -sc.e, x);
                        const int mf = max(M, F[k]);
                        x = mf - sc.oe;
                        Hn[k] = max(mf, e);
                    }
                } else {
                    uint32_t dw = 0;
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const int Fin = F[k], Ein = e;
                        F[k] = __viaddmax_s32(F[k], -sc.e, Hc[k] - sc.oe);
                        const int M = D[k] + scr.s(k);
                        e = __viaddmax_s32(e, -sc.e, up - sc.oe);
                        const int H = __vimax3_s32(M, F[k], e);
                        if (TB) dw |= semi_nib(M, D[k], H, F[k], Fin, Hc[k], Ein, up, sc) << (28 - 4 * k);
                        Hn[k] = H;
                        up = H;
                    }
                    if (TB) dir[b] = dw;
                }
                rb.st(c, pack_he(Hn[7], e));
                D[0] = up0;
#pragma unroll
                for (int k = 1; k < 8; k++) D[k] = Hn[k - 1];
#pragma unroll
                for (int k = 0; k < 8; k++) Hc[k] = Hn[k];
                if (free_tail_t && c == qlen - 1) {
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const int row = (T << 3) + k, H = Hn[k];
                        if (H > a.best && row < tlen) a.best = H, a.brow = row;
                        if (SECOND && H > a.sec && H < a.best && row < tlen) a.sec = H, a.srow = row;
                    }
                }
            }
            if (TB) {
                uint4 *tp = tb + (size_t)T * (2 * qregs) + 2 * j;
                tp[0] = make_uint4(dir[0], dir[1], dir[2], dir[3]);
                tp[1] = make_uint4(dir[4], dir[5], dir[6], dir[7]);
            }
        }
    }
}

/* free query tail: scan of the last (padded) row, :185-213 */
template <bool SECOND>
__device__ void semi_tail_query(int head, int q8, int qlen, int tlen, int mql, const Scores &sc, RowBuf rb,
                                SemiAcc &a)
{
    const int lim = SECOND ? max(qlen, min(mql, tlen)) : qlen;
    for (int m = 0; m < lim && m < mql; m++) {
        const int v = m < q8 ? sext16(rb.ld(m)) : semi_init_h(head, m, sc);
        if (v > a.best && m < qlen) a.bcol = m, a.best = v;
        if (SECOND && v > a.sec && v < a.best && m < tlen) a.scol = m, a.sec = v;
    }
    if (a.bcol != tlen) a.brow = qlen;
    if (SECOND && a.scol != tlen) a.srow = qlen;
}

/* The start pass alone: both sequences reversed base by base, pads as code
 * 0 (:227-381), from the forward pass's score (best), end row (brow) and end
 * column (bcol). */
template <class SC>
__device__ void semi_start(const uint32_t *q, int qregs, int qlen, const uint32_t *t, int tregs, int tlen,
                           const Scores &sc, int head, int tail, int mql, RowBuf rb, SC &scr, int best, int brow,
                           int bcol, Res &r)
{
    const int q8 = qregs << 3;
    const int x = tregs - ((brow >> 3) + 1);
    int gend_reg = x > 0 ? x - 1 : x;
    if (gend_reg < 0) gend_reg = 0; /* reference reads before its array here */
    const int fwd = best;
    SemiAcc b = {NEG16, 0, bcol, NEG16, 0, 0};
    semi_init_rows(head, q8, sc, rb);
    auto rq = [&](int j) { return rev_window(q, qlen - 8 - (j << 3)); };
    auto rt = [&](int T) { return rev_window(t, tlen - 8 - (T << 3)); };
    if (sc.o >= 0)
        semi_sweep<false, true>(rq, qregs, qlen, rt, tregs, tlen, sc, head, tail, gend_reg, fwd, rb, scr, b);
    else
        semi_sweep<false, false>(rq, qregs, qlen, rt, tregs, tlen, sc, head, tail, gend_reg, fwd, rb, scr, b);
    if (tail == QUERY_ || tail == BOTH_) semi_tail_query<false>(head, q8, qlen, tlen, mql, sc, rb, b);
    r.t_start = (tlen - 1) - b.brow;
    r.q_start = (qlen - 1) - b.bcol;
}

template <bool SECOND, bool START, class SC, bool TB = false>
__device__ void semi_global(const uint32_t *q, int qregs, int qlen, const uint32_t *t, int tregs, int tlen,
                            const Scores &sc, int head, int tail, int mql, RowBuf rb, SC scr, Res &r,
                            uint4 *tb = nullptr)
{
    const int q8 = qregs << 3;
    SemiAcc a = {NEG16, qlen, tlen, NEG16, qlen, tlen};
    semi_init_rows(head, q8, sc, rb);
    auto qf = [&](int j) { return q[j]; };
    auto tf = [&](int T) { return t[T]; };
    if (TB) /* the traceback reads the H-open recurrence's own gap bits: no OPEN_NN form */
        semi_sweep<SECOND, false, SC, decltype(qf), decltype(tf), true>(qf, qregs, qlen, tf, tregs, tlen, sc, head,
                                                                        tail, 0, 0x7fffffff, rb, scr, a, tb);
    else if (sc.o >= 0)
        semi_sweep<SECOND, true>([&](int j) { return q[j]; }, qregs, qlen, [&](int T) { return t[T]; }, tregs, tlen,
                                 sc, head, tail, 0, 0x7fffffff, rb, scr, a);
    else
        semi_sweep<SECOND, false>([&](int j) { return q[j]; }, qregs, qlen, [&](int T) { return t[T]; }, tregs,
                                  tlen, sc, head, tail, 0, 0x7fffffff, rb, scr, a);
    if (tail == QUERY_ || tail == BOTH_) semi_tail_query<SECOND>(head, q8, qlen, tlen, mql, sc, rb, a);
    r.score = a.best, r.t_end = a.brow, r.q_end = a.bcol;
    if (SECOND) r.score2 = a.sec, r.t_end2 = a.srow, r.q_end2 = a.scol;
    if (!START) return;
    semi_start(q, qregs, qlen, t, tregs, tlen, sc, head, tail, mql, rb, scr, a.best, a.brow, a.bcol, r);
}

/* =========================== BANDED ===================================== */
/* Reference src/kernels/banded.h:10-139: local, gaps opened from H, swept
 * per band T over query words max(0,T-k_other+1) .. min(k+T,qregs)-1. */
template <class SC>
__device__ void banded(const uint32_t *q, int qregs, const uint32_t *t, int tregs, int kw, const Scores &sc,
                       RowBuf rb, SC scr, Res &r)
{
    const int q8 = qregs << 3;
    const int k_other = tregs - (qregs - kw);
    for (int c = 0; c < q8; c++) rb.st(c, 0u);
    int best = 0, brow = 0, bcol = 0;
    for (int T = 0; T < tregs; T++) {
        scr.band(t[T], sc, true);
        int F[8], D[8], Hc[8];
#pragma unroll
        for (int k = 0; k < 8; k++) F[k] = 0, D[k] = 0, Hc[k] = 0;
        const int j_lo = max(0, T - k_other + 1), j_hi = min(kw + T, qregs);
        for (int j = j_lo; j < j_hi; j++) {
            const uint32_t qw = q[j];
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int c = (j << 3) + b;
                scr.column(code(qw, b));
                const uint32_t v = rb.ld(c);
                const int up0 = sext16(v);
                int e = hi16(v), up = up0;
                int Hn[8], key[8];
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    F[k] = __viaddmax_s32(F[k], -sc.e, Hc[k] - sc.oe);
                    int H = __vimax3_s32_relu(D[k] + scr.s(k), F[k], 0);
                    e = __viaddmax_s32(e, -sc.e, up - sc.oe);
                    H = max(H, e);
                    key[k] = key8(H, 7 - k);
                    Hn[k] = H;
                    up = H;
                }
                rb.st(c, pack_he(Hn[7], e));
                D[0] = up0;
#pragma unroll
                for (int k = 1; k < 8; k++) D[k] = Hn[k - 1];
#pragma unroll
                for (int k = 0; k < 8; k++) Hc[k] = Hn[k];
                const int ck = col_key(key);
                if ((ck >> 3) > best) best = ck >> 3, brow = (T << 3) + 7 - (ck & 7), bcol = c;
            }
        }
    }
    r.score = best, r.q_end = bcol, r.t_end = brow;
}

/* BANDED start position, an extension: the reference's banded kernel reports
 * ends only (src/kernels/banded.h:10-139).  Defined as the LOCAL start pass
 * (local_start): the banded recurrence run backwards from the 8-base words
 * holding the end cell over the reversed words, on the forward pass's band
 * tiles (band T's words [max(0, T-k_other+1), min(kw+T, qregs)), clipped to
 * the end word, visited in reverse), leaving after the column in which the
 * score reaches the forward score.  The start is reported as the forward row
 * and column of the cell where that maximum was first reached. */
template <class SC>
__device__ void banded_start(const uint32_t *q, int qregs, const uint32_t *t, int tregs, int kw, const Scores &sc,
                             RowBuf rb, SC scr, Res &r)
{
    const int rend_reg = min((r.q_end >> 3) + 1, qregs);
    const int gend_reg = min((r.t_end >> 3) + 1, tregs);
    const int k_other = tregs - (qregs - kw);
    const int fwd = r.score;
    const int qn = rend_reg << 3;
    int best = 0, xs = 0, ys = 0;
    for (int c = 0; c < qn; c++) rb.st(c, 0u);
    for (int T = 0; T < gend_reg && best < fwd; T++) {
        const int Tf = gend_reg - 1 - T;       /* the forward band */
        const int gidx = (Tf << 3) + 7;        /* forward row of the reversed band's first row */
        scr.band(nib_rev(t[Tf]), sc, true);
        int F[8], D[8], Hc[8];
#pragma unroll
        for (int k = 0; k < 8; k++) F[k] = 0, D[k] = 0, Hc[k] = 0;
        const int j_lo = max(0, Tf - k_other + 1), j_hi = min(min(kw + Tf, qregs), rend_reg);
        for (int j = rend_reg - j_hi; j < rend_reg - j_lo && best < fwd; j++) {
            const uint32_t qw = nib_rev(q[rend_reg - 1 - j]);
#pragma unroll
            for (int b = 0; b < 8; b++) {
                if (best >= fwd) break;
                const int c = (j << 3) + b;
                scr.column(code(qw, b));
                const uint32_t v = rb.ld(c);
                const int up0 = sext16(v);
                int e = hi16(v), up = up0;
                int Hn[8], key[8];
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    F[k] = __viaddmax_s32(F[k], -sc.e, Hc[k] - sc.oe);
                    int H = __vimax3_s32_relu(D[k] + scr.s(k), F[k], 0);
                    e = __viaddmax_s32(e, -sc.e, up - sc.oe);
                    H = max(H, e);
                    key[k] = key8(H, 7 - k);
                    Hn[k] = H;
                    up = H;
                }
                rb.st(c, pack_he(Hn[7], e));
                D[0] = up0;
#pragma unroll
                for (int k = 1; k < 8; k++) D[k] = Hn[k - 1];
#pragma unroll
                for (int k = 0; k < 8; k++) Hc[k] = Hn[k];
                const int ck = col_key(key);
                if ((ck >> 3) > best) best = ck >> 3, ys = gidx - (7 - (ck & 7)), xs = qn - 1 - c;
            }
        }
    }
    r.q_start = xs, r.t_start = ys;
}

/* ============================= KSW ====================================== */
/* BWA-style extension (reference src/kernels/ksw_kernel_template.h:46-199).
 * eh[j] = (H(i-1,j-1) before the update / H(i,j-1) after, E(i,j)) lives in
 * the row buffer as two words per column.  Reference traits kept: a row whose
 * maximum is 0 (or that triggers z-drop) ends only the current 8-row target
 * tile; the end-to-end score is taken when the tiled column loop's final
 * index equals qlen (end == qlen or qlen a multiple of 8); exclusive ends. */
__device__ void ksw(const uint32_t *q, int qlen, const uint32_t *t, int tlen, uint32_t h0u, int zdrop,
                    const Scores &sc, RowBuf rb, Res &r)
{
    const int e_del = sc.e, e_ins = sc.e, oe_del = sc.oe, oe_ins = sc.oe, o_del = sc.o;
    const int h0 = (int)h0u;
    const int L8 = (qlen >> 3) << 3;
    for (int j = 0; j <= qlen + 1; j++) rb.st(2 * j, 0u), rb.st(2 * j + 1, 0u);
    rb.st(0, (uint32_t)h0);
    int prevh = h0u > (uint32_t)oe_ins ? (int)(h0u - (uint32_t)oe_ins) : 0;
    rb.st(2, (uint32_t)prevh);
    for (int j = 2; j <= qlen && prevh > e_ins; ++j) {
        prevh -= e_ins;
        rb.st(2 * j, (uint32_t)prevh);
    }
    int mx = h0, max_i = -1, max_j = -1, max_ie = -1, gscore = -1, mo = 0;
    int beg = 0, end = qlen;
    for (int i = 0; i < tlen;) {
        int f = 0, h1, m = 0, mj = -1;
        if (beg == 0) {
            h1 = (int)(h0u - (uint32_t)(o_del + e_del * (i + 1)));
            if (h1 < 0) h1 = 0;
        } else {
            h1 = 0;
        }
        const int g = code(t[i >> 3], i & 7);
        const bool gN = g == N_CODE4;
        for (int j = beg; j < end; ++j) {
            int M = (int)rb.ld(2 * j), e = (int)rb.ld(2 * j + 1);
            rb.st(2 * j, (uint32_t)h1);
            const int rbase = code(q[j >> 3], j & 7);
            const int s = (gN || rbase == N_CODE4) ? 0 : (rbase == g ? sc.match : -sc.mismatch);
            M = M ? M + s : 0;
            int h = max(M, e);
            h = max(h, f);
            h1 = h;
            mj = m > h ? mj : j;
            m = max(m, h);
            const int tdel = max(M - oe_del, 0);
            e = max(e - e_del, tdel);
            rb.st(2 * j + 1, (uint32_t)e);
            const int tins = max(M - oe_ins, 0);
            f = max(f - e_ins, tins);
        }
        rb.st(2 * end, (uint32_t)h1);
        rb.st(2 * end + 1, 0u);
        if (max(L8, end) == qlen) {
            max_ie = gscore > h1 ? max_ie : i;
            gscore = max(gscore, h1);
        }
        bool leave = false;
        if (m == 0) {
            leave = true;
        } else if (m > mx) {
            mx = m, max_i = i, max_j = mj;
            mo = max(mo, abs(mj - i));
        } else if (zdrop > 0) {
            if (i - max_i > mj - max_j) {
                if (mx - m - ((i - max_i) - (mj - max_j)) * e_del > zdrop) leave = true;
            } else {
                if (mx - m - ((mj - max_j) - (i - max_i)) * e_ins > zdrop) leave = true;
            }
        }
        if (leave) {
            i = ((i >> 3) + 1) << 3;
            continue;
        }
        int j;
        for (j = beg; j < end && rb.ld(2 * j) == 0u && rb.ld(2 * j + 1) == 0u; ++j)
            ;
        beg = j;
        for (j = end; j >= beg && rb.ld(2 * j) == 0u && rb.ld(2 * j + 1) == 0u; --j)
            ;
        end = j + 2 < qlen ? j + 2 : qlen;
        i++;
    }
    if (gscore <= 0 || gscore <= mx - 5) {
        r.score = mx, r.q_end = max_j + 1, r.t_end = max_i + 1;
    } else {
        r.score = gscore, r.q_end = qlen, r.t_end = max_ie + 1;
    }
    r.score2 = mo; /* ksw has no second best: the slot carries max_off */
}


} // namespace
} // namespace gb

#endif
