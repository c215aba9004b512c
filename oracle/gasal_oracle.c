/*
 * gasal_oracle.c -- scalar C restatement of GASAL2's alignment path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline); the
 * product never links it.  Parity of every routine here is pinned against the
 * reference library compiled for sm_100a (the .npz fixtures in tests/golden); see
 * gasal_oracle.h.
 *
 * All citations are reference paths (src/...).  Conventions used throughout:
 *   - a pair is aligned on its PADDED grid: target rows 0..8*tregs-1 and query
 *     columns 0..8*qregs-1, padding bases being N (code 0xE), exactly as the
 *     reference kernels sweep whole packed words;
 *   - rows are processed in bands of 8 ("tile rows"); inside a band the sweep
 *     is column by column, and inside a column row by row.  Every
 *     first-maximum / second-best rule below depends on that order;
 *   - H and E leave a band through a row buffer that the reference stores as
 *     short2, so they are truncated to int16 there (ORC_INT16_ROWS);
 *   - D[k] is the diagonal predecessor of row k in the current column,
 *     Hc[k] the H of row k in the previous column, F[k] the horizontal gap
 *     state of row k.
 */
#include "gasal_oracle.h"

#include <stdlib.h>
#include <string.h>
#include <omp.h>

/* enum values of gasal.h (src/gasal.h:50-65) */
enum { SRC_NONE = 0, SRC_QUERY = 1, SRC_TARGET = 2, SRC_BOTH = 3 };
enum { A_GLOBAL = 1, A_SEMI_GLOBAL = 2, A_LOCAL = 3, A_BANDED = 5, A_KSW = 6 };
enum { S_WITHOUT_START = 0, S_WITH_START = 1, S_WITH_TB = 2 };

#define NEG16 (-32768) /* MINUS_INF = SHRT_MIN, src/gasal_kernels.h:35 */
#define N_NIBBLE 0xE   /* N_VALUE = N_CODE & 0xF, src/gasal_kernels.h:37 */

typedef struct {
    int match, mismatch, o, e, oe;
    int compat;
    int mql;
} sc_t;

typedef struct {
    int score, q_end, t_end, q_start, t_start, score2, q_end2, t_end2;
    uint32_t n_ops;
} res_t;

typedef struct { uint32_t w[4]; } tile_t; /* one uint4 of direction nibbles */

static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int row16(int v, const sc_t *s) { return (s->compat & ORC_INT16_ROWS) ? (int)(int16_t)v : v; }

/* Substitution scores.  LOCAL variant (used by local, semi-global, banded and
 * ksw) scores N against anything as 0; GLOBAL variant treats N as an ordinary
 * base (src/gasal_kernels.h:47-56, no N_PENALTY). */
static inline int sub_local(int r, int g, const sc_t *s)
{
    if (r == N_NIBBLE || g == N_NIBBLE) return 0;
    return r == g ? s->match : -s->mismatch;
}
static inline int sub_global(int r, int g, const sc_t *s) { return r == g ? s->match : -s->mismatch; }

/* ------------------------------------------------------------------------ */
/* K1 pack: 8 ASCII bytes -> one word of 4-bit codes (low nibble of each
 * byte), first base in bits 31..28 (src/kernels/pack_rc_seqs.h:19-31). */
void oracle_pack(const uint8_t *ascii, uint32_t nbytes, uint32_t *words)
{
    for (uint32_t w = 0; w < nbytes / 8; w++) {
        uint32_t v = 0;
        for (int k = 0; k < 8; k++) v |= (uint32_t)(ascii[8 * w + k] & 15) << (28 - 4 * k);
        words[w] = v;
    }
}

static inline uint32_t nib_reverse(uint32_t v)
{
    uint32_t r = 0;
    for (int k = 0; k < 8; k++) r |= ((v >> (4 * k)) & 15u) << (28 - 4 * k);
    return r;
}

/* K2 reverse / complement of one sequence in place
 * (src/kernels/pack_rc_seqs.h:56-212).  op bit 0 reverses, bit 1 complements
 * A<->T, C<->G (codes 1<->4, 3<->7); other codes are left alone.
 * Reverse (ORC_RC_REF_REVERSE): the reference counts pad nibbles by comparing
 * 4-bit nibbles with the 8-bit N_CODE (:115), never a match, and then shifts
 * 32-bit words by 32 (:286,303), which is undefined.  Its sm_100a build
 * (nvcc 12.9), run on a B200 over every length 1..48 (fixture rc.npz), swaps
 * word pairs i <-> regs-1-i for i < ceil(regs/2) such that word regs-1-i
 * becomes the nibble-reversed original word i while word i becomes 0, the
 * middle word of an odd run ending up reversed in place.  Off = reverse the
 * real bases only, pads staying at the end. */
void oracle_revcomp(uint32_t *words, uint32_t word_off, uint32_t len, int op, int compat)
{
    uint32_t regs = (len + 7) / 8;
    uint32_t *w = words + word_off;
    if (op & 1) {
        if (compat & ORC_RC_REF_REVERSE) {
            const uint32_t half = (regs + 1) / 2;
            for (uint32_t i = 0; i < half; i++) {
                const uint32_t head = w[i];
                w[i] = 0;
                w[regs - 1 - i] = nib_reverse(head);
            }
        } else {
            uint8_t codes[8 * 64];
            uint8_t *c = len <= 8 * 64 ? codes : (uint8_t *)malloc(8 * regs);
            for (uint32_t k = 0; k < 8 * regs; k++) c[k] = (w[k >> 3] >> (28 - 4 * (k & 7))) & 15;
            for (uint32_t k = 0; k < len / 2; k++) {
                uint8_t t = c[k];
                c[k] = c[len - 1 - k];
                c[len - 1 - k] = t;
            }
            for (uint32_t i = 0; i < regs; i++) {
                uint32_t v = 0;
                for (int k = 0; k < 8; k++) v |= (uint32_t)c[8 * i + k] << (28 - 4 * k);
                w[i] = v;
            }
            if (c != codes) free(c);
        }
    }
    if (op & 2) {
        for (uint32_t i = 0; i < regs; i++) {
            uint32_t v = w[i], r = 0;
            for (int k = 0; k < 8; k++) {
                uint32_t c = (v >> (28 - 4 * k)) & 15;
                if (c == 1) c = 4;
                else if (c == 4) c = 1;
                else if (c == 3) c = 7;
                else if (c == 7) c = 3;
                r |= c << (28 - 4 * k);
            }
            w[i] = r;
        }
    }
}

/* Direction nibble of one cell (src/kernels/local_kernel_template.h:45-60,
 * src/kernels/global.h:14-26): bits 1..0 = where H came from (0 diagonal with
 * M >= diagonal predecessor, 1 diagonal with a drop, 3 horizontal gap F, 2
 * anything else -- E, or the zero floor of local); bit 3 = F at the next
 * column extends rather than opens; bit 2 = same for E at the next row.
 * Ties favour extension. */
static inline uint32_t dir_nibble(int M, int diag, int H, int F, int E, const sc_t *s)
{
    uint32_t d = (H == M) ? (M >= diag ? 0u : 1u) : (H == F ? 3u : 2u);
    if (!((M - s->oe) > (F - s->e))) d |= 8u;
    if (!((M - s->oe) > (E - s->e))) d |= 4u;
    return d;
}

static inline void tb_put(tile_t *tb, int qregs, int T, int c, int k, uint32_t nib)
{
    tile_t *t = &tb[(size_t)T * (2 * qregs) + (c >> 2)];
    t->w[c & 3] |= nib << (28 - 4 * k);
}

/* ------------------------------------------------------------------------ */
/* LOCAL (Smith-Waterman, gaps opened from M; E and F start at 0).
 * src/kernels/local_kernel_template.h:71-438.  Also records the first-best
 * cell in sweep order, and with `second` the second best: the largest value
 * lower than the running maximum at the moment its cell is swept (:145-164). */
static void local_fwd(const uint8_t *qc, int qregs, const uint8_t *tc, int tregs, const sc_t *s,
                      int second, tile_t *tb, int *Hb, int *Eb, res_t *r)
{
    const int q8 = 8 * qregs;
    int best = 0, brow = 0, bcol = 0, prev = 0;
    int sec = 0, srow = 0, scol = 0, sprev = 0;
    for (int c = 0; c < q8; c++) Hb[c] = 0, Eb[c] = 0;
    for (int T = 0; T < tregs; T++) {
        int F[8] = {0}, D[8] = {0}, Hn[8];
        const uint8_t *g = tc + 8 * T;
        for (int c = 0; c < q8; c++) {
            const int rb = qc[c];
            const int up0 = Hb[c];
            int e = Eb[c];
            for (int k = 0; k < 8; k++) {
                const int M = D[k] + sub_local(rb, g[k], s);
                int H = imax(imax(M, F[k]), imax(e, 0));
                if (tb) tb_put(tb, qregs, T, c, k, dir_nibble(M, D[k], H, F[k], e, s));
                F[k] = imax(M - s->oe, F[k] - s->e);
                e = imax(M - s->oe, e - s->e);
                if (best < H) best = H, brow = 8 * T + k;
                if (second && sec < H && best > H) sec = H, srow = 8 * T + k;
                Hn[k] = H;
            }
            Hb[c] = row16(Hn[7], s);
            Eb[c] = row16(e, s);
            D[0] = up0;
            for (int k = 1; k < 8; k++) D[k] = Hn[k - 1];
            if (prev < best) bcol = c;
            if (second) {
                if (sprev < best) scol = c;
                sprev = imax(sec, sprev);
            }
            prev = imax(best, prev);
        }
    }
    r->score = best, r->q_end = bcol, r->t_end = brow;
    if (second) r->score2 = sec, r->q_end2 = scol, r->t_end2 = srow;
}

/* LOCAL start position: the same recurrence run backwards from the 8-base
 * words holding the end cell, over the reversed padded sequences, stopping
 * after the column in which the score reaches the forward score
 * (src/kernels/local_kernel_template.h:441-509). */
static void local_start(const uint8_t *qc, int qregs, const uint8_t *tc, int tregs, const sc_t *s,
                        int *Hb, int *Eb, res_t *r)
{
    const int rend_reg = imin((r->q_end >> 3) + 1, qregs);
    const int gend_reg = imin((r->t_end >> 3) + 1, tregs);
    const int fwd = r->score;
    const int qn = 8 * rend_reg;
    int best = 0, prev = 0, xs = 0, ys = 0;
    for (int c = 0; c < qn; c++) Hb[c] = 0, Eb[c] = 0;
    for (int T = 0; T < gend_reg && best < fwd; T++) {
        const int gidx = 8 * gend_reg - 1 - 8 * T; /* original row of the band's first reversed row */
        int F[8] = {0}, D[8] = {0}, Hn[8];
        for (int c = 0; c < qn && best < fwd; c++) {
            const int qpos = qn - 1 - c;
            const int rb = qc[qpos];
            const int up0 = Hb[c];
            int e = Eb[c];
            for (int k = 0; k < 8; k++) {
                const int M = D[k] + sub_local(rb, tc[gidx - k], s);
                int H = imax(imax(M, F[k]), imax(e, 0));
                F[k] = imax(M - s->oe, F[k] - s->e);
                e = imax(M - s->oe, e - s->e);
                if (best < H) best = H, ys = (s->compat & ORC_LOCAL_START_ROW) ? gidx + k : gidx - k;
                Hn[k] = H;
            }
            Hb[c] = row16(Hn[7], s);
            Eb[c] = row16(e, s);
            D[0] = up0;
            for (int k = 1; k < 8; k++) D[k] = Hn[k - 1];
            if (prev < best) xs = qpos;
            prev = imax(best, prev);
        }
    }
    r->q_start = xs, r->t_start = ys;
}

/* ------------------------------------------------------------------------ */
/* GLOBAL (Needleman-Wunsch, gaps opened from M).  src/kernels/global.h:30-303.
 * Boundaries: the row buffer starts as H(-1,c) = 0 for c = 0 and -(o+e*c)
 * after, E = MINUS_INF (:57-60); column 0 of row R sees the diagonal
 * 0 (R = 0) or -(o+e*R) and F = MINUS_INF (:63-71).  The score is H at the
 * last real cell (:98-103,299). */
static void global_fwd(const uint8_t *qc, int qregs, int qlen, const uint8_t *tc, int tregs, int tlen,
                       const sc_t *s, tile_t *tb, int *Hb, int *Eb, res_t *r)
{
    const int q8 = 8 * qregs;
    int cap[8] = {0};
    Hb[0] = 0;
    for (int c = 1; c < q8; c++) Hb[c] = row16(-(s->o + s->e * c), s);
    for (int c = 0; c < q8; c++) Eb[c] = NEG16;
    for (int T = 0; T < tregs; T++) {
        int F[8], D[8], Hn[8];
        for (int k = 0; k < 8; k++) {
            const int R = 8 * T + k;
            F[k] = NEG16;
            D[k] = R == 0 ? 0 : -(s->o + s->e * R);
        }
        const uint8_t *g = tc + 8 * T;
        for (int c = 0; c < q8; c++) {
            const int rb = qc[c];
            const int up0 = Hb[c];
            int e = Eb[c];
            for (int k = 0; k < 8; k++) {
                const int M = D[k] + sub_global(rb, g[k], s);
                const int H = imax(imax(M, F[k]), e);
                if (tb) tb_put(tb, qregs, T, c, k, dir_nibble(M, D[k], H, F[k], e, s));
                F[k] = imax(M - s->oe, F[k] - s->e);
                e = imax(M - s->oe, e - s->e);
                Hn[k] = H;
            }
            Hb[c] = row16(Hn[7], s);
            Eb[c] = row16(e, s);
            D[0] = up0;
            for (int k = 1; k < 8; k++) D[k] = Hn[k - 1];
            if (c == qlen - 1)
                for (int k = 0; k < 8; k++) cap[k] = Hn[k];
        }
    }
    r->score = cap[tlen - 1 - 8 * (tregs - 1)];
}

/* ------------------------------------------------------------------------ */
/* SEMI_GLOBAL (standard Gotoh: gaps opened from H; N scores 0).
 * src/kernels/semiglobal_kernel_template.h:39-226 (forward) and :227-382
 * (start).  `head`/`tail` select which end gaps are free. */
typedef struct {
    int best, brow, bcol, sec, srow, scol;
} semi_acc_t;

/* Row buffer before the first band (:87-99): all zero when the query head is
 * free, else H(-1,c) = 0, -(o+e*c) and E = MINUS_INF. */
static void semi_init_rows(int head, int n, int *Hb, int *Eb, const sc_t *s)
{
    if (head == SRC_QUERY || head == SRC_BOTH) {
        for (int c = 0; c < n; c++) Hb[c] = 0, Eb[c] = 0;
    } else {
        Hb[0] = 0;
        Eb[0] = NEG16;
        for (int c = 1; c < n; c++) Hb[c] = row16(-(s->o + s->e * c), s), Eb[c] = NEG16;
    }
}

/* One sweep over bands T0..tregs-1, leaving whenever acc->best reaches
 * stop_at (checked per band and per 8-column word, :301,323).  Left edge of a
 * band (:114-129): free target head -> H(R,-1) = 0 and diagonal 0; otherwise
 * H(R,-1) = -(o+e*R) and diagonal 0 for R = 0 else -(o+e*R), R counting rows
 * from the start of this sweep.  The free-target-tail maximum is taken over
 * the last real query column, real rows only (:160-178). */
/* Direction nibble of a SEMI_GLOBAL cell for the traceback extension (the
 * reference instantiates semi-global WITH_TB empty,
 * semiglobal_kernel_template.h:227): bits 0-1 the source of H (0 diagonal
 * with M >= its diagonal predecessor, 1 diagonal with a drop, 3 F, 2 E; ties
 * in that order); bit 3 set when F(r,c) extends F(r,c-1)
 * (F(r,c-1) - e >= H(r,c-1) - (o+e)); bit 2 the same for E(r,c) from the row
 * above.  The gap bits describe the cell's own F and E (gaps open from H). */
static inline uint32_t semi_nibble(int M, int diag, int H, int F, int Fin, int Hleft, int Ein, int Hup,
                                   const sc_t *s)
{
    uint32_t d = (H == M) ? (M >= diag ? 0u : 1u) : (H == F ? 3u : 2u);
    if (Fin - s->e >= Hleft - s->oe) d |= 8u;
    if (Ein - s->e >= Hup - s->oe) d |= 4u;
    return d;
}

static void semi_sweep(const uint8_t *qc, int qregs, int qlen, const uint8_t *tc, int tregs, int tlen,
                       const sc_t *s, int head, int tail, int second, int T0, int stop_at, int *Hb, int *Eb,
                       semi_acc_t *a, tile_t *tb)
{
    const int free_head_t = (head == SRC_TARGET || head == SRC_BOTH);
    const int free_tail_t = (tail == SRC_TARGET || tail == SRC_BOTH);
    int R = 0;
    for (int T = T0; T < tregs && a->best < stop_at; T++, R += 8) {
        int F[8], D[8], Hc[8], Hn[8];
        for (int k = 0; k < 8; k++) {
            F[k] = NEG16;
            if (free_head_t) {
                Hc[k] = 0, D[k] = 0;
            } else {
                Hc[k] = -(s->o + s->e * (R + k));
                D[k] = (R + k) == 0 ? 0 : -(s->o + s->e * (R + k));
            }
        }
        const uint8_t *g = tc + 8 * T;
        for (int j = 0; j < qregs && a->best < stop_at; j++) {
            for (int c = 8 * j; c < 8 * j + 8; c++) {
                const int rb = qc[c];
                const int up0 = Hb[c];
                int e = Eb[c], up = up0;
                for (int k = 0; k < 8; k++) {
                    const int Fin = F[k], Ein = e;
                    F[k] = imax(Hc[k] - s->oe, F[k] - s->e);
                    const int M = D[k] + sub_local(rb, g[k], s);
                    e = imax(up - s->oe, e - s->e);
                    const int H = imax(imax(M, F[k]), e);
                    if (tb) tb_put(tb, qregs, T, c, k, semi_nibble(M, D[k], H, F[k], Fin, Hc[k], Ein, up, s));
                    Hn[k] = H;
                    up = H;
                }
                Hb[c] = row16(Hn[7], s);
                Eb[c] = row16(e, s);
                D[0] = up0;
                for (int k = 1; k < 8; k++) D[k] = Hn[k - 1];
                for (int k = 0; k < 8; k++) Hc[k] = Hn[k];
                if (free_tail_t && c == qlen - 1) {
                    for (int k = 0; k < 8; k++) {
                        const int row = 8 * T + k, H = Hn[k];
                        if (H > a->best && row < tlen) a->best = H, a->brow = row;
                        if (second && H > a->sec && H < a->best && row < tlen) a->sec = H, a->srow = row;
                    }
                }
            }
        }
    }
}

/* Free query tail: maximum over the row buffer, i.e. the last PADDED row,
 * for columns below the query length; the scan runs to MAX_QUERY_LEN and the
 * second-best test bounds the column by the target length (:185-213). */
static void semi_tail_query(int qlen, int tlen, int mql, const int *Hb, int second, semi_acc_t *a)
{
    for (int m = 0; m < mql; m++) {
        const int v = Hb[m];
        if (v > a->best && m < qlen) a->bcol = m, a->best = v;
        if (second && v > a->sec && v < a->best && m < tlen) a->scol = m, a->sec = v;
    }
    if (a->bcol != tlen) a->brow = qlen;
    if (second && a->scol != tlen) a->srow = qlen;
}

static void semi_global(const uint8_t *qc, int qregs, int qlen, const uint8_t *tc, int tregs, int tlen,
                        const sc_t *s, int head, int tail, int second, int with_start, int nrow,
                        uint8_t *rq, uint8_t *rt, int *Hb, int *Eb, res_t *r, tile_t *tb)
{
    /* end positions start as (row = query length, column = target length),
     * :63-64,73-74 */
    semi_acc_t a = {NEG16, qlen, tlen, NEG16, qlen, tlen};
    semi_init_rows(head, nrow, Hb, Eb, s);
    semi_sweep(qc, qregs, qlen, tc, tregs, tlen, s, head, tail, second, 0, 0x7fffffff, Hb, Eb, &a, tb);
    if (tail == SRC_QUERY || tail == SRC_BOTH) semi_tail_query(qlen, tlen, s->mql, Hb, second, &a);
    r->score = a.best, r->t_end = a.brow, r->q_end = a.bcol;
    if (second) r->score2 = a.sec, r->t_end2 = a.srow, r->q_end2 = a.scol;
    if (!with_start) return;

    /* Start (:227-381): both sequences reversed base by base into zeroed
     * words (pads become code 0), then the same sweep from word
     * gend_reg of the reversed target, keeping the forward column. */
    for (int k = 0; k < 8 * qregs; k++) rq[k] = k < qlen ? qc[qlen - 1 - k] : 0;
    for (int k = 0; k < 8 * tregs; k++) rt[k] = k < tlen ? tc[tlen - 1 - k] : 0;
    const int x = tregs - ((a.brow >> 3) + 1);
    int gend_reg = x > 0 ? x - 1 : x;
    if (gend_reg < 0) gend_reg = 0; /* the reference indexes before its array here */
    const int fwd = a.best;
    semi_acc_t b = {NEG16, 0, a.bcol, NEG16, 0, 0};
    semi_init_rows(head, nrow, Hb, Eb, s);
    semi_sweep(rq, qregs, qlen, rt, tregs, tlen, s, head, tail, 0, gend_reg, fwd, Hb, Eb, &b, NULL);
    if (tail == SRC_QUERY || tail == SRC_BOTH) {
        for (int m = 0; m < s->mql; m++) {
            if (Hb[m] > b.best && m < qlen) b.bcol = m, b.best = Hb[m];
        }
        if (b.bcol != tlen) b.brow = qlen;
    }
    r->t_start = (tlen - 1) - b.brow;
    r->q_start = (qlen - 1) - b.bcol;
}

/* ------------------------------------------------------------------------ */
/* BANDED: local alignment (gaps opened from H, E/F from 0) restricted, per
 * band of 8 target rows T, to query words max(0,T-k_other+1) ..
 * min(k+T,qregs)-1 with k = k_band>>3 and k_other = tregs-(qregs-k).  Columns
 * outside the band keep whatever the row buffer held.
 * src/kernels/banded.h:10-139. */
static void banded(const uint8_t *qc, int qregs, const uint8_t *tc, int tregs, int kw, const sc_t *s,
                   int *Hb, int *Eb, res_t *r)
{
    const int q8 = 8 * qregs;
    const int k_other = tregs - (qregs - kw);
    int best = 0, brow = 0, bcol = 0, prev = 0;
    for (int c = 0; c < q8; c++) Hb[c] = 0, Eb[c] = 0;
    for (int T = 0; T < tregs; T++) {
        int F[8] = {0}, D[8] = {0}, Hc[8] = {0}, Hn[8];
        const uint8_t *g = tc + 8 * T;
        const int c_lo = imax(0, T - k_other + 1) * 8;
        const int c_hi = imin(kw + T, qregs) * 8;
        for (int c = c_lo; c < c_hi; c++) {
            const int rb = qc[c];
            const int up0 = Hb[c];
            int e = Eb[c], up = up0;
            for (int k = 0; k < 8; k++) {
                F[k] = imax(Hc[k] - s->oe, F[k] - s->e);
                int H = imax(imax(D[k] + sub_local(rb, g[k], s), F[k]), 0);
                e = imax(up - s->oe, e - s->e);
                H = imax(H, e);
                if (best < H) best = H, brow = 8 * T + k;
                Hn[k] = H;
                up = H;
            }
            Hb[c] = row16(Hn[7], s);
            Eb[c] = row16(e, s);
            D[0] = up0;
            for (int k = 1; k < 8; k++) D[k] = Hn[k - 1];
            for (int k = 0; k < 8; k++) Hc[k] = Hn[k];
            if (prev < best) bcol = c;
            prev = imax(best, prev);
        }
    }
    r->score = best, r->q_end = bcol, r->t_end = brow;
}

/* BANDED start position (an extension of this project: the reference's
 * banded kernel reports ends only, src/kernels/banded.h:10-139).  Defined as
 * the LOCAL start pass (local_start above): the banded recurrence run
 * backwards from the 8-base words holding the end cell over the reversed
 * padded sequences, on the forward pass's band tiles (forward band T's words
 * clipped to the end word, visited in reverse), stopping after the column in
 * which the score reaches the forward score.  The start is the forward row
 * and column of the cell where that maximum was first reached. */
static void banded_start(const uint8_t *qc, int qregs, const uint8_t *tc, int tregs, int kw, const sc_t *s,
                         int *Hb, int *Eb, res_t *r)
{
    const int rend_reg = imin((r->q_end >> 3) + 1, qregs);
    const int gend_reg = imin((r->t_end >> 3) + 1, tregs);
    const int k_other = tregs - (qregs - kw);
    const int fwd = r->score;
    const int qn = 8 * rend_reg;
    int best = 0, prev = 0, xs = 0, ys = 0;
    for (int c = 0; c < qn; c++) Hb[c] = 0, Eb[c] = 0;
    for (int T = 0; T < gend_reg && best < fwd; T++) {
        const int Tf = gend_reg - 1 - T;   /* forward band */
        const int gidx = 8 * Tf + 7;       /* forward row of the reversed band's first row */
        int F[8] = {0}, D[8] = {0}, Hc[8] = {0}, Hn[8];
        const int j_lo = imax(0, Tf - k_other + 1), j_hi = imin(imin(kw + Tf, qregs), rend_reg);
        for (int c = 8 * (rend_reg - j_hi); c < 8 * (rend_reg - j_lo) && best < fwd; c++) {
            const int qpos = qn - 1 - c;
            const int rb = qc[qpos];
            const int up0 = Hb[c];
            int e = Eb[c], up = up0;
            for (int k = 0; k < 8; k++) {
                F[k] = imax(Hc[k] - s->oe, F[k] - s->e);
                int H = imax(imax(D[k] + sub_local(rb, tc[gidx - k], s), F[k]), 0);
                e = imax(up - s->oe, e - s->e);
                H = imax(H, e);
                if (best < H) best = H, ys = gidx - k;
                Hn[k] = H;
                up = H;
            }
            Hb[c] = row16(Hn[7], s);
            Eb[c] = row16(e, s);
            D[0] = up0;
            for (int k = 1; k < 8; k++) D[k] = Hn[k - 1];
            for (int k = 0; k < 8; k++) Hc[k] = Hn[k];
            if (prev < best) xs = qpos;
            prev = imax(best, prev);
        }
    }
    r->q_start = xs, r->t_start = ys;
}

/* ------------------------------------------------------------------------ */
/* KSW: BWA-style seed extension from score h0.
 * src/kernels/ksw_kernel_template.h:46-199.  Rows are target bases, columns
 * query bases; only columns [beg, end) are swept per row.  Reference traits
 * kept: (1) "m == 0" (and a z-drop trigger) leave only the current 8-row
 * target tile (ORC_KSW_TILE_BREAK), the next tile resumes with the old
 * beg/end; (2) the end-to-end score is taken whenever the column loop's last
 * index equals qlen, which for the tiled loop means end == qlen or qlen a
 * multiple of 8 (:56,113-123,155-158); (3) ends are exclusive. */
typedef struct { int h, e; } eh_t;

static void ksw(const uint8_t *qc, int qlen, const uint8_t *tc, int tlen, uint32_t h0u, int zdrop,
                const sc_t *s, eh_t *eh, res_t *r)
{
    const int o_del = s->o, e_del = s->e, o_ins = s->o, e_ins = s->e;
    const int oe_del = o_del + e_del, oe_ins = o_ins + e_ins;
    const int h0 = (int)h0u;
    const int L8 = (qlen >> 3) << 3;
    for (int j = 0; j <= qlen + 1; j++) eh[j].h = 0, eh[j].e = 0;
    eh[0].h = h0;
    eh[1].h = h0u > (uint32_t)oe_ins ? (int)(h0u - (uint32_t)oe_ins) : 0;
    for (int j = 2; j <= qlen && eh[j - 1].h > e_ins; ++j) eh[j].h = eh[j - 1].h - e_ins;
    int max = h0, max_i = -1, max_j = -1, max_ie = -1, gscore = -1, max_off = 0;
    int beg = 0, end = qlen;
    for (int i = 0; i < tlen;) {
        int f = 0, h1, m = 0, mj = -1;
        if (beg == 0) {
            h1 = (int)(h0u - (uint32_t)(o_del + e_del * (i + 1)));
            if (h1 < 0) h1 = 0;
        } else {
            h1 = 0;
        }
        const int g = tc[i];
        for (int j = beg; j < end; ++j) {
            eh_t *p = &eh[j];
            int h, M = p->h, e = p->e, t;
            p->h = h1;
            M = M ? M + sub_local(qc[j], g, s) : 0;
            h = M > e ? M : e;
            h = h > f ? h : f;
            h1 = h;
            mj = m > h ? mj : j;
            m = m > h ? m : h;
            t = M - oe_del;
            t = t > 0 ? t : 0;
            e -= e_del;
            e = e > t ? e : t;
            p->e = e;
            t = M - oe_ins;
            t = t > 0 ? t : 0;
            f -= e_ins;
            f = f > t ? f : t;
        }
        eh[end].h = h1;
        eh[end].e = 0;
        if (imax(L8, end) == qlen) {
            max_ie = gscore > h1 ? max_ie : i;
            gscore = gscore > h1 ? gscore : h1;
        }
        int leave = 0;
        if (m == 0) {
            leave = 1;
        } else if (m > max) {
            max = m, max_i = i, max_j = mj;
            max_off = max_off > abs(mj - i) ? max_off : abs(mj - i);
        } else if (zdrop > 0) {
            if (i - max_i > mj - max_j) {
                if (max - m - ((i - max_i) - (mj - max_j)) * e_del > zdrop) leave = 1;
            } else {
                if (max - m - ((mj - max_j) - (i - max_i)) * e_ins > zdrop) leave = 1;
            }
        }
        if (leave) {
            if (!(s->compat & ORC_KSW_TILE_BREAK)) break;
            i = ((i >> 3) + 1) << 3;
            continue;
        }
        int j;
        for (j = beg; j < end && eh[j].h == 0 && eh[j].e == 0; ++j)
            ;
        beg = j;
        for (j = end; j >= beg && eh[j].h == 0 && eh[j].e == 0; --j)
            ;
        end = j + 2 < qlen ? j + 2 : qlen;
        i++;
    }
    r->score2 = max_off; /* ksw has no second best: the slot carries max_off (checker of the band labels) */
    if (gscore <= 0 || gscore <= max - 5) { /* PEN_CLIP5, :20,188-197 */
        r->score = max, r->q_end = max_j + 1, r->t_end = max_i + 1;
    } else {
        r->score = gscore, r->q_end = qlen, r->t_end = max_ie + 1;
    }
}

/* ------------------------------------------------------------------------ */
/* Traceback to run-length CIGAR bytes ((count << 2) | op, op 0 match, 1
 * mismatch, 2 deletion (consumes target), 3 insertion (consumes query)),
 * written last operation first.  src/kernels/get_tb.h:4-149.
 * LOCAL starts at the end cell and stops once the ops re-score to the
 * alignment score; GLOBAL starts at (tlen, qlen), one past the last cell, and
 * flushes any remaining target / query bases as 63-long runs. */
static uint32_t traceback(const tile_t *tb, int qregs, int algo, int i, int j, int total, const sc_t *s,
                          uint8_t *out, int *si, int *sj)
{
    const int q8 = 8 * qregs;
    uint32_t prev_op = 0, n_ops = 0, op_fill;
    int prev_tile = -1, op_select = 3, op_shift = 0, count = 0, curr = 0;
    tile_t tile = {{0, 0, 0, 0}};
    while (i >= 0 && j >= 0) {
        const int cell = (((i >> 3) * q8) << 3) + (j << 3) + (i & 7);
        const int tile_no = cell >> 5;
        if (tile_no != prev_tile) tile = tb[tile_no];
        prev_tile = tile_no;
        const int in_tile = cell & 31;
        const uint32_t nib = (tile.w[in_tile >> 3] >> (28 - ((in_tile & 7) << 2))) & 15u;
        const uint32_t op = (nib >> op_shift) & (uint32_t)op_select;
        op_fill = (op == 0 || op_select == 3) ? op : (uint32_t)op_shift;
        op_select = (op == 0 || (op == 1 && op_select == 3)) ? 3 : 1;
        op_shift = (op == 0 || (op == 1 && op_select == 3)) ? 0 : ((op == 2 || op == 3) ? (int)op : op_shift);
        if (count < 63 && op_fill == prev_op) {
            count++;
        } else {
            if (count > 0) out[n_ops++] = (uint8_t)(prev_op | ((uint32_t)count << 2));
            count = 1;
        }
        if (algo == A_LOCAL) {
            const int gap = (op_fill == 2 || op_fill == 3);
            curr += (gap && prev_op != op_fill) ? -s->oe : (gap ? -s->e : (op_fill == 1 ? -s->mismatch : s->match));
            if (curr == total) break;
        }
        prev_op = op_fill;
        if (op_fill == 0 || op_fill == 1 || op_fill == 2) i--;
        if (op_fill == 0 || op_fill == 1 || op_fill == 3) j--;
    }
    out[n_ops++] = (uint8_t)(prev_op | ((uint32_t)count << 2));
    if (algo == A_GLOBAL) {
        for (; i >= 0; i -= 63) out[n_ops++] = (uint8_t)(2u | ((uint32_t)imin(i + 1, 63) << 2));
        for (; j >= 0; j -= 63) out[n_ops++] = (uint8_t)(3u | ((uint32_t)imin(j + 1, 63) << 2));
    }
    *si = i, *sj = j;
    return n_ops;
}

/* SEMI_GLOBAL traceback for a free target tail (the extension above): from
 * the end cell (t_end, qlen - 1), in H the nibble's two low bits give a
 * diagonal move or the gap (E / F) H came from at the same cell; in a gap the
 * cell's own extend bit says whether the gap continues or was opened from H
 * of the cell the move reaches.  At a free leading edge (target for head
 * TARGET or BOTH, query for QUERY or BOTH) the walk stops; at a closed one
 * the remaining bases become one gap.  Runs as in traceback(), at most 63
 * long, last operation first.  si / sj: the first aligned target row and
 * query column. */
static uint32_t semi_traceback(const tile_t *tb, int qregs, int head, int i, int j, uint8_t *out, int *si,
                               int *sj)
{
    const int q8 = 8 * qregs;
    uint32_t n_ops = 0, run_op = 0;
    int run = 0, state = 0; /* 0 H, 2 E (deletion), 3 F (insertion) */
#define SEMI_PUT(o)                                                                                                \
    do {                                                                                                           \
        if (run > 0 && run < 63 && (uint32_t)(o) == run_op) {                                                      \
            run++;                                                                                                 \
        } else {                                                                                                   \
            if (run > 0) out[n_ops++] = (uint8_t)(run_op | ((uint32_t)run << 2));                                  \
            run_op = (uint32_t)(o), run = 1;                                                                       \
        }                                                                                                          \
    } while (0)
    while (i >= 0 && j >= 0) {
        const int cell = (((i >> 3) * q8) << 3) + (j << 3) + (i & 7);
        const tile_t *t = &tb[cell >> 5];
        const int in_tile = cell & 31;
        const uint32_t nib = (t->w[in_tile >> 3] >> (28 - ((in_tile & 7) << 2))) & 15u;
        if (state == 0) {
            const uint32_t src = nib & 3u;
            if (src <= 1) {
                SEMI_PUT(src);
                i--, j--;
                continue;
            }
            state = (int)src;
        }
        if (state == 2) {
            SEMI_PUT(2);
            state = (nib & 4u) ? 2 : 0;
            i--;
        } else {
            SEMI_PUT(3);
            state = (nib & 8u) ? 3 : 0;
            j--;
        }
    }
    const int free_t = head == SRC_TARGET || head == SRC_BOTH, free_q = head == SRC_QUERY || head == SRC_BOTH;
    int ts = i + 1, qs = j + 1;
    if (j < 0 && i >= 0 && !free_t) {
        for (; i >= 0; i--) SEMI_PUT(2);
        ts = 0;
    }
    if (i < 0 && j >= 0 && !free_q) {
        for (; j >= 0; j--) SEMI_PUT(3);
        qs = 0;
    }
    if (run > 0) out[n_ops++] = (uint8_t)(run_op | ((uint32_t)run << 2));
#undef SEMI_PUT
    *si = ts, *sj = qs;
    return n_ops;
}

/* ------------------------------------------------------------------------ */
static void unpack_codes(const uint32_t *words, uint32_t word_off, int n, uint8_t *codes)
{
    for (int k = 0; k < n; k++) codes[k] = (words[word_off + (k >> 3)] >> (28 - ((k & 7) << 2))) & 15u;
}

int oracle_align(const gb_params_t *p, const gb_batch_t *b, gb_out_t *o, int threads, int compat)
{
    return oracle_align_ex(p, b, o, threads, compat, 0);
}

int oracle_align_ex(const gb_params_t *p, const gb_batch_t *b, gb_out_t *o, int threads, int compat, int mql)
{
    if (!p || !b || !o || b->n <= 0 || (b->q_bytes & 7) || (b->t_bytes & 7)) return GB_ERR_ARG;
    const int algo = p->algo;
    if (algo != A_GLOBAL && algo != A_SEMI_GLOBAL && algo != A_LOCAL && algo != A_BANDED && algo != A_KSW)
        return GB_ERR_ARG;
    const int n = b->n;
    sc_t s = {p->match, p->mismatch, p->gap_open, p->gap_extend, p->gap_open + p->gap_extend, compat,
              mql > 0 ? mql : 2048};
    if (threads <= 0) threads = omp_get_max_threads();

    uint32_t *pq = (uint32_t *)calloc(b->q_bytes / 8 + 2, 4);
    uint32_t *pt = (uint32_t *)calloc(b->t_bytes / 8 + 2, 4);
    if (!pq || !pt) return GB_ERR_ALLOC;
    oracle_pack(b->q, b->q_bytes, pq);
    oracle_pack(b->t, b->t_bytes, pt);
    if (p->reverse_complement) {
        for (int i = 0; i < n; i++) {
            if (b->q_op && (b->q_op[i] & 3)) oracle_revcomp(pq, b->q_off[i] >> 3, b->q_len[i], b->q_op[i], compat);
            if (b->t_op && (b->t_op[i] & 3)) oracle_revcomp(pt, b->t_off[i] >> 3, b->t_len[i], b->t_op[i], compat);
        }
    }
    if (o->packed_q) memcpy(o->packed_q, pq, (b->q_bytes / 8) * 4);
    if (o->packed_t) memcpy(o->packed_t, pt, (b->t_bytes / 8) * 4);

    uint32_t maxq = 8, maxt = 8;
    for (int i = 0; i < n; i++) {
        if (b->q_len[i] > maxq) maxq = b->q_len[i];
        if (b->t_len[i] > maxt) maxt = b->t_len[i];
    }
    const int maxq8 = (int)((maxq + 7) & ~7u) + 8, maxt8 = (int)((maxt + 7) & ~7u) + 8;
    const int nrow = imax(maxq8, s.mql);
    const int with_tb = (p->start_pos == S_WITH_TB) &&
                        (algo == A_LOCAL || algo == A_GLOBAL || (algo == A_SEMI_GLOBAL && p->tail == SRC_TARGET));
    uint8_t **ops = with_tb ? (uint8_t **)calloc(n, sizeof(uint8_t *)) : NULL;
    uint32_t *nops = with_tb ? (uint32_t *)calloc(n, 4) : NULL;
    int err = 0;

#pragma omp parallel num_threads(threads)
    {
        int *Hb = (int *)malloc(sizeof(int) * nrow);
        int *Eb = (int *)malloc(sizeof(int) * nrow);
        uint8_t *qc = (uint8_t *)malloc(maxq8), *tc = (uint8_t *)malloc(maxt8);
        uint8_t *rq = (uint8_t *)malloc(maxq8), *rt = (uint8_t *)malloc(maxt8);
        eh_t *eh = (eh_t *)malloc(sizeof(eh_t) * (maxq + 2));
        if (!Hb || !Eb || !qc || !tc || !rq || !rt || !eh) {
#pragma omp atomic write
            err = 1;
        } else {
#pragma omp for schedule(dynamic, 16)
            for (int i = 0; i < n; i++) {
                const int qlen = (int)b->q_len[i], tlen = (int)b->t_len[i];
                res_t r;
                memset(&r, 0, sizeof(r));
                /* ksw runs on empty sequences too: the reference then returns the
                 * seed score h0 (src/kernels/ksw_kernel_template.h:176-186) */
                if ((qlen > 0 && tlen > 0) || algo == A_KSW) {
                    const int qregs = (qlen + 7) >> 3, tregs = (tlen + 7) >> 3;
                    const int sb = p->second_best != 0;
                    unpack_codes(pq, b->q_off[i] >> 3, 8 * qregs, qc);
                    unpack_codes(pt, b->t_off[i] >> 3, 8 * tregs, tc);
                    tile_t *tb = NULL;
                    if (with_tb) tb = (tile_t *)calloc((size_t)(tregs + 2) * 2 * qregs, sizeof(tile_t));
                    switch (algo) {
                    case A_LOCAL:
                        local_fwd(qc, qregs, tc, tregs, &s, sb, tb, Hb, Eb, &r);
                        if (p->start_pos == S_WITH_START) local_start(qc, qregs, tc, tregs, &s, Hb, Eb, &r);
                        break;
                    case A_GLOBAL:
                        global_fwd(qc, qregs, qlen, tc, tregs, tlen, &s, tb, Hb, Eb, &r);
                        break;
                    case A_SEMI_GLOBAL:
                        semi_global(qc, qregs, qlen, tc, tregs, tlen, &s, p->head, p->tail, sb,
                                    p->start_pos == S_WITH_START, nrow, rq, rt, Hb, Eb, &r, tb);
                        break;
                    case A_BANDED:
                        banded(qc, qregs, tc, tregs, p->k_band >> 3, &s, Hb, Eb, &r);
                        if (p->start_pos == S_WITH_START) banded_start(qc, qregs, tc, tregs, p->k_band >> 3, &s, Hb, Eb, &r);
                        break;
                    case A_KSW:
                        ksw(qc, qlen, tc, tlen, b->seed ? b->seed[i] : 0u, p->zdrop, &s, eh, &r);
                        break;
                    }
                    if (tb) {
                        uint8_t *buf = (uint8_t *)malloc((size_t)8 * (qregs + tregs) + 256);
                        int si, sj;
                        if (algo == A_LOCAL)
                            nops[i] = traceback(tb, qregs, algo, r.t_end, r.q_end, r.score, &s, buf, &si, &sj);
                        else if (algo == A_SEMI_GLOBAL)
                            nops[i] = semi_traceback(tb, qregs, p->head, r.t_end, qlen - 1, buf, &si, &sj);
                        else
                            nops[i] = traceback(tb, qregs, algo, tlen, qlen, 0, &s, buf, &si, &sj);
                        if (algo == A_LOCAL || algo == A_SEMI_GLOBAL) r.t_start = si, r.q_start = sj;
                        ops[i] = buf;
                        free(tb);
                    }
                }
                if (o->score) o->score[i] = r.score;
                if (algo != A_GLOBAL) {
                    if (o->q_end) o->q_end[i] = r.q_end;
                    if (o->t_end) o->t_end[i] = r.t_end;
                    if (p->start_pos == S_WITH_START || (with_tb && algo != A_GLOBAL)) {
                        if (o->q_start) o->q_start[i] = r.q_start;
                        if (o->t_start) o->t_start[i] = r.t_start;
                    }
                    if (algo == A_KSW && o->score2) o->score2[i] = r.score2; /* max_off */
                    if (p->second_best && (algo == A_LOCAL || algo == A_SEMI_GLOBAL)) {
                        if (o->score2) o->score2[i] = r.score2;
                        if (o->q_end2) o->q_end2[i] = r.q_end2;
                        if (o->t_end2) o->t_end2[i] = r.t_end2;
                    }
                }
            }
        }
        free(Hb), free(Eb), free(qc), free(tc), free(rq), free(rt), free(eh);
    }

    if (with_tb) {
        /* CIGAR bytes go over the unpacked query batch at each pair's offset,
         * in pair order (a CIGAR longer than its slot runs into the next). */
        if (o->cigar) memcpy(o->cigar, b->q, b->q_bytes);
        for (int i = 0; i < n; i++) {
            if (o->cigar && ops[i]) {
                for (uint32_t k = 0; k < nops[i] && b->q_off[i] + k < b->q_bytes; k++) o->cigar[b->q_off[i] + k] = ops[i][k];
            }
            if (o->n_cigar) o->n_cigar[i] = nops[i];
            free(ops[i]);
        }
        free(ops), free(nops);
    }
    free(pq), free(pt);
    return err ? GB_ERR_ALLOC : GB_OK;
}

/* ---------------- forward CIGAR text (test_prog/test_prog.cpp:382-428) ---------------- */
void oracle_cigar_text(const uint8_t *cigar, const uint32_t *q_off, const uint32_t *n_cigar, int n, char *text,
                       int stride, int32_t *text_len)
{
    static const char OPS[4] = {'M', 'X', 'D', 'I'};
    for (int i = 0; i < n; i++) {
        char *out = text + (size_t)i * stride;
        const uint8_t *c = cigar + q_off[i];
        int len = 0, ok = 1;
        /* runs in forward order: the bytes from last to first */
        int u = (int)n_cigar[i] - 1;
        while (u >= 0 && ok) {
            const int op = c[u] & 3;
            long count = 0;
            while (u >= 0 && (c[u] & 3) == op) count += c[u--] >> 2;
            char digits[24];
            int nd = 0;
            do {
                digits[nd++] = (char)('0' + count % 10);
                count /= 10;
            } while (count > 0);
            if (len + nd + 1 > stride - 1) {
                ok = 0;
                break;
            }
            while (nd > 0) out[len++] = digits[--nd];
            out[len++] = OPS[op];
        }
        if (stride > 0) out[ok ? len : 0] = 0;
        text_len[i] = ok ? len : -1;
    }
}
