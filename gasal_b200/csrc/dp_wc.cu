/*
 * dp_wc.cu -- warp-cooperative DP for long pairs (LOCAL and GLOBAL).
 *
 * One warp aligns one pair.  Lane L sweeps the pair's 8-row bands L, L+32,
 * L+64, ... one 8-column query word per step, lane L lagging lane L-1 by one
 * step, so the H/E leaving the bottom of band b at word w are produced by
 * lane b%32 exactly one step before lane (b+1)%32 needs them; they travel by
 * __shfl_up_sync as int16 pairs (the reference's short2 row buffer, so the
 * truncation is unchanged).  Lane 31's outputs reach lane 0, one round later,
 * through a shared-memory ring of one word per query column per warp.  Every
 * cell is computed from exactly the operands the one-pair-per-thread sweep
 * uses, so scores are identical; positions follow the reference's sweep order
 * (bands, then columns, then rows) through per-lane records of
 * (value, band, column, row) reduced first by value and then by band.
 *
 * Replaces, for long pairs, reference src/kernels/local_kernel_template.h and
 * src/kernels/global.h (one thread per pair there).  The pairs handled here
 * need at least 32 query words (the ring's reader must trail its writer).
 */
#include "dp_core.cuh"

namespace gb {

namespace {

constexpr int NEG16W = -32768;

__device__ __forceinline__ int sx16(uint32_t v) { return (int)(int16_t)(v & 0xFFFFu); }
__device__ __forceinline__ int hx16(uint32_t v) { return (int)v >> 16; }
__device__ __forceinline__ uint32_t pk(int h, int e) { return (uint32_t)(uint16_t)h | ((uint32_t)e << 16); }
__device__ __forceinline__ int cd(uint32_t w, int k) { return (int)((w >> (28 - 4 * k)) & 15u); }

__device__ __forceinline__ uint32_t nrev(uint32_t x)
{
    const uint32_t r = __byte_perm(x, 0, 0x0123);
    return ((r >> 4) & 0x0F0F0F0Fu) | ((r << 4) & 0xF0F0F0F0u);
}

__device__ __forceinline__ uint32_t wprmt(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

constexpr uint64_t WC_CLASS = (5ull << 0) | (0ull << 4) | (6ull << 8) | (1ull << 12) | (3ull << 16) | (6ull << 20) |
                              (6ull << 24) | (2ull << 28) | (6ull << 32) | (6ull << 36) | (6ull << 40) |
                              (6ull << 44) | (6ull << 48) | (6ull << 52) | (4ull << 56) | (6ull << 60);
constexpr uint32_t WC_PLAIN = (1u << 0) | (1u << 1) | (1u << 3) | (1u << 4) | (1u << 7) | (1u << 14);

__device__ bool wc_plain(const uint32_t *w, int n)
{
    uint32_t bad = 0;
    for (int i = threadIdx.x & 31; i < n; i += 32) {
        const uint32_t x = w[i];
#pragma unroll
        for (int k = 0; k < 8; k++) bad |= ~(WC_PLAIN >> ((x >> (4 * k)) & 15u)) & 1u;
    }
    return __all_sync(0xFFFFFFFFu, bad == 0);
}

__device__ void wc_score_table(uint2 *tab, const Scores &sc, bool local)
{
    const int rep[8] = {1, 3, 7, 4, 14, 0, 2, 2};
    for (int r = threadIdx.x; r < 16; r += blockDim.x) {
        uint32_t lo = 0, hi = 0;
        for (int j = 0; j < 8; j++) {
            const int g = rep[j];
            int v = (local && (r == 14 || g == 14)) ? 0 : ((r == g) ? sc.match : -sc.mismatch);
            if (j >= 6) v = 0;
            const uint32_t byte = (uint32_t)(v & 0xFF);
            if (j < 4) lo |= byte << (8 * j);
            else hi |= byte << (8 * (j - 4));
        }
        tab[r] = make_uint2(lo, hi);
    }
}

/* substitution for one band: prmt table (plain codes) or compares */
struct WcScore {
    bool fast, local;
    uint32_t sel[8];
    int g[8], ma[8], mm[8];
    const uint2 *tab;
    __device__ __forceinline__ void band(uint32_t gw, const Scores &sc)
    {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint32_t code = (gw >> (28 - 4 * k)) & 15u;
            const uint32_t c = (uint32_t)(WC_CLASS >> (4 * code)) & 15u;
            sel[k] = c | ((c | 8u) * 0x1110u);
            g[k] = (int)code;
            const bool n = local && code == 14u;
            ma[k] = n ? 0 : sc.match;
            mm[k] = n ? 0 : -sc.mismatch;
        }
    }
};

struct WcRec { /* first maximum of a lane's bands in sweep order */
    int v, band, col, row;
};

__device__ __forceinline__ bool rec_before(const WcRec &a, const WcRec &b)
{
    return a.v > b.v || (a.v == b.v && a.band < b.band);
}

__device__ __forceinline__ WcRec rec_reduce(WcRec r)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        WcRec o;
        o.v = __shfl_xor_sync(0xFFFFFFFFu, r.v, off);
        o.band = __shfl_xor_sync(0xFFFFFFFFu, r.band, off);
        o.col = __shfl_xor_sync(0xFFFFFFFFu, r.col, off);
        o.row = __shfl_xor_sync(0xFFFFFFFFu, r.row, off);
        if (rec_before(o, r)) r = o;
    }
    return r;
}

__device__ __forceinline__ int key_max8(const int *k)
{
    int m = __vimax3_s32(k[0], k[1], k[2]);
    m = __vimax3_s32(m, k[3], k[4]);
    m = __vimax3_s32(m, k[5], k[6]);
    return max(m, k[7]);
}

__device__ __forceinline__ uint32_t dnib(int M, int diag, int H, int F, int E, const Scores &sc)
{
    uint32_t d = (H == M) ? (M >= diag ? 0u : 1u) : (H == F ? 3u : 2u);
    d |= ((M - sc.oe) > (F - sc.e)) ? 0u : 8u;
    d |= ((M - sc.oe) > (E - sc.e)) ? 0u : 4u;
    return d;
}

/*
 * One sweep of a pair by the warp.
 *   MODE 0: LOCAL forward       (first max; optional second-best pass 2)
 *   MODE 1: LOCAL start pass    (reversed words, stops after the first round
 *                                whose bands reach `stop`)
 *   MODE 2: GLOBAL forward
 * qword(j), tword(T): the words the sweep reads (reversed for MODE 1).
 * bandmax: per-band maxima (written when SECOND pass 1, read in pass 2).
 */
template <int MODE, bool TB, bool SECOND_PASS2, class QW, class TW>
__device__ void wc_sweep(QW qword, int qregs, TW tword, int tregs, int qlen, int tlen, const Scores &sc,
                         WcScore &S, uint32_t *ring, uint4 *tb, int stop, int *bandmax, bool write_bandmax,
                         WcRec &best_out, WcRec &sec_out, int &gscore)
{
    const int lane = threadIdx.x & 31;
    const int rounds = (tregs + 31) >> 5;
    const bool local = MODE != 2;
    const int last_band = tregs - 1, last_row_in_band = tlen - 1 - ((tregs - 1) << 3);
    uint32_t out[8];
#pragma unroll
    for (int k = 0; k < 8; k++) out[k] = 0;
    int F[8], D[8];
    int up_prev = 0; /* bottom H of the band above at the previous column (diagonal of row 0) */
    int run = 0;     /* second best: running max before the cell */
    WcRec best = {0, 0x7fffffff, 0, 0}, sec = {0, 0x7fffffff, 0, 0};
    if (MODE == 2) best.v = 0;
    int bandbest = 0;
    int hit_round = 0x7fffffff;
    const long steps = (long)rounds * qregs + 31;
    for (long s = 0; s < steps; s++) {
        const long rel = s - lane;
        const int r = rel >= 0 ? (int)(rel / qregs) : -1;
        const int w = rel >= 0 ? (int)(rel - (long)r * qregs) : 0;
        const int band = (r << 5) + lane;
        const bool active = rel >= 0 && r < rounds && band < tregs;
        /* stop once every lane is past the first round with a hit (s-based,
         * so the whole warp leaves together) */
        if (MODE == 1 && hit_round != 0x7fffffff && s >= (long)(hit_round + 1) * qregs + 31) break;
        /* inputs: bottom H/E of the band above at the 8 columns of word w */
        uint32_t in[8];
#pragma unroll
        for (int k = 0; k < 8; k++) in[k] = __shfl_up_sync(0xFFFFFFFFu, out[k], 1);
        if (lane == 0 && active) {
            if (r == 0) {
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int c = (w << 3) + k;
                    in[k] = local ? 0u : pk(c == 0 ? 0 : -(sc.o + sc.e * c), NEG16W);
                }
            } else {
#pragma unroll
                for (int k = 0; k < 8; k++) in[k] = ring[(w << 3) + k];
            }
        }
        __syncwarp();
        if (active) {
            if (w == 0) { /* new band: left boundary */
                S.band(tword(band), sc);
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int R = (band << 3) + k;
                    F[k] = local ? 0 : NEG16W;
                    D[k] = local ? 0 : (R == 0 ? 0 : -(sc.o + sc.e * R));
                }
                up_prev = 0;
                bandbest = 0;
                if (SECOND_PASS2) run = band == 0 ? 0 : bandmax[band - 1];
            }
            const uint32_t qw = qword(w);
            uint32_t dir[8];
            int colkey_best = -1, colkey_sec = -1, colc = 0;
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int c = (w << 3) + b;
                const int rbase = cd(qw, b);
                uint2 tcol = make_uint2(0, 0);
                if (S.fast) tcol = S.tab[rbase];
                const bool rz = local && rbase == 14;
                const uint32_t v = in[b];
                const int up0 = sx16(v);
                int e = hx16(v);
                if (b > 0 || w > 0) D[0] = up_prev;
                else D[0] = local ? 0 : D[0];
                int Hn[8], key[8], cand[8];
                uint32_t dw = 0;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    int s_;
                    if (S.fast) s_ = (int)wprmt(tcol.x, tcol.y, S.sel[k]);
                    else s_ = rz ? 0 : ((rbase == S.g[k]) ? S.ma[k] : S.mm[k]);
                    const int M = D[k] + s_;
                    const int H = local ? __vimax3_s32_relu(M, F[k], e) : __vimax3_s32(M, F[k], e);
                    if (TB) dw |= dnib(M, D[k], H, F[k], e, sc) << (28 - 4 * k);
                    const int t0 = M - sc.oe;
                    F[k] = __viaddmax_s32(F[k], -sc.e, t0);
                    e = __viaddmax_s32(e, -sc.e, t0);
                    key[k] = (H << 3) + (7 - k);
                    if (SECOND_PASS2) {
                        bool ge;
                        run = __vibmax_s32(H, run, &ge);
                        cand[k] = ge ? -1 : key[k];
                    }
                    Hn[k] = H;
                }
                out[b] = pk(Hn[7], e);
#pragma unroll
                for (int k = 7; k > 0; k--) D[k] = Hn[k - 1];
                up_prev = up0;
                if (TB) dir[b] = dw;
                if (MODE == 2) {
                    if (band == last_band && c == qlen - 1) {
#pragma unroll
                        for (int k = 0; k < 8; k++)
                            if (k == last_row_in_band) gscore = Hn[k];
                    }
                } else {
                    const int ck = key_max8(key);
                    if ((ck >> 3) > bandbest) bandbest = ck >> 3;
                    if ((ck >> 3) > best.v) {
                        best.v = ck >> 3, best.band = band, best.col = c, best.row = (band << 3) + 7 - (ck & 7);
                    }
                    if (SECOND_PASS2) {
                        const int cs = key_max8(cand);
                        if (cs >= 0 && (cs >> 3) > sec.v) {
                            sec.v = cs >> 3, sec.band = band, sec.col = c, sec.row = (band << 3) + 7 - (cs & 7);
                        }
                    }
                }
                (void)colkey_best, (void)colkey_sec, (void)colc;
            }
            D[0] = up_prev;
            if (TB) {
                uint4 *tp = tb + (size_t)band * (2 * qregs) + 2 * w;
                tp[0] = make_uint4(dir[0], dir[1], dir[2], dir[3]);
                tp[1] = make_uint4(dir[4], dir[5], dir[6], dir[7]);
            }
            if (lane == 31) {
#pragma unroll
                for (int k = 0; k < 8; k++) ring[(w << 3) + k] = out[k];
            }
            if (w == qregs - 1 && write_bandmax) bandmax[band] = bandbest;
        }
        __syncwarp();
        if (MODE == 1) {
            /* a band reaching the forward score ends the sweep after its round */
            const bool hit = active && w == qregs - 1 && bandbest >= stop;
            const unsigned m = __ballot_sync(0xFFFFFFFFu, hit);
            if (m) {
                const int hr = __shfl_sync(0xFFFFFFFFu, r, __ffs(m) - 1);
                if (hr < hit_round) hit_round = hr;
            }
        }
    }
    best_out = best;
    sec_out = sec;
}

/*
 * SEMI_GLOBAL (reference src/kernels/semiglobal_kernel_template.h:39-388)
 * with the target tail free (tail TARGET): one sweep of bands T0..tregs-1,
 * gaps opened from H, the H of the last query column of every row kept in
 * `lastcol` (indexed by absolute row).  FWD = false: the start pass over the
 * reversed words, bands counted from T0 for the left boundary, leaving after
 * the first round whose bands reach `stop` at the last column.
 */
template <bool START_PASS, bool OPEN_NN, class QW, class TW>
__device__ void wc_semi_sweep(QW qword, int qregs, TW tword, int tregs, int T0, int qlen, const Scores &sc,
                              int head, WcScore &S, uint32_t *ring, int *lastcol, int stop)
{
    const int lane = threadIdx.x & 31;
    const int nb = tregs - T0;
    if (nb <= 0) return;
    const int rounds = (nb + 31) >> 5;
    const bool free_head_t = (head == TARGET_ || head == BOTH_);
    const bool zero_rows = (head == QUERY_ || head == BOTH_);
    uint32_t out[8];
#pragma unroll
    for (int k = 0; k < 8; k++) out[k] = 0;
    int F[8], D[8], Hc[8];
#pragma unroll
    for (int k = 0; k < 8; k++) F[k] = NEG16W, D[k] = 0, Hc[k] = 0;
    int up_prev = 0;
    int hit_round = 0x7fffffff;
    const int lastw = (qlen - 1) >> 3, lastb = (qlen - 1) & 7;
    const long steps = (long)rounds * qregs + 31;
    for (long st = 0; st < steps; st++) {
        const long rel = st - lane;
        const int r = rel >= 0 ? (int)(rel / qregs) : -1;
        const int w = rel >= 0 ? (int)(rel - (long)r * qregs) : 0;
        const int brel = (r << 5) + lane;
        const bool active = rel >= 0 && r < rounds && brel < nb;
        if (START_PASS && hit_round != 0x7fffffff && st >= (long)(hit_round + 1) * qregs + 31) break;
        uint32_t in[8];
#pragma unroll
        for (int k = 0; k < 8; k++) in[k] = __shfl_up_sync(0xFFFFFFFFu, out[k], 1);
        if (lane == 0 && active) {
            if (r == 0) {
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int c = (w << 3) + k;
                    in[k] = zero_rows ? 0u : pk(c == 0 ? 0 : (int)(int16_t)(-(sc.o + sc.e * c)), NEG16W);
                }
            } else {
#pragma unroll
                for (int k = 0; k < 8; k++) in[k] = ring[(w << 3) + k];
            }
        }
        __syncwarp();
        bool hit = false;
        if (active) {
            const int band = T0 + brel;
            if (w == 0) { /* new band: left boundary (rows counted from T0) */
                S.band(tword(band), sc);
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int R = (brel << 3) + k;
                    F[k] = NEG16W;
                    if (free_head_t) {
                        Hc[k] = 0, D[k] = 0;
                    } else {
                        Hc[k] = -(sc.o + sc.e * R);
                        D[k] = R == 0 ? 0 : -(sc.o + sc.e * R);
                    }
                }
                up_prev = 0;
            }
            const uint32_t qw = qword(w);
#pragma unroll
            for (int b = 0; b < 8; b++) {
                const int rbase = cd(qw, b);
                uint2 tcol = make_uint2(0, 0);
                if (S.fast) tcol = S.tab[rbase];
                const bool rz = rbase == 14;
                const uint32_t v = in[b];
                const int up0 = sx16(v);
                int e = hx16(v);
                if (b > 0 || w > 0) D[0] = up_prev;
                int Hn[8];
                int x = up0 - sc.oe, up = up0;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    int s_;
                    if (S.fast) s_ = (int)wprmt(tcol.x, tcol.y, S.sel[k]);
                    else s_ = rz ? 0 : ((rbase == S.g[k]) ? S.ma[k] : S.mm[k]);
                    F[k] = __viaddmax_s32(F[k], -sc.e, Hc[k] - sc.oe);
                    const int M = D[k] + s_;
                    if (OPEN_NN) {
                        e = __viaddmax_s32(e, -sc.e, x);
                        const int mf = max(M, F[k]);
                        x = mf - sc.oe;
                        Hn[k] = max(mf, e);
                    } else {
                        e = __viaddmax_s32(e, -sc.e, up - sc.oe);
                        Hn[k] = __vimax3_s32(M, F[k], e);
                        up = Hn[k];
                    }
                }
                out[b] = pk(Hn[7], e);
#pragma unroll
                for (int k = 7; k > 0; k--) D[k] = Hn[k - 1];
#pragma unroll
                for (int k = 0; k < 8; k++) Hc[k] = Hn[k];
                up_prev = up0;
                if (w == lastw && b == lastb) {
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        lastcol[(band << 3) + k] = Hn[k];
                        if (START_PASS && Hn[k] >= stop) hit = true;
                    }
                }
            }
            D[0] = up_prev;
            if (lane == 31) {
#pragma unroll
                for (int k = 0; k < 8; k++) ring[(w << 3) + k] = out[k];
            }
        }
        __syncwarp();
        if (START_PASS) {
            const unsigned m = __ballot_sync(0xFFFFFFFFu, hit);
            if (m) {
                const int hr = __shfl_sync(0xFFFFFFFFu, r, __ffs(m) - 1);
                if (hr < hit_round) hit_round = hr;
            }
        }
    }
    __syncwarp();
}

/* First maximum (strict >, row order) of lastcol over rows [r0, r1) with the
 * reference's initial best NEG16 / row `row0`; with SECOND also its second
 * best (a row qualifies when below every earlier row's value). */
template <bool SECOND>
__device__ void wc_lastcol_scan(const int *lastcol, int r0, int r1, int row0, int &best, int &brow, int &sec,
                                int &srow)
{
    const int lane = threadIdx.x & 31;
    best = NEG16W, brow = row0, sec = NEG16W, srow = row0;
    int carry = NEG16W; /* max of the rows before the chunk */
    for (int base = r0; base < r1; base += 32) {
        const int row = base + lane;
        const int h = row < r1 ? lastcol[row] : NEG16W - 1;
        int pm = h; /* inclusive prefix max within the chunk */
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int o = __shfl_up_sync(0xFFFFFFFFu, pm, off);
            if (lane >= off) pm = max(pm, o);
        }
        int before = __shfl_up_sync(0xFFFFFFFFu, pm, 1);
        before = lane == 0 ? carry : max(before, carry);
        /* chunk argmax, first row on ties */
        int bv = h, br = row;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const int ov = __shfl_xor_sync(0xFFFFFFFFu, bv, off), orow = __shfl_xor_sync(0xFFFFFFFFu, br, off);
            if (ov > bv || (ov == bv && orow < br)) bv = ov, br = orow;
        }
        if (bv > best) best = bv, brow = br;
        if (SECOND) {
            const bool q = row < r1 && h < before && h > NEG16W;
            int sv = q ? h : NEG16W - 1, sr = row;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const int ov = __shfl_xor_sync(0xFFFFFFFFu, sv, off), orow = __shfl_xor_sync(0xFFFFFFFFu, sr, off);
                if (ov > sv || (ov == sv && orow < sr)) sv = ov, sr = orow;
            }
            if (sv > sec) sec = sv, srow = sr;
        }
        carry = max(carry, __shfl_sync(0xFFFFFFFFu, pm, 31));
    }
}

template <bool SECOND, bool START>
__global__ void __launch_bounds__(128) dp_wc_semi_kernel(DpArgs a, const uint32_t *list, int nlist, int ring_cols)
{
    extern __shared__ uint32_t wc_smem[];
    __shared__ uint2 tab[16];
    wc_score_table(tab, a.sc, true);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int warps_per_block = blockDim.x >> 5;
    uint32_t *ring = wc_smem + (size_t)warp * ring_cols;
    int *lastcol = (int *)(wc_smem + (size_t)warps_per_block * ring_cols) + (size_t)warp * a.scratch_cols;
    const bool fast_scores = a.sc.match >= -128 && a.sc.match <= 127 && a.sc.mismatch >= -127 && a.sc.mismatch <= 128;
    const bool open_nn = a.sc.o >= 0;
    for (int item = blockIdx.x * warps_per_block + warp; item < nlist; item += gridDim.x * warps_per_block) {
        const int i = (int)list[item];
        const int qlen = (int)a.q_len[i], tlen = (int)a.t_len[i];
        const uint32_t *q = a.pq + (a.q_off[i] >> 3);
        const uint32_t *t = a.pt + (a.t_off[i] >> 3);
        const int qregs = (qlen + 7) >> 3, tregs = (tlen + 7) >> 3;
        WcScore S;
        S.local = true;
        S.tab = tab;
        S.fast = fast_scores && wc_plain(q, qregs) && wc_plain(t, tregs);
        auto qf = [&](int j) { return q[j]; };
        auto tf = [&](int T) { return t[T]; };
        if (open_nn) wc_semi_sweep<false, true>(qf, qregs, tf, tregs, 0, qlen, a.sc, a.head, S, ring, lastcol, 0);
        else wc_semi_sweep<false, false>(qf, qregs, tf, tregs, 0, qlen, a.sc, a.head, S, ring, lastcol, 0);
        int best, brow, sec, srow;
        wc_lastcol_scan<SECOND>(lastcol, 0, tlen, qlen, best, brow, sec, srow);
        int t_start = 0, q_start = 0;
        if (START) {
            const int x = tregs - ((brow >> 3) + 1);
            int gend_reg = x > 0 ? x - 1 : x;
            if (gend_reg < 0) gend_reg = 0;
            auto rq = [&](int j) { return rev_window(q, qlen - 8 - (j << 3)); };
            auto rt = [&](int T) { return rev_window(t, tlen - 8 - (T << 3)); };
            __syncwarp();
            if (open_nn)
                wc_semi_sweep<true, true>(rq, qregs, rt, tregs, gend_reg, qlen, a.sc, a.head, S, ring, lastcol, best);
            else
                wc_semi_sweep<true, false>(rq, qregs, rt, tregs, gend_reg, qlen, a.sc, a.head, S, ring, lastcol,
                                           best);
            /* rows up to the end of the first band that reached the forward score */
            const int r0 = gend_reg << 3;
            int r1 = min(tregs << 3, tlen);
            for (int base = r0; base < r1; base += 32) {
                const int row = base + lane;
                const unsigned m = __ballot_sync(0xFFFFFFFFu, row < r1 && lastcol[row] >= best);
                if (m) {
                    const int hit = base + __ffs(m) - 1;
                    r1 = min(r1, ((hit >> 3) + 1) << 3);
                    break;
                }
            }
            int bb, bbrow, s2, s2r;
            wc_lastcol_scan<false>(lastcol, r0, r1, 0, bb, bbrow, s2, s2r);
            t_start = (tlen - 1) - bbrow;
            q_start = (qlen - 1) - tlen;
        }
        if (lane == 0) {
            if (a.score) a.score[i] = best;
            if (a.t_end) a.t_end[i] = brow;
            if (a.q_end) a.q_end[i] = tlen;
            if (SECOND) {
                if (a.score2) a.score2[i] = sec;
                if (a.t_end2) a.t_end2[i] = srow;
                if (a.q_end2) a.q_end2[i] = tlen;
            }
            if (START) {
                if (a.t_start) a.t_start[i] = t_start;
                if (a.q_start) a.q_start[i] = q_start;
            }
        }
        __syncwarp();
    }
}

} // namespace

/* ---------------------------------------------------------------------- */

template <int ALGO, int START, bool SECOND>
__global__ void __launch_bounds__(128) dp_wc_kernel(DpArgs a, const uint32_t *list, int nlist, int ring_cols)
{
    extern __shared__ uint32_t wc_smem[];
    __shared__ uint2 tab[16];
    wc_score_table(tab, a.sc, ALGO == LOCAL_);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int warps_per_block = blockDim.x >> 5;
    uint32_t *ring = wc_smem + (size_t)warp * ring_cols;
    int *bandmax = (int *)(wc_smem + (size_t)warps_per_block * ring_cols) + (size_t)warp * a.scratch_cols;
    const bool fast_scores = a.sc.match >= -128 && a.sc.match <= 127 && a.sc.mismatch >= -127 && a.sc.mismatch <= 128;
    for (int item = blockIdx.x * warps_per_block + warp; item < nlist; item += gridDim.x * warps_per_block) {
        const int i = (int)list[item];
        const int qlen = (int)a.q_len[i], tlen = (int)a.t_len[i];
        const uint32_t *q = a.pq + (a.q_off[i] >> 3);
        const uint32_t *t = a.pt + (a.t_off[i] >> 3);
        const int qregs = (qlen + 7) >> 3, tregs = (tlen + 7) >> 3;
        WcScore S;
        S.local = ALGO == LOCAL_;
        S.tab = tab;
        S.fast = fast_scores && wc_plain(q, qregs) && wc_plain(t, tregs);
        uint4 *tb = nullptr;
        if (START == WITH_TB_) {
            tb = a.tb + a.tb_off[i];
            uint4 *z = tb + (size_t)tregs * 2 * qregs;
            for (int k = lane; k < 4 * qregs; k += 32) z[k] = make_uint4(0, 0, 0, 0);
        }
        auto qf = [&](int j) { return q[j]; };
        auto tf = [&](int T) { return t[T]; };
        WcRec best, sec;
        int gscore = 0;
        if (ALGO == GLOBAL_) {
            wc_sweep<2, START == WITH_TB_, false>(qf, qregs, tf, tregs, qlen, tlen, a.sc, S, ring, tb, 0, bandmax,
                                                  false, best, sec, gscore);
            /* the owner lane of the last band holds the score */
            const int owner = (tregs - 1) & 31;
            gscore = __shfl_sync(0xFFFFFFFFu, gscore, owner);
            if (lane == 0 && a.score) a.score[i] = gscore;
            continue;
        }
        /* LOCAL forward (pass 1 also records per-band maxima for second best) */
        wc_sweep<0, START == WITH_TB_, false>(qf, qregs, tf, tregs, qlen, tlen, a.sc, S, ring, tb, 0, bandmax,
                                              SECOND, best, sec, gscore);
        best = rec_reduce(best);
        WcRec secr = {0, 0x7fffffff, 0, 0};
        if (SECOND) {
            __syncwarp();
            /* exclusive prefix maximum over bands, in place */
            int carry = 0;
            for (int base = 0; base < tregs; base += 32) {
                const int b = base + lane;
                int v = b < tregs ? bandmax[b] : 0;
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const int o = __shfl_up_sync(0xFFFFFFFFu, v, off);
                    if (lane >= off) v = max(v, o);
                }
                v = max(v, carry);
                if (b < tregs) bandmax[b] = v;
                carry = __shfl_sync(0xFFFFFFFFu, v, 31);
            }
            __syncwarp();
            WcRec b2, s2;
            int g2 = 0;
            wc_sweep<0, false, true>(qf, qregs, tf, tregs, qlen, tlen, a.sc, S, ring, nullptr, 0, bandmax, false,
                                     b2, s2, g2);
            secr = rec_reduce(s2);
        }
        int qs = 0, ts = 0;
        if (START == WITH_START_ && best.v > 0) {
            const int rend_reg = min((best.col >> 3) + 1, qregs);
            const int gend_reg = min((best.row >> 3) + 1, tregs);
            auto qr = [&](int j) { return nrev(q[rend_reg - 1 - j]); };
            auto tr = [&](int T) { return nrev(t[gend_reg - 1 - T]); };
            WcRec bs, ss;
            int g3 = 0;
            if (rend_reg >= 32) {
                wc_sweep<1, false, false>(qr, rend_reg, tr, gend_reg, 0, 0, a.sc, S, ring, nullptr, best.v, bandmax,
                                          false, bs, ss, g3);
                bs = rec_reduce(bs);
                /* reversed coordinates -> what the reference records */
                const int gidx = (gend_reg << 3) - 1 - (bs.band << 3);
                ts = gidx + (bs.row - (bs.band << 3));
                qs = (rend_reg << 3) - 1 - bs.col;
            } else {
                /* reverse region narrower than 32 words (the ring's reader
                 * must trail its writer): lane 0 runs the one-thread start
                 * pass with the warp's ring as row buffer.  It stops at the
                 * first cell reaching the score -- for the short local hits
                 * that end this early, a few bands -- where the warp would
                 * finish a 32-band round. */
                if (lane == 0) {
                    RowBuf rb{ring, 1u};
                    Res rr = {best.v, best.col, best.row, 0, 0, 0, 0, 0};
                    if (S.fast) {
                        ScFast sf;
                        sf.tab = tab;
                        local_start(q, qregs, t, tregs, a.sc, rb, sf, rr);
                    } else {
                        ScCmp sc2{};
                        local_start(q, qregs, t, tregs, a.sc, rb, sc2, rr);
                    }
                    qs = rr.q_start, ts = rr.t_start;
                }
                __syncwarp();
            }
        }
        if (lane == 0) {
            if (a.score) a.score[i] = best.v;
            if (a.q_end) a.q_end[i] = best.v > 0 ? best.col : 0;
            if (a.t_end) a.t_end[i] = best.v > 0 ? best.row : 0;
            if (SECOND) {
                if (a.score2) a.score2[i] = secr.v;
                if (a.q_end2) a.q_end2[i] = best.v > 0 ? (qregs << 3) - 1 : 0;
                if (a.t_end2) a.t_end2[i] = secr.v > 0 ? secr.row : 0;
            }
            if (START == WITH_START_) {
                if (a.q_start) a.q_start[i] = best.v > 0 ? qs : 0;
                if (a.t_start) a.t_start[i] = best.v > 0 ? ts : 0;
            }
        }
    }
}

template <int ALGO, int START, bool SECOND>
static cudaError_t launch_wc_one(const DpArgs &a, const uint32_t *list, int nlist, int max_q8, int max_t8,
                                 cudaStream_t s)
{
    const int warps = 4, block = warps * 32;
    const int ring_cols = max_q8;
    const size_t smem = (size_t)warps * ring_cols * 4 + (size_t)warps * (max_t8 / 8 + 1) * 4;
    DpArgs b = a;
    b.scratch_cols = (uint32_t)(max_t8 / 8 + 1); /* bandmax stride per warp */
    auto k = dp_wc_kernel<ALGO, START, SECOND>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int blocks = (nlist + warps - 1) / warps;
    if (blocks > sms * 16) blocks = sms * 16;
    k<<<blocks, block, smem, s>>>(b, list, nlist, ring_cols);
    return cudaGetLastError();
}

template <bool SECOND, bool START>
static cudaError_t launch_wc_semi(const DpArgs &a, const uint32_t *list, int nlist, int max_q8, int max_t8,
                                  cudaStream_t s)
{
    const int warps = 4, block = warps * 32;
    const int ring_cols = max_q8;
    DpArgs b = a;
    b.scratch_cols = (uint32_t)(max_t8 + 8); /* lastcol stride per warp */
    const size_t smem = (size_t)warps * ring_cols * 4 + (size_t)warps * b.scratch_cols * 4;
    auto k = dp_wc_semi_kernel<SECOND, START>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int blocks = (nlist + warps - 1) / warps;
    if (blocks > sms * 16) blocks = sms * 16;
    k<<<blocks, block, smem, s>>>(b, list, nlist, ring_cols);
    return cudaGetLastError();
}

cudaError_t launch_dp_wc(int algo, int start, bool second, const DpArgs &a, const uint32_t *list, int nlist,
                         int max_q8, int max_t8, cudaStream_t s)
{
    if (nlist <= 0) return cudaSuccess;
    if (algo == SEMI_GLOBAL_) {
        if (start == WITH_START_)
            return second ? launch_wc_semi<true, true>(a, list, nlist, max_q8, max_t8, s)
                          : launch_wc_semi<false, true>(a, list, nlist, max_q8, max_t8, s);
        return second ? launch_wc_semi<true, false>(a, list, nlist, max_q8, max_t8, s)
                      : launch_wc_semi<false, false>(a, list, nlist, max_q8, max_t8, s);
    }
    if (algo == GLOBAL_)
        return start == WITH_TB_ ? launch_wc_one<GLOBAL_, WITH_TB_, false>(a, list, nlist, max_q8, max_t8, s)
                                 : launch_wc_one<GLOBAL_, WITHOUT_START_, false>(a, list, nlist, max_q8, max_t8, s);
    if (algo == LOCAL_) {
        if (start == WITH_START_)
            return second ? launch_wc_one<LOCAL_, WITH_START_, true>(a, list, nlist, max_q8, max_t8, s)
                          : launch_wc_one<LOCAL_, WITH_START_, false>(a, list, nlist, max_q8, max_t8, s);
        if (start == WITH_TB_)
            return second ? launch_wc_one<LOCAL_, WITH_TB_, true>(a, list, nlist, max_q8, max_t8, s)
                          : launch_wc_one<LOCAL_, WITH_TB_, false>(a, list, nlist, max_q8, max_t8, s);
        return second ? launch_wc_one<LOCAL_, WITHOUT_START_, true>(a, list, nlist, max_q8, max_t8, s)
                      : launch_wc_one<LOCAL_, WITHOUT_START_, false>(a, list, nlist, max_q8, max_t8, s);
    }
    return cudaErrorInvalidValue;
}

} // namespace gb
