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
 * Lane groups: with G = 16 or 8 a warp sweeps 32/G pairs side by side, each
 * on its own G lanes with its own ring (shuffles of width G, ballots masked
 * to the group).  A pair's sweep takes rounds*qregs + G-1 steps on G lanes,
 * so the G-1 steps of pipeline fill and drain cost less: on w2's 250-1000 bp
 * pairs 72% of lane-steps do work at G = 32, 88% at 16, 95% at 8.
 * Neighbouring pairs of the length-ordered list have about the same lengths,
 * so the groups of a warp finish together.  Every loop that contains a warp
 * operation runs the same trip count on all lanes (the warp's maximum) with
 * per-group predicates.
 *
 * Replaces, for long pairs, reference src/kernels/local_kernel_template.h and
 * src/kernels/global.h (one thread per pair there).  The pairs handled here
 * need at least G query words (the ring's reader must trail its writer).
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

/* lanes of a group of G <= 32: its first lane and its ballot mask (a group
 * of 64 is a whole block of two warps: every lane of each warp) */
template <int G> __device__ __forceinline__ int gbase_of(int lane) { return G >= 32 ? 0 : lane & ~(G - 1); }
template <int G> __device__ __forceinline__ unsigned gmask_of(int lane)
{
    return G >= 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << (lane & ~(G - 1)));
}
/* a lane's index in its group */
template <int G> __device__ __forceinline__ int glane_of() { return G > 32 ? (int)threadIdx.x : (int)(threadIdx.x & (G - 1)); }

/* Block-wide pieces of the 64-lane (two-warp) groups; each ends with the
 * block barrier so its shared slots can be reused at once. */
/* inclusive prefix maximum over the group's lanes in lane order */
template <int G> __device__ __forceinline__ int grp_prefix_max(int v)
{
    const int gl = glane_of<G>(), wl = threadIdx.x & 31;
#pragma unroll
    for (int off = 1; off < (G > 32 ? 32 : G); off <<= 1) {
        const int o = __shfl_up_sync(0xFFFFFFFFu, v, off, G > 32 ? 32 : G);
        if ((G > 32 ? wl : gl) >= off) v = max(v, o);
    }
    if constexpr (G > 32) {
        __shared__ int x;
        if (threadIdx.x == 31) x = v;
        __syncthreads();
        if (threadIdx.x >= 32) v = max(v, x);
        __syncthreads();
    }
    return v;
}
/* value of lane `src` of the group */
template <int G> __device__ __forceinline__ int grp_bcast(int v, int src)
{
    if constexpr (G > 32) {
        __shared__ int x;
        if ((int)threadIdx.x == src) x = v;
        __syncthreads();
        v = x;
        __syncthreads();
        return v;
    } else {
        return __shfl_sync(0xFFFFFFFFu, v, gbase_of<G>(threadIdx.x & 31) + src);
    }
}
/* the value of the group's previous lane (`fill` for lane 0) */
template <int G> __device__ __forceinline__ int grp_shift_up1(int v, int fill)
{
    const int gl = glane_of<G>();
    int o = __shfl_up_sync(0xFFFFFFFFu, v, 1, G > 32 ? 32 : G);
    if constexpr (G > 32) {
        __shared__ int x;
        if (threadIdx.x == 31) x = v;
        __syncthreads();
        if (threadIdx.x == 32) o = x;
        __syncthreads();
    }
    return gl == 0 ? fill : o;
}
/* largest value, then smallest index, over the group */
template <int G> __device__ __forceinline__ void grp_argmax(int &v, int &idx)
{
#pragma unroll
    for (int off = (G > 32 ? 32 : G) / 2; off > 0; off >>= 1) {
        const int ov = __shfl_xor_sync(0xFFFFFFFFu, v, off), oi = __shfl_xor_sync(0xFFFFFFFFu, idx, off);
        if (ov > v || (ov == v && oi < idx)) v = ov, idx = oi;
    }
    if constexpr (G > 32) {
        __shared__ int xv[2], xi[2];
        if ((threadIdx.x & 31) == 0) xv[threadIdx.x >> 5] = v, xi[threadIdx.x >> 5] = idx;
        __syncthreads();
        const int o = (threadIdx.x >> 5) ^ 1;
        if (xv[o] > v || (xv[o] == v && xi[o] < idx)) v = xv[o], idx = xi[o];
        __syncthreads();
    }
}
/* first lane of the group (lowest index) with `hit`, or -1 */
template <int G> __device__ __forceinline__ int grp_first(bool hit)
{
    const unsigned m = __ballot_sync(0xFFFFFFFFu, hit) & gmask_of<G>(threadIdx.x & 31);
    if constexpr (G > 32) {
        __shared__ int x[2];
        if ((threadIdx.x & 31) == 0) x[threadIdx.x >> 5] = m ? (int)(threadIdx.x & ~31u) + __ffs(m) - 1 : -1;
        __syncthreads();
        const int f = x[0] >= 0 ? x[0] : x[1];
        __syncthreads();
        return f;
    } else {
        return m ? __ffs(m) - 1 - gbase_of<G>(threadIdx.x & 31) : -1;
    }
}

/* all codes of the group's words plain (A, C, G, T and the like)? */
template <int G> __device__ bool wc_plain(const uint32_t *w, int n)
{
    const int lane = threadIdx.x & 31;
    uint32_t bad = 0;
    for (int i = glane_of<G>(); i < n; i += G) {
        const uint32_t x = w[i];
#pragma unroll
        for (int k = 0; k < 8; k++) bad |= ~(WC_PLAIN >> ((x >> (4 * k)) & 15u)) & 1u;
    }
    if constexpr (G > 32) return grp_first<G>(bad != 0) < 0;
    return (__ballot_sync(0xFFFFFFFFu, bad != 0) & gmask_of<G>(lane)) == 0;
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

template <int G> __device__ __forceinline__ WcRec rec_reduce(WcRec r)
{
#pragma unroll
    for (int off = (G > 32 ? 32 : G) / 2; off > 0; off >>= 1) {
        WcRec o;
        o.v = __shfl_xor_sync(0xFFFFFFFFu, r.v, off);
        o.band = __shfl_xor_sync(0xFFFFFFFFu, r.band, off);
        o.col = __shfl_xor_sync(0xFFFFFFFFu, r.col, off);
        o.row = __shfl_xor_sync(0xFFFFFFFFu, r.row, off);
        if (rec_before(o, r)) r = o;
    }
    if constexpr (G > 32) {
        __shared__ WcRec x[2];
        if ((threadIdx.x & 31) == 0) x[threadIdx.x >> 5] = r;
        __syncthreads();
        const WcRec o = x[(threadIdx.x >> 5) ^ 1];
        if (rec_before(o, r)) r = o;
        __syncthreads();
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
template <int G, int MODE, bool TB, bool SECOND_PASS2, bool FAST, class QW, class TW>
__device__ void wc_sweep(QW qword, int qregs, TW tword, int tregs, int qlen, int tlen, const Scores &sc,
                         WcScore &S, uint32_t *ring, uint4 *tb, int stop, int *bandmax, bool write_bandmax,
                         WcRec &best_out, WcRec &sec_out, int &gscore)
{
    const int lane = threadIdx.x & 31, gl = glane_of<G>();
    const unsigned gmask = gmask_of<G>(lane);
    constexpr int SW = G > 32 ? 32 : G; /* shuffle width */
    /* G = 64: warp 0's last lane hands its outputs to warp 1's first lane
     * through shared memory, double-buffered by step parity, one block
     * barrier per step; hits are combined the same way */
    __shared__ uint32_t xch[2][8];
    __shared__ int xhit[2][2];
    const int rounds = (tregs + G - 1) / G; /* 0 for a group without a pair */
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
    const long gsteps = rounds > 0 && qregs > 0 ? (long)rounds * qregs + G - 1 : 0;
    const long steps = G >= 32 ? gsteps : (long)__reduce_max_sync(0xFFFFFFFFu, (unsigned)gsteps);
    /* this lane's position: word cw of round cr (cw < 0 before its first
     * step); step s puts the lane at s - gl words into its sweep */
    int cw = -gl, cr = 0;
    for (long s = 0; s < steps; s++) {
        const bool started = cw >= 0;
        const int r = started ? cr : -1;
        const int w = started ? cw : 0;
        const int band = r * G + gl;
        /* a group is done once its lanes are past the first round with a
         * hit (MODE 1) or its sweep has ended; the warp (block for G = 64)
         * leaves together */
        const bool gdone = s >= gsteps || (MODE == 1 && hit_round != 0x7fffffff &&
                                           s >= (long)(hit_round + 1) * qregs + G - 1);
        if (MODE == 1 && (G >= 32 ? gdone : __all_sync(0xFFFFFFFFu, gdone))) break;
        const bool active = !gdone && started && r < rounds && band < tregs;
        /* inputs: bottom H/E of the band above at the 8 columns of word w */
        uint32_t in[8];
#pragma unroll
        for (int k = 0; k < 8; k++) in[k] = __shfl_up_sync(0xFFFFFFFFu, out[k], 1, SW);
        if (G > 32 && gl == 32) {
#pragma unroll
            for (int k = 0; k < 8; k++) in[k] = xch[(s + 1) & 1][k];
        }
        if (gl == 0 && active) {
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
                if (FAST) tcol = S.tab[rbase];
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
                    if (FAST) s_ = (int)wprmt(tcol.x, tcol.y, S.sel[k]);
                    else s_ = rz ? 0 : ((rbase == S.g[k]) ? S.ma[k] : S.mm[k]);
                    const int M = D[k] + s_;
                    const int H = local ? __vimax3_s32_relu(M, F[k], e) : __vimax3_s32(M, F[k], e);
                    if (TB) dw |= dnib(M, D[k], H, F[k], e, sc) << (28 - 4 * k);
                    const int t0 = M - sc.oe;
                    F[k] = __viaddmax_s32(F[k], -sc.e, t0);
                    e = __viaddmax_s32(e, -sc.e, t0);
                    key[k] = key8(H, 7 - k);
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
            if (gl == G - 1) {
#pragma unroll
                for (int k = 0; k < 8; k++) ring[(w << 3) + k] = out[k];
            }
            if (w == qregs - 1 && write_bandmax) bandmax[band] = bandbest;
        }
        __syncwarp();
        if constexpr (G > 32) {
            if (gl == 31) {
#pragma unroll
                for (int k = 0; k < 8; k++) xch[s & 1][k] = out[k];
            }
            if (MODE == 1) {
                const bool hit = active && w == qregs - 1 && bandbest >= stop;
                const unsigned m = __ballot_sync(0xFFFFFFFFu, hit);
                const int hr = __shfl_sync(0xFFFFFFFFu, r, m ? __ffs(m) - 1 : lane);
                if (lane == 0) xhit[s & 1][threadIdx.x >> 5] = m ? hr : 0x7fffffff;
            }
            __syncthreads();
            if (MODE == 1) {
                const int h0 = xhit[s & 1][0], h1 = xhit[s & 1][1];
                const int hr = h0 != 0x7fffffff ? h0 : h1;
                if (hr < hit_round) hit_round = hr;
            }
        } else if (MODE == 1) {
            /* a band reaching the forward score ends the group's sweep after its round */
            const bool hit = active && w == qregs - 1 && bandbest >= stop;
            const unsigned m = __ballot_sync(0xFFFFFFFFu, hit) & gmask;
            const int hr = __shfl_sync(0xFFFFFFFFu, r, m ? __ffs(m) - 1 : lane);
            if (m && hr < hit_round) hit_round = hr;
        }
        if (++cw == qregs) cw = 0, ++cr;
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
template <int G, bool START_PASS, bool OPEN_NN, bool FAST, class QW, class TW>
__device__ void wc_semi_sweep(QW qword, int qregs, TW tword, int tregs, int T0, int qlen, const Scores &sc,
                              int head, WcScore &S, uint32_t *ring, int *lastcol, int stop)
{
    const int lane = threadIdx.x & 31, gl = glane_of<G>();
    const unsigned gmask = gmask_of<G>(lane);
    constexpr int SW = G > 32 ? 32 : G; /* shuffle width */
    __shared__ uint32_t xch[2][8];      /* G = 64: warp 0's last lane -> warp 1's first, by step parity */
    __shared__ int xhit[2][2];
    const int nb = tregs - T0;
    if (G >= 32 && nb <= 0) return;
    const int rounds = nb > 0 ? (nb + G - 1) / G : 0;
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
    const long gsteps = rounds > 0 && qregs > 0 ? (long)rounds * qregs + G - 1 : 0;
    const long steps = G >= 32 ? gsteps : (long)__reduce_max_sync(0xFFFFFFFFu, (unsigned)gsteps);
    int cw = -gl, cr = 0; /* word and round of this lane's step (cw < 0: not started) */
    for (long st = 0; st < steps; st++) {
        const bool started = cw >= 0;
        const int r = started ? cr : -1;
        const int w = started ? cw : 0;
        const int brel = r * G + gl;
        const bool gdone = st >= gsteps || (START_PASS && hit_round != 0x7fffffff &&
                                            st >= (long)(hit_round + 1) * qregs + G - 1);
        if (START_PASS && (G >= 32 ? gdone : __all_sync(0xFFFFFFFFu, gdone))) break;
        const bool active = !gdone && started && r < rounds && brel < nb;
        uint32_t in[8];
#pragma unroll
        for (int k = 0; k < 8; k++) in[k] = __shfl_up_sync(0xFFFFFFFFu, out[k], 1, SW);
        if (G > 32 && gl == 32) {
#pragma unroll
            for (int k = 0; k < 8; k++) in[k] = xch[(st + 1) & 1][k];
        }
        if (gl == 0 && active) {
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
                if (FAST) tcol = S.tab[rbase];
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
                    if (FAST) s_ = (int)wprmt(tcol.x, tcol.y, S.sel[k]);
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
            if (gl == G - 1) {
#pragma unroll
                for (int k = 0; k < 8; k++) ring[(w << 3) + k] = out[k];
            }
        }
        __syncwarp();
        if constexpr (G > 32) {
            if (gl == 31) {
#pragma unroll
                for (int k = 0; k < 8; k++) xch[st & 1][k] = out[k];
            }
            if (START_PASS) {
                const unsigned m = __ballot_sync(0xFFFFFFFFu, hit);
                const int hr = __shfl_sync(0xFFFFFFFFu, r, m ? __ffs(m) - 1 : lane);
                if (lane == 0) xhit[st & 1][threadIdx.x >> 5] = m ? hr : 0x7fffffff;
            }
            __syncthreads();
            if (START_PASS) {
                const int h0 = xhit[st & 1][0], h1 = xhit[st & 1][1];
                const int hr = h0 != 0x7fffffff ? h0 : h1;
                if (hr < hit_round) hit_round = hr;
            }
        } else if (START_PASS) {
            const unsigned m = __ballot_sync(0xFFFFFFFFu, hit) & gmask;
            const int hr = __shfl_sync(0xFFFFFFFFu, r, m ? __ffs(m) - 1 : lane);
            if (m && hr < hit_round) hit_round = hr;
        }
        if (++cw == qregs) cw = 0, ++cr;
    }
    if constexpr (G > 32) __syncthreads();
    else __syncwarp();
}

/* First maximum (strict >, row order) of lastcol over rows [r0, r1) with the
 * reference's initial best NEG16 / row `row0`; with SECOND also its second
 * best (a row qualifies when below every earlier row's value). */
template <int G, bool SECOND>
__device__ void wc_lastcol_scan(const int *lastcol, int r0, int r1, int row0, int &best, int &brow, int &sec,
                                int &srow)
{
    const int gl = glane_of<G>();
    best = NEG16W, brow = row0, sec = NEG16W, srow = row0;
    int carry = NEG16W; /* max of the rows before the chunk */
    const int chunks = r1 > r0 ? (r1 - r0 + G - 1) / G : 0;
    const int nchunks = G >= 32 ? chunks : (int)__reduce_max_sync(0xFFFFFFFFu, (unsigned)chunks);
    for (int ch = 0; ch < nchunks; ch++) {
        const int base = r0 + ch * G;
        const int row = base + gl;
        const int h = row < r1 ? lastcol[row] : NEG16W - 1;
        const int pm = grp_prefix_max<G>(h); /* inclusive prefix max within the chunk */
        const int before = max(grp_shift_up1<G>(pm, carry), carry);
        /* chunk argmax, first row on ties */
        int bv = h, br = row;
        grp_argmax<G>(bv, br);
        if (bv > best) best = bv, brow = br;
        if (SECOND) {
            const bool q = row < r1 && h < before && h > NEG16W;
            int sv = q ? h : NEG16W - 1, sr = row;
            grp_argmax<G>(sv, sr);
            if (sv > sec) sec = sv, srow = sr;
        }
        carry = max(carry, grp_bcast<G>(pm, G - 1));
    }
}

/* The first list position of this warp's groups (G <= 32: 32/G of them) or
 * of this block's two-warp group (G = 64) for the next pass of a kernel's
 * pair loop: taken from the launch's zeroed work counter (a.queue), so a
 * group that finishes early takes the next pair -- the order lists the
 * longest pairs first -- or, without one, by grid stride. */
template <int G> __device__ __forceinline__ int wc_next(const DpArgs &a, int gpb, int iter)
{
    if (a.queue) {
        if constexpr (G > 32) {
            __shared__ int next;
            __syncthreads(); /* both warps are done with the previous pair */
            if (threadIdx.x == 0) next = (int)atomicAdd(a.queue, 1u);
            __syncthreads();
            return next;
        } else {
            unsigned v = 0;
            if ((threadIdx.x & 31) == 0) v = atomicAdd(a.queue, (unsigned)(32 / G));
            return (int)__shfl_sync(0xFFFFFFFFu, v, 0);
        }
    }
    if constexpr (G > 32) __syncthreads(); /* both warps are done with the previous pair */
    return (int)(blockIdx.x + iter * gridDim.x) * gpb + (G > 32 ? 0 : (int)(threadIdx.x >> 5) * (32 / G));
}

template <int G, bool SECOND, bool START, bool FAST>
__global__ void __launch_bounds__(128) dp_wc_semi_kernel(DpArgs a, const uint32_t *list, int nlist, int ring_cols)
{
    extern __shared__ uint32_t wc_smem[];
    __shared__ uint2 tab[16];
    wc_score_table(tab, a.sc, true);
    __syncthreads();
    const int gl = glane_of<G>();
    /* groups per block: 32/G per warp, or one two-warp group (G = 64) */
    const int gpb = G > 32 ? 1 : (int)(blockDim.x >> 5) * (32 / G);
    const int slot = G > 32 ? 0 : (int)(threadIdx.x / G); /* this group's ring and last-column buffer */
    uint32_t *ring = wc_smem + (size_t)slot * ring_cols;
    int *lastcol = a.lastcol + ((size_t)blockIdx.x * gpb + slot) * a.scratch_cols;
    const bool fast_scores = a.sc.match >= -128 && a.sc.match <= 127 && a.sc.mismatch >= -127 && a.sc.mismatch <= 128;
    const bool open_nn = a.sc.o >= 0;
    const int nl = a.n_dev ? min((int)*a.n_dev, nlist) : nlist;
    const int wslot = G > 32 ? 0 : (int)((threadIdx.x & 31) / G); /* this group's place in its warp */
    for (int iter = 0;; iter++) {
        const int item0 = wc_next<G>(a, gpb, iter);
        if (item0 >= nl) break; /* the same for every lane of a warp (and of a two-warp group) */
        const int item = item0 + wslot;
        const bool listed = item < nl; /* the last warp may have groups without a pair */
        const int i = listed ? (int)list[item] : 0;
        const int qlen0 = listed ? (int)a.q_len[i] : 0, tlen0 = listed ? (int)a.t_len[i] : 0;
        const uint32_t *q = a.pq + (listed ? (a.q_off[i] >> 3) : 0);
        const uint32_t *t = a.pt + (listed ? (a.t_off[i] >> 3) : 0);
        /* FAST: this launch scores with the prmt table; a pair with another
         * code or scores beyond a byte goes to the compare-scoring launch
         * that follows (a.defer), and this launch skips it */
        const bool plain_q = wc_plain<G>(q, (qlen0 + 7) >> 3); /* warp collectives: every lane calls both */
        const bool plain_t = wc_plain<G>(t, (tlen0 + 7) >> 3);
        const bool fast_pair = fast_scores && plain_q && plain_t;
        const bool has = listed && (!FAST || fast_pair);
        if (FAST && listed && !fast_pair && gl == 0) a.defer[atomicAdd(a.ndefer, 1u)] = (uint32_t)i;
        const int qlen = has ? qlen0 : 0, tlen = has ? tlen0 : 0;
        const int qregs = (qlen + 7) >> 3, tregs = (tlen + 7) >> 3;
        WcScore S;
        S.local = true;
        S.tab = tab;
        S.fast = fast_pair;
        auto qf = [&](int j) { return q[j]; };
        auto tf = [&](int T) { return t[T]; };
        if (open_nn)
            wc_semi_sweep<G, false, true, FAST>(qf, qregs, tf, tregs, 0, qlen, a.sc, a.head, S, ring, lastcol, 0);
        else
            wc_semi_sweep<G, false, false, FAST>(qf, qregs, tf, tregs, 0, qlen, a.sc, a.head, S, ring, lastcol, 0);
        int best, brow, sec, srow;
        wc_lastcol_scan<G, SECOND>(lastcol, 0, tlen, qlen, best, brow, sec, srow);
        int t_start = 0, q_start = 0;
        if (START) {
            const int x = tregs - ((brow >> 3) + 1);
            int gend_reg = x > 0 ? x - 1 : x;
            if (gend_reg < 0) gend_reg = 0;
            auto rq = [&](int j) { return rev_window(q, qlen - 8 - (j << 3)); };
            auto rt = [&](int T) { return rev_window(t, tlen - 8 - (T << 3)); };
            if constexpr (G > 32) __syncthreads();
            else __syncwarp();
            if (open_nn)
                wc_semi_sweep<G, true, true, FAST>(rq, qregs, rt, tregs, gend_reg, qlen, a.sc, a.head, S, ring, lastcol,
                                             best);
            else
                wc_semi_sweep<G, true, false, FAST>(rq, qregs, rt, tregs, gend_reg, qlen, a.sc, a.head, S, ring,
                                                    lastcol, best);
            /* rows up to the end of the first band that reached the forward score */
            const int r0 = gend_reg << 3;
            int r1 = min(tregs << 3, tlen);
            const int chunks = r1 > r0 ? (r1 - r0 + G - 1) / G : 0;
            const int nchunks = G >= 32 ? chunks : (int)__reduce_max_sync(0xFFFFFFFFu, (unsigned)chunks);
            bool found = false;
            for (int ch = 0; ch < nchunks; ch++) {
                const int base = r0 + ch * G;
                const int row = base + gl;
                const int f = grp_first<G>(!found && row < r1 && lastcol[row] >= best);
                if (f >= 0 && !found) {
                    const int hit = base + f;
                    r1 = min(r1, ((hit >> 3) + 1) << 3);
                    found = true;
                }
                if (G >= 32 && found) break;
            }
            int bb, bbrow, s2, s2r;
            wc_lastcol_scan<G, false>(lastcol, r0, r1, 0, bb, bbrow, s2, s2r);
            t_start = (tlen - 1) - bbrow;
            q_start = (qlen - 1) - tlen;
        }
        if (tlen == 0) /* an empty target: every result 0, as on the one-pair-per-thread path */
            best = 0, brow = 0, sec = 0, srow = 0, t_start = 0, q_start = 0;
        if (gl == 0 && has) {
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

template <int G, int ALGO, int START, bool SECOND, bool FAST>
__global__ void __launch_bounds__(128) dp_wc_kernel(DpArgs a, const uint32_t *list, int nlist, int ring_cols)
{
    extern __shared__ uint32_t wc_smem[];
    __shared__ uint2 tab[16];
    wc_score_table(tab, a.sc, ALGO == LOCAL_);
    __syncthreads();
    const int gl = glane_of<G>();
    /* groups per block: 32/G per warp, or one two-warp group (G = 64) */
    const int gpb = G > 32 ? 1 : (int)(blockDim.x >> 5) * (32 / G);
    const int slot = G > 32 ? 0 : (int)(threadIdx.x / G); /* this group's ring and band maxima */
    uint32_t *ring = wc_smem + (size_t)slot * ring_cols;
    int *bandmax = (int *)(wc_smem + (size_t)gpb * ring_cols) + (size_t)slot * a.scratch_cols;
    const bool fast_scores = a.sc.match >= -128 && a.sc.match <= 127 && a.sc.mismatch >= -127 && a.sc.mismatch <= 128;
    const int nl = a.n_dev ? min((int)*a.n_dev, nlist) : nlist;
    const int wslot = G > 32 ? 0 : (int)((threadIdx.x & 31) / G); /* this group's place in its warp */
    for (int iter = 0;; iter++) {
        const int item0 = wc_next<G>(a, gpb, iter);
        if (item0 >= nl) break; /* the same for every lane of a warp (and of a two-warp group) */
        const int item = item0 + wslot;
        const bool listed = item < nl; /* the last warp may have groups without a pair */
        const int i = listed ? (int)list[item] : 0;
        const int qlen0 = listed ? (int)a.q_len[i] : 0, tlen0 = listed ? (int)a.t_len[i] : 0;
        const uint32_t *q = a.pq + (listed ? (a.q_off[i] >> 3) : 0);
        const uint32_t *t = a.pt + (listed ? (a.t_off[i] >> 3) : 0);
        /* FAST: this launch scores with the prmt table; a pair with another
         * code or scores beyond a byte goes to the compare-scoring launch
         * that follows (a.defer), and this launch skips it */
        const bool plain_q = wc_plain<G>(q, (qlen0 + 7) >> 3); /* warp collectives: every lane calls both */
        const bool plain_t = wc_plain<G>(t, (tlen0 + 7) >> 3);
        const bool fast_pair = fast_scores && plain_q && plain_t;
        const bool has = listed && (!FAST || fast_pair);
        if (FAST && listed && !fast_pair && gl == 0) a.defer[atomicAdd(a.ndefer, 1u)] = (uint32_t)i;
        const int qlen = has ? qlen0 : 0, tlen = has ? tlen0 : 0;
        const int qregs = (qlen + 7) >> 3, tregs = (tlen + 7) >> 3;
        WcScore S;
        S.local = ALGO == LOCAL_;
        S.tab = tab;
        S.fast = fast_pair;
        uint4 *tb = nullptr;
        if (START == WITH_TB_ && has) {
            tb = a.tb + a.tb_off[i];
            uint4 *z = tb + (size_t)tregs * 2 * qregs;
            for (int k = gl; k < 4 * qregs; k += G) z[k] = make_uint4(0, 0, 0, 0);
        }
        auto qf = [&](int j) { return q[j]; };
        auto tf = [&](int T) { return t[T]; };
        WcRec best, sec;
        int gscore = 0;
        if (ALGO == GLOBAL_) {
            wc_sweep<G, 2, START == WITH_TB_, false, FAST>(qf, qregs, tf, tregs, qlen, tlen, a.sc, S, ring, tb, 0,
                                                     bandmax, false, best, sec, gscore);
            /* the owner lane of the last band holds the score */
            gscore = grp_bcast<G>(gscore, (tregs - 1) & (G - 1));
            if (gl == 0 && has && a.score) a.score[i] = gscore;
            continue;
        }
        /* LOCAL forward (pass 1 also records per-band maxima for second best) */
        wc_sweep<G, 0, START == WITH_TB_, false, FAST>(qf, qregs, tf, tregs, qlen, tlen, a.sc, S, ring, tb, 0, bandmax,
                                                 SECOND, best, sec, gscore);
        best = rec_reduce<G>(best);
        WcRec secr = {0, 0x7fffffff, 0, 0};
        if (SECOND) {
            if constexpr (G > 32) __syncthreads();
            else __syncwarp();
            /* inclusive prefix maximum over bands, in place */
            int carry = 0;
            const int chunks = (tregs + G - 1) / G;
            const int nchunks = G >= 32 ? chunks : (int)__reduce_max_sync(0xFFFFFFFFu, (unsigned)chunks);
            for (int ch = 0; ch < nchunks; ch++) {
                const int b = ch * G + gl;
                int v = grp_prefix_max<G>(b < tregs ? bandmax[b] : 0);
                v = max(v, carry);
                if (b < tregs) bandmax[b] = v;
                carry = grp_bcast<G>(v, G - 1);
            }
            if constexpr (G > 32) __syncthreads();
            else __syncwarp();
            WcRec b2, s2;
            int g2 = 0;
            wc_sweep<G, 0, false, true, FAST>(qf, qregs, tf, tregs, qlen, tlen, a.sc, S, ring, nullptr, 0, bandmax,
                                              false, b2, s2, g2);
            secr = rec_reduce<G>(s2);
        }
        int qs = 0, ts = 0;
        if (START == WITH_START_) {
            /* groups whose reverse region spans at least G words sweep it;
             * the others (and groups without a hit) pass an empty sweep */
            const int rend_reg = best.v > 0 ? min((best.col >> 3) + 1, qregs) : 0;
            const int gend_reg = best.v > 0 ? min((best.row >> 3) + 1, tregs) : 0;
            const bool sweep = rend_reg >= G;
            auto qr = [&](int j) { return nrev(q[rend_reg - 1 - j]); };
            auto tr = [&](int T) { return nrev(t[gend_reg - 1 - T]); };
            WcRec bs, ss;
            int g3 = 0;
            wc_sweep<G, 1, false, false, FAST>(qr, sweep ? rend_reg : 0, tr, sweep ? gend_reg : 0, 0, 0, a.sc, S, ring,
                                         nullptr, best.v, bandmax, false, bs, ss, g3);
            bs = rec_reduce<G>(bs);
            if (sweep) {
                /* reversed coordinates -> what the reference records */
                const int gidx = (gend_reg << 3) - 1 - (bs.band << 3);
                ts = gidx + (bs.row - (bs.band << 3));
                qs = (rend_reg << 3) - 1 - bs.col;
            } else if (best.v > 0) {
                bool done = false;
                if constexpr (G > 32) {
                    /* a two-warp group with a reverse region of 32-63 words:
                     * warp 0 sweeps it alone on 32 lanes */
                    if (rend_reg >= 32) {
                        done = true;
                        if (threadIdx.x < 32) {
                            WcRec b2, s2;
                            int g4 = 0;
                            wc_sweep<32, 1, false, false, FAST>(qr, rend_reg, tr, gend_reg, 0, 0, a.sc, S, ring,
                                                                nullptr, best.v, bandmax, false, b2, s2, g4);
                            b2 = rec_reduce<32>(b2);
                            const int gidx = (gend_reg << 3) - 1 - (b2.band << 3);
                            ts = gidx + (b2.row - (b2.band << 3));
                            qs = (rend_reg << 3) - 1 - b2.col;
                        }
                    }
                }
                /* reverse region narrower than 32 words (the ring's reader
                 * must trail its writer): the group's first lane runs the
                 * one-thread start pass with the group's ring as row buffer.
                 * It stops at the first cell reaching the score -- for the
                 * short local hits that end this early, a few bands -- where
                 * the group would finish a 32-band round. */
                if (!done && gl == 0) {
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
            }
            if constexpr (G > 32) __syncthreads();
            else __syncwarp();
        }
        if (gl == 0 && has) {
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

/* Shared memory of one warp-cooperative block: `warps` warps x 32/G groups,
 * each with a ring of max_q8 words and, for LOCAL/GLOBAL, band maxima
 * (max_t8/8 + 1 words).  SEMI_GLOBAL's last-column rows live in global
 * scratch (`DpArgs::lastcol`), one slot per group of the grid. */
size_t wc_smem_bytes(int algo, int group, int warps, int max_q8, int max_t8)
{
    const size_t per = (size_t)max_q8 + (algo == SEMI_GLOBAL_ ? 0 : (size_t)max_t8 / 8 + 1);
    return (size_t)warps * 32 / group * per * 4; /* groups per block x per group */
}

/* one kernel instantiation per (group, algo, start, second best) */
template <int G, bool FAST, class F> static cudaError_t with_wc_kernel(int algo, int start, bool second, F &&f)
{
    if (algo == SEMI_GLOBAL_) {
        if (start == WITH_START_)
            return second ? f(dp_wc_semi_kernel<G, true, true, FAST>) : f(dp_wc_semi_kernel<G, false, true, FAST>);
        return second ? f(dp_wc_semi_kernel<G, true, false, FAST>) : f(dp_wc_semi_kernel<G, false, false, FAST>);
    }
    if (algo == GLOBAL_)
        return start == WITH_TB_ ? f(dp_wc_kernel<G, GLOBAL_, WITH_TB_, false, FAST>)
                                 : f(dp_wc_kernel<G, GLOBAL_, WITHOUT_START_, false, FAST>);
    if (algo == LOCAL_) {
        if (start == WITH_START_)
            return second ? f(dp_wc_kernel<G, LOCAL_, WITH_START_, true, FAST>)
                          : f(dp_wc_kernel<G, LOCAL_, WITH_START_, false, FAST>);
        if (start == WITH_TB_)
            return second ? f(dp_wc_kernel<G, LOCAL_, WITH_TB_, true, FAST>)
                          : f(dp_wc_kernel<G, LOCAL_, WITH_TB_, false, FAST>);
        return second ? f(dp_wc_kernel<G, LOCAL_, WITHOUT_START_, true, FAST>)
                      : f(dp_wc_kernel<G, LOCAL_, WITHOUT_START_, false, FAST>);
    }
    return cudaErrorInvalidValue;
}
/* fast: the table-scoring kernels (the ones that run nearly every pair) */
template <class F>
static cudaError_t with_wc_kernel(int group, int algo, int start, bool second, F &&f, bool fast = true)
{
    if (fast) {
        if (group == 64) return with_wc_kernel<64, true>(algo, start, second, f);
        if (group == 8) return with_wc_kernel<8, true>(algo, start, second, f);
        if (group == 16) return with_wc_kernel<16, true>(algo, start, second, f);
        if (group == 32) return with_wc_kernel<32, true>(algo, start, second, f);
    } else {
        if (group == 64) return with_wc_kernel<64, false>(algo, start, second, f);
        if (group == 8) return with_wc_kernel<8, false>(algo, start, second, f);
        if (group == 16) return with_wc_kernel<16, false>(algo, start, second, f);
        if (group == 32) return with_wc_kernel<32, false>(algo, start, second, f);
    }
    return cudaErrorInvalidValue;
}

/* resident blocks per SM of one launch shape (0: it cannot run) */
static int wc_blocks_per_sm(int algo, int start, bool second, int group, int warps, size_t smem)
{
    if (smem > (200u << 10)) return 0;
    int n = 0;
    const cudaError_t e = with_wc_kernel(group, algo, start, second, [&](auto k) {
        cudaError_t r = allow_dyn_smem(k);
        if (r == cudaSuccess) r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, 32 * warps, smem);
        return r;
    });
    if (e != cudaSuccess) {
        cudaGetLastError(); /* a size the kernel cannot take: no resident block */
        return 0;
    }
    return n;
}

/* the shape with the most resident warps for this group (4, 2 or 1 warps
 * per block; long rings fit better in small blocks) */
static WcLaunch wc_shape(int algo, int start, bool second, int group, int max_q8, int max_t8)
{
    WcLaunch best;
    int best_res = 0;
    for (int warps : {4, 2, 1}) {
        if (group == 64 && warps != 2) continue; /* one two-warp group per block */
        const size_t smem = wc_smem_bytes(algo, group, warps, max_q8, max_t8);
        const int res = wc_blocks_per_sm(algo, start, second, group, warps, smem) * warps;
        if (res > best_res) {
            best_res = res;
            best.group = group, best.warps = warps, best.smem = smem, best.resident_warps = res;
        }
    }
    return best;
}

WcLaunch wc_plan(int algo, int start, bool second, int nlist, int max_q8, int max_t8, int forced_group,
                 int max_group)
{
    WcLaunch l;
    if (nlist <= 0) return l;
    if (forced_group > 0) {
        l = wc_shape(algo, start, second, forced_group, max_q8, max_t8);
    } else if (max_group >= 64) {
        /* queries of 64+ words (the launch of the longest pairs): a few
         * hundred pairs of very unequal length, so the launch lasts as long
         * as its longest pair's sweep; two-warp groups halve that */
        l = wc_shape(algo, start, second, 64, max_q8, max_t8);
        if (l.group == 0) l = wc_shape(algo, start, second, 32, max_q8, max_t8);
    } else {
        /* the narrowest group that keeps 3/4 of the 32-lane kernel's
         * resident warps: narrower groups waste fewer lanes on each pair's
         * pipeline fill and drain but hold one ring per pair */
        const WcLaunch w32 = max_group >= 32 ? wc_shape(algo, start, second, 32, max_q8, max_t8) : WcLaunch{};
        for (int g : {8, 16}) {
            if (g > max_group) break;
            /* SEMI_GLOBAL measured slower at 8 lanes than at 16 (250-1000 bp:
             * 93 against 87 ms), its last-column writes and row scans
             * weighing more on narrow groups */
            if (algo == SEMI_GLOBAL_ && g == 8 && max_group >= 16) continue;
            const WcLaunch wg = wc_shape(algo, start, second, g, max_q8, max_t8);
            if (wg.group > 0 && (w32.group == 0 || 4 * wg.resident_warps >= 3 * w32.resident_warps)) {
                l = wg;
                break;
            }
        }
        if (l.group == 0) l = w32;
    }
    if (l.group == 0) return l;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int per_block = l.warps * 32 / l.group;
    l.blocks = (nlist + per_block - 1) / per_block;
    const int cap = sms * 64 / l.warps; /* at most 64 warps per SM's worth of blocks; warps loop over pairs */
    if (l.blocks > cap) l.blocks = cap;
    return l;
}

size_t wc_scratch_words(int algo, const WcLaunch &l, int max_t8)
{
    if (algo != SEMI_GLOBAL_ || l.group == 0) return 0;
    return (size_t)l.blocks * l.warps * 32 / l.group * ((size_t)max_t8 + 8);
}

cudaError_t launch_dp_wc(int algo, int start, bool second, const DpArgs &a, const uint32_t *list, int nlist,
                         int max_q8, int max_t8, const WcLaunch &l, int32_t *rows, uint32_t *defer, uint32_t *ndefer,
                         uint32_t *wq, cudaStream_t s)
{
    if (nlist <= 0) return cudaSuccess;
    if (l.group == 0) return cudaErrorInvalidValue;
    DpArgs b = a;
    /* the launches' own work counters (a.queue is the one-thread kernel's) */
    b.queue = wq;
    if (wq) {
        const cudaError_t z = cudaMemsetAsync(wq, 0, 2 * sizeof(uint32_t), s);
        if (z != cudaSuccess) return z;
    }
    if (algo == SEMI_GLOBAL_) {
        b.scratch_cols = (uint32_t)(max_t8 + 8); /* last-column rows per group */
        b.lastcol = rows;
    } else {
        b.scratch_cols = (uint32_t)(max_t8 / 8 + 1); /* band maxima per group */
    }
    const int ring_cols = max_q8;
    auto launch = [&](const DpArgs &args, const uint32_t *lst, int blocks, bool fast) {
        return with_wc_kernel(l.group, algo, start, second, [&](auto k) {
            cudaError_t e = allow_dyn_smem(k);
            if (e != cudaSuccess) return e;
            k<<<blocks, 32 * l.warps, l.smem, s>>>(args, lst, nlist, ring_cols);
            return cudaGetLastError();
        }, fast);
    };
    const bool byte_scores = a.sc.match >= -128 && a.sc.match <= 127 && a.sc.mismatch >= -127 && a.sc.mismatch <= 128;
    if (!byte_scores || !defer || !ndefer) return launch(b, list, l.blocks, false);
    /* the table-scoring launch, then the compare-scoring one over the pairs
     * it left (usually none: its grid only checks an empty count) */
    cudaError_t e = cudaMemsetAsync(ndefer, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    b.defer = defer, b.ndefer = ndefer, b.n_dev = nullptr;
    e = launch(b, list, l.blocks, true);
    if (e != cudaSuccess) return e;
    DpArgs c = b;
    c.defer = nullptr, c.ndefer = nullptr, c.n_dev = ndefer;
    c.queue = wq ? wq + 1 : nullptr;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return launch(c, defer, l.blocks < sms ? l.blocks : sms, false);
}

} // namespace gb
