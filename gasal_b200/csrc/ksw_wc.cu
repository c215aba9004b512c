/*
 * ksw_wc.cu -- ksw seed extension, one warp per pair, row-parallel.
 *
 * Replaces reference src/kernels/ksw_kernel_template.h:46-199 (one thread per
 * pair there, its eh[] row array in local memory).  The reference's loop is
 * kept exactly -- rows in target order, each row over the trimmed column range
 * [beg, end) that the previous row's zero/non-zero eh entries decide, a row
 * whose maximum is 0 (or that meets z-drop) ending its 8-row target tile, the
 * end-to-end score taken when the column loop's final index equals qlen -- but
 * the columns of one row are spread over the 32 lanes:
 *
 *   eh[] (H of the previous row's column j-1, E entering row i at column j)
 *   lives in shared memory, one 32-bit word per column (H low, E high half;
 *   both lie in [0, h0 + match*qlen], so pairs where that reaches 2^15 go to
 *   the one-thread kernel), in slots of 256 columns; within a row's tile lane
 *   L takes 8 consecutive columns, stored k-major (slot = (j & ~255) | k*32 |
 *   (j/8 mod 32)) so each of the tile's 8 loads/stores is one conflict-free
 *   warp access whatever multiple of 8 the tile starts at.
 *
 *   Within a row, M' (the diagonal score, 0 when the diagonal predecessor is
 *   0) and the E update are per column.  F -- the only left-to-right
 *   dependency -- opens from M' rather than H in ksw, so it is a max-plus
 *   prefix over t_j = max(M'_j - (o+e), 0) decaying by e per column: each
 *   lane folds its 8 columns, a 5-step shuffle scan combines the lanes, and
 *   the lane applies its carry in a second pass over the same registers.
 *
 *   The row maximum and its last column come from one warp max-reduction of
 *   the key H*8192 + j; the trimming scan from one ballot per tile and a
 *   broadcast re-read of the boundary lane's 8 entries.
 *
 * Columns left of beg are computed too (they hold zeros and stay zero, which
 * is exactly what skipping them leaves); columns at or right of end are not
 * written, so the entries the reference leaves stale stay stale.
 */
#include "dp_core.cuh"

namespace gb {

namespace {

constexpr int KT = 256;                 /* columns per tile (32 lanes x 8) */
constexpr int KSW_WC_COLS0 = 2048;      /* length class 0: queries up to 2046 bases */
constexpr int KSW_WC_COLS1 = 8192;      /* length class 1: up to 8190 */
constexpr int EH_LIMIT = 1 << 15;       /* H and E are stored as 16-bit halves */
constexpr int KEY_BITS = 13;            /* key = H << 13 | column: columns up to 8191, H below EH_LIMIT */
static_assert((1 << KEY_BITS) >= KSW_WC_COLS1, "the row-maximum key must hold every column of a length class");
static_assert((long long)EH_LIMIT << KEY_BITS <= 0x7FFFFFFFll, "the row-maximum key must fit in 32 bits");
constexpr unsigned FULL = 0xFFFFFFFFu;

__device__ __forceinline__ int kslot(int j) { return (j & ~255) | ((j & 7) << 5) | ((j >> 3) & 31); }

/* 16-bit prmt selector that sign-extends byte c (class c < 8) */
__device__ __forceinline__ uint32_t sel16(uint32_t c) { return c * 0x1111u | 0x8880u; }

/* The row loop is bound by the ALU pipe (min/max, permutes, logic): the
 * 16-bit split and merge of the eh words and the row-maximum keys are
 * written as integer multiply-adds so they issue on the FMA pipe. */
__device__ __forceinline__ uint32_t high16(uint32_t x)
{
    uint32_t d;
    asm("mul.hi.u32 %0, %1, %2;" : "=r"(d) : "r"(x), "r"(65536u));
    return d;
}

/* Per-row values shared by the tiles of one row, and the state they carry. */
struct TileConst {
    uint32_t *eh;
    const uint4 *selw;
    int slots;
    uint2 tab;
    int sm, sx, g, lane, end, Cmul, oe, e_del;
};
struct TileState {
    int fcarry, hcarry, kmax, hlast, flast; /* F and H entering the next tile, row-maximum key, H/F at end-1 */
    int fcol, fcnt;                         /* columns of the first lane holding a non-zero eh entry */
    int lcol, lcnt;                         /* ... and of the last one */
};

/* One tile of a row starting at column pos (a multiple of 8): lane L owns the
 * CPL columns pos + CPL*L ..  (CPL = 8: 256 columns; 4 and 2: the narrower
 * tiles that finish a row whose remaining range is at most 128 or 64
 * columns, so a trimmed row does not run whole 256-column tiles).  The eh
 * slots keep the 8-column layout of kslot(); with CPL = 4 / 2, two / four
 * lanes share a bank, which costs no more shared-memory cycles than the
 * 8-column tile's eight conflict-free accesses.  FULLT: every column lies
 * before the row's end (no per-column checks; the row's last column, if in
 * this tile, is lane 31's last). */
template <bool FAST, bool BAND, bool FULLT, int CPL>
__device__ __forceinline__ void ksw_tile(const TileConst &c, int pos, TileState &ts)
{
    static_assert(CPL == 8 || CPL == 4 || CPL == 2, "columns per lane");
    const int lane = c.lane;
    const int j0 = pos + lane * CPL;
    const int nv = FULLT ? CPL : min(max(c.end - j0, 0), CPL);
    /* lanes past the row (nv == 0) read slot group 0 and store nothing */
    const int jr = (FULLT || j0 < c.slots) ? j0 : 0;
    const int sub0 = jr & 7; /* first column of the lane within its 8-column word */
    const int sb = (jr & ~255) | ((jr >> 3) & 31);
    const uint4 sw = c.selw[jr >> 3];
    uint32_t swk[CPL / 2];
    if (CPL == 8) {
        swk[0] = sw.x, swk[1] = sw.y, swk[2] = sw.z, swk[3] = sw.w;
    } else if (CPL == 4) {
        const bool hi = sub0 != 0;
        swk[0] = hi ? sw.z : sw.x;
        swk[1] = hi ? sw.w : sw.y;
    } else {
        const int q4 = sub0 >> 1;
        swk[0] = q4 == 0 ? sw.x : q4 == 1 ? sw.y : q4 == 2 ? sw.z : sw.w;
    }
    int vh[CPL], ve[CPL];
#pragma unroll
    for (int k = 0; k < CPL; k++) {
        const uint32_t pv = c.eh[sb + 32 * (sub0 + k)];
        const uint32_t hi = high16(pv);
        ve[k] = (int)hi;
        vh[k] = (int)mad_lo_u32(hi, 0xFFFF0000u, pv); /* pv - (hi << 16) */
    }
    /* pass 1: M', t and the lane's F fold */
    int Mp[CPL], tv[CPL];
    int agg = 0;
#pragma unroll
    for (int k = 0; k < CPL; k++) {
        int s;
        if (FAST) {
            s = (int)prmt(c.tab.x, c.tab.y, (k & 1) ? (swk[k >> 1] >> 16) : swk[k >> 1]);
        } else {
            const int cd = (int)((sw.x >> (28 - 4 * (sub0 + k))) & 15u);
            s = cd == N_CODE4 ? 0 : (cd == c.g ? c.sm : c.sx);
        }
        Mp[k] = __viaddmin_s32(vh[k], s, vh[k] * c.Cmul);
        tv[k] = __viaddmax_s32(Mp[k], -c.oe, 0);
        agg = k == 0 ? tv[0] : __viaddmax_s32(agg, -c.e_del, tv[k]);
    }
    /* F entering each lane: max-plus scan over lanes, decay e per column.
     * A lane below the shift gets its own value back from the shuffle, and
     * max(x, x - eK*d) = x (e >= 0), so every lane takes the fused step. */
    const int eK = c.e_del * CPL;
    int x = agg;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(FULL, x, d);
        x = __viaddmax_s32(y, -eK * d, x);
    }
    const int ex = __shfl_up_sync(FULL, x, 1);
    int f = lane == 0 ? ts.fcarry : __viaddmax_s32(ts.fcarry, -eK * lane, ex);
    ts.fcarry = __shfl_sync(FULL, __viaddmax_s32(ts.fcarry, -eK * (lane + 1), x), 31);
    /* pass 2: H, E, F, row maximum key */
    int H[CPL];
    int lkey = -1; /* FULLT: this lane's best H * 8 + k (the last column on ties) */
#pragma unroll
    for (int k = 0; k < CPL; k++) {
        H[k] = __vimax3_s32(Mp[k], ve[k], f);
        ve[k] = __viaddmax_s32(ve[k], -c.e_del, tv[k]);
        f = __viaddmax_s32(f, -c.e_del, tv[k]);
        if (FULLT) {
            if (k & 1) lkey = __vimax3_s32(lkey, (int)mad_lo_u32((uint32_t)H[k - 1], 8u, (uint32_t)(k - 1)),
                                           (int)mad_lo_u32((uint32_t)H[k], 8u, (uint32_t)k));
        } else if (k < nv) {
            ts.kmax = max(ts.kmax, (int)mad_lo_u32((uint32_t)H[k], 1u << KEY_BITS, (uint32_t)(j0 + k)));
            ts.hlast = H[k];
            if (BAND) ts.flast = f;
        }
    }
    if (FULLT) {
        ts.kmax = max(ts.kmax, (int)mad_lo_u32((uint32_t)(lkey >> 3), 1u << KEY_BITS, (uint32_t)(j0 + (lkey & 7))));
        ts.hlast = H[CPL - 1];
        if (BAND) ts.flast = f;
    }
    int hp = __shfl_up_sync(FULL, H[CPL - 1], 1);
    if (lane == 0) hp = ts.hcarry;
    ts.hcarry = __shfl_sync(FULL, H[CPL - 1], 31);
    uint32_t nz = 0;
#pragma unroll
    for (int k = 0; k < CPL; k++) {
        const int hs = k == 0 ? hp : H[k - 1];
        if (FULLT || k < nv) {
            const uint32_t pv = mad_lo_u32((uint32_t)ve[k], 65536u, (uint32_t)hs);
            c.eh[sb + 32 * (sub0 + k)] = pv;
            nz |= pv;
        }
    }
    const unsigned bm = __ballot_sync(FULL, nz != 0);
    if (bm) {
        if (ts.fcol < 0) ts.fcol = pos + (__ffs(bm) - 1) * CPL, ts.fcnt = CPL;
        ts.lcol = pos + (31 - __clz(bm)) * CPL, ts.lcnt = CPL;
    }
}

/* Band certificate state (BAND mode).  C bounds every value of the
 * unbanded computation that the banded one does not have: cells outside the
 * band and band cells whose unbanded value was raised from outside.  Paths
 * leave the band only through the F chain past its right edge and the E of
 * its leftmost column (the band moves one column right per row), or start
 * outside it (the first row's seed-derived entries, the first column's
 * h0-derived values); a positive value gains at most max(match, 0) per row
 * and a zero one none ("M ? M + s : 0").  The unbanded computation then has
 * the banded one's row maximum and position whenever that maximum exceeds C
 * (or C is 0), the same trimmed range whenever the banded range ends inside
 * the band only while C is 0, and an end-to-end score that is either known or
 * bounded by C. */
struct Cert {
    int C = 0;          /* carried bound, after the last processed row */
    int gcert = -1;     /* largest end-to-end score the unbanded run surely took */
    int gie = -1;       /* its (last) row */
    int gunc = -1;      /* bound on every end-to-end candidate not known exactly */
};

/* One pair; `slots` shared-memory columns hold its eh row.  FAST: every
 * code is plain and the scores fit a signed byte (prmt table lookup),
 * otherwise nibble compares.  BAND: half-width w >= 0, returns false when
 * the certificate cannot vouch for the banded result (nothing is written). */
template <bool FAST, bool BAND>
__device__ bool ksw_pair(const DpArgs &a, uint32_t pid, uint32_t *eh, const uint4 *selw, int slots, const uint2 *stab,
                         int lane, int qlen, int tlen, const uint32_t *q, const uint32_t *t, int h0, int w,
                         unsigned long long &ncells)
{
    const int e_del = a.sc.e, oe = a.sc.oe, o_del = a.sc.o;
    const int mpos = max(a.sc.match, 0);
    /* C bounds every substitution score so that min(M + s, M*C) is M + s for
     * M >= 1 and <= 0 for M = 0 (0 and a negative value act alike below:
     * every later use is max(., e>=0, f>=0) or max(. - (o+e), 0)) */
    const int Cmul = max(max(a.sc.match, -a.sc.mismatch), 0) + 1;

    /* the reference's first row (ksw_kernel_template.h:75-79) */
    for (int s = lane; s < slots; s += 32) eh[s] = 0u;
    __syncwarp();
    const long long v1 = (uint32_t)h0 > (uint32_t)oe ? (long long)h0 - oe : 0;
    auto init_h = [&](int j) -> long long {
        if (j == 0) return h0;
        if (j == 1) return v1;
        if (j <= qlen && v1 - (long long)(j - 2) * e_del > e_del) return v1 - (long long)(j - 1) * e_del;
        return 0;
    };
    for (int j = lane; j <= qlen + 1; j += 32) {
        const long long h = init_h(j);
        if (h) eh[kslot(j)] = (uint32_t)h;
    }
    __syncwarp();

    Cert ct;
    if (BAND) ct.C = (int)init_h(w + 1); /* the seed-derived entries right of the first row's band */

    const int L8 = (qlen >> 3) << 3;
    int mx = h0, max_i = -1, max_j = -1, max_ie = -1, gscore = -1, mo = 0;
    int beg = 0, end = qlen;
    ncells = 0;
    for (int i = 0; i < tlen;) {
        bool clipped_r = false;
        int Cprev = 0;
        if (BAND) {
            Cprev = ct.C;
            /* a trimmed end inside the band is the unbanded end only while C is 0 */
            if (Cprev > 0 && end < min(i + w + 1, qlen)) return false;
            clipped_r = end > i + w + 1;
            if (beg < i - w) beg = i - w;
            if (end > i + w + 1) end = i + w + 1;
        }
        const int g = code(__ldg(t + (i >> 3)), i & 7);
        int h1 = 0;
        if (beg == 0) {
            h1 = (int)((uint32_t)h0 - (uint32_t)(o_del + e_del * (i + 1)));
            if (h1 < 0) h1 = 0;
        }
        int m = 0, mj = -1, fout = 0;
        int fcol = -1, fcnt = 0, lcol = -1, lcnt = 0;
        if (beg < end) {
            ncells += (unsigned long long)(end - beg);
            uint2 tab = make_uint2(0, 0);
            int sm = 0, sx = 0;
            if (FAST) {
                tab = stab[g];
            } else {
                sm = g == N_CODE4 ? 0 : a.sc.match;
                sx = g == N_CODE4 ? 0 : -a.sc.mismatch;
            }
            TileState ts{0, h1, -1, 0, 0, -1, 0, -1, 0};
            const TileConst tc{eh, selw, slots, tab, sm, sx, g, lane, end, Cmul, oe, e_del};
            /* 256-column tiles while more than 128 columns remain, then one
             * 128- or 64-column tile for the rest; FULLT when the whole tile
             * lies inside the row */
            int pos = beg & ~7, lpos = pos, lcpl = 8;
            while (pos < end) {
                const int rem = end - pos;
                lpos = pos;
                if (rem > 128) {
                    lcpl = 8;
                    if (rem >= 256) ksw_tile<FAST, BAND, true, 8>(tc, pos, ts);
                    else ksw_tile<FAST, BAND, false, 8>(tc, pos, ts);
                    pos += 256;
                } else if (rem > 64) {
                    lcpl = 4;
                    if (rem == 128) ksw_tile<FAST, BAND, true, 4>(tc, pos, ts);
                    else ksw_tile<FAST, BAND, false, 4>(tc, pos, ts);
                    pos += 128;
                } else {
                    lcpl = 2;
                    if (rem == 64) ksw_tile<FAST, BAND, true, 2>(tc, pos, ts);
                    else ksw_tile<FAST, BAND, false, 2>(tc, pos, ts);
                    pos += 64;
                }
            }
            int kmax = ts.kmax;
            const int hlast = ts.hlast, flast = ts.flast;
            fcol = ts.fcol, fcnt = ts.fcnt, lcol = ts.lcol, lcnt = ts.lcnt;
            kmax = __reduce_max_sync(FULL, kmax);
            m = kmax >> KEY_BITS;
            mj = kmax & ((1 << KEY_BITS) - 1);
            const int owner = (end - 1 - lpos) / lcpl;
            h1 = __shfl_sync(FULL, hlast, owner);
            if (BAND) fout = __shfl_sync(FULL, flast, owner);
        }
        if (lane == 0) eh[kslot(end)] = (uint32_t)h1;
        __syncwarp();
        if (BAND) {
            /* bound on this row's values the banded run does not have */
            int Crow = Cprev > 0 ? Cprev + mpos : 0;
            if (i > w) { /* the h0-derived column left of the matrix, outside the band */
                const int hv = h0 - o_del - e_del * i;
                if (hv > 0) Crow = max(Crow, hv + mpos);
            }
            if (end == i + w + 1 && end < qlen) Crow = max(Crow, fout);            /* F past the right edge */
            if (!(Crow == 0 || m > Crow)) return false;
            /* end-to-end score candidates (the unbanded end is known when the
             * row reached qlen, or when nothing was clipped or contaminated) */
            const bool end_known = end == qlen || (!clipped_r && Cprev == 0);
            const bool val_known = Crow == 0 || h1 > Crow;
            bool upd_known = false, upd_maybe = false;
            if (L8 == qlen) {
                if (end_known) upd_known = true;
                else ct.gunc = max(ct.gunc, max(h1, Crow));
            } else if (end == qlen) {
                upd_known = true;
            } else if (!end_known) {
                upd_maybe = true;
            }
            if (upd_known) {
                if (val_known) {
                    ct.gie = ct.gcert > h1 ? ct.gie : i;
                    ct.gcert = max(ct.gcert, h1);
                } else {
                    ct.gunc = max(ct.gunc, Crow);
                }
            }
            if (upd_maybe) ct.gunc = max(ct.gunc, Crow);
            /* E leaving the band's leftmost column into the next row */
            int Cnext = Crow;
            if (beg < end && beg == i - w) Cnext = max(Cnext, (int)(eh[kslot(i - w)] >> 16));
            ct.C = Cnext;
        } else if (max(L8, end) == qlen) {
            max_ie = gscore > h1 ? max_ie : i;
            gscore = max(gscore, h1);
        }
        bool leave = false;
        if (m == 0) {
            leave = true;
        } else if (m > mx) {
            mx = m, max_i = i, max_j = mj;
            mo = max(mo, abs(mj - i));
        } else if (a.zdrop > 0) {
            if (i - max_i > mj - max_j) {
                if (mx - m - ((i - max_i) - (mj - max_j)) * e_del > a.zdrop) leave = true;
            } else {
                if (mx - m - ((mj - max_j) - (i - max_i)) * e_del > a.zdrop) leave = true;
            }
        }
        if (leave) {
            __syncwarp();
            i = ((i >> 3) + 1) << 3;
            continue;
        }
        /* trimming (ksw_kernel_template.h:188-196): the first non-zero entry
         * lies among the columns of the first lane (over the row's tiles)
         * whose stores were non-zero, the last one (unless eh[end] = h1 is
         * non-zero) among those of the last such lane; lanes 0-7 read the
         * first group, lanes 8-15 the second, and one ballot gives both */
        int jj = -1;
        if (lane < 8) {
            if (fcol >= 0 && lane < fcnt) jj = fcol + lane;
        } else if (lane < 16) {
            if (h1 == 0 && lcol >= 0 && lane - 8 < lcnt) jj = lcol + (lane - 8);
        }
        const bool nzj = jj >= 0 && jj < end && eh[kslot(jj)] != 0u;
        const unsigned bal = __ballot_sync(FULL, nzj);
        const int nbeg = (bal & 0xFFu) ? fcol + __ffs(bal & 0xFFu) - 1 : end;
        int lastnz = nbeg - 1;
        if (h1 != 0) lastnz = end;
        else if (bal & 0xFF00u) lastnz = lcol + (31 - __clz(bal & 0xFF00u)) - 8;
        beg = nbeg;
        end = lastnz + 2 < qlen ? lastnz + 2 : qlen;
        __syncwarp(); /* the scans above read slots their owners rewrite next row */
        i++;
    }
    if (BAND) {
        const int gmax = max(ct.gcert, ct.gunc);
        if (gmax <= 0 || gmax <= mx - 5) {
            gscore = -1; /* the maximum is the answer */
        } else if (ct.gcert > ct.gunc) {
            gscore = ct.gcert, max_ie = ct.gie;
        } else {
            return false;
        }
    }
    if (lane == 0) {
        int sc, qe, te;
        if (gscore <= 0 || gscore <= mx - 5) {
            sc = mx, qe = max_j + 1, te = max_i + 1;
        } else {
            sc = gscore, qe = qlen, te = max_ie + 1;
        }
        if (a.score) a.score[pid] = sc;
        if (a.q_end) a.q_end[pid] = qe;
        if (a.t_end) a.t_end[pid] = te;
        if (!BAND && a.max_off) a.max_off[pid] = mo;
    }
    __syncwarp();
    return true;
}

/* band: per-pair half-width (negative = none) or null; retry/nretry collect
 * the pairs whose banded result the certificate did not accept. */
struct BandArgs {
    const int32_t *w;
    uint32_t *retry, *nretry;
    unsigned long long *cells; /* computed cells (rows x trimmed range), or null */
    int q_lo;                  /* shorter queries belong to an earlier class launch: skipped */
    int handback;              /* queries too long for this launch: 1 = to fb, 0 = skipped (next class) */
};

template <bool BAND>
__global__ void __launch_bounds__(32) ksw_wc_kernel(DpArgs a, const uint32_t *list, int nlist, int slots,
                                                     uint32_t *fb, uint32_t *fbn, uint32_t *wq, BandArgs ba)
{
    extern __shared__ __align__(16) uint32_t ksw_smem[];
    __shared__ uint2 stab[16];
    build_score_table(stab, a.sc, true);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    uint32_t *eh = ksw_smem + (size_t)warp * slots;
    uint4 *selw = reinterpret_cast<uint4 *>(ksw_smem + (size_t)warps * slots) + (size_t)warp * (slots / 8);
    const bool fast_scores = a.sc.match >= -128 && a.sc.match <= 127 && a.sc.mismatch >= -127 && a.sc.mismatch <= 128;
    const long long mpos = a.sc.match > 0 ? a.sc.match : 0;
    const uint32_t n = a.n_dev ? min(*a.n_dev, (uint32_t)nlist) : (uint32_t)nlist;
    for (;;) {
        uint32_t idx = 0;
        if (lane == 0) idx = atomicAdd(wq, 1u);
        idx = __shfl_sync(FULL, idx, 0);
        if (idx >= n) break;
        const uint32_t pid = list ? list[idx] : idx;
        const int qlen = (int)a.q_len[pid], tlen = (int)a.t_len[pid];
        const uint32_t h0u = a.seed ? a.seed[pid] : 0u;
        if (qlen < ba.q_lo) continue;
        if (qlen + 2 > slots) {
            if (ba.handback && lane == 0) fb[atomicAdd(fbn, 1u)] = pid;
            continue;
        }
        if ((long long)h0u + mpos * qlen >= EH_LIMIT) {
            if (lane == 0) fb[atomicAdd(fbn, 1u)] = pid;
            continue;
        }
        const uint32_t *q = a.pq + (a.q_off[pid] >> 3), *t = a.pt + (a.t_off[pid] >> 3);
        bool plain = fast_scores;
        const int qregs = (qlen + 7) >> 3;
        if (plain) {
            const int tregs = (tlen + 7) >> 3;
            uint32_t bad = 0;
            for (int x = lane; x < qregs + tregs; x += 32) {
                const uint32_t y = x < qregs ? q[x] : t[x - qregs];
#pragma unroll
                for (int k = 0; k < 8; k++) bad |= ~(PLAIN_CODES >> ((y >> (4 * k)) & 15u)) & 1u;
            }
            plain = __all_sync(FULL, bad == 0);
        }
        /* per 8 query columns: eight 16-bit prmt selectors (plain), or the packed word */
        for (int gi = lane; gi < slots / 8; gi += 32) {
            const uint32_t y = gi < qregs ? q[gi] : 0u;
            uint4 sw;
            if (plain) {
                uint32_t c[8];
#pragma unroll
                for (int k = 0; k < 8; k++) c[k] = sel16(class_of((y >> (28 - 4 * k)) & 15u));
                sw = make_uint4(c[0] | (c[1] << 16), c[2] | (c[3] << 16), c[4] | (c[5] << 16), c[6] | (c[7] << 16));
            } else {
                sw = make_uint4(y, 0u, 0u, 0u);
            }
            selw[gi] = sw;
        }
        __syncwarp();
        const int w = BAND && ba.w ? min(ba.w[pid], 1 << 20) : -1; /* wider than any matrix = unbanded */
        bool ok;
        unsigned long long nc = 0;
        if (BAND && w >= 0) {
            ok = plain ? ksw_pair<true, true>(a, pid, eh, selw, slots, stab, lane, qlen, tlen, q, t, (int)h0u, w, nc)
                       : ksw_pair<false, true>(a, pid, eh, selw, slots, stab, lane, qlen, tlen, q, t, (int)h0u, w, nc);
        } else {
            ok = plain ? ksw_pair<true, false>(a, pid, eh, selw, slots, stab, lane, qlen, tlen, q, t, (int)h0u, -1, nc)
                       : ksw_pair<false, false>(a, pid, eh, selw, slots, stab, lane, qlen, tlen, q, t, (int)h0u, -1,
                                               nc);
        }
        if (ba.cells && lane == 0) atomicAdd(ba.cells, nc);
        if (!ok && lane == 0) ba.retry[atomicAdd(ba.nretry, 1u)] = pid;
        __syncwarp();
    }
}

/* ---- lane groups: 32/G short pairs per warp ----------------------------
 *
 * A pair whose query fits one 256-column slot row runs on a group of G lanes
 * (8 columns per lane, 8G-column tiles), 32/G pairs side by side in a warp.
 * The groups step their pairs' rows in lockstep: every pass of the kernel's
 * loop runs one row of every group that holds a pair (a group whose pair
 * ended fetches the next one first), so the per-row work -- row maximum,
 * trimming, z-drop -- is shared by 32/G pairs instead of paid by a whole warp
 * for one, and a short trimmed row no longer spans a 256-column tile.  The
 * collectives are the warp kernel's at width G with the group's lane mask.
 * Group g's eh row starts 8g words past a multiple of 32 so that the groups'
 * accesses of one tile step fall in different banks. */
constexpr int GRP_SLOTS = 256;  /* eh columns per group: queries up to GRP_QMAX bases */
constexpr int GRP_QMAX = 248;   /* 31 query words: the suffix of the length order */
constexpr int GRP_PAD = 8;

template <int G> __device__ __forceinline__ int kslot_g(int j)
{
    return (j & ~(8 * G - 1)) | ((j & 7) * G) | ((j >> 3) & (G - 1));
}

struct GrpConst {
    uint32_t *eh;
    const uint4 *selw;
    uint2 tab;
    int sm, sx, g, gl, end, Cmul, oe, e_del;
    unsigned gmask;
    int gbase;
};

/* one 8G-column tile of a group's row starting at column pos (a multiple of
 * 8); lane gl owns pos + 8gl .. +7.  FULLT: the whole tile lies before end. */
template <int G, bool FAST, bool FULLT>
__device__ __forceinline__ void grp_tile(const GrpConst &c, int pos, TileState &ts)
{
    const int gl = c.gl;
    const int j0 = pos + gl * 8;
    const int nv = FULLT ? 8 : min(max(c.end - j0, 0), 8);
    const int jr = (FULLT || j0 < GRP_SLOTS) ? j0 : 0;
    const int sb = (jr & ~(8 * G - 1)) | ((jr >> 3) & (G - 1));
    const uint4 sw = c.selw[jr >> 3];
    const uint32_t swk[4] = {sw.x, sw.y, sw.z, sw.w};
    int vh[8], ve[8], Mp[8], tv[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const uint32_t pv = c.eh[sb + G * k];
        const uint32_t hi = high16(pv);
        ve[k] = (int)hi;
        vh[k] = (int)mad_lo_u32(hi, 0xFFFF0000u, pv);
    }
    int agg = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        int s;
        if (FAST) {
            s = (int)prmt(c.tab.x, c.tab.y, (k & 1) ? (swk[k >> 1] >> 16) : swk[k >> 1]);
        } else {
            const int cd = (int)((sw.x >> (28 - 4 * k)) & 15u);
            s = cd == N_CODE4 ? 0 : (cd == c.g ? c.sm : c.sx);
        }
        Mp[k] = __viaddmin_s32(vh[k], s, vh[k] * c.Cmul);
        tv[k] = __viaddmax_s32(Mp[k], -c.oe, 0);
        agg = k == 0 ? tv[0] : __viaddmax_s32(agg, -c.e_del, tv[k]);
    }
    const int eK = c.e_del * 8;
    int x = agg;
#pragma unroll
    for (int d = 1; d < G; d <<= 1) { /* as in ksw_tile: lanes below the shift keep their value */
        const int y = __shfl_up_sync(c.gmask, x, d, G);
        x = __viaddmax_s32(y, -eK * d, x);
    }
    const int ex = __shfl_up_sync(c.gmask, x, 1, G);
    int f = gl == 0 ? ts.fcarry : __viaddmax_s32(ts.fcarry, -eK * gl, ex);
    ts.fcarry = __shfl_sync(c.gmask, __viaddmax_s32(ts.fcarry, -eK * (gl + 1), x), G - 1, G);
    int H[8];
    int lkey = -1;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        H[k] = __vimax3_s32(Mp[k], ve[k], f);
        ve[k] = __viaddmax_s32(ve[k], -c.e_del, tv[k]);
        f = __viaddmax_s32(f, -c.e_del, tv[k]);
        if (FULLT) {
            if (k & 1) lkey = __vimax3_s32(lkey, (int)mad_lo_u32((uint32_t)H[k - 1], 8u, (uint32_t)(k - 1)),
                                           (int)mad_lo_u32((uint32_t)H[k], 8u, (uint32_t)k));
        } else if (k < nv) {
            ts.kmax = max(ts.kmax, (int)mad_lo_u32((uint32_t)H[k], 1u << KEY_BITS, (uint32_t)(j0 + k)));
            ts.hlast = H[k];
        }
    }
    if (FULLT) {
        ts.kmax = max(ts.kmax, (int)mad_lo_u32((uint32_t)(lkey >> 3), 1u << KEY_BITS, (uint32_t)(j0 + (lkey & 7))));
        ts.hlast = H[7];
    }
    int hp = __shfl_up_sync(c.gmask, H[7], 1, G);
    if (gl == 0) hp = ts.hcarry;
    ts.hcarry = __shfl_sync(c.gmask, H[7], G - 1, G);
    uint32_t nz = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int hs = k == 0 ? hp : H[k - 1];
        if (FULLT || k < nv) {
            const uint32_t pv = mad_lo_u32((uint32_t)ve[k], 65536u, (uint32_t)hs);
            c.eh[sb + G * k] = pv;
            nz |= pv;
        }
    }
    const unsigned bm = (__ballot_sync(c.gmask, nz != 0) >> c.gbase) & ((G >= 32) ? 0xFFFFFFFFu : ((1u << G) - 1u));
    if (bm) {
        if (ts.fcol < 0) ts.fcol = pos + (__ffs(bm) - 1) * 8, ts.fcnt = 8;
        ts.lcol = pos + (31 - __clz(bm)) * 8, ts.lcnt = 8;
    }
}

/* The unbanded ksw on lane groups, for pairs of at most GRP_QMAX query bases.
 * Pairs with longer queries are skipped (the 32-lane class launches take
 * them); pairs whose seed + match * qlen reaches 2^15 go to fb.  With `split`
 * >= 0 the list is length-ordered and its short pairs are exactly
 * list[split, n): the launch visits only those. */
template <int G>
__global__ void __launch_bounds__(32) ksw_grp_kernel(DpArgs a, const uint32_t *list, int nlist, int split,
                                                      uint32_t *fb, uint32_t *fbn, uint32_t *wq,
                                                      unsigned long long *cells)
{
    static_assert(G == 8 || G == 16, "lane group");
    constexpr int NG = 32 / G;
    extern __shared__ __align__(16) uint32_t kg_smem[];
    __shared__ uint2 stab[16];
    build_score_table(stab, a.sc, true);
    __syncthreads();
    const int lane = threadIdx.x & 31, grp = lane / G, gl = lane & (G - 1), gbase = grp * G;
    const unsigned gmask = (G >= 32) ? FULL : (((1u << G) - 1u) << gbase);
    /* one warp per block: group grp's eh row, then the groups' selector rows */
    uint32_t *eh = kg_smem + grp * (GRP_SLOTS + GRP_PAD);
    uint4 *selw = reinterpret_cast<uint4 *>(kg_smem + NG * (GRP_SLOTS + GRP_PAD)) + grp * (GRP_SLOTS / 8);
    const bool fast_scores = a.sc.match >= -128 && a.sc.match <= 127 && a.sc.mismatch >= -127 && a.sc.mismatch <= 128;
    const long long mpos_ll = a.sc.match > 0 ? a.sc.match : 0;
    const uint32_t n = a.n_dev ? min(*a.n_dev, (uint32_t)nlist) : (uint32_t)nlist;
    const uint32_t first = split > 0 ? (uint32_t)split : 0u;
    const int e_del = a.sc.e, oe = a.sc.oe, o_del = a.sc.o;
    const int Cmul = max(max(a.sc.match, -a.sc.mismatch), 0) + 1;

    bool have = false, done = false, plain = false;
    uint32_t pid = 0;
    int qlen = 0, tlen = 0, h0 = 0, i = 0, beg = 0, end = 0, L8 = 0;
    int mx = 0, max_i = -1, max_j = -1, max_ie = -1, gscore = -1, mo = 0;
    const uint32_t *t = nullptr;
    unsigned long long nc = 0;
    for (;;) {
        if (!have && !done) {
            /* this group fetches its next pair */
            uint32_t idx = 0;
            if (gl == 0) idx = first + atomicAdd(wq, 1u);
            idx = __shfl_sync(gmask, idx, 0, G);
            if (idx >= n) {
                done = true;
            } else {
                pid = list ? list[idx] : idx;
                qlen = (int)a.q_len[pid];
                tlen = (int)a.t_len[pid];
                const uint32_t h0u = a.seed ? a.seed[pid] : 0u;
                if (qlen <= GRP_QMAX) {
                    if ((long long)h0u + mpos_ll * qlen >= EH_LIMIT) {
                        if (gl == 0) fb[atomicAdd(fbn, 1u)] = pid;
                    } else {
                        const uint32_t *q = a.pq + (a.q_off[pid] >> 3);
                        t = a.pt + (a.t_off[pid] >> 3);
                        h0 = (int)h0u;
                        const int qregs = (qlen + 7) >> 3, tregs = (tlen + 7) >> 3;
                        uint32_t bad = fast_scores ? 0u : 1u;
                        for (int x = gl; x < qregs + tregs; x += G) {
                            const uint32_t y = x < qregs ? q[x] : t[x - qregs];
#pragma unroll
                            for (int k = 0; k < 8; k++) bad |= ~(PLAIN_CODES >> ((y >> (4 * k)) & 15u)) & 1u;
                        }
                        plain = __all_sync(gmask, bad == 0);
                        for (int gi = gl; gi < GRP_SLOTS / 8; gi += G) {
                            const uint32_t y = gi < qregs ? q[gi] : 0u;
                            uint4 sw;
                            if (plain) {
                                uint32_t cc[8];
#pragma unroll
                                for (int k = 0; k < 8; k++) cc[k] = sel16(class_of((y >> (28 - 4 * k)) & 15u));
                                sw = make_uint4(cc[0] | (cc[1] << 16), cc[2] | (cc[3] << 16), cc[4] | (cc[5] << 16),
                                                cc[6] | (cc[7] << 16));
                            } else {
                                sw = make_uint4(y, 0u, 0u, 0u);
                            }
                            selw[gi] = sw;
                        }
                        /* the reference's first row (ksw_kernel_template.h:75-79) */
                        for (int s2 = gl; s2 < GRP_SLOTS; s2 += G) eh[s2] = 0u;
                        __syncwarp(gmask);
                        const int v1 = h0u > (uint32_t)oe ? h0 - oe : 0;
                        for (int j = gl; j <= qlen + 1; j += G) {
                            int h = 0;
                            if (j == 0) h = h0;
                            else if (j == 1) h = v1;
                            else if (j <= qlen && v1 - (j - 2) * e_del > e_del) h = v1 - (j - 1) * e_del;
                            if (h) eh[kslot_g<G>(j)] = (uint32_t)h;
                        }
                        __syncwarp(gmask);
                        have = true;
                        i = 0, beg = 0, end = qlen, L8 = (qlen >> 3) << 3;
                        mx = h0, max_i = -1, max_j = -1, max_ie = -1, gscore = -1, mo = 0;
                        nc = 0;
                    }
                }
            }
        }
        if (__all_sync(FULL, done)) break;
        if (have && i < tlen) {
            /* one row of this group's pair */
            const int g = code(__ldg(t + (i >> 3)), i & 7);
            int h1 = 0;
            if (beg == 0) {
                h1 = (int)((uint32_t)h0 - (uint32_t)(o_del + e_del * (i + 1)));
                if (h1 < 0) h1 = 0;
            }
            int m = 0, mj = -1;
            int fcol = -1, lcol = -1;
            if (beg < end) {
                nc += (unsigned long long)(end - beg);
                uint2 tab = make_uint2(0, 0);
                int sm = 0, sx = 0;
                if (plain) {
                    tab = stab[g];
                } else {
                    sm = g == N_CODE4 ? 0 : a.sc.match;
                    sx = g == N_CODE4 ? 0 : -a.sc.mismatch;
                }
                TileState ts{0, h1, -1, 0, 0, -1, 0, -1, 0};
                const GrpConst gc{eh, selw, tab, sm, sx, g, gl, end, Cmul, oe, e_del, gmask, gbase};
                int pos = beg & ~7, lpos = pos;
                while (pos < end) {
                    lpos = pos;
                    const bool full = end - pos >= 8 * G;
                    if (plain) {
                        if (full) grp_tile<G, true, true>(gc, pos, ts);
                        else grp_tile<G, true, false>(gc, pos, ts);
                    } else {
                        if (full) grp_tile<G, false, true>(gc, pos, ts);
                        else grp_tile<G, false, false>(gc, pos, ts);
                    }
                    pos += 8 * G;
                }
                int kmax = ts.kmax;
#pragma unroll
                for (int o = G / 2; o > 0; o >>= 1) kmax = max(kmax, __shfl_xor_sync(gmask, kmax, o, G));
                m = kmax >> KEY_BITS;
                mj = kmax & ((1 << KEY_BITS) - 1);
                h1 = __shfl_sync(gmask, ts.hlast, (end - 1 - lpos) >> 3, G);
                fcol = ts.fcol, lcol = ts.lcol;
            }
            if (gl == 0) eh[kslot_g<G>(end)] = (uint32_t)h1;
            __syncwarp(gmask);
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
            } else if (a.zdrop > 0) {
                if (i - max_i > mj - max_j) {
                    if (mx - m - ((i - max_i) - (mj - max_j)) * e_del > a.zdrop) leave = true;
                } else {
                    if (mx - m - ((mj - max_j) - (i - max_i)) * e_del > a.zdrop) leave = true;
                }
            }
            if (leave) {
                i = ((i >> 3) + 1) << 3;
            } else {
                /* trimming (ksw_kernel_template.h:188-196): the first and last
                 * non-zero entries lie among the 8 columns of the first and the
                 * last group lane whose stores were non-zero */
                const int jf = fcol >= 0 ? fcol + gl : -1;
                const int jl = (h1 == 0 && lcol >= 0) ? lcol + gl : -1;
                const bool nzf = gl < 8 && jf >= 0 && jf < end && eh[kslot_g<G>(jf)] != 0u;
                const bool nzl = gl < 8 && jl >= 0 && jl < end && eh[kslot_g<G>(jl)] != 0u;
                const unsigned bf = (__ballot_sync(gmask, nzf) >> gbase) & 0xFFu;
                const unsigned bl = (__ballot_sync(gmask, nzl) >> gbase) & 0xFFu;
                const int nbeg = bf ? fcol + __ffs(bf) - 1 : end;
                int lastnz = nbeg - 1;
                if (h1 != 0) lastnz = end;
                else if (bl) lastnz = lcol + (31 - __clz(bl));
                beg = nbeg;
                end = lastnz + 2 < qlen ? lastnz + 2 : qlen;
                i++;
            }
            __syncwarp(gmask); /* the scans above read slots their owners rewrite next row */
        }
        if (have && i >= tlen) {
            if (gl == 0) {
                int sc, qe, te;
                if (gscore <= 0 || gscore <= mx - 5) {
                    sc = mx, qe = max_j + 1, te = max_i + 1;
                } else {
                    sc = gscore, qe = qlen, te = max_ie + 1;
                }
                if (a.score) a.score[pid] = sc;
                if (a.q_end) a.q_end[pid] = qe;
                if (a.t_end) a.t_end[pid] = te;
                if (a.max_off) a.max_off[pid] = mo;
                if (cells) atomicAdd(cells, nc);
            }
            have = false;
            __syncwarp(gmask);
        }
    }
}

template <int G> size_t grp_smem() { return (size_t)(32 / G) * ((GRP_SLOTS + GRP_PAD) * 4 + (GRP_SLOTS / 8) * 16); }

cudaError_t launch_grp(const DpArgs &a, const uint32_t *list, int nlist, int split, uint32_t *fb, uint32_t *fbn,
                       uint32_t *wq, unsigned long long *cells, cudaStream_t s)
{
    constexpr int G = 8;
    const int nshort = split >= 0 ? nlist - split : nlist;
    if (nshort <= 0) return cudaSuccess;
    const size_t smem = grp_smem<G>();
    int dev = 0, sms = 148, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ksw_grp_kernel<G>, 32, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int blocks = (nshort + 32 / G - 1) / (32 / G);
    if (blocks > per_sm * sms) blocks = per_sm * sms;
    ksw_grp_kernel<G><<<blocks, 32, smem, s>>>(a, list, nlist, split, fb, fbn, wq, cells);
    return cudaGetLastError();
}

/* shared-memory slots per warp for queries up to max_qlen (whole tiles) */
int slots_for(int max_qlen) { return ((max_qlen + 2 + KT - 1) / KT) * KT; }

cudaError_t launch_slots(const DpArgs &a, const uint32_t *list, int nlist, int slots, uint32_t *fb, uint32_t *fbn,
                         uint32_t *wq, const BandArgs &ba, bool band, cudaStream_t s)
{
    const int block = 32, warps = block / 32; /* one warp per block packs shared memory tightest */
    const size_t smem = (size_t)warps * slots * (sizeof(uint32_t) + 2);
    auto k = band ? ksw_wc_kernel<true> : ksw_wc_kernel<false>;
    cudaError_t e = allow_dyn_smem(k);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int blocks = (nlist + warps - 1) / warps;
    if (blocks > per_sm * sms) blocks = per_sm * sms;
    if (blocks < 1) blocks = 1;
    k<<<blocks, block, smem, s>>>(a, list, nlist, slots, fb, fbn, wq, ba);
    return cudaGetLastError();
}

} // namespace

bool ksw_wc_scores_ok(const Scores &sc)
{
    return sc.e >= 0 && sc.oe >= 0 && sc.match < 4095 && sc.match > -4095 && sc.mismatch < 4095 &&
           sc.mismatch > -4095;
}

void ksw_wc_classes(const uint32_t *h_q_len, int n, int slots[2])
{
    int m0 = 0, m1 = -1;
    for (int i = 0; i < n; i++) {
        const int q = (int)h_q_len[i];
        if (q + 2 <= KSW_WC_COLS0) m0 = q > m0 ? q : m0;
        else if (q + 2 <= KSW_WC_COLS1) m1 = q > m1 ? q : m1;
    }
    slots[0] = slots_for(m0);
    slots[1] = m1 >= 0 ? slots_for(m1) : 0;
}

/* the class launches over one list; wq[c] is class c's zeroed work counter;
 * class 0 skips queries shorter than q_lo0 (the lane-group launch's) */
static cudaError_t launch_classes(const DpArgs &a, const uint32_t *list, int nlist, const int slots[2], uint32_t *fb,
                                  uint32_t *fbn, uint32_t *wq, BandArgs ba, bool band, cudaStream_t s, int q_lo0 = 0)
{
    if (nlist <= 0) return cudaSuccess;
    ba.q_lo = q_lo0;
    ba.handback = slots[1] == 0;
    cudaError_t e = launch_slots(a, list, nlist, slots[0], fb, fbn, wq, ba, band, s);
    if (e != cudaSuccess || slots[1] == 0) return e;
    ba.q_lo = slots[0] - 1;
    ba.handback = 1;
    return launch_slots(a, list, nlist, slots[1], fb, fbn, wq + 1, ba, band, s);
}

cudaError_t launch_ksw_wc(const DpArgs &a, const uint32_t *list, int nlist, const int slots[2], uint32_t *fb,
                          uint32_t *fbn, uint32_t *wq, unsigned long long *cells, cudaStream_t s, int split,
                          uint32_t *gq)
{
    BandArgs ba{nullptr, nullptr, nullptr, cells, 0, 1};
    if (split < -1) return launch_classes(a, list, nlist, slots, fb, fbn, wq, ba, false, s);
    /* short queries on lane groups: the order's suffix [split, nlist), or
     * every pair of an unordered list skipping the longer ones */
    const cudaError_t e = launch_grp(a, list, nlist, split, fb, fbn, gq, cells, s);
    if (e != cudaSuccess) return e;
    if (split >= 0) return launch_classes(a, list, split, slots, fb, fbn, wq, ba, false, s);
    return launch_classes(a, list, nlist, slots, fb, fbn, wq, ba, false, s, GRP_QMAX + 1);
}

int ksw_grp_short(const uint32_t *h_q_len, int n)
{
    int c = 0;
    for (int i = 0; i < n; i++) c += ((h_q_len[i] + 7) >> 3) <= (uint32_t)(GRP_QMAX / 8) ? 1 : 0;
    return c;
}

cudaError_t launch_ksw_band(const DpArgs &a, const uint32_t *list, int nlist, const int slots[2],
                            const int32_t *band_w, uint32_t *fb, uint32_t *fbn, uint32_t *retry, uint32_t *nretry,
                            unsigned long long *cells, uint32_t *wq, cudaStream_t s)
{
    BandArgs ba{band_w, retry, nretry, cells, 0, 1};
    return launch_classes(a, list, nlist, slots, fb, fbn, wq, ba, true, s);
}

} // namespace gb
