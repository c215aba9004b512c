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
 *   lives in shared memory, one int2 per column, tiles of 256 columns; lane L
 *   owns columns 8L..8L+7 of every tile, stored k-major (slot = tile*256 +
 *   k*32 + L) so each of the 8 loads/stores of a tile is one conflict-free
 *   warp access.
 *
 *   Within a row, M' (the diagonal score, 0 when the diagonal predecessor is
 *   0) and the E update are per column.  F -- the only left-to-right
 *   dependency -- opens from M' rather than H in ksw, so it is a max-plus
 *   prefix over t_j = max(M'_j - (o+e), 0) decaying by e per column: each
 *   lane folds its 8 columns, a 5-step shuffle scan combines the lanes, and
 *   the lane applies its carry in a second pass over the same registers.
 *
 *   The row maximum and its last column come from one warp max-reduction of
 *   the key H*4096 + j; the trimming scan from one ballot per tile and a
 *   broadcast re-read of the boundary lane's 8 entries.
 *
 * Columns left of beg are computed too (they hold zeros and stay zero, which
 * is exactly what skipping them leaves); columns at or right of end are not
 * written, so the entries the reference leaves stale stay stale.
 */
#include "dp_core.cuh"

namespace gb {

namespace {

constexpr int KT = 256;                 /* columns per tile */
constexpr int KEY_BITS = 12;            /* key = H << 12 | column */
constexpr int KEY_H_LIMIT = 1 << 19;    /* H must stay below this for the key */
constexpr unsigned FULL = 0xFFFFFFFFu;

__device__ __forceinline__ int kslot(int j) { return (j & ~255) | ((j & 7) << 5) | ((j >> 3) & 31); }

/* 16-bit prmt selector that sign-extends byte c (class c < 8) */
__device__ __forceinline__ uint32_t sel16(uint32_t c) { return c * 0x1111u | 0x8880u; }

/* One pair.  NT tiles cover the query (qlen + 2 <= NT*256).  FAST: every code
 * is plain and the scores fit a signed byte (prmt table lookup); otherwise
 * nibble compares. */
template <int NT, bool FAST>
__device__ void ksw_pair(const DpArgs &a, uint32_t pid, int2 *eh, const uint2 *stab, int lane, int qlen, int tlen,
                         const uint32_t *q, const uint32_t *t, int h0)
{
    const int e_del = a.sc.e, oe = a.sc.oe, o_del = a.sc.o;
    const int eK = e_del * 8;
    /* C bounds every substitution score so that min(M + s, M*C) is M + s for
     * M >= 1 and <= 0 for M = 0 (0 and a negative value act alike below:
     * every later use is max(., e>=0, f>=0) or max(. - (o+e), 0)) */
    const int C = max(max(a.sc.match, -a.sc.mismatch), 0) + 1;

    /* per-lane column codes: FAST = two 16-bit prmt selectors per register,
     * otherwise the raw packed word */
    uint32_t cw[NT][4];
    const int qregs = (qlen + 7) >> 3;
#pragma unroll
    for (int tt = 0; tt < NT; tt++) {
        const int wi = tt * 32 + lane;
        const uint32_t w = wi < qregs ? q[wi] : 0u;
        if (FAST) {
#pragma unroll
            for (int p = 0; p < 4; p++) {
                const uint32_t c0 = class_of((w >> (28 - 8 * p)) & 15u), c1 = class_of((w >> (24 - 8 * p)) & 15u);
                cw[tt][p] = sel16(c0) | (sel16(c1) << 16);
            }
        } else {
            cw[tt][0] = w;
        }
    }

    /* the reference's first row (ksw_kernel_template.h:75-79) */
    for (int s = lane; s < NT * KT; s += 32) eh[s] = make_int2(0, 0);
    __syncwarp();
    {
        const long long v1 = (uint32_t)h0 > (uint32_t)oe ? (long long)h0 - oe : 0;
        for (int j = lane; j <= qlen + 1; j += 32) {
            long long h = 0;
            if (j == 0) h = h0;
            else if (j == 1) h = v1;
            else if (j <= qlen && v1 - (long long)(j - 2) * e_del > e_del) h = v1 - (long long)(j - 1) * e_del;
            if (h) eh[kslot(j)].x = (int)h;
        }
    }
    __syncwarp();

    const int L8 = (qlen >> 3) << 3;
    int mx = h0, max_i = -1, max_j = -1, max_ie = -1, gscore = -1;
    int beg = 0, end = qlen;
    for (int i = 0; i < tlen;) {
        const int g = code(__ldg(t + (i >> 3)), i & 7);
        int h1 = 0;
        if (beg == 0) {
            h1 = (int)((uint32_t)h0 - (uint32_t)(o_del + e_del * (i + 1)));
            if (h1 < 0) h1 = 0;
        }
        int m = 0, mj = -1;
        int tf = -1, tl = -1;
        unsigned mf = 0, ml = 0;
        if (beg < end) {
            uint2 tab = make_uint2(0, 0);
            int sm = 0, sx = 0;
            if (FAST) {
                tab = stab[g];
            } else {
                sm = g == N_CODE4 ? 0 : a.sc.match;
                sx = g == N_CODE4 ? 0 : -a.sc.mismatch;
            }
            int fcarry = 0, hcarry = h1, kmax = -1, hlast = 0;
            const int tlo = beg >> 8, thi = (end - 1) >> 8;
#pragma unroll
            for (int tt = 0; tt < NT; tt++) {
                if (tt < tlo || tt > thi) continue;
                const int j0 = tt * KT + lane * 8;
                const int nv = min(max(end - j0, 0), 8);
                int2 v[8];
                int Mp[8], tv[8];
#pragma unroll
                for (int k = 0; k < 8; k++) v[k] = eh[tt * KT + k * 32 + lane];
                /* pass 1: M', t and the lane's F fold */
                int agg = 0;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    int s;
                    if (FAST) {
                        s = (int)prmt(tab.x, tab.y, (k & 1) ? (cw[tt][k >> 1] >> 16) : cw[tt][k >> 1]);
                    } else {
                        const int c = (int)((cw[tt][0] >> (28 - 4 * k)) & 15u);
                        s = c == N_CODE4 ? 0 : (c == g ? sm : sx);
                    }
                    Mp[k] = __viaddmin_s32(v[k].x, s, v[k].x * C);
                    tv[k] = __viaddmax_s32(Mp[k], -oe, 0);
                    agg = k == 0 ? tv[0] : __viaddmax_s32(agg, -e_del, tv[k]);
                }
                /* F entering each lane: max-plus scan over lanes, decay e per column */
                int x = agg;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int y = __shfl_up_sync(FULL, x, d);
                    if (lane >= d) x = max(x, y - eK * d);
                }
                const int ex = __shfl_up_sync(FULL, x, 1);
                int f = lane == 0 ? fcarry : max(ex, fcarry - eK * lane);
                fcarry = __shfl_sync(FULL, max(x, fcarry - eK * (lane + 1)), 31);
                /* pass 2: H, E, F, row maximum key */
                int H[8];
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    H[k] = __vimax3_s32(Mp[k], v[k].y, f);
                    v[k].y = __viaddmax_s32(v[k].y, -e_del, tv[k]);
                    f = __viaddmax_s32(f, -e_del, tv[k]);
                    if (k < nv) {
                        kmax = max(kmax, H[k] * (1 << KEY_BITS) + (j0 + k));
                        hlast = H[k];
                    }
                }
                int hp = __shfl_up_sync(FULL, H[7], 1);
                if (lane == 0) hp = hcarry;
                hcarry = __shfl_sync(FULL, H[7], 31);
                uint32_t nz = 0;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int hs = k == 0 ? hp : H[k - 1];
                    if (k < nv) {
                        eh[tt * KT + k * 32 + lane] = make_int2(hs, v[k].y);
                        nz |= (uint32_t)(hs | v[k].y);
                    }
                }
                const unsigned bm = __ballot_sync(FULL, nz != 0);
                if (bm) {
                    if (tf < 0) tf = tt, mf = bm;
                    tl = tt, ml = bm;
                }
            }
            kmax = __reduce_max_sync(FULL, kmax);
            m = kmax >> KEY_BITS;
            mj = kmax & ((1 << KEY_BITS) - 1);
            h1 = __shfl_sync(FULL, hlast, ((end - 1) >> 3) & 31);
        }
        if (lane == 0) eh[kslot(end)] = make_int2(h1, 0);
        __syncwarp();
        if (max(L8, end) == qlen) {
            max_ie = gscore > h1 ? max_ie : i;
            gscore = max(gscore, h1);
        }
        bool leave = false;
        if (m == 0) {
            leave = true;
        } else if (m > mx) {
            mx = m, max_i = i, max_j = mj;
        } else if (a.zdrop > 0) {
            if (i - max_i > mj - max_j) {
                if (mx - m - ((i - max_i) - (mj - max_j)) * e_del > a.zdrop) leave = true;
            } else {
                if (mx - m - ((mj - max_j) - (i - max_i)) * e_del > a.zdrop) leave = true;
            }
        }
        if (leave) {
            i = ((i >> 3) + 1) << 3;
            continue;
        }
        /* trimming (ksw_kernel_template.h:188-196) */
        int nbeg = end;
        if (tf >= 0) {
            const int base = tf * KT + (__ffs(mf) - 1) * 8;
            for (int k = 7; k >= 0; k--) {
                const int j = base + k;
                if (j < end) {
                    const int2 w = eh[kslot(j)];
                    if (w.x | w.y) nbeg = j;
                }
            }
        }
        int lastnz = nbeg - 1;
        if (h1 != 0) {
            lastnz = end;
        } else if (tl >= 0) {
            const int base = tl * KT + (31 - __clz(ml)) * 8;
            for (int k = 0; k < 8; k++) {
                const int j = base + k;
                if (j < end) {
                    const int2 w = eh[kslot(j)];
                    if (w.x | w.y) lastnz = j;
                }
            }
        }
        beg = nbeg;
        end = lastnz + 2 < qlen ? lastnz + 2 : qlen;
        __syncwarp(); /* the scans above read slots their owners rewrite next row */
        i++;
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
    }
    __syncwarp();
}

template <int NT>
__global__ void __launch_bounds__(128) ksw_wc_kernel(DpArgs a, const uint32_t *list, int nlist, uint32_t *fb,
                                                     uint32_t *fbn, uint32_t *wq)
{
    extern __shared__ int2 ksw_smem[];
    __shared__ uint2 stab[16];
    build_score_table(stab, a.sc, true);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int2 *eh = ksw_smem + (size_t)warp * NT * KT;
    const bool fast_scores = a.sc.match >= -128 && a.sc.match <= 127 && a.sc.mismatch >= -127 && a.sc.mismatch <= 128;
    const long long mpos = a.sc.match > 0 ? a.sc.match : 0;
    for (;;) {
        uint32_t idx = 0;
        if (lane == 0) idx = atomicAdd(wq, 1u);
        idx = __shfl_sync(FULL, idx, 0);
        if (idx >= (uint32_t)nlist) break;
        const uint32_t pid = list ? list[idx] : idx;
        const int qlen = (int)a.q_len[pid], tlen = (int)a.t_len[pid];
        const uint32_t h0u = a.seed ? a.seed[pid] : 0u;
        if (qlen + 2 > NT * KT || (long long)h0u + mpos * qlen >= KEY_H_LIMIT) {
            if (lane == 0) fb[atomicAdd(fbn, 1u)] = pid;
            continue;
        }
        const uint32_t *q = a.pq + (a.q_off[pid] >> 3), *t = a.pt + (a.t_off[pid] >> 3);
        bool plain = fast_scores;
        if (plain) {
            const int qregs = (qlen + 7) >> 3, tregs = (tlen + 7) >> 3;
            uint32_t bad = 0;
            for (int w = lane; w < qregs + tregs; w += 32) {
                const uint32_t x = w < qregs ? q[w] : t[w - qregs];
#pragma unroll
                for (int k = 0; k < 8; k++) bad |= ~(PLAIN_CODES >> ((x >> (4 * k)) & 15u)) & 1u;
            }
            plain = __all_sync(FULL, bad == 0);
        }
        if (plain) ksw_pair<NT, true>(a, pid, eh, stab, lane, qlen, tlen, q, t, (int)h0u);
        else ksw_pair<NT, false>(a, pid, eh, stab, lane, qlen, tlen, q, t, (int)h0u);
    }
}

template <int NT>
cudaError_t launch_nt(const DpArgs &a, const uint32_t *list, int nlist, uint32_t *fb, uint32_t *fbn, uint32_t *wq,
                      cudaStream_t s)
{
    const int block = 128;
    const size_t smem = (size_t)(block / 32) * NT * KT * sizeof(int2);
    auto k = ksw_wc_kernel<NT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int blocks = (nlist + 3) / 4;
    if (blocks > per_sm * sms) blocks = per_sm * sms;
    if (blocks < 1) blocks = 1;
    k<<<blocks, block, smem, s>>>(a, list, nlist, fb, fbn, wq);
    return cudaGetLastError();
}

} // namespace

bool ksw_wc_scores_ok(const Scores &sc)
{
    return sc.e >= 0 && sc.oe >= 0 && sc.match < 4095 && sc.match > -4095 && sc.mismatch < 4095 &&
           sc.mismatch > -4095;
}

int ksw_wc_tiles(int max_qlen)
{
    for (int nt = 1; nt <= 8; nt <<= 1)
        if (max_qlen + 2 <= nt * KT) return nt;
    return 0;
}

cudaError_t launch_ksw_wc(const DpArgs &a, const uint32_t *list, int nlist, int tiles, uint32_t *fb, uint32_t *fbn,
                          uint32_t *wq, cudaStream_t s)
{
    if (nlist <= 0) return cudaSuccess;
    switch (tiles) {
    case 1: return launch_nt<1>(a, list, nlist, fb, fbn, wq, s);
    case 2: return launch_nt<2>(a, list, nlist, fb, fbn, wq, s);
    case 4: return launch_nt<4>(a, list, nlist, fb, fbn, wq, s);
    case 8: return launch_nt<8>(a, list, nlist, fb, fbn, wq, s);
    default: return cudaErrorInvalidValue;
    }
}

} // namespace gb
