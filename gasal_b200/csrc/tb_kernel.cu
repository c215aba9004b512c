/*
 * tb_kernel.cu -- traceback of the direction tiles into GASAL2's CIGAR bytes.
 *
 * Replaces reference src/kernels/get_tb.h:4-149.  One thread per pair walks
 * its tiles backwards.  Output format: one byte per run, (count << 2) | op
 * with op 0 match, 1 mismatch, 2 deletion (consumes target), 3 insertion
 * (consumes query), count <= 63, written last operation first at the pair's
 * query offset of the device query batch; the run count replaces nothing else
 * (n_cigar is written to its own array).  LOCAL starts at the end cell and
 * stops once the operations re-score to the alignment score, reporting the
 * start; GLOBAL starts at (target length, query length) -- one past the last
 * cell, as the reference does -- and flushes leftover target / query bases as
 * 63-long runs.  The state machine (normal mode reads the 2 direction bits,
 * gap mode reads the extend bit of the gap's kind) is the reference's.
 * Target-tail SEMI_GLOBAL (an extension) has its own walk, semi_walk.
 */
#include "gb_internal.h"

namespace gb {

/* Run-length CIGAR writer: runs of one operation up to 63 long, last
 * operation first, bytes past `room` counted but not written. */
struct CigarOut {
    uint8_t *out;
    uint32_t room, n = 0, op = 0;
    int count = 0;
    __device__ __forceinline__ void put(uint32_t o)
    {
        if (count > 0 && count < 63 && o == op) {
            count++;
            return;
        }
        flush();
        op = o, count = 1;
    }
    __device__ __forceinline__ void flush()
    {
        if (count > 0) {
            if (n < room) out[n] = (uint8_t)(op | ((uint32_t)count << 2));
            n++;
        }
        count = 0;
    }
};

/* SEMI_GLOBAL traceback, an extension (the reference instantiates semi-global
 * WITH_TB empty, semiglobal_kernel_template.h:227), for a free target tail:
 * from the end cell (t_end, qlen - 1), an affine state machine over the
 * nibbles of semi_nib -- in H the two low bits give the move (diagonal, or
 * enter E / F at the same cell), in E (deletion) and F (insertion) the
 * cell's own extend bit says whether the gap continues or was opened from H
 * of the cell it came from.  At a free leading edge (target for head TARGET
 * or BOTH, query for QUERY or BOTH) the walk stops; at a closed one the
 * remaining bases become one gap.  Starts: the first aligned target row and
 * query column. */
__device__ uint32_t semi_walk(const uint4 *tb, int q8, int i, int j, int head, uint8_t *out, uint32_t room,
                              int *si, int *sj)
{
    CigarOut c{out, room};
    int state = 0; /* 0 H, 2 E (deletion), 3 F (insertion) */
    while (i >= 0 && j >= 0) {
        const int cell = (((i >> 3) * q8) << 3) + (j << 3) + (i & 7);
        const uint4 tile = tb[cell >> 5];
        const int in_tile = cell & 31, reg = in_tile >> 3;
        const uint32_t word = reg == 0 ? tile.x : (reg == 1 ? tile.y : (reg == 2 ? tile.z : tile.w));
        const uint32_t nib = (word >> (28 - ((in_tile & 7) << 2))) & 15u;
        if (state == 0) {
            const uint32_t src = nib & 3u;
            if (src <= 1) {
                c.put(src);
                i--, j--;
                continue;
            }
            state = (int)src;
        }
        if (state == 2) {
            c.put(2);
            state = (nib & 4u) ? 2 : 0;
            i--;
        } else {
            c.put(3);
            state = (nib & 8u) ? 3 : 0;
            j--;
        }
    }
    const bool free_t = head == TARGET_ || head == BOTH_, free_q = head == QUERY_ || head == BOTH_;
    int ts = i + 1, qs = j + 1;
    if (j < 0 && i >= 0 && !free_t) {
        for (; i >= 0; i--) c.put(2);
        ts = 0;
    }
    if (i < 0 && j >= 0 && !free_q) {
        for (; j >= 0; j--) c.put(3);
        qs = 0;
    }
    c.flush();
    *si = ts, *sj = qs;
    return c.n;
}

__global__ void __launch_bounds__(128) traceback_kernel(TbArgs a)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const int qlen = (int)a.q_len[p], tlen = (int)a.t_len[p];
    uint32_t n_ops = 0;
    if (a.algo == SEMI_GLOBAL_) {
        int si = 0, sj = 0;
        if (qlen > 0 && tlen > 0) {
            const uint32_t room = a.q_off[p] < a.cigar_bytes ? a.cigar_bytes - a.q_off[p] : 0u;
            n_ops = semi_walk(a.tb + a.tb_off[p], ((qlen + 7) >> 3) << 3, a.t_end[p], qlen - 1, a.head,
                              a.cigar + a.q_off[p], room, &si, &sj);
        }
        if (a.t_start) a.t_start[p] = si;
        if (a.q_start) a.q_start[p] = sj;
        if (a.n_cigar) a.n_cigar[p] = n_ops;
        return;
    }
    if (qlen > 0 && tlen > 0) {
        const uint4 *tb = a.tb + a.tb_off[p];
        const int q8 = ((qlen + 7) >> 3) << 3;
        int i, j, total = 0;
        if (a.algo == LOCAL_) {
            i = a.t_end[p], j = a.q_end[p], total = a.score[p];
        } else {
            i = tlen, j = qlen;
        }
        uint8_t *out = a.cigar + a.q_off[p];
        const uint32_t room = a.q_off[p] < a.cigar_bytes ? a.cigar_bytes - a.q_off[p] : 0u;
        uint32_t prev_op = 0, op_fill;
        int prev_tile = -1, op_select = 3, op_shift = 0, count = 0, curr = 0;
        uint4 tile = make_uint4(0, 0, 0, 0);
        while (i >= 0 && j >= 0) {
            const int cell = (((i >> 3) * q8) << 3) + (j << 3) + (i & 7);
            const int tile_no = cell >> 5;
            if (tile_no != prev_tile) tile = tb[tile_no];
            prev_tile = tile_no;
            const int in_tile = cell & 31;
            const int reg = in_tile >> 3;
            const uint32_t word = reg == 0 ? tile.x : (reg == 1 ? tile.y : (reg == 2 ? tile.z : tile.w));
            const uint32_t nib = (word >> (28 - ((in_tile & 7) << 2))) & 15u;
            const uint32_t op = (nib >> op_shift) & (uint32_t)op_select;
            op_fill = (op == 0 || op_select == 3) ? op : (uint32_t)op_shift;
            op_select = (op == 0 || (op == 1 && op_select == 3)) ? 3 : 1;
            op_shift = (op == 0 || (op == 1 && op_select == 3)) ? 0 : ((op == 2 || op == 3) ? (int)op : op_shift);
            if (count < 63 && op_fill == prev_op) {
                count++;
            } else {
                if (count > 0) {
                    if (n_ops < room) out[n_ops] = (uint8_t)(prev_op | ((uint32_t)count << 2));
                    n_ops++;
                }
                count = 1;
            }
            if (a.algo == LOCAL_) {
                const bool gap = (op_fill == 2 || op_fill == 3);
                curr += (gap && prev_op != op_fill) ? -a.sc.oe
                                                    : (gap ? -a.sc.e : (op_fill == 1 ? -a.sc.mismatch : a.sc.match));
                if (curr == total) break;
            }
            prev_op = op_fill;
            if (op_fill == 0 || op_fill == 1 || op_fill == 2) i--;
            if (op_fill == 0 || op_fill == 1 || op_fill == 3) j--;
        }
        if (n_ops < room) out[n_ops] = (uint8_t)(prev_op | ((uint32_t)count << 2));
        n_ops++;
        if (a.algo == GLOBAL_) {
            for (; i >= 0; i -= 63, n_ops++)
                if (n_ops < room) out[n_ops] = (uint8_t)(2u | ((uint32_t)min(i + 1, 63) << 2));
            for (; j >= 0; j -= 63, n_ops++)
                if (n_ops < room) out[n_ops] = (uint8_t)(3u | ((uint32_t)min(j + 1, 63) << 2));
        }
        if (a.algo == LOCAL_) {
            if (a.t_start) a.t_start[p] = i;
            if (a.q_start) a.q_start[p] = j;
        }
    } else if (a.algo == LOCAL_) {
        /* an empty query or target: no operations and start 0, like every
         * other result of such a pair (nothing else writes the starts) */
        if (a.t_start) a.t_start[p] = 0;
        if (a.q_start) a.q_start[p] = 0;
    }
    if (a.n_cigar) a.n_cigar[p] = n_ops;
}

cudaError_t launch_traceback(const TbArgs &a, cudaStream_t s)
{
    if (a.n <= 0) return cudaSuccess;
    traceback_kernel<<<(a.n + 127) / 128, 128, 0, s>>>(a);
    return cudaGetLastError();
}

} // namespace gb
