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
 */
#include "gb_internal.h"

namespace gb {

__global__ void __launch_bounds__(128) traceback_kernel(TbArgs a)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const int qlen = (int)a.q_len[p], tlen = (int)a.t_len[p];
    uint32_t n_ops = 0;
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
