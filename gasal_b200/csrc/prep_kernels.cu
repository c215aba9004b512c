/*
 * prep_kernels.cu -- sequence packing and reverse/complement on sm_100a.
 *
 * Pack (replaces reference src/kernels/pack_rc_seqs.h:13-53): ASCII bases ->
 * 4-bit codes, 8 per 32-bit word, first base in bits 31..28, code = low nibble
 * of the byte.  HBM-bound (1 B read + 0.5 B written per base): each thread
 * moves 32 input bytes with two 128-bit loads and one 128-bit store, in a
 * grid-stride loop sized to the SM count, so every warp access is a fully
 * coalesced 512 B / 256 B transaction.  Two byte permutes gather the even and
 * odd bases of 8 bytes, one shift and one 3-input logic op merge them.
 *
 * Reverse / complement (replaces src/kernels/pack_rc_seqs.h:56-212): per
 * sequence, op bit 0 reverses and bit 1 complements (A<->T, C<->G; other
 * codes unchanged).  The reference's reversal shifts 32-bit words by 32; the
 * sm_100a build of it zeroes the first floor(regs/2) words and writes the
 * nibble-reversed word i to word regs-1-i for i < ceil(regs/2).  That is the
 * default here (ref_reverse = 1) so results stay identical to the reference;
 * ref_reverse = 0 reverses the real bases and keeps the N pad at the end.
 */
#include "gb_internal.h"

namespace gb {

__device__ __forceinline__ uint32_t pack8(uint32_t lo, uint32_t hi)
{
    /* lo = bytes b0..b3, hi = b4..b7 (little endian) */
    const uint32_t ev = __byte_perm(lo, hi, 0x0246); /* b0 b2 b4 b6 into bytes 3..0 */
    const uint32_t od = __byte_perm(lo, hi, 0x1357); /* b1 b3 b5 b7 */
    /* even base -> high nibble, odd base -> low nibble of each byte */
    return ((ev << 4) & 0xF0F0F0F0u) | (od & 0x0F0F0F0Fu);
}

__global__ void __launch_bounds__(256) pack_kernel(const uint8_t *__restrict__ ascii, uint32_t nbytes,
                                                   uint32_t *__restrict__ words)
{
    const uint32_t n32 = nbytes >> 5; /* 32-byte chunks */
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint4 *in = reinterpret_cast<const uint4 *>(ascii);
    uint4 *out = reinterpret_cast<uint4 *>(words);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n32; i += stride) {
        const uint4 a = __ldcs(in + 2 * i);
        const uint4 b = __ldcs(in + 2 * i + 1);
        uint4 w;
        w.x = pack8(a.x, a.y);
        w.y = pack8(a.z, a.w);
        w.z = pack8(b.x, b.y);
        w.w = pack8(b.z, b.w);
        out[i] = w;
    }
    /* tail: up to three 8-byte groups */
    const uint32_t done = n32 << 2, total = nbytes >> 3;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < total - done) {
        const uint2 v = reinterpret_cast<const uint2 *>(ascii)[done + t];
        words[done + t] = pack8(v.x, v.y);
    }
}

cudaError_t launch_pack(const uint8_t *ascii, uint32_t nbytes, uint32_t *words, cudaStream_t s)
{
    if (nbytes == 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t chunks = (nbytes >> 5) + 1;
    uint32_t blocks = (chunks + 255) / 256;
    const uint32_t cap = (uint32_t)sms * 8;
    if (blocks > cap) blocks = cap;
    pack_kernel<<<blocks, 256, 0, s>>>(ascii, nbytes, words);
    return cudaGetLastError();
}

__device__ __forceinline__ uint32_t nib_reverse(uint32_t x)
{
    const uint32_t r = __byte_perm(x, 0, 0x0123);
    return ((r >> 4) & 0x0F0F0F0Fu) | ((r << 4) & 0xF0F0F0F0u);
}

__device__ __forceinline__ uint32_t complement_word(uint32_t x)
{
    /* per nibble: 1<->4, 3<->7, everything else unchanged.  Nibble-wise masks:
     * lo bit patterns 0001 (A) 0100 (T) 0011 (C) 0111 (G). */
    uint32_t r = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        uint32_t c = (x >> (4 * k)) & 15u;
        c = (c == 1u) ? 4u : (c == 4u) ? 1u : (c == 3u) ? 7u : (c == 7u) ? 3u : c;
        r |= c << (4 * k);
    }
    return r;
}

__device__ void revcomp_one(uint32_t *w, uint32_t len, int op, int ref_reverse)
{
    const uint32_t regs = (len + 7) >> 3;
    if (op & 1) {
        if (ref_reverse) {
            const uint32_t half = (regs + 1) >> 1;
            for (uint32_t i = 0; i < half; i++) {
                const uint32_t head = w[i];
                w[i] = 0u;
                w[regs - 1 - i] = nib_reverse(head);
            }
        } else {
            /* reverse the real bases: reverse the whole padded run (pads move
             * to the front), then shift the run left by the pad count and
             * refill the tail with N codes */
            for (uint32_t i = 0; i < regs / 2; i++) {
                const uint32_t x = w[i], y = w[regs - 1 - i];
                w[i] = nib_reverse(y);
                w[regs - 1 - i] = nib_reverse(x);
            }
            if (regs & 1) w[regs >> 1] = nib_reverse(w[regs >> 1]);
            const uint32_t pad = 8 * regs - len;
            if (pad) {
                const uint32_t sh = 4 * pad;
                for (uint32_t i = 0; i + 1 < regs; i++) w[i] = (w[i] << sh) | (w[i + 1] >> (32 - sh));
                w[regs - 1] = (w[regs - 1] << sh) | (0xEEEEEEEEu >> (32 - sh));
            }
        }
    }
    if (op & 2) {
        for (uint32_t i = 0; i < regs; i++) w[i] = complement_word(w[i]);
    }
}

/* Reference-identical reversal, word-parallel: blockDim = (32, 8), one row of
 * 32 threads per pair, thread x handling word pairs (x, regs-1-x) for
 * x < ceil(regs/2) in steps of 32.  Each word is read by at most one thread
 * (its own index, below ceil(regs/2)) and written only after that read, so
 * the in-place update is race-free; the complement of the untouched words
 * runs after a row barrier. */
__device__ __forceinline__ void revcomp_ref_row(uint32_t *w, uint32_t len, int op)
{
    const uint32_t regs = (len + 7) >> 3;
    if (op & 1) {
        const uint32_t half = (regs + 1) >> 1;
        for (uint32_t i = threadIdx.x; i < half; i += 32) {
            const uint32_t head = w[i];
            uint32_t rev = nib_reverse(head);
            if (op & 2) rev = complement_word(rev);
            if (i != regs - 1 - i) w[i] = 0u;
            w[regs - 1 - i] = rev;
        }
    } else if (op & 2) {
        for (uint32_t i = threadIdx.x; i < regs; i += 32) w[i] = complement_word(w[i]);
    }
}

__global__ void __launch_bounds__(256) revcomp_ref_kernel(uint32_t *pq, uint32_t *pt, const uint32_t *q_off,
                                                          const uint32_t *t_off, const uint32_t *q_len,
                                                          const uint32_t *t_len, const uint8_t *q_op,
                                                          const uint8_t *t_op, int32_t n)
{
    const int i = blockIdx.x * blockDim.y + threadIdx.y;
    if (i >= n) return;
    const int qo = q_op ? q_op[i] : 0, to = t_op ? t_op[i] : 0;
    if (qo & 3) revcomp_ref_row(pq + (q_off[i] >> 3), q_len[i], qo);
    if (to & 3) revcomp_ref_row(pt + (t_off[i] >> 3), t_len[i], to);
}

__global__ void revcomp_kernel(uint32_t *pq, uint32_t *pt, const uint32_t *q_off, const uint32_t *t_off,
                               const uint32_t *q_len, const uint32_t *t_len, const uint8_t *q_op,
                               const uint8_t *t_op, int32_t n, int ref_reverse)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int qo = q_op ? q_op[i] : 0, to = t_op ? t_op[i] : 0;
    if (qo & 3) revcomp_one(pq + (q_off[i] >> 3), q_len[i], qo, ref_reverse);
    if (to & 3) revcomp_one(pt + (t_off[i] >> 3), t_len[i], to, ref_reverse);
}

cudaError_t launch_revcomp(uint32_t *pq, uint32_t *pt, const uint32_t *q_off, const uint32_t *t_off,
                           const uint32_t *q_len, const uint32_t *t_len, const uint8_t *q_op,
                           const uint8_t *t_op, int32_t n, int ref_reverse, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    if (ref_reverse) {
        const dim3 blk(32, 8);
        revcomp_ref_kernel<<<(n + 7) / 8, blk, 0, s>>>(pq, pt, q_off, t_off, q_len, t_len, q_op, t_op, n);
    } else {
        revcomp_kernel<<<(n + 127) / 128, 128, 0, s>>>(pq, pt, q_off, t_off, q_len, t_len, q_op, t_op, n, 0);
    }
    return cudaGetLastError();
}

} // namespace gb
