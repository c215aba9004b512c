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

/* Complement of every A/C/G/T nibble (codes 1, 3, 7, 4: A<->T, C<->G), other
 * codes unchanged, without branches: per code an exact zero-nibble test of
 * x ^ code marks its nibbles, and the swap is one XOR per class (A and T differ
 * by 0x5, C and G by 0x4). */
__device__ __forceinline__ uint32_t nib_eq(uint32_t x, uint32_t rep)
{
    uint32_t t = x ^ rep;
    t |= t >> 1;
    t |= t >> 2;
    return (~t & 0x11111111u) * 0xFu; /* 0xF in every nibble equal to the code */
}

__device__ __forceinline__ uint32_t complement_flat(uint32_t x)
{
    const uint32_t at = nib_eq(x, 0x11111111u) | nib_eq(x, 0x44444444u);
    const uint32_t cg = nib_eq(x, 0x33333333u) | nib_eq(x, 0x77777777u);
    return x ^ (at & 0x55555555u) ^ (cg & 0x44444444u);
}

/* Reference-identical reversal, flat over the batch.  A warp takes 32
 * sequences (queries, then targets, in groups of 32), prefix-sums their word
 * tasks across lanes -- ceil(regs/2) word pairs when reversing, regs words when
 * only complementing, none otherwise -- cut into chunks of RC_CHUNK
 * consecutive tasks of one sequence, and sweeps the concatenated chunk list 32
 * chunks at a time: a lane finds its chunk's sequence with one 5-step search
 * over the lanes' inclusive counts, then issues the chunk's loads together
 * (RC_CHUNK independent loads in flight per lane) before its stores.  Task i
 * of a reversed sequence reads word i, writes its nibble-reversed (and, for
 * op 3, complemented) value to word regs-1-i and zeroes word i (the sm_100a
 * build's result); no other task touches those words, so the update in place
 * is race-free. */
constexpr uint32_t RC_CHUNK = 4;

__global__ void __launch_bounds__(256) revcomp_flat_kernel(uint32_t *pq, uint32_t *pt, const uint32_t *q_off,
                                                           const uint32_t *t_off, const uint32_t *q_len,
                                                           const uint32_t *t_len, const uint8_t *q_op,
                                                           const uint8_t *t_op, int32_t n)
{
    const int lane = threadIdx.x & 31;
    const int groups_q = q_op ? (n + 31) >> 5 : 0;
    const int groups = groups_q + (t_op ? (n + 31) >> 5 : 0);
    const int warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    /* the op, offset and length of a group's 32 sequences: independent loads,
     * issued together, and for the warp's next group before this one's words */
    auto meta = [&](int g, uint32_t &o8, uint32_t &off, uint32_t &len) {
        o8 = 0, off = 0, len = 0;
        if (g >= groups) return;
        const bool ts = g >= groups_q;
        const int p = ((ts ? g - groups_q : g) << 5) + lane;
        if (p < n) {
            o8 = __ldg((ts ? t_op : q_op) + p);
            off = __ldg((ts ? t_off : q_off) + p);
            len = __ldg((ts ? t_len : q_len) + p);
        }
    };
    uint32_t n_o8, n_off, n_len;
    meta(warp0, n_o8, n_off, n_len);
    for (int g = warp0; g < groups; g += nwarps) {
        const bool tside = g >= groups_q;
        uint32_t *words = tside ? pt : pq;
        const int op = (int)(n_o8 & 3u);
        const uint32_t base = op ? n_off >> 3 : 0u, regs = op ? (n_len + 7) >> 3 : 0u;
        meta(g + nwarps, n_o8, n_off, n_len);
        const uint32_t tasks = (op & 1) ? (regs + 1) >> 1 : (op == 2 ? regs : 0u);
        const uint32_t chunks = (tasks + RC_CHUNK - 1) / RC_CHUNK;
        uint32_t incl = chunks;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (lane >= d) incl += y;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        for (uint32_t k0 = 0; k0 < total; k0 += 32) {
            const uint32_t k = k0 + lane;
            /* owner: the first lane whose inclusive count exceeds k */
            int owner = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const uint32_t c = __shfl_sync(0xFFFFFFFFu, incl, owner + step - 1);
                if (c <= k) owner += step;
            }
            const uint32_t o_incl = __shfl_sync(0xFFFFFFFFu, incl, owner & 31);
            const uint32_t o_chunks = __shfl_sync(0xFFFFFFFFu, chunks, owner & 31);
            const uint32_t o_tasks = __shfl_sync(0xFFFFFFFFu, tasks, owner & 31);
            const uint32_t o_base = __shfl_sync(0xFFFFFFFFu, base, owner & 31);
            const uint32_t o_regs = __shfl_sync(0xFFFFFFFFu, regs, owner & 31);
            const int o_op = __shfl_sync(0xFFFFFFFFu, op, owner & 31);
            if (k >= total) continue;
            const uint32_t i0 = (k - (o_incl - o_chunks)) * RC_CHUNK;
            const uint32_t nt = min(RC_CHUNK, o_tasks - i0);
            uint32_t *w = words + o_base;
            uint32_t v[RC_CHUNK];
#pragma unroll
            for (uint32_t u = 0; u < RC_CHUNK; u++) v[u] = u < nt ? w[i0 + u] : 0u;
            if (o_op & 1) {
#pragma unroll
                for (uint32_t u = 0; u < RC_CHUNK; u++) {
                    if (u < nt) {
                        const uint32_t i = i0 + u, mirror = o_regs - 1 - i;
                        uint32_t rev = nib_reverse(v[u]);
                        if (o_op & 2) rev = complement_flat(rev);
                        if (i != mirror) w[i] = 0u;
                        w[mirror] = rev;
                    }
                }
            } else {
#pragma unroll
                for (uint32_t u = 0; u < RC_CHUNK; u++)
                    if (u < nt) w[i0 + u] = complement_flat(v[u]);
            }
        }
    }
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
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int groups = ((q_op ? (n + 31) / 32 : 0) + (t_op ? (n + 31) / 32 : 0));
        if (groups == 0) return cudaSuccess;
        int blocks = (groups + 7) / 8; /* 8 warps per block */
        if (blocks > sms * 8) blocks = sms * 8;
        revcomp_flat_kernel<<<blocks, 256, 0, s>>>(pq, pt, q_off, t_off, q_len, t_len, q_op, t_op, n);
    } else {
        revcomp_kernel<<<(n + 127) / 128, 128, 0, s>>>(pq, pt, q_off, t_off, q_len, t_len, q_op, t_op, n, 0);
    }
    return cudaGetLastError();
}

} // namespace gb
