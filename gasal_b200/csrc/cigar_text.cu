/*
 * cigar_text.cu -- forward CIGAR strings on the device.
 *
 * The traceback leaves each pair's CIGAR as run-length bytes (count << 2 |
 * op, last operation first) at the pair's query offset, as the reference
 * does (src/kernels/get_tb.h); turning them into text is left to the caller
 * there (test_prog/test_prog.cpp:382-428 reads the bytes from last to first,
 * merges neighbouring runs of one operation and prints count and M/X/D/I).
 * This kernel does that decode for the whole batch on the GPU, one thread
 * per pair, into fixed-stride slots, so results can leave the device as
 * text.  No counterpart in the reference library.
 */
#include "gb_internal.h"

namespace gb {

namespace {

__global__ void __launch_bounds__(128) cigar_text_kernel(const uint8_t *cigar, const uint32_t *q_off,
                                                         const uint32_t *n_cigar, int n, char *text, int stride,
                                                         int32_t *text_len)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    char *out = text + (size_t)i * stride;
    const uint8_t *c = cigar + q_off[i];
    int u = (int)n_cigar[i] - 1;
    int len = 0;
    bool ok = true;
    while (u >= 0) {
        const uint32_t op = c[u] & 3u;
        uint32_t count = 0;
        while (u >= 0 && (c[u] & 3u) == op) count += c[u--] >> 2;
        /* digits of count, most significant first */
        uint32_t p10 = 1;
        int nd = 1;
        while (count / p10 >= 10u) p10 *= 10u, nd++;
        if (len + nd + 1 > stride - 1) {
            ok = false;
            break;
        }
        for (; p10 > 0; p10 /= 10u) out[len++] = (char)('0' + (count / p10) % 10u);
        out[len++] = "MXDI"[op];
    }
    if (stride > 0) out[ok ? len : 0] = 0;
    text_len[i] = ok ? len : -1;
}

} // namespace

cudaError_t launch_cigar_text(const uint8_t *cigar, const uint32_t *q_off, const uint32_t *n_cigar, int n,
                              char *text, int stride, int32_t *text_len, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    cigar_text_kernel<<<(n + 127) / 128, 128, 0, s>>>(cigar, q_off, n_cigar, n, text, stride, text_len);
    return cudaGetLastError();
}

} // namespace gb
