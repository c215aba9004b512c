/*
 * mlband.h -- learned ksw band width: feature and MLP kernels (mlband.cu).
 */
#ifndef GB_MLBAND_H
#define GB_MLBAND_H

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace gb {

constexpr int BAND_FEATS = 67;      /* 3 scalars + 64-bin diagonal histogram */
constexpr int BAND_FEATS_PAD = 68;  /* floats per pair in the feature matrix */
constexpr int MLP_HIDDEN = 64;
constexpr int MLP_PARAMS = MLP_HIDDEN * BAND_FEATS + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN + MLP_HIDDEN + 1;

cudaError_t launch_band_features(const uint32_t *pq, const uint32_t *pt, const uint32_t *q_off, const uint32_t *t_off,
                                 const uint32_t *q_len, const uint32_t *t_len, int n, float *feat, cudaStream_t s);
cudaError_t launch_mlp_forward(const __nv_bfloat16 *w, const float *feat, int n, float *out, cudaStream_t s);
cudaError_t launch_mlp_grad(const float *w, const float *feat, const float *label, int n, float tau, float *grad,
                            float *loss, cudaStream_t s);
cudaError_t launch_mlp_adam(float *w, float *m, float *v, const float *g, __nv_bfloat16 *wb, float lr, int step,
                            cudaStream_t s);
cudaError_t launch_to_bf16(const float *w, __nv_bfloat16 *wb, cudaStream_t s);
cudaError_t launch_band_from_pred(const float *pred, const uint32_t *q_len, const uint32_t *t_len, int n, int bmin,
                                  int bmax, int32_t *band, cudaStream_t s);
cudaError_t launch_band_ok(uint8_t *ok, int n, const uint32_t *retry, const uint32_t *nretry, cudaStream_t s);

} // namespace gb

#endif
