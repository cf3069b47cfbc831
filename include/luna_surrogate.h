/*
 * libluna_surrogate — training and inference kernels of the learned surrogate of the
 * capillary scan (sm_100a). No counterpart in the reference: the surrogate maps the scan
 * parameters and z to the log spectrum and temporal envelope that the batched solver
 * (libluna_b200) produces, and the solver is its fallback and its judge.
 *
 * Every pointer is device memory; BF16 arrays hold __nv_bfloat16 (passed as void*).
 * Arrays of an ensemble are stacked along a leading member index with the stated member
 * strides; `members` ensemble members are processed by one launch. Batch sizes and layer
 * widths must be multiples of 128 and the reduction dimension a multiple of 64
 * (LUNA_ERR_BAD_ARG, 16, otherwise). `err` (device int) is set nonzero when a bounded
 * tensor-core wait gave up (the result is then invalid). Calls are enqueued on `stream`
 * (a cudaStream_t, may be NULL) and return 0 or 18 (a CUDA launch error).
 */
#ifndef LUNA_SURROGATE_H
#define LUNA_SURROGATE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Linear layer forward: Z = X W^T + b, Y = act(Z) (act 1: SiLU, 0: identity). X [B x K]
 * BF16 (member stride sX, 0 to share one input), W [N x K] BF16 (stride N*K), b [N] FP32
 * (stride N); outputs [B x N] (stride B*N): Y BF16, Zout BF16, Yf FP32, each may be NULL. */
int luna_sg_linear_fwd(const void* X, long long sX, const void* W, const float* b, int B, int K, int N, int act,
                       void* Y, void* Zout, float* Yf, int members, int* err, void* stream);
/* Backward through the layer's input: dXpre = (dZ W) * silu'(Zprev), [B x K] BF16. */
int luna_sg_linear_bwd_data(const void* dZ, const void* W, const void* Zprev, int B, int K, int N, void* dXpre,
                            int members, int* err, void* stream);
/* Weight and bias gradients: dW = dZ^T X [N x K] FP32, db = sum over the batch of dZ [N]. */
int luna_sg_linear_bwd_weight(const void* dZ, const void* X, long long sX, int B, int K, int N, float* dW, float* db,
                              int members, int* err, void* stream);
/* Fourier-feature input: x [B x 8] FP32 -> out [B x (8 + 2 nf)] BF16 = (x, sin 2πFx, cos 2πFx). */
int luna_sg_features(const float* x, int B, const float* f, int nf, void* out, int ld, void* stream);
/* Mean squared error of Y [members x B x N] against T (member stride sT): dY BF16 and
 * loss[member] += MSE (FP64). */
int luna_sg_mse(const float* Y, const float* T, long long sT, int B, int N, void* dY, double* loss, int members,
                void* stream);
/* One Adam step t >= 1 on n FP32 parameters with gradient g; wbf (may be NULL) receives BF16. */
int luna_sg_adam(float* p, float* m, float* v, const float* g, long long n, float lr, float b1, float b2, float eps,
                 int t, void* wbf, void* stream);
/* Ensemble mean [B x N] and per-point spread (largest standard deviation over the members
 * among the first nspec outputs) of Y [members x B x N]. */
int luna_sg_ensemble(const float* Y, int members, int B, int N, int nspec, float* mean, float* spread, void* stream);

#ifdef __cplusplus
}
#endif
#endif
