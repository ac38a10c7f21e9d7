/*
 * ttcb200_mlp.h -- device kernels of the learned schedule selector (a 3-layer fp32 MLP that ranks
 * transposition schedules). No counterpart in TTC, which times every generated variant instead
 * (ttc.py:847-1022). All matrices are row-major fp32 device arrays; every call is stream-ordered and
 * returns a ttcb_status.
 */
#ifndef TTCB200_MLP_H
#define TTCB200_MLP_H

#include "ttcb200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* C[M x N] = op(A) * op(B) (+ bias[N]) (then ReLU if relu != 0), op = transpose when trans* != 0.
 * op(A) is M x K, op(B) is K x N; lda/ldb/ldc are row strides of the stored matrices. */
ttcb_status ttcb_mlp_gemm(int transA, int transB, int M, int N, int K, const float* A, int lda, const float* B,
                          int ldb, float* C, int ldc, const float* bias, int relu, ttcb_stream_t stream);

/* dZ = dY * (Y > 0), elementwise over n values (backward of ReLU, given the ReLU output Y). */
ttcb_status ttcb_mlp_relu_grad(const float* Y, const float* dY, float* dZ, int n, ttcb_stream_t stream);

/* out[N] = sum over rows of X[M x N] (the bias gradient). */
ttcb_status ttcb_mlp_colsum(const float* X, int M, int N, float* out, ttcb_stream_t stream);

/* Mean squared error: dpred = 2 (pred - target) / n, loss[0] = mean (pred - target)^2. */
ttcb_status ttcb_mlp_mse(const float* pred, const float* target, int n, float* dpred, float* loss,
                         ttcb_stream_t stream);

/* One Adam step (Kingma & Ba, 2015) on n parameters, step t >= 1. */
ttcb_status ttcb_mlp_adam(float* param, const float* grad, float* m, float* v, int n, float lr, float beta1,
                          float beta2, float eps, int t, ttcb_stream_t stream);

/* The same step with L2 weight decay: the gradient used is grad + weight_decay * param. */
ttcb_status ttcb_mlp_adam_l2(float* param, const float* grad, float* m, float* v, int n, float lr, float beta1,
                             float beta2, float eps, float weight_decay, int t, ttcb_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* TTCB200_MLP_H */
