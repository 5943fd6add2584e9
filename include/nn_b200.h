/*
 * nn_b200.h -- C ABI of the warm-start network's training and inference
 * kernels (diffswe2d_b200/_lib/libswe_b200.so).
 *
 * No counterpart in the reference: the network (a 1D-conv encoder plus an
 * MLP that maps gauge waveforms to inflow spline controls) is the learned
 * warm start of the boundary inversion, whose plain form is the reference's
 * Examples/inverse/Monai_Valley/Monai_Velley_BC_inversion_spline_lr002/
 * bc_inversion_train.py:648-768.
 *
 * Conventions as in swe_b200.h: device pointers, caller-owned buffers, work
 * on `stream`, SWE_OK or SWE_E* returned.  bf16 buffers are passed as
 * uint16_t (IEEE bfloat16 bit patterns).
 */
#ifndef NN_B200_H
#define NN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NN_ACT_NONE 0
#define NN_ACT_GELU 1 /* x * Phi(x), Phi the standard normal CDF (erf form) */

/*
 * C = act(A B^T + bias) on the tcgen05 tensor cores: A [M, K] and B [N, K]
 * bf16, row-major with leading dimensions lda, ldb (elements; multiples of
 * 8, 16-byte aligned rows), K a multiple of 16; fp32 accumulation in tensor
 * memory.  Outputs (each optional, leading dimension ldc): out_f32 = the
 * activation (fp32), out_bf16 = the same rounded to bf16, pre_f32 = the
 * pre-activation (A B^T + bias).  bias [N] fp32 or NULL.
 * ksplit > 1 splits K over that many CTAs (for small M, N and long K); the
 * partial sums go to `workspace` (ksplit * M * N floats) and a second kernel
 * adds them in a fixed order and applies the epilogue.
 * Every wait of a CTA for its tensor-core work inside the K loop gives up
 * after wait_ns nanoseconds (>= 0; the time is checked before each probe,
 * so 0 gives up at once; NN_GEMM_WAIT_NS is the normal limit); the CTA then
 * stops, waits up to 2 s for the MMAs it issued, frees its tensor memory and
 * returns without writing its tile.  err (one word, may be NULL) receives
 * bit 1 when a wait gave up and bit 2 when the MMAs had still not completed
 * when the tensor memory was freed (the context is then suspect).
 */
#define NN_GEMM_WAIT_NS 1000000000LL
int nn_gemm_bf16(const uint16_t* A, int lda, const uint16_t* B, int ldb, int M, int N, int K,
                 const float* bias, int act, float* out_f32, uint16_t* out_bf16, float* pre_f32,
                 int ldc, int ksplit, float* workspace, long long wait_ns, uint32_t* err,
                 void* stream);

/*
 * Conv1d as a matrix: cols[(n*Lout + l), kk*Cin + ci] = scale * X[n, l*stride - pad + kk, ci]
 * + shift (0 outside [0, Lin)), bf16, columns kk*Cin + ci < k*Cin, zero up
 * to ldcols.  X is NLC: fp32 if x_f32, else bf16 (x_bf16); x_stride_l and
 * x_stride_c give its layout ([N, L, C]: C, 1; [N, C, L]: 1, L).
 */
int nn_im2col(const float* x_f32, const uint16_t* x_bf16, int Nb, int Lin, int Cin, int x_stride_n,
              int x_stride_l, int x_stride_c, int k, int stride, int pad, int Lout, float scale,
              float shift, uint16_t* cols, int ldcols, void* stream);

/*
 * Adjoint of nn_im2col (scale 1, no shift): dX[n, l, ci] (NLC fp32, overwritten) = sum
 * over (lo, kk) with lo*stride - pad + kk = l of dcols[(n*Lout + lo), kk*Cin + ci].
 * Gather form, deterministic.
 */
int nn_col2im(const float* dcols, int lddcols, int Nb, int Lin, int Cin, int k, int stride,
              int pad, int Lout, float* dX, void* stream);

/*
 * Activation adjoint and operand preparation of a layer's backward pass:
 * d = dact * act'(pre) (act NONE: d = dact), written as bf16 [M, ldd] (d_bf16)
 * and transposed bf16 [N, ldt] (dT_bf16, columns >= M zero up to ldt);
 * either output may be NULL.
 */
int nn_act_backward(const float* dact, const float* pre, int M, int N, int ld_in, int act,
                    uint16_t* d_bf16, int ldd, uint16_t* dT_bf16, int ldt, float* d_f32,
                    void* stream);

/* Column sums: out[n] = sum over m < M of x[m*ld + n] (fixed order). */
int nn_colsum(const float* x, int M, int N, int ld, float* out, void* stream);

/* bf16 transpose: out[c*ldo + r] = in[r*ldi + c] for r < R, c < C; columns
 * R..ldo-1 of out are zeroed. */
int nn_transpose_bf16(const uint16_t* in, int R, int C, int ldi, uint16_t* out, int ldo,
                      void* stream);

/* fp32 [R, C] (ld ldi) -> bf16 [R, ldo] (columns >= C zeroed) and, if
 * outT != NULL, its transpose bf16 [C, ldt] (columns >= R zeroed). */
int nn_cast_bf16(const float* in, int R, int C, int ldi, uint16_t* out, int ldo, uint16_t* outT,
                 int ldt, void* stream);

/*
 * Mean squared error over an [M, N] prediction: loss[0] = mean((pred - target)^2)
 * (fixed-order sum), grad = 2 (pred - target) / (M N).  One block.
 */
int nn_mse(const float* pred, const float* target, int M, int N, float* loss, float* grad,
           void* stream);

/*
 * Adam (Kingma and Ba, 2015) over a flat fp32 parameter vector:
 * m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2;
 * p -= lr * (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps).
 */
int nn_adam(float* params, const float* grads, float* m, float* v, long long count, float lr,
            float beta1, float beta2, float eps, int step, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NN_B200_H */
