// krylov.cuh -- FP64 vector kernels of the outer flexible GMRES and the set-up dense inverse.
#pragma once
#include <algorithm>

#include "mgm_internal.cuh"

namespace mgm {

constexpr int kMaxKrylov = 128;

void resid64(int n, int k, const int *idx, const double *A, const double *b, const double *x, double *r, double *part,
             cudaStream_t s);
template <class T>
void apply64(int n, int k, const int *idx, const double *A, const T *z, double *w, cudaStream_t s);
int dot_blocks(int n);
void multidot(int n, int cnt, const double *V, long ldv, const double *w, double *part, double *out, cudaStream_t s);
void reduce_parts(const double *part, int nblk, int cnt, double *out, cudaStream_t s);
void orth_update(int n, int cnt, const double *V, long ldv, const double *h, double *w, cudaStream_t s);
// w -= sum_c h[c] V_c and *norm2 = |w|^2 of the result (device scalar)
void orth_norm(int n, int cnt, const double *V, long ldv, const double *h, double *w, double *part, double *norm2,
               cudaStream_t s);
void scale_by(int n, const double *in, double *out, const double *nrm, int is_sq, cudaStream_t s);
template <class T>
void combine(int n, int cnt, const T *Z, long ldz, const double *y, double *x, cudaStream_t s);
template <class T>
void copy_convert(long n, const double *in, T *out, cudaStream_t s);
template <class T>
void copy_out(long n, const T *in, T *out, cudaStream_t s);
void dense_inverse(int n, int k, const int *idx, const double *A, double *inv64, float *inv32, cudaStream_t s);

}  // namespace mgm
