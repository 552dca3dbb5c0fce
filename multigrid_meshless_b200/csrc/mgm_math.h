/*
 * mgm_math.h -- rounding-exact scalar helpers shared by the CUDA kernels and
 * by a host-side self-check (compiled with gcc -ffp-contract=off).
 *
 * The reference evaluates its RBF matrices with libm's pow() (rbf.h:35, 39,
 * 68-72, 108-110; mesh_functions.h:585-587), whose results are the correctly
 * rounded value of x^y in all but vanishingly rare cases.  CUDA's pow() is
 * only accurate to 2 ulp, which the ill-conditioned saddle-point solves would
 * amplify.  The functions below therefore compute the two kinds of powers the
 * reference uses -- small integer powers of a coordinate difference and
 * half-integer powers r^(phs/2) of a squared distance -- in double-double
 * arithmetic (error-free products via fused multiply-add, Dekker/Knuth style)
 * and round once at the end, which gives the correctly rounded result except
 * when x^y lies within ~2^-100 relative of a rounding midpoint.
 *
 * Every product and sum that must follow the reference's rounding sequence
 * uses MGM_MUL / MGM_ADD / MGM_SUB, which never contract into an FMA.
 */
#ifndef MGM_MATH_H
#define MGM_MATH_H

#include <math.h>

#if defined(__CUDACC__)
#define MGM_HD __host__ __device__ __forceinline__
#ifdef __CUDA_ARCH__
#define MGM_MUL(a, b) __dmul_rn((a), (b))
#define MGM_ADD(a, b) __dadd_rn((a), (b))
#define MGM_SUB(a, b) __dsub_rn((a), (b))
#define MGM_FMA(a, b, c) __fma_rn((a), (b), (c))
#define MGM_SQRT(a) __dsqrt_rn(a)
#define MGM_DIV(a, b) __ddiv_rn((a), (b))
#else
#define MGM_MUL(a, b) ((a) * (b))
#define MGM_ADD(a, b) ((a) + (b))
#define MGM_SUB(a, b) ((a) - (b))
#define MGM_FMA(a, b, c) fma((a), (b), (c))
#define MGM_SQRT(a) sqrt(a)
#define MGM_DIV(a, b) ((a) / (b))
#endif
#else
#define MGM_HD static inline
#define MGM_MUL(a, b) ((a) * (b))
#define MGM_ADD(a, b) ((a) + (b))
#define MGM_SUB(a, b) ((a) - (b))
#define MGM_FMA(a, b, c) fma((a), (b), (c))
#define MGM_SQRT(a) sqrt(a)
#define MGM_DIV(a, b) ((a) / (b))
#endif

/* (hi, lo) unevaluated sum, |lo| <= ulp(hi)/2 */
typedef struct { double hi, lo; } mgm_dd;

MGM_HD mgm_dd mgm_dd_mul_d(mgm_dd a, double b)
{
    double p = MGM_MUL(a.hi, b);
    double e = MGM_FMA(a.hi, b, -p);          /* exact error of hi*b */
    e = MGM_FMA(a.lo, b, e);                  /* + lo*b (lower order) */
    double s = MGM_ADD(p, e);                 /* fast two-sum renormalisation */
    mgm_dd r;
    r.hi = s;
    r.lo = MGM_SUB(e, MGM_SUB(s, p));
    return r;
}

/* pow(d, e) for a small non-negative integer e (the monomial powers). */
MGM_HD double mgm_pow_int(double d, int e)
{
    if (e == 0) return 1.0;
    if (e == 1) return d;
    if (e == 2) return MGM_MUL(d, d);
    mgm_dd acc;
    acc.hi = MGM_MUL(d, d);
    acc.lo = MGM_FMA(d, d, -acc.hi);
    for (int i = 3; i <= e; i++) acc = mgm_dd_mul_d(acc, d);
    return MGM_ADD(acc.hi, acc.lo);
}

/* pow(s, phs * 0.5) for s > 0 and a small non-negative integer phs. */
MGM_HD double mgm_pow_half(double s, int phs)
{
    if ((phs & 1) == 0) return mgm_pow_int(s, phs >> 1);
    double r = MGM_SQRT(s);
    if (phs == 1) return r;
    mgm_dd acc;
    acc.hi = r;
    acc.lo = MGM_DIV(MGM_FMA(-r, r, s), MGM_MUL(2.0, r)); /* sqrt(s) - r, to ~2^-106 relative */
    for (int i = 0; i < (phs >> 1); i++) acc = mgm_dd_mul_d(acc, s);
    return MGM_ADD(acc.hi, acc.lo);
}

/* calculate_phs_rbf (rbf.h:32-40): sum of pow(diff, 2) over `dim` coordinates,
 * 0 at zero distance, else pow(sum, phs * 0.5). */
MGM_HD double mgm_phs_rbf(const double *p1, const double *p2, int phs, int dim)
{
    double s = 0;
    for (int i = 0; i < dim; i++) {
        double d = MGM_SUB(p1[i], p2[i]);
        s = MGM_ADD(s, MGM_MUL(d, d));
    }
    if (s == 0) return 0;
    return mgm_pow_half(s, phs);
}

/* sqrt(dist_sq) of kdtree_functions.h:28-35, 84 (always 3 coordinates). */
MGM_HD double mgm_ref_distance(double px, double py, double pz, double qx, double qy, double qz)
{
    double s = 0, d;
    d = MGM_SUB(px, qx); s = MGM_ADD(s, MGM_MUL(d, d));
    d = MGM_SUB(py, qy); s = MGM_ADD(s, MGM_MUL(d, d));
    d = MGM_SUB(pz, qz); s = MGM_ADD(s, MGM_MUL(d, d));
    return MGM_SQRT(s);
}

#endif
