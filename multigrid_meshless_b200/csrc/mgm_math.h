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
 * and round once at the end.  That alone is correctly rounded unless x^y lies
 * within ~2^-100 relative of a rounding midpoint -- rare for arguments in
 * general position, but systematic for squared distances a few ulps from a
 * power of four or from the square of a short dyadic number (two nodes on
 * concentric circles, one gap apart: s = 0.25 (1 - 2^-53), s^1.5 within
 * 2^-107 of a midpoint).  There the midpoint is compared with the exact
 * power in integer arithmetic (mgm_round_near_midpoint), so the result is
 * the correctly rounded value for every finite positive argument.
 *
 * Every product and sum that must follow the reference's rounding sequence
 * uses MGM_MUL / MGM_ADD / MGM_SUB, which never contract into an FMA.
 */
#ifndef MGM_MATH_H
#define MGM_MATH_H

#include <math.h>
#include <stdint.h>
#if !defined(__CUDA_ARCH__)
#include <string.h>
#endif

#if defined(__CUDACC__)
#define MGM_HD __host__ __device__ __forceinline__
#define MGM_HD_COLD static __host__ __device__ __noinline__
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
#define MGM_HD_COLD static
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

/* ---- exact comparison with a rounding midpoint --------------------------
 * A value A * 2^ea with A a non-negative integer of up to MGM_BIGW 64-bit
 * words.  Only the rare near-midpoint branch of the powers below uses it. */
#define MGM_BIGW 9

typedef struct { uint64_t w[MGM_BIGW]; int n, e; } mgm_big;

MGM_HD uint64_t mgm_bits(double x)
{
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t b;
    memcpy(&b, &x, sizeof b);
    return b;
#endif
}

MGM_HD double mgm_from_bits(uint64_t b)
{
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double x;
    memcpy(&x, &b, sizeof x);
    return x;
#endif
}

MGM_HD int mgm_clz64(uint64_t v)
{
#ifdef __CUDA_ARCH__
    return __clzll((long long)v);
#else
    return __builtin_clzll(v);
#endif
}

/* x = m * 2^e for finite x > 0 (m < 2^53) */
MGM_HD void mgm_split(double x, uint64_t *m, int *e)
{
    uint64_t b = mgm_bits(x);
    int ef = (int)((b >> 52) & 0x7ff);
    uint64_t f = b & ((1ULL << 52) - 1);
    if (ef == 0) { *m = f; *e = -1074; }
    else { *m = f | (1ULL << 52); *e = ef - 1075; }
}

/* a *= v; returns 0 when the product would not fit in MGM_BIGW words */
MGM_HD int mgm_big_mul(mgm_big *a, uint64_t v)
{
    uint64_t carry = 0;
    for (int i = 0; i < a->n; i++) {
        uint64_t lo, hi;
#ifdef __CUDA_ARCH__
        lo = a->w[i] * v;
        hi = __umul64hi(a->w[i], v);
#else
        unsigned __int128 p = (unsigned __int128)a->w[i] * v;
        lo = (uint64_t)p;
        hi = (uint64_t)(p >> 64);
#endif
        lo += carry;
        hi += lo < carry;
        a->w[i] = lo;
        carry = hi;
    }
    if (carry) {
        if (a->n == MGM_BIGW) return 0;
        a->w[a->n++] = carry;
    }
    return 1;
}

/* m^k * 2^(k e) exactly; 0 when it does not fit */
MGM_HD int mgm_big_pow(uint64_t m, int e, int k, mgm_big *r)
{
    r->w[0] = m;
    r->n = 1;
    r->e = e * k;
    for (int i = 1; i < k; i++)
        if (!mgm_big_mul(r, m)) return 0;
    return 1;
}

MGM_HD int mgm_big_len(const mgm_big *a)
{
    int n = a->n;
    while (n > 0 && a->w[n - 1] == 0) n--;
    return n == 0 ? 0 : 64 * n - mgm_clz64(a->w[n - 1]);
}

/* word i of a shifted left by sh bits */
MGM_HD uint64_t mgm_big_word(const mgm_big *a, int sh, int i)
{
    int q = sh >> 6, r = sh & 63, j = i - q;
    uint64_t hi = (j >= 0 && j < a->n) ? a->w[j] : 0;
    uint64_t lo = (j - 1 >= 0 && j - 1 < a->n) ? a->w[j - 1] : 0;
    return r == 0 ? hi : (hi << r) | (lo >> (64 - r));
}

/* sign of A * 2^ea - B * 2^eb (both non-zero) */
MGM_HD int mgm_big_cmp(const mgm_big *a, const mgm_big *b)
{
    int la = mgm_big_len(a), lb = mgm_big_len(b);
    int ta = la + a->e, tb = lb + b->e;
    if (ta != tb) return ta > tb ? 1 : -1;
    /* same leading bit position: align both tops at bit 64 MGM_BIGW - 1 */
    int sa = 64 * MGM_BIGW - la, sb = 64 * MGM_BIGW - lb;
    for (int i = MGM_BIGW - 1; i >= 0; i--) {
        uint64_t wa = mgm_big_word(a, sa, i), wb = mgm_big_word(b, sb, i);
        if (wa != wb) return wa > wb ? 1 : -1;
    }
    return 0;
}

/* The near-midpoint branch, kept out of line: y = x^k (k_den == 1) or
 * x^(k/2) (k_den == 2) lies within the evaluation error of the midpoint
 * between lower and upper = nextup(lower); returns the one that the exact
 * comparison of y with that midpoint selects (r when the powers do not fit). */
MGM_HD_COLD double mgm_round_exact(double x, int k, int k_den, double lower, double upper, double r)
{
    uint64_t lm;
    int le;
    mgm_split(lower, &lm, &le);
    /* midpoint (2 lm + 1) 2^(le - 1); compare y^k_den with it^k_den */
    mgm_big mid, pw;
    mid.w[0] = 2 * lm + 1;
    mid.n = 1;
    mid.e = le - 1;
    if (k_den == 2) {
        if (!mgm_big_mul(&mid, 2 * lm + 1)) return r;
        mid.e = 2 * (le - 1);
    }
    uint64_t xm;
    int xe;
    mgm_split(x, &xm, &xe);
    if (xm == 0 || !mgm_big_pow(xm, xe, k, &pw)) return r;
    const int c = mgm_big_cmp(&pw, &mid);
    if (c > 0) return upper;
    if (c < 0) return lower;
    return (lm & 1) ? upper : lower;   /* exact tie: to even */
}

/* The exact value y = x^k (k_den == 1) or x^(k/2) (k_den == 2), x > 0, has
 * the double-double approximation hi + lo, and r = RN(hi + lo).  Returns r
 * when no midpoint lies within the approximation's error bound (2^-96 r,
 * well above the 2^-100 the evaluations below reach), else the neighbour of
 * r that the exact comparison of y with that midpoint selects. */
MGM_HD double mgm_round_near_midpoint(double x, int k, int k_den, double hi, double lo, double r)
{
    if (!(r > 0) || !(r < 1.7e308)) return r;
    const uint64_t br = mgm_bits(r);
    const double up = mgm_from_bits(br + 1), dn = mgm_from_bits(br - 1);
    const double diff = MGM_ADD(MGM_SUB(hi, r), lo);     /* ~ y - r; hi - r is exact */
    const double half = diff >= 0 ? MGM_MUL(0.5, MGM_SUB(up, r)) : MGM_MUL(0.5, MGM_SUB(r, dn));
    if (fabs(MGM_SUB(fabs(diff), half)) > MGM_MUL(1.2621774483536189e-29 /* 2^-96 */, r)) return r;
    return diff >= 0 ? mgm_round_exact(x, k, k_den, r, up, r) : mgm_round_exact(x, k, k_den, dn, r, r);
}

/* |d|^e, d != 0, e >= 3, as a double-double rounded once */
MGM_HD double mgm_pow_int_pos(double a, int e)
{
    mgm_dd acc;
    acc.hi = MGM_MUL(a, a);
    acc.lo = MGM_FMA(a, a, -acc.hi);
    for (int i = 3; i <= e; i++) acc = mgm_dd_mul_d(acc, a);
    const double r = MGM_ADD(acc.hi, acc.lo);
    return mgm_round_near_midpoint(a, e, 1, acc.hi, acc.lo, r);
}

/* pow(d, e) for a small non-negative integer e (the monomial powers). */
MGM_HD double mgm_pow_int(double d, int e)
{
    if (e == 0) return 1.0;
    if (e == 1) return d;
    if (e == 2) return MGM_MUL(d, d);
    if (d == 0) return (e & 1) ? d : 0.0;
    const double r = mgm_pow_int_pos(fabs(d), e);
    return (d < 0 && (e & 1)) ? -r : r;
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
    return mgm_round_near_midpoint(s, phs, 2, acc.hi, acc.lo, MGM_ADD(acc.hi, acc.lo));
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
