// Device-side building blocks of the HigFlow step on sm_100a: recorded-query
// evaluation, the reference's point formulas, the cyclic Jacobi eigensolver
// and the cell CUBISTA flux.  Each function states the reference routine it
// follows; the arithmetic is written in the reference's evaluation order and
// the translation unit is compiled without FMA contraction, so the FP64 form
// reproduces the reference's rounding sequence.
#pragma once
#include <cstdint>
#include "higflow_b200.h"

#define HF_EPSMACH 1.0e-12
#define HF_FLT_EQ(x, y) (fabs((x) - (y)) < HF_EPSMACH)  // higtree/src/utils.h:40

// pi to double precision (the reference's pi, hig-flow-mittag-leffler.h:8,
// rounds to the same double)
#define HF_PI 3.141592653589793238462643383279502884

namespace hf {

// General stencil rows, in FP64 or FP32 storage.
template <typename W>
struct Rows {
    const int32_t *tmpl;    // per row: template
    const int32_t *base;    // per row: offset added to the template's columns
    const W *rhs;           // per row: boundary term
    const int64_t *tptr;    // per template: CSR pointer
    const int32_t *col;
    const W *w;
};

// Value of one recorded query (dp_interpolate_from_stencil, pdomain.c:1026-1053):
// code >= 0 is a centre hit, otherwise -rhs + sum_k w_k * f[base + col_k] in
// template order.
template <typename W, typename F>
__device__ __forceinline__ W query(const Rows<W> &R, int32_t code, const F *__restrict__ f)
{
    if (code >= 0) return (W)__ldg(f + code);
    const int64_t r = -(int64_t)code - 1;
    const int32_t t = __ldg(R.tmpl + r);
    const F *__restrict__ fb = f + __ldg(R.base + r);
    W res = (W)0;
    res += -__ldg(R.rhs + r);
    const int64_t e = __ldg(R.tptr + t + 1);
    for (int64_t k = __ldg(R.tptr + t); k < e; k++)
        res += (W)__ldg(fb + __ldg(R.col + k)) * __ldg(R.w + k);
    return res;
}

// hig_flow_jacobi (hig-flow-step-viscoelastic.c:1517-1600): cyclic Jacobi with
// the reference's thresholds and sweep limit.
template <int D>
__device__ void jacobi(double A[D][D], double d[D], double V[D][D])
{
    double bb[D], z[D];
    const int NMAX = 500;
#pragma unroll
    for (int ip = 0; ip < D; ip++) {
#pragma unroll
        for (int iq = 0; iq < D; iq++) V[ip][iq] = 0.0;
        V[ip][ip] = 1.0;
        bb[ip] = A[ip][ip];
        d[ip] = bb[ip];
        z[ip] = 0.0;
    }
    for (int i = 1; i <= NMAX; i++) {
        double tresh, sm = 0.0;
#pragma unroll
        for (int ip = 0; ip < D - 1; ip++)
#pragma unroll
            for (int iq = ip + 1; iq < D; iq++) sm += fabs(A[ip][iq]);
        if (sm == 0.0) return;
        if (i < 4) tresh = 0.2 * sm / (D * D);
        else tresh = 0.0;
#pragma unroll
        for (int ip = 0; ip < D - 1; ip++) {
#pragma unroll
            for (int iq = ip + 1; iq < D; iq++) {
                double g = 100.0 * fabs(A[ip][iq]);
                if ((i > 4) && (fabs(d[ip]) + g == fabs(d[ip])) && (fabs(d[iq]) + g == fabs(d[iq]))) {
                    A[ip][iq] = 0.0;
                } else if (fabs(A[ip][iq]) > tresh) {
                    double t, theta;
                    double h = d[iq] - d[ip];
                    if (fabs(h) + g == fabs(h)) {
                        t = A[ip][iq] / h;
                    } else {
                        theta = 0.5 * h / A[ip][iq];
                        t = 1.0 / (fabs(theta) + sqrt(1.0 + theta * theta));
                        if (theta < 0.0) t = -t;
                    }
                    double c = 1.0 / sqrt(1.0 + t * t);
                    double s = t * c;
                    double tau = s / (1.0 + c);
                    h = t * A[ip][iq];
                    z[ip] = z[ip] - h;
                    z[iq] = z[iq] + h;
                    d[ip] = d[ip] - h;
                    d[iq] = d[iq] + h;
                    A[ip][iq] = 0.0;
#pragma unroll
                    for (int j = 0; j <= ip - 1; j++) {
                        g = A[j][ip]; h = A[j][iq];
                        A[j][ip] = g - s * (h + g * tau);
                        A[j][iq] = h + s * (g - h * tau);
                    }
#pragma unroll
                    for (int j = ip + 1; j <= iq - 1; j++) {
                        g = A[ip][j]; h = A[j][iq];
                        A[ip][j] = g - s * (h + g * tau);
                        A[j][iq] = h + s * (g - h * tau);
                    }
#pragma unroll
                    for (int j = iq + 1; j < D; j++) {
                        g = A[ip][j]; h = A[iq][j];
                        A[ip][j] = g - s * (h + g * tau);
                        A[iq][j] = h + s * (g - h * tau);
                    }
#pragma unroll
                    for (int j = 0; j < D; j++) {
                        g = V[j][ip]; h = V[j][iq];
                        V[j][ip] = g - s * (h + g * tau);
                        V[j][iq] = h + s * (g - h * tau);
                    }
                }
            }
        }
#pragma unroll
        for (int ip = 0; ip < D; ip++) {
            bb[ip] = bb[ip] + z[ip];
            d[ip] = bb[ip];
            z[ip] = 0.0;
        }
    }
}

// R^t A R (hig_flow_matrix_product, :1603)
template <int D>
__device__ __forceinline__ void mprod(const double A[D][D], const double R[D][D], double B[D][D])
{
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) {
            B[i][j] = 0.0;
#pragma unroll
            for (int k = 0; k < D; k++)
#pragma unroll
                for (int l = 0; l < D; l++) B[i][j] += R[k][i] * A[k][l] * R[l][j];
        }
}

// R A R^t (hig_flow_matrix_transpose_product, :1617)
template <int D>
__device__ __forceinline__ void mtprod(const double A[D][D], const double R[D][D], double B[D][D])
{
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) {
            B[i][j] = 0.0;
#pragma unroll
            for (int k = 0; k < D; k++)
#pragma unroll
                for (int l = 0; l < D; l++) B[i][j] += R[i][k] * A[k][l] * R[j][l];
        }
}

// kernel-conformation transforms, selected from the case's callbacks at
// attach (commented variants in higflow/example2d_Oldroyd/ns-example-2d.c:21-56)
__device__ __forceinline__ double kernel_inverse(int kind, double l)
{
    if (kind == HF_KERNEL_LOG) return exp(l);
    if (kind == HF_KERNEL_SQRT) return l * l;
    return l;
}

__device__ __forceinline__ double kernel_jacobian(int kind, double l, double tol)
{
    if (kind == HF_KERNEL_LOG) return l < tol ? 1.0 / tol : 1.0 / l;
    if (kind == HF_KERNEL_SQRT) return l < tol ? 0.5 / sqrt(tol) : 0.5 / sqrt(l);
    return 1.0;
}

// The implicit constitutive step's per-cell system: the matrix of
// hig_flow_kernel_system_matrix (hig-flow-step-viscoelastic.c:1964-1989) for
// Omega (row-major D x D) and dt, solved for the right-hand side x (n = D*D,
// overwritten by the solution) by hig_flow_solve_system_constitutive_equation
// (:1912-1953): Gauss elimination with partial pivoting, in its order.  Out of
// line: only cells of instances with the implicit form call it.
template <int D>
__device__ __noinline__ void implicit_kernel_solve(const double *Om, double dt, double *x)
{
    constexpr int n = D * D;
    double A[n][n + 1];
    for (int i = 0; i < D; i++)
        for (int j = i; j < D; j++)
            for (int k = 0; k < D; k++)
                for (int l = 0; l < D; l++) {
                    const double I = k == l ? 1.0 : 0.0;
                    if (i == j) {
                        A[i * D + k][j * D + l] = I - dt * Om[k * D + l] - dt * Om[i * D + i] * I;
                    } else {
                        A[i * D + k][j * D + l] = dt * Om[j * D + i] * I;
                        A[j * D + l][i * D + k] = -dt * Om[j * D + i] * I;
                    }
                }
    for (int j = 0; j < n; j++) A[j][n] = x[j];
    for (int k = 0; k < n - 1; k++) {
        double mx = fabs(A[k][k]);
        int l = k;
        for (int i = k + 1; i < n; i++)
            if (fabs(A[i][k]) > mx) {
                mx = fabs(A[i][k]);
                l = i;
            }
        if (l != k)
            for (int j = k; j <= n; j++) {
                const double aux = A[k][j];
                A[k][j] = A[l][j];
                A[l][j] = aux;
            }
        for (int i = k + 1; i < n; i++) {
            const double s = A[i][k] / A[k][k];
            A[i][k] = 0;
            for (int j = k + 1; j <= n; j++) A[i][j] -= s * A[k][j];
        }
    }
    x[n - 1] = A[n - 1][n] / A[n - 1][n - 1];
    for (int i = n - 2; i >= 0; i--) {
        double s = 0;
        for (int j = i + 1; j < n; j++) s += A[i][j] * x[j];
        x[i] = (A[i][n] - s) / A[i][i];
    }
}

// FLT_EQ of higtree/src/utils.h:40 in the arithmetic type
template <typename T>
__device__ __forceinline__ bool flt_eq(T x, T y)
{
    return fabs(x - y) < T(HF_EPSMACH);
}

// hig_flow_convective_cell_term_cubista (hig-flow-step.c:1185-1358).  Out of
// line: the VE cell stage calls it D(D+1)/2 x D times, and six inlined copies
// of its branches made that kernel instruction-fetch bound (1.74 -> 1.38 ms on
// 4.29 M cells with one shared copy).
template <typename T>
__device__ __noinline__ T cubista_cell_t(T kl, T kr, T kll, T krr, int il, int ir, int ill, int irr, T vl, T vr, T kc,
                                       T cdelta)
{
    const T a = T(1.7500), b = T(0.3750), c = T(0.7500), d = T(0.1250), e = T(0.2500);
    T vbar, fi, conv1 = T(0), conv2 = T(0);
    vbar = vr;
    if (vbar > T(0)) {
        if (flt_eq(kr, kl)) {
            conv1 = vbar * kc;
        } else {
            fi = (kc - kl) / (kr - kl);
            if ((fi <= T(0)) || (fi >= T(1))) {
                conv1 = vbar * kc;
            } else {
                if (fi < b) conv1 = il == 1 ? vbar * (a * kc - c * kl) : vbar * kc;
                if ((fi >= b) && (fi <= c)) conv1 = ((il == 1) && (ir == 1)) ? vbar * (c * kc + b * kr - d * kl) : vbar * kc;
                if (fi > c) conv1 = ir == 1 ? vbar * (e * kc + c * kr) : vbar * kc;
            }
        }
    } else {
        if ((ir == 1) && (irr == 1)) {
            if (flt_eq(kc, krr)) {
                conv1 = vbar * kr;
            } else {
                fi = (kr - krr) / (kc - krr);
                if ((fi <= T(0)) || (fi >= T(1))) {
                    conv1 = vbar * kr;
                } else {
                    if (fi < b) conv1 = vbar * (a * kr - c * krr);
                    if ((fi >= b) && (fi <= c)) conv1 = vbar * (c * kr + b * kc - d * krr);
                    if (fi > c) conv1 = vbar * (c * kc + e * kr);
                }
            }
        } else if ((ir == 1) && (irr == 0)) {
            if (flt_eq(kc, krr)) {
                conv1 = vbar * kr;
            } else {
                fi = (kr - krr) / (kc - krr);
                if ((fi <= T(0)) || (fi >= T(1))) {
                    conv1 = vbar * kr;
                } else {
                    if (fi <= c) conv1 = vbar * kr;
                    if (fi > c) conv1 = vbar * (c * kc + e * kr);
                }
            }
        } else {
            conv1 = vr * kc;
            vbar = vl;
            conv2 = vbar > T(0) ? vbar * kl : vbar * kc;
            return ((conv1 - conv2) / cdelta);
        }
    }
    vbar = vl;
    if (vbar > T(0)) {
        if ((il == 1) && (ill == 1)) {
            if (flt_eq(kc, kll)) {
                conv2 = vbar * kl;
            } else {
                fi = (kl - kll) / (kc - kll);
                if ((fi <= T(0)) || (fi >= T(1))) {
                    conv2 = vbar * kl;
                } else {
                    if (fi < b) conv2 = vbar * (a * kl - c * kll);
                    if ((fi >= b) && (fi <= c)) conv2 = vbar * (b * kc + c * kl - d * kll);
                    if (fi > c) conv2 = vbar * (c * kc + e * kl);
                }
            }
        } else if ((il == 1) && (ill == 0)) {
            if (flt_eq(kc, kll)) {
                conv2 = vbar * kl;
            } else {
                fi = (kl - kll) / (kc - kll);
                if ((fi <= T(0)) || (fi >= T(1))) {
                    conv2 = vbar * kl;
                } else {
                    if (fi <= c) conv2 = vbar * kl;
                    if (fi > c) conv2 = vbar * (c * kc + e * kl);
                }
            }
        } else {
            conv1 = vr > T(0) ? vr * kc : vr * kr;
            conv2 = vl * kc;
            return ((conv1 - conv2) / cdelta);
        }
    } else {
        if (flt_eq(kl, kr)) {
            conv2 = vbar * kc;
        } else {
            fi = (kc - kr) / (kl - kr);
            if ((fi <= T(0)) || (fi >= T(1))) {
                conv2 = vbar * kc;
            } else {
                if (fi < b) conv2 = ir == 1 ? vbar * (a * kc - c * kr) : vbar * kc;
                if ((fi >= b) && (fi <= c)) conv2 = ((il == 1) && (ir == 1)) ? vbar * (c * kc + b * kl - d * kr) : vbar * kc;
                if (fi > c) conv2 = il == 1 ? vbar * (e * kc + c * kl) : vbar * kc;
            }
        }
    }
    return ((conv1 - conv2) / cdelta);
}

// (the FP64 instantiation is the reference's arithmetic; the mixed form
// takes the FP32 one)
__device__ __forceinline__ double cubista_cell(double kl, double kr, double kll, double krr, int il, int ir, int ill,
                                               int irr, double vl, double vr, double kc, double cdelta)
{
    return cubista_cell_t<double>(kl, kr, kll, krr, il, ir, ill, irr, vl, vr, kc, cdelta);
}

// ---------------------------------------------------------------------------
// Mittag-Leffler function E_{a,b}(z) for the GPTT model (hig_flow_calculate_m_
// gptt, hig-flow-step-viscoelastic.c:1771-1830; the reference evaluates it with
// mlfv, hig-flow-mittag-leffler.c:117-366).  The published algorithm of
// Gorenflo, Loutchko and Luchko (Fract. Calc. Appl. Anal. 5, 2002): power
// series near the origin, the integral representation (ray integral of K, arc
// integral of P, Romberg's rule) in the middle, the asymptotic series far out
// for a <= 1, and for a > 1 the reduction to smaller a over roots of z.  rho =
// 10^-fi sets the region bounds and the arc's Romberg levels (the ray takes
// six, as the reference's rombint does, :53-56).  Powers of z are polar,
// |z|^p e^{i p arg z}.  Only real parts enter the model; the leading term's
// imaginary part is the true one (the reference's differs in sign, which never
// reaches a real part).  The recursion depth is static: a >= 2 reduces to
// [1, 2), which halves to below 1, where nothing recurses (level L = 2 at the
// top).  Every loop is bounded.
// ---------------------------------------------------------------------------
struct Cx { double re, im; };

__device__ inline Cx cx_make(double re, double im) { Cx z; z.re = re; z.im = im; return z; }
__device__ inline Cx cx_polar(double r, double t) { return cx_make(r * cos(t), r * sin(t)); }
__device__ inline Cx cx_add(Cx a, Cx b) { return cx_make(a.re + b.re, a.im + b.im); }
__device__ inline Cx cx_div(Cx a, Cx b)
{
    const double d = b.re * b.re + b.im * b.im;
    return cx_make((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}

struct MlArgs { double a, b, eps; Cx z; };

// ray integrand: r^((1-b)/a) e^(-r^(1/a)) / (pi a)
//   * (r sin(pi(1-b)) - z sin(pi(1-b+a))) / (r^2 - 2 r z cos(pi a) + z^2)
__device__ inline Cx ml_ray(const MlArgs &c, double r)
{
    const double a = c.a, b = c.b;
    const double A = pow(r, (1.0 - b) / a) * exp(-pow(r, 1.0 / a)) / (HF_PI * a);
    const double s1 = r * sin(HF_PI * (1.0 - b)), s2 = sin(HF_PI * (1.0 - b + a));
    const double e = 2.0 * r * cos(HF_PI * a);
    const Cx num = cx_make(s1 - s2 * c.z.re, -s2 * c.z.im);
    const Cx den = cx_make(r * r - e * c.z.re + (c.z.re * c.z.re - c.z.im * c.z.im), -e * c.z.im + 2.0 * c.z.re * c.z.im);
    const Cx q = cx_div(num, den);
    return cx_make(A * q.re, A * q.im);
}

// arc integrand on |zeta| = eps: eps^(1+(1-b)/a) e^(eps^(1/a) cos(phi/a))
//   e^{i w} / (2 pi a (eps e^{i phi} - z)), w = eps^(1/a) sin(phi/a) + phi (1+(1-b)/a)
__device__ inline Cx ml_arc(const MlArgs &c, double phi)
{
    const double a = c.a, b = c.b, eps = c.eps;
    const double p = 1.0 + (1.0 - b) / a, er = pow(eps, 1.0 / a);
    const double A = pow(eps, p) * exp(er * cos(phi / a)) / (2.0 * HF_PI * a);
    const double w = er * sin(phi / a) + phi * p;
    return cx_div(cx_polar(A, w), cx_make(eps * cos(phi) - c.z.re, eps * sin(phi) - c.z.im));
}

// Romberg's rule, one row kept in place: R[k] of the new row needs R[k-1] of
// the new row and R[k-1] of the old one.  At most eight levels (the
// reference's table holds eight, rombint :46-50)
template <bool RAY>
__device__ __noinline__ Cx ml_romberg(MlArgs c, double lo, double hi, int n)
{
    if (RAY) n = 6;
    n = n < 1 ? 1 : (n > 8 ? 8 : n);
    Cx R[8];
    for (int k = 0; k < 8; k++) R[k] = cx_make(0.0, 0.0);
    double h = hi - lo;
    const Cx fa = RAY ? ml_ray(c, lo) : ml_arc(c, lo);
    const Cx fb = RAY ? ml_ray(c, hi) : ml_arc(c, hi);
    R[0] = cx_make(h * (fa.re + fb.re) / 2.0, h * (fa.im + fb.im) / 2.0);
    int npts = 1;
    for (int i = 1; i < n; i++) {
        Cx s = cx_make(0.0, 0.0);
        for (int j = 1; j <= npts; j++) s = cx_add(s, RAY ? ml_ray(c, lo + h * (j - 0.5)) : ml_arc(c, lo + h * (j - 0.5)));
        Cx old = R[0];
        R[0] = cx_make((R[0].re + h * s.re) / 2.0, (R[0].im + h * s.im) / 2.0);
        double q = 1.0;
        for (int k = 1; k <= i; k++) {
            q *= 4.0;
            const Cx ok = R[k];
            R[k] = cx_make((q * R[k - 1].re - old.re) / (q - 1.0), (q * R[k - 1].im - old.im) / (q - 1.0));
            old = ok;
        }
        npts *= 2;
        h /= 2.0;
    }
    return R[n - 1];
}

// z^((1-b)/a) e^(z^(1/a)) / a
__device__ inline Cx ml_lead(double a, double b, double az, double th)
{
    const double ra = pow(az, 1.0 / a);
    const double mag = (pow(az, (1.0 - b) / a) / a) * exp(ra * cos(th / a));
    return cx_polar(mag, th * (1.0 - b) / a + ra * sin(th / a));
}

template <int L>
__device__ __noinline__ Cx mittag_leffler(double a, double b, Cx z, int fi)
{
    const double az = sqrt(z.re * z.re + z.im * z.im);
    const double th = atan2(z.im, z.re), ath = fabs(th);
    const double rho = pow(10.0, (double)-fi);
    const bool series = (a < 1.0 && az <= 1.0) ||
                        (1.0 <= a && a < 2.0 && az <= floor(20.0 / pow(2.1 - a, 5.5 - 2.0 * a))) ||
                        (a >= 2.0 && az <= 50.0);
    if (series) {
        int k = 0;
        while (a * k + b <= 0.0 && k < 1000000) k++;
        Cx s = cx_make(pow(az, (double)k) * cos(th * k) / tgamma(a * k + b),
                       pow(az, (double)k) * sin(th * k) / tgamma(a * k + b));
        for (int it = 0; it < 100000; it++) {
            const Cx old = s;
            for (int t = 0; t < 2; t++) {
                k++;
                const double g = tgamma(a * k + b), pk = pow(az, (double)k);
                s = cx_make(s.re + pk * cos(th * k) / g, s.im + pk * sin(th * k) / g);
            }
            if (s.re == old.re && s.im == old.im) break;
        }
        return s;
    }
    if (a <= 1.0 && az <= floor(5.0 * a + 10.0)) {
        const double r0 = fmax(fmax(1.0, 2.0 * az), pow(-2.0 * log(rho * HF_PI / 6.0), a));
        MlArgs c;
        c.a = a; c.b = b; c.eps = 0.0; c.z = z;
        const double pa = HF_PI * a;
        if (ath > pa && fabs(ath - pa) > rho) {
            if (b <= 1.0) return ml_romberg<true>(c, 0.0, r0, fi);
            c.eps = 1.0;
            return cx_add(ml_romberg<true>(c, c.eps, r0, fi), ml_romberg<false>(c, -pa, pa, fi));
        }
        if (ath < pa && fabs(ath - pa) > rho) {
            if (b <= 1.0) return cx_add(ml_romberg<true>(c, 0.0, r0, fi), ml_lead(a, b, az, th));
            c.eps = az / 2.0;
            const Cx arc = ml_romberg<false>(c, -pa, pa, fi);
            return cx_add(cx_add(arc, ml_romberg<true>(c, c.eps, r0, fi)), ml_lead(a, b, az, th));
        }
        c.eps = az + 0.5;
        return cx_add(ml_romberg<true>(c, c.eps, r0, fi), ml_romberg<false>(c, -pa, pa, fi));
    }
    if (a <= 1.0) {
        Cx s = cx_make(0.0, 0.0);
        if (ath < (HF_PI * a / 2.0 + fmin(HF_PI, HF_PI * a)) / 2.0) s = ml_lead(a, b, az, th);
        const double kmax = floor(fi / log10(az));
        for (int k = 1; k <= kmax && k <= 64; k++) {
            const double g = b - a * k;
            if (ceil(g) == floor(g)) continue;
            const double pk = pow(az, (double)-k);
            s = cx_make(s.re - pk * cos(th * k) / tgamma(g), s.im - (-(pk * sin(th * k))) / tgamma(g));
        }
        return s;
    }
    if constexpr (L > 0) {
        if (a >= 2.0) {
            const int m = (int)floor(a / 2.0);
            Cx s = cx_make(0.0, 0.0);
            for (int h = 0; h <= m && h < 64; h++) {
                const double r = pow(az, 1.0 / (m + 1.0));
                s = cx_add(s, mittag_leffler<L - 1>(a / (m + 1), b, cx_polar(r, (2.0 * HF_PI * h + th) / (m + 1.0)), fi));
            }
            const double w = 1.0 / (m + 1.0);
            return cx_make(w * s.re, w * s.im);
        }
        const double r = sqrt(az);
        const Cx z1 = cx_make(r * cos(th / 2.0), r * sin(th / 2.0));
        const Cx e1 = mittag_leffler<L - 1>(a / 2.0, b, z1, fi);
        const Cx e2 = mittag_leffler<L - 1>(a / 2.0, b, cx_make(-z1.re, -z1.im), fi);
        return cx_make((e1.re + e2.re) / 2.0, (e1.im + e2.im) / 2.0);
    } else {
        // unreachable: at the last level a < 1
        return cx_make(nan(""), nan(""));
    }
}

// E_{a_g,b_g}(z) for real z with fi = 6, as the GPTT M term takes it (:1805)
__device__ __noinline__ double gptt_ml(double alpha_g, double beta_g, double z)
{
    return mittag_leffler<2>(alpha_g, beta_g, cx_make(z, 0.0), 6).re;
}

}  // namespace hf
