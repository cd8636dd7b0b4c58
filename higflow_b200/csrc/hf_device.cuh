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

// The same value with the general-row evaluation out of line, for call sites
// where general rows are rare (cells away from boundaries hit centres): the
// caller's code stays small, which matters in kernels with many query sites.
template <typename W, typename F>
__device__ __noinline__ W query_row(const Rows<W> R, int32_t code, const F *__restrict__ f)
{
    return query<W, F>(R, code, f);
}

template <typename W, typename F>
__device__ __forceinline__ W query_cold(const Rows<W> &R, int32_t code, const F *__restrict__ f)
{
    if (code >= 0) return (W)__ldg(f + code);
    return query_row<W, F>(R, code, f);
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

// hig_flow_convective_cell_term_cubista (hig-flow-step.c:1185-1358).  Out of
// line: the VE cell stage calls it D(D+1)/2 x D times, and six inlined copies
// of its branches made that kernel instruction-fetch bound (1.74 -> 1.38 ms on
// 4.29 M cells with one shared copy).
__device__ __noinline__ double cubista_cell(double kl, double kr, double kll, double krr, int il, int ir,
                                      int ill, int irr, double vl, double vr, double kc, double cdelta)
{
    const double a = 1.7500, b = 0.3750, c = 0.7500, d = 0.1250, e = 0.2500;
    double vbar, fi, conv1 = 0.0, conv2 = 0.0;
    vbar = vr;
    if (vbar > 0.0) {
        if (HF_FLT_EQ(kr, kl)) {
            conv1 = vbar * kc;
        } else {
            fi = (kc - kl) / (kr - kl);
            if ((fi <= 0.0) || (fi >= 1.0)) {
                conv1 = vbar * kc;
            } else {
                if (fi < b) conv1 = il == 1 ? vbar * (a * kc - c * kl) : vbar * kc;
                if ((fi >= b) && (fi <= c)) conv1 = ((il == 1) && (ir == 1)) ? vbar * (c * kc + b * kr - d * kl) : vbar * kc;
                if (fi > c) conv1 = ir == 1 ? vbar * (e * kc + c * kr) : vbar * kc;
            }
        }
    } else {
        if ((ir == 1) && (irr == 1)) {
            if (HF_FLT_EQ(kc, krr)) {
                conv1 = vbar * kr;
            } else {
                fi = (kr - krr) / (kc - krr);
                if ((fi <= 0.0) || (fi >= 1.0)) {
                    conv1 = vbar * kr;
                } else {
                    if (fi < b) conv1 = vbar * (a * kr - c * krr);
                    if ((fi >= b) && (fi <= c)) conv1 = vbar * (c * kr + b * kc - d * krr);
                    if (fi > c) conv1 = vbar * (c * kc + e * kr);
                }
            }
        } else if ((ir == 1) && (irr == 0)) {
            if (HF_FLT_EQ(kc, krr)) {
                conv1 = vbar * kr;
            } else {
                fi = (kr - krr) / (kc - krr);
                if ((fi <= 0.0) || (fi >= 1.0)) {
                    conv1 = vbar * kr;
                } else {
                    if (fi <= c) conv1 = vbar * kr;
                    if (fi > c) conv1 = vbar * (c * kc + e * kr);
                }
            }
        } else {
            conv1 = vr * kc;
            vbar = vl;
            conv2 = vbar > 0.0 ? vbar * kl : vbar * kc;
            return ((conv1 - conv2) / cdelta);
        }
    }
    vbar = vl;
    if (vbar > 0.0) {
        if ((il == 1) && (ill == 1)) {
            if (HF_FLT_EQ(kc, kll)) {
                conv2 = vbar * kl;
            } else {
                fi = (kl - kll) / (kc - kll);
                if ((fi <= 0.0) || (fi >= 1.0)) {
                    conv2 = vbar * kl;
                } else {
                    if (fi < b) conv2 = vbar * (a * kl - c * kll);
                    if ((fi >= b) && (fi <= c)) conv2 = vbar * (b * kc + c * kl - d * kll);
                    if (fi > c) conv2 = vbar * (c * kc + e * kl);
                }
            }
        } else if ((il == 1) && (ill == 0)) {
            if (HF_FLT_EQ(kc, kll)) {
                conv2 = vbar * kl;
            } else {
                fi = (kl - kll) / (kc - kll);
                if ((fi <= 0.0) || (fi >= 1.0)) {
                    conv2 = vbar * kl;
                } else {
                    if (fi <= c) conv2 = vbar * kl;
                    if (fi > c) conv2 = vbar * (c * kc + e * kl);
                }
            }
        } else {
            conv1 = vr > 0.0 ? vr * kc : vr * kr;
            conv2 = vl * kc;
            return ((conv1 - conv2) / cdelta);
        }
    } else {
        if (HF_FLT_EQ(kl, kr)) {
            conv2 = vbar * kc;
        } else {
            fi = (kc - kr) / (kl - kr);
            if ((fi <= 0.0) || (fi >= 1.0)) {
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

}  // namespace hf
