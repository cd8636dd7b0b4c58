// Persistent per-instance Poisson solver for batched cases.
//
// One CTA owns one instance of a batch program for the whole projection: it
// forms the divergence right-hand side of its cells (higflow_pressure,
// hig-flow-step.c:58-120, with the instance's own dt and pressure pin), then
// runs CG preconditioned by the instance's own smoothed-aggregation V-cycle
// (hf_amg.cuh) until its own residual test passes, and writes the pressure
// increment back.  Each instance therefore keeps its own Krylov scalars and
// convergence test, so a result does not depend on which other instances share
// the launch.  Vectors live in global memory (the working set of an instance
// stays in L2); phases are separated by __syncthreads().
//
// Precision: T = double is the plain form.  The mixed form runs the
// preconditioned CG in float (float matrices, vectors and dot products) inside
// an FP64 iterative-refinement loop whose residual b - A x is formed in FP64
// against the same convergence test as the plain form.
#pragma once

constexpr int kPB = 512;   // threads per instance

template <typename T>
struct ILevel {
    int n;
    const int32_t *Ap, *Ac;
    const T *Av;
    const int32_t *Pp, *Pc;
    const T *Pv;
    const int32_t *Rp, *Rc;
    const T *Rv;
    const T *dinv;
    T *x, *b, *r, *out;
};

struct InstSolve {
    int inst;              // instance index in the batch
    int n, coff;           // rows, first global cell
    int nlev;              // smoothed levels (the coarsest has a dense inverse)
    int lev;               // first entry of this instance in the level tables
    int cn;                // coarsest rows
    const double *cinv64;
    const float *cinv32;
    double *cb64, *cx64;
    float *cb32, *cx32;
    const int32_t *Mp, *Mc;   // reduced fine operator, local columns
    const double *Mv;
    const double *apin;       // A[i][pin] of the original rows
    const double *brhs;       // boundary part of the rhs
    int pin;                  // local pin row or -1
    double *b, *r, *z, *p, *q;         // FP64 work (b: reduced rhs)
    float *r32, *e32;                  // FP32 inner rhs and solution (mixed form)
    float *t32, *z32, *p32, *q32;      // FP32 inner CG work
    int *iters, *outer, *status;        // per-instance results
    double *res;
};

namespace batch {

__device__ __forceinline__ double block_sum(double v, double *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = threadIdx.x < kPB / 32 ? sh[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[kPB / 32] = v;
    }
    __syncthreads();
    return sh[kPB / 32];
}

__device__ __forceinline__ float block_sumf(float v, float *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = threadIdx.x < kPB / 32 ? sh[threadIdx.x] : 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[kPB / 32] = v;
    }
    __syncthreads();
    return sh[kPB / 32];
}

template <typename T>
__device__ __forceinline__ T row(const int32_t *p, const int32_t *c, const T *v, int i, const T *x)
{
    T s = T(0);
    for (int k = p[i]; k < p[i + 1]; k++) s += v[k] * x[c[k]];
    return s;
}

// z = V(b0), level 0 operator is L[0].A; all passes are CTA-wide loops
template <typename T>
__device__ void vcycle(const ILevel<T> *L, int nlev, int cn, const T *cinv, T *cb, T *cx, const T *b0, T *z0)
{
    const T w = T(2.0 / 3.0);
    for (int l = 0; l < nlev; l++) {
        const ILevel<T> &lv = L[l];
        const T *b = l == 0 ? b0 : lv.b;
        for (int i = threadIdx.x; i < lv.n; i += kPB) lv.x[i] = w * lv.dinv[i] * b[i];
        __syncthreads();
        for (int i = threadIdx.x; i < lv.n; i += kPB) lv.r[i] = b[i] - row(lv.Ap, lv.Ac, lv.Av, i, (const T *)lv.x);
        __syncthreads();
        T *bn = l + 1 < nlev ? L[l + 1].b : cb;
        const int nn = l + 1 < nlev ? L[l + 1].n : cn;
        for (int i = threadIdx.x; i < nn; i += kPB) bn[i] = row(lv.Rp, lv.Rc, lv.Rv, i, (const T *)lv.r);
        __syncthreads();
    }
    for (int i = threadIdx.x; i < cn; i += kPB) {
        T s = T(0);
        for (int k = 0; k < cn; k++) s += cinv[(size_t)i * cn + k] * cb[k];
        cx[i] = s;
    }
    __syncthreads();
    for (int l = nlev - 1; l >= 0; l--) {
        const ILevel<T> &lv = L[l];
        const T *e = l + 1 < nlev ? (const T *)L[l + 1].out : (const T *)cx;
        const T *b = l == 0 ? b0 : lv.b;
        for (int i = threadIdx.x; i < lv.n; i += kPB) lv.x[i] += row(lv.Pp, lv.Pc, lv.Pv, i, e);
        __syncthreads();
        T *out = l == 0 ? z0 : lv.out;
        for (int i = threadIdx.x; i < lv.n; i += kPB)
            out[i] = lv.x[i] + w * lv.dinv[i] * (b[i] - row(lv.Ap, lv.Ac, lv.Av, i, (const T *)lv.x));
        __syncthreads();
    }
    if (nlev == 0) {   // the whole operator is the coarsest level: z = inv b
        for (int i = threadIdx.x; i < cn; i += kPB) z0[i] = cx[i];
        __syncthreads();
    }
}

// z = V(b0) including the case where the operator itself is the coarsest level
template <typename T>
__device__ void precondition(const ILevel<T> *L, int nlev, int cn, const T *cinv, T *cb, T *cx, const T *b0, T *z0)
{
    if (nlev == 0) {
        for (int i = threadIdx.x; i < cn; i += kPB) cb[i] = b0[i];
        __syncthreads();
    }
    vcycle<T>(L, nlev, cn, cinv, cb, cx, b0, z0);
}

template <typename T>
__device__ void precondition(const ILevel<T> *L, int nlev, int cn, const T *cinv, T *cb, T *cx, const T *b0, T *z0);

// PCG in precision T on L[0].A x = b from x (x updated in place); returns
// iterations; stops at ||r|| <= tol or maxit; status 0 / HF_ERR_*
template <typename T, typename S>
__device__ int pcg(const ILevel<T> *L, int nlev, int cn, const T *cinv, T *cb, T *cx, int n, const T *b, T *x,
                   T *r, T *z, T *p, T *q, S tol, int maxit, int *status, S (*dot)(const T *, const T *, int, S *),
                   S *sh)
{
    const ILevel<T> &A = L[0];
    for (int i = threadIdx.x; i < n; i += kPB) r[i] = b[i] - row(A.Ap, A.Ac, A.Av, i, (const T *)x);
    __syncthreads();
    S rr = dot(r, r, n, sh);
    if (!isfinite((double)rr)) { *status = HF_ERR_NAN; return 0; }
    if (!(rr > tol * tol)) return 0;
    precondition<T>(L, nlev, cn, cinv, cb, cx, r, z);
    S rz = dot(r, z, n, sh);
    for (int i = threadIdx.x; i < n; i += kPB) p[i] = z[i];
    __syncthreads();
    int it = 0;
    while (it < maxit) {
        for (int i = threadIdx.x; i < n; i += kPB) q[i] = row(A.Ap, A.Ac, A.Av, i, (const T *)p);
        __syncthreads();
        S pq = dot(p, q, n, sh);
        if (!(pq > S(0)) || !isfinite((double)pq)) {
            if (!isfinite((double)pq)) *status = HF_ERR_NAN;
            else if (rr > S(1e4) * tol * tol) *status = HF_ERR_NOT_CONVERGED;
            return it;
        }
        const T alpha = T(rz / pq);
        for (int i = threadIdx.x; i < n; i += kPB) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
        }
        __syncthreads();
        it++;
        rr = dot(r, r, n, sh);
        if (!isfinite((double)rr)) { *status = HF_ERR_NAN; return it; }
        if (!(rr > tol * tol)) return it;
        precondition<T>(L, nlev, cn, cinv, cb, cx, r, z);
        const S rz2 = dot(r, z, n, sh);
        const T beta = T(rz2 / rz);
        rz = rz2;
        for (int i = threadIdx.x; i < n; i += kPB) p[i] = z[i] + beta * p[i];
        __syncthreads();
    }
    *status = HF_ERR_NOT_CONVERGED;
    return it;
}

__device__ double dot64(const double *a, const double *b, int n, double *sh)
{
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += kPB) s += a[i] * b[i];
    return block_sum(s, sh);
}

__device__ float dot32(const float *a, const float *b, int n, float *sh)
{
    float s = 0.0f;
    for (int i = threadIdx.x; i < n; i += kPB) s += a[i] * b[i];
    return block_sumf(s, sh);
}

}  // namespace batch

// One CTA per instance: rhs, solve, write the pressure increment (or pressure).
template <int D>
__global__ void __launch_bounds__(kPB) k_batch_poisson(DevProg P, DevFields F, const InstSolve *IS,
                                                      const ILevel<double> *L64, const ILevel<float> *L32,
                                                      int mixed, double rtol, double atol, int maxit)
{
    __shared__ double sh[kPB / 32 + 1];
    __shared__ float shf[kPB / 32 + 1];
    const InstSolve &S = IS[blockIdx.x];
    const hf_params &par = P.ipar[S.inst];
    const int n = S.n;
    const int nglob = P.ncell;
    double *xg = (par.projtype == HF_INCREMENTAL ? F.dp : F.p) + S.coff;
    const double pinv = S.pin >= 0
        ? (par.projtype == HF_INCREMENTAL ? P.ipinv[S.inst] - F.p[S.coff + S.pin] : P.ipinv[S.inst]) : 0.0;
    // divergence rhs (the original system's b, for the tolerance) and reduced rhs
    double bb = 0.0;
    for (int i = threadIdx.x; i < n; i += kPB) {
        const int cc = S.coff + i;
        double borig;
        if (i == S.pin) {
            borig = pinv;
        } else {
            const double *cd = P.delta + (size_t)__ldg(P.cdelta + cc) * D;
            double sumdudx = 0.0;
#pragma unroll
            for (int dim = 0; dim < D; dim++) {
                const double ustarl = hf::query(P.rows, __ldg(P.dslots + (size_t)HF_P_UL(dim) * nglob + cc), F.us[dim]);
                const double ustarr = hf::query(P.rows, __ldg(P.dslots + (size_t)HF_P_UR(dim) * nglob + cc), F.us[dim]);
                sumdudx += (ustarr - ustarl) / (2.0 * 0.5 * cd[dim]);
            }
            borig = sumdudx / par.dt + S.brhs[i];
        }
        S.b[i] = i == S.pin ? pinv : -(borig - S.apin[i] * pinv);
        bb += borig * borig;
    }
    bb = batch::block_sum(bb, sh);
    const double tol = fmax(rtol * sqrt(bb), atol);
    int status = 0, iters = 0, outer = 0;
    if (!mixed) {
        iters = batch::pcg<double, double>(L64 + S.lev, S.nlev, S.cn, S.cinv64, S.cb64, S.cx64, n, S.b, xg, S.r, S.z,
                                           S.p, S.q, tol, maxit, &status, batch::dot64, sh);
        outer = 1;
    } else {
        // FP64 iterative refinement around an FP32 preconditioned CG
        const ILevel<double> &A = L64[S.lev];
        for (outer = 0; outer < 30; outer++) {
            for (int i = threadIdx.x; i < n; i += kPB) S.r[i] = S.b[i] - batch::row(A.Ap, A.Ac, A.Av, i, (const double *)xg);
            __syncthreads();
            const double rr = batch::dot64(S.r, S.r, n, sh);
            if (!isfinite(rr)) { status = HF_ERR_NAN; break; }
            if (!(rr > tol * tol)) break;
            if (iters >= maxit) { status = HF_ERR_NOT_CONVERGED; break; }
            const double scale = sqrt(rr);
            for (int i = threadIdx.x; i < n; i += kPB) {
                S.r32[i] = (float)(S.r[i] / scale);
                S.e32[i] = 0.0f;
            }
            __syncthreads();
            int st = 0;
            // inner target: 1e-4 of the current (unit-scaled) residual; a
            // NOT_CONVERGED inner solve is tolerated, the outer test decides
            iters += batch::pcg<float, float>(L32 + S.lev, S.nlev, S.cn, S.cinv32, S.cb32, S.cx32, n, S.r32, S.e32,
                                              S.t32, S.z32, S.p32, S.q32, 1e-4f, maxit, &st, batch::dot32, shf);
            if (st == HF_ERR_NAN) { status = HF_ERR_NAN; break; }
            for (int i = threadIdx.x; i < n; i += kPB) xg[i] += scale * (double)S.e32[i];
            __syncthreads();
        }
        if (outer == 30 && status == 0) status = HF_ERR_NOT_CONVERGED;
    }
    // true relative residual of the original system at exit
    const ILevel<double> &A0 = L64[S.lev];
    for (int i = threadIdx.x; i < n; i += kPB) S.r[i] = S.b[i] - batch::row(A0.Ap, A0.Ac, A0.Av, i, (const double *)xg);
    __syncthreads();
    const double rr = batch::dot64(S.r, S.r, n, sh);
    if (threadIdx.x == 0) {
        *S.iters = iters;
        *S.outer = outer;
        *S.status = status;
        *S.res = bb > 0.0 ? sqrt(rr / bb) : sqrt(rr);
    }
}
