// HigFlow per-time-step hot path on NVIDIA B200 (sm_100a).
//
// The step engine executes a flattened step program (include/higflow_b200.h)
// with every field resident in HBM:
//
//   ve_cell      one thread per cell: velocity-derivative tensor, explicit
//                kernel-conformation update and polymeric tensor, fused
//                (hig-flow-step-generalized-newtonian.c:14-97,
//                 hig-flow-step-viscoelastic.c:212-544)
//   velocity     one thread per interior facet, all directions in one launch:
//                computational cell + terms + explicit Euler
//                (hig-flow-discret.c:86-259, :541-569; hig-flow-terms.c;
//                 hig-flow-step.c:613-660; hig-flow-step-viscoelastic.c:931-980)
//   cg_init      divergence right-hand side of the Poisson rows fused with the
//                first residual of the solve (hig-flow-step.c:48-131)
//   cg_dir_spmv, cg_update
//                Jacobi-preconditioned CG, two launches per iteration, with
//                block partial sums finished by the last block to arrive
//                (deterministic order); BiCGStab (five launches per iteration)
//                when the reduced Poisson matrix is not symmetric
//   final        u = u* - dt dp/dx on facets and p += dp on cells, one launch
//                (hig-flow-step.c:242-340)
//
// The pinned pressure row (remove_pressure_singularity, hig-flow-step.c:14-45;
// slv_impose_value, solver.c:142-150) is eliminated from the other rows at
// create time, so the remaining matrix is symmetric on uniform meshes and the
// system is negated to make it positive definite for CG.
//
// Kernels that evaluate the reference's formulas are compiled without FMA
// contraction (-fmad=false), so the plain FP64 form reproduces the reference
// rounding sequence; only reduction order in the solver differs.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "hf_amg.cuh"
#include "hf_device.cuh"
#include "higflow_b200.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

#define HF_CK(x)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (x);                                                             \
        if (e_ != cudaSuccess) return fail(HF_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr int kBlock = 256;

// ---------------------------------------------------------------------------
// device data
// ---------------------------------------------------------------------------
struct DevProg {
    int D, ncell, nf[3], off[4];
    hf_params par;
    const double *delta;
    hf::Rows<double> rows;
    hf::Rows<float> rows32;
    const int32_t *vslots[3];
    const uint32_t *vflags[3];
    const uint16_t *vdelta[3];
    int vns;
    const int32_t *dslots;
    const uint16_t *cdelta;
    const int32_t *cslots;
    const uint32_t *cflags;
    int cns;
    int pin;               // single-instance path: instance 0's pin and parameters (par)
    double pin_value;
    // per-instance parameters and element -> instance maps (batches)
    int ninst;
    const hf_params *ipar;
    const int32_t *cinst;
    const int32_t *finst[3];
    const double *ipinv;
};

struct DevFields {
    double *u[3], *us[3], *p, *dp, *F, *FU[3];
    double *K[9], *Knew[9], *S[9], *Du[9];
};

// Poisson operator in the reduced, negated form (see header comment).
struct DevMat {
    int n;
    const int32_t *ptr;
    const int32_t *col;
    const double *val;
    const float *val32;
    const double *dinv;
    const float *dinv32;
    const double *apin;   // A[i][pin] of the original rows (moved to the rhs)
    const double *brhs;   // boundary part of the original rhs
};

struct Scal {
    double rz, alpha, beta, pq, rr, bb, tol2, rho, rho1, omega, ts, tt;
    int done, iters, maxit, status;
    unsigned counter;
};

// ---------------------------------------------------------------------------
// reductions: block partials, finished by the last block in a fixed order
// ---------------------------------------------------------------------------
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (*sh)[kBlock / 32])
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[k][wid] = x;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double x = threadIdx.x < kBlock / 32 ? sh[k][threadIdx.x] : 0.0;
        if (wid == 0) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        }
        v[k] = x;  // valid in thread 0
    }
    __syncthreads();
}

// Returns true in every thread of the last block, with tot[] = grid sums.
template <int NV>
__device__ bool grid_sum(double (&v)[NV], double *partials, unsigned *counter, double (&tot)[NV])
{
    __shared__ double sh[NV][kBlock / 32];
    __shared__ bool last;
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) partials[(size_t)blockIdx.x * NV + k] = v[k];
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) acc[k] = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += kBlock) {
#pragma unroll
        for (int k = 0; k < NV; k++) acc[k] += ((volatile double *)partials)[(size_t)b * NV + k];
    }
    block_sum<NV>(acc, sh);
    __shared__ double bc[NV];
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) bc[k] = acc[k];
        *counter = 0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) tot[k] = bc[k];
    return true;
}

__device__ __forceinline__ bool finite(double x) { return isfinite(x); }

// ---------------------------------------------------------------------------
// velocity stage
// ---------------------------------------------------------------------------
template <int D, bool VE>
__global__ void __launch_bounds__(kBlock) k_velocity(DevProg P, DevFields F)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= P.off[D]) return;
    int d = 0;
#pragma unroll
    for (int k = 1; k < D; k++) d += (e >= P.off[k]);
    const int f = e - P.off[d];
    const int nf = P.nf[d];
    const int32_t *__restrict__ sl = P.vslots[d];
#define SL(s) __ldg(sl + (size_t)(s) * nf + f)
    const double *fd = P.delta + (size_t)__ldg(P.vdelta[d] + f) * D;
    const uint32_t fl = __ldg(P.vflags[d] + f);
    const hf::Rows<double> &R = P.rows;
    const hf_params &par = P.ipar[__ldg(P.finst[d] + f)];
    const double a = 1.7500, b = 0.3750, c = 0.7500, dd = 0.1250, ee = 0.2500;
    int convec = par.convecdiscrtype;
    const int second = par.secondconvecdiscrtype;
    double conv1 = 0.0, conv2 = 0.0;
    const double ufacet = F.u[d][f];
    double Fs = hf::query(R, SL(HF_V_FU), F.FU[d]);
    const double pl = hf::query(R, SL(HF_V_PL), F.p);
    const double pr = hf::query(R, SL(HF_V_PR), F.p);
    const double dpdx = (pr - pl) / (2.0 * 0.5 * fd[d]);
    const double Fl = hf::query(R, SL(HF_V_FL), F.F);
    const double Fr = hf::query(R, SL(HF_V_FR), F.F);
    Fs += (Fr + Fl) / 2.0;
    double v[D], dudxc[D], dudxr[D], dudxl[D], dudxrr[D], dudxll[D], du2dx2[D], vc[D];
#pragma unroll
    for (int d2 = 0; d2 < D; d2++) {
        dudxrr[d2] = 0.0;
        dudxll[d2] = 0.0;
        vc[d2] = 0.0;
        const int B = HF_V_BLK0 + HF_V_NB * d2;
        if (d2 == d) {
            v[d2] = ufacet;
        } else {
            const double vrr = hf::query(R, SL(B + HF_V_V4 + 0), F.u[d2]);
            const double vlr = hf::query(R, SL(B + HF_V_V4 + 1), F.u[d2]);
            const double vrl = hf::query(R, SL(B + HF_V_V4 + 2), F.u[d2]);
            const double vll = hf::query(R, SL(B + HF_V_V4 + 3), F.u[d2]);
            v[d2] = 0.25 * (vll + vlr + vrl + vrr);
        }
        const double ul = hf::query(R, SL(B + HF_V_UL), F.u[d]);
        const int infl = (fl >> (4 * d2 + 0)) & 1;
        if (infl == 0 && convec == HF_SECOND_ORDER) convec = HF_FIRST_ORDER;
        const double ur = hf::query(R, SL(B + HF_V_UR), F.u[d]);
        const int infr = (fl >> (4 * d2 + 1)) & 1;
        if (infr == 0 && convec == HF_SECOND_ORDER) convec = HF_FIRST_ORDER;
        dudxc[d2] = (ur - ul) / (2.0 * 1.0 * fd[d2]);
        dudxr[d2] = (ur - ufacet) / (1.0 * fd[d2]);
        dudxl[d2] = (ufacet - ul) / (1.0 * fd[d2]);
        const double urr = hf::query(R, SL(B + HF_V_URR), F.u[d]);
        const int infrr = (fl >> (4 * d2 + 3)) & 1;
        const double ull = hf::query(R, SL(B + HF_V_ULL), F.u[d]);
        const int infll = (fl >> (4 * d2 + 2)) & 1;
        if (convec == HF_SECOND_ORDER) {
            if (second == HF_QUICK) {
                dudxrr[d2] = (urr - ur) / (1.0 * fd[d2]);
                dudxll[d2] = (ul - ull) / (1.0 * fd[d2]);
            } else if (second == HF_CUBISTA) {
                const double vcr = hf::query(R, SL(B + HF_V_VCR), F.u[d2]);
                if (vcr > 0.0) {
                    if (HF_FLT_EQ(ur, ul)) {
                        conv1 = vcr * ufacet;
                    } else {
                        const double fi = (ufacet - ul) / (ur - ul);
                        if ((fi <= 0.0) || (fi >= 1.0)) {
                            conv1 = vcr * ufacet;
                        } else {
                            if (fi < b) conv1 = vcr * (a * ufacet - c * ul);
                            if ((fi >= b) && (fi <= c)) conv1 = vcr * (c * ufacet + b * ur - dd * ul);
                            if (fi > c) conv1 = vcr * (ee * ufacet + c * ur);
                        }
                    }
                } else {
                    if (HF_FLT_EQ(ufacet, urr)) {
                        conv1 = vcr * ur;
                    } else {
                        const double fi = (ur - urr) / (ufacet - urr);
                        if ((fi <= 0.0) || (fi >= 1.0)) {
                            conv1 = vcr * ur;
                        } else {
                            if (fi < b) conv1 = infrr == 1 ? vcr * (a * ur - c * urr) : vcr * ur;
                            if ((fi >= b) && (fi <= c)) conv1 = infrr == 1 ? vcr * (c * ur + b * ufacet - dd * urr) : vcr * ur;
                            if (fi > c) conv1 = vcr * (c * ufacet + ee * ur);
                        }
                    }
                }
                const double vcl = hf::query(R, SL(B + HF_V_VCL), F.u[d2]);
                if (vcl > 0.0) {
                    if (HF_FLT_EQ(ufacet, ull)) {
                        conv2 = vcl * ul;
                    } else {
                        const double fi = (ul - ull) / (ufacet - ull);
                        if ((fi <= 0.0) || (fi >= 1.0)) {
                            conv2 = vcl * ul;
                        } else {
                            if (fi < b) conv2 = infll == 1 ? vcl * (a * ul - c * ull) : vcl * ul;
                            if ((fi >= b) && (fi <= c)) conv2 = infll == 1 ? vcl * (b * ufacet + c * ul - dd * ull) : vcl * ul;
                            if (fi > c) conv2 = vcl * (c * ufacet + ee * ul);
                        }
                    }
                } else {
                    if (HF_FLT_EQ(ul, ur)) {
                        conv2 = vcl * ufacet;
                    } else {
                        const double fi = (ufacet - ur) / (ul - ur);
                        if ((fi <= 0.0) || (fi >= 1.0)) {
                            conv2 = vcl * ufacet;
                        } else {
                            if (fi < b) conv2 = vcl * (a * ufacet - c * ur);
                            if ((fi >= b) && (fi <= c)) conv2 = vcl * (b * ul + c * ufacet - dd * ur);
                            if (fi > c) conv2 = vcl * (c * ul + ee * ufacet);
                        }
                    }
                }
                vc[d2] = ((conv1 - conv2) / fd[d]);
            }
        }
        du2dx2[d2] = (ul - 2.0 * ufacet + ur) / (fd[d2] * fd[d2] * 1.0 * 1.0);
    }
    double tens = 0.0;
    if (VE) {
        double dSdx[D];
#pragma unroll
        for (int d2 = 0; d2 < D; d2++) {
            const int B = HF_V_NSLOT_NEWT(D) + HF_V_NS * d2;
            const double *Sf = F.S[d * D + d2];
            if (d2 == d) {
                const double Sl = hf::query(R, SL(B + 0), Sf);
                const double Sr = hf::query(R, SL(B + 2), Sf);
                dSdx[d2] = (Sr - Sl) / (2.0 * 0.5 * fd[d2]);
            } else {
                const double l1 = hf::query(R, SL(B + 0), Sf);
                const double l2 = hf::query(R, SL(B + 1), Sf);
                const double Sl = 0.5 * (l1 + l2);
                const double r1 = hf::query(R, SL(B + 2), Sf);
                const double r2 = hf::query(R, SL(B + 3), Sf);
                const double Sr = 0.5 * (r1 + r2);
                dSdx[d2] = (Sr - Sl) / (2.0 * 1.0 * fd[d2]);
            }
        }
#pragma unroll
        for (int d2 = 0; d2 < D; d2++) tens += dSdx[d2];
    }
#undef SL
    const double pterm = par.projtype == HF_INCREMENTAL ? dpdx : 0.0;
    double conv = 0.0;
    if (convec == HF_CENTRAL) {
#pragma unroll
        for (int d2 = 0; d2 < D; d2++) conv += v[d2] * dudxc[d2];
    } else if (convec == HF_FIRST_ORDER) {
#pragma unroll
        for (int d2 = 0; d2 < D; d2++) {
            conv += 0.5 * (v[d2] + fabs(v[d2])) * dudxl[d2];
            conv += 0.5 * (v[d2] - fabs(v[d2])) * dudxr[d2];
        }
    } else if (second == HF_CUBISTA) {
#pragma unroll
        for (int d2 = 0; d2 < D; d2++) conv += vc[d2];
    } else if (second == HF_QUICK) {
#pragma unroll
        for (int d2 = 0; d2 < D; d2++) {
            conv += (v[d2] + fabs(v[d2])) * 0.1875 * dudxl[d2];
            conv += (v[d2] + fabs(v[d2])) * 0.3750 * dudxr[d2];
            conv -= (v[d2] + fabs(v[d2])) * 0.0625 * dudxrr[d2];
            conv += (v[d2] - fabs(v[d2])) * 0.3750 * dudxl[d2];
            conv += (v[d2] - fabs(v[d2])) * 0.1875 * dudxr[d2];
            conv -= (v[d2] - fabs(v[d2])) * 0.0625 * dudxll[d2];
        }
    } else {
#pragma unroll
        for (int d2 = 0; d2 < D; d2++) {
            conv += 0.5 * (v[d2] + fabs(v[d2])) * dudxl[d2];
            conv += 0.5 * (v[d2] - fabs(v[d2])) * dudxr[d2];
            if (v[d2] > 0.0) {
                if (fabs(dudxl[d2]) > 1.0e-8) conv += 0.5 * v[d2] * fd[d2] * du2dx2[d2] / dudxl[d2];
            } else {
                if (fabs(dudxr[d2]) > 1.0e-8) conv -= 0.5 * v[d2] * fd[d2] * du2dx2[d2] / dudxr[d2];
            }
        }
    }
    double diff = 0.0;
#pragma unroll
    for (int d2 = 0; d2 < D; d2++) diff += du2dx2[d2];
    diff /= par.Re;
    double rhs = 0.0;
    if (!VE) {
        rhs -= pterm;
        rhs -= conv;
        rhs += diff;
        rhs += Fs;
    } else {
        rhs += Fs;
        rhs -= pterm;
        rhs += tens;
        rhs -= conv;
        rhs += diff;
    }
    F.us[d][f] = ufacet + par.dt * rhs;
}

// ---------------------------------------------------------------------------
// viscoelastic cell stage (Du, constitutive update, polymeric tensor)
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(kBlock) k_ve_cell(DevProg P, DevFields F)
{
    const int cc = blockIdx.x * blockDim.x + threadIdx.x;
    if (cc >= P.ncell) return;
    const int n = P.ncell;
    const hf::Rows<double> &R = P.rows;
#define CS(s) __ldg(P.cslots + (size_t)(s) * n + cc)
    const double *cd = P.delta + (size_t)__ldg(P.cdelta + cc) * D;
    const uint32_t fl = __ldg(P.cflags + cc);
    const hf_params &pr = P.ipar[__ldg(P.cinst + cc)];
    // velocity at the faces of this cell, shared by Du, u_c and the CUBISTA flux
    double vl[D], vr[D];
#pragma unroll
    for (int dim = 0; dim < D; dim++) {
        const int B = HF_C_BLK0 + HF_C_NB * dim;
        vl[dim] = hf::query(R, CS(B + HF_C_UVL), F.u[dim]);
        vr[dim] = hf::query(R, CS(B + HF_C_UVR), F.u[dim]);
    }
    // Du (hig-flow-step-generalized-newtonian.c:30-64)
    double Du[D][D];
    {
        int pair = 0;
#pragma unroll
        for (int dim = 0; dim < D; dim++) {
#pragma unroll
            for (int dim2 = 0; dim2 < D; dim2++) {
                double ul, ur;
                if (dim == dim2) {
                    ul = vl[dim];
                    ur = vr[dim];
                } else {
                    const int Q = HF_C_BLK0 + HF_C_NB * D + HF_C_NQ * pair;
                    pair++;
                    double vrr = hf::query(R, CS(Q + 0), F.u[dim]);
                    double vll = hf::query(R, CS(Q + 1), F.u[dim]);
                    ul = 0.25 * (vll + vl[dim] + vr[dim] + vrr);
                    vrr = hf::query(R, CS(Q + 2), F.u[dim]);
                    vll = hf::query(R, CS(Q + 3), F.u[dim]);
                    ur = 0.25 * (vll + vl[dim] + vr[dim] + vrr);
                }
                Du[dim][dim2] = (ur - ul) / (2.0 * 0.5 * cd[dim2]);
                F.Du[dim * D + dim2][cc] = Du[dim][dim2];
            }
        }
    }
    // constitutive step (hig-flow-step-viscoelastic.c:384-521); the self slot
    // is the cell's own index (checked at create)
    const double Re = pr.Re, De = pr.De, tol = pr.kernel_tol, small = HF_EPSMACH;
    double S[D][D], K[D][D], KC[D][D];
    double trS = 0.0;
#pragma unroll
    for (int i = 0; i < D; i++) {
#pragma unroll
        for (int j = 0; j < D; j++) {
            S[i][j] = F.S[i * D + j][cc];
            K[i][j] = F.K[i * D + j][cc];
            KC[i][j] = K[i][j];
        }
        trS += S[i][i];
    }
    double Rm[D][D], Kl[D], lam[D];
    hf::jacobi<D>(KC, Kl, Rm);
#pragma unroll
    for (int dim = 0; dim < D; dim++) lam[dim] = hf::kernel_inverse(pr.kernel, Kl[dim]);
    double Mt[D][D], M[D][D];
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) {
            Mt[i][j] = Du[i][j];
            if (pr.ve_model == HF_LPTT) Mt[i][j] -= pr.xi * 0.5 * (Du[i][j] + Du[j][i]);
        }
    hf::mprod<D>(Mt, Rm, M);
    double Oa[D][D], Om[D][D];
#pragma unroll
    for (int i = 0; i < D - 1; i++) {
#pragma unroll
        for (int j = i + 1; j < D; j++) {
            Oa[i][j] = (M[i][j] * lam[j] + M[j][i] * lam[i]) / (lam[j] - lam[i] + small);
            Oa[j][i] = -Oa[i][j];
        }
        Oa[i][i] = 0.0;
    }
    Oa[D - 1][D - 1] = 0.0;
    hf::mtprod<D>(Oa, Rm, Om);
    double jl[D];
#pragma unroll
    for (int i = 0; i < D; i++) jl[i] = hf::kernel_jacobian(pr.kernel, lam[i], tol);
    double Ba[D][D], BB[D][D], Ma[D][D], MM[D][D];
#pragma unroll
    for (int i = 0; i < D; i++) {
#pragma unroll
        for (int j = i + 1; j < D; j++) {
            Ba[i][j] = 0.0; Ba[j][i] = 0.0;
            Ma[i][j] = 0.0; Ma[j][i] = 0.0;
        }
        Ba[i][i] = M[i][i] * lam[i] * jl[i];
        if (pr.ve_model == HF_GIESEKUS) {
            const double aux = 1.0 - lam[i];
            Ma[i][i] = (aux - pr.alpha * aux * aux) * jl[i];
        } else if (pr.ve_model == HF_LPTT) {
            Ma[i][i] = (1.0 - lam[i]) * (1.0 + (pr.epsilon * Re * De * trS) / (1.0 - pr.beta)) * jl[i];
        } else {
            Ma[i][i] = (1.0 - lam[i]) * jl[i];
        }
    }
    hf::mtprod<D>(Ba, Rm, BB);
    hf::mtprod<D>(Ma, Rm, MM);
    double RHS[D][D];
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) {
            double ok = 0.0, ko = 0.0;
#pragma unroll
            for (int k = 0; k < D; k++) {
                ok += Om[i][k] * K[k][j];
                ko += K[i][k] * Om[k][j];
            }
            RHS[i][j] = ok - ko + 2.0 * BB[i][j] + MM[i][j] / De;
        }
    double Knew[D][D];
#pragma unroll
    for (int i = 0; i < D; i++) {
#pragma unroll
        for (int j = i; j < D; j++) {
            const double *Kf = F.K[i * D + j];
            double rhs = 0.0;
#pragma unroll
            for (int dim = 0; dim < D; dim++) {
                const int B = HF_C_BLK0 + HF_C_NB * dim;
                const int il = (fl >> (4 * dim + 0)) & 1, ir = (fl >> (4 * dim + 1)) & 1;
                const int ill = (fl >> (4 * dim + 2)) & 1, irr = (fl >> (4 * dim + 3)) & 1;
                const double kl = hf::query(R, CS(B + HF_C_KL), Kf);
                const double kr = hf::query(R, CS(B + HF_C_KR), Kf);
                if (pr.ve_convecdiscrtype == HF_CELL_CUBISTA) {
                    const double kll = hf::query(R, CS(B + HF_C_KLL), Kf);
                    const double krr = hf::query(R, CS(B + HF_C_KRR), Kf);
                    rhs -= hf::cubista_cell(kl, kr, kll, krr, il, ir, ill, irr, vl[dim], vr[dim], K[i][j], cd[dim]);
                } else {
                    double dk;
                    if ((il == 1) && (ir == 1)) dk = (kr - kl) / (2.0 * 1.0 * cd[dim]);
                    else if (ir == 1) dk = (kr - K[i][j]) / (1.0 * cd[dim]);
                    else dk = (K[i][j] - kl) / (1.0 * cd[dim]);
                    const double uc = 0.5 * (vl[dim] + vr[dim]);
                    rhs -= uc * dk;
                }
            }
            rhs += RHS[i][j];
            const double kernel = K[i][j] + pr.dt * rhs;
            Knew[i][j] = kernel;
            Knew[j][i] = kernel;
        }
    }
#undef CS
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) F.Knew[i * D + j][cc] = Knew[i][j];
    // polymeric tensor from the new kernel (hig-flow-step-viscoelastic.c:244-318)
    double lam2[D], R2[D][D], Bk[D][D], A[D][D];
    hf::jacobi<D>(Knew, lam2, R2);
#pragma unroll
    for (int i = 0; i < D; i++) {
#pragma unroll
        for (int j = i + 1; j < D; j++) { Bk[i][j] = 0.0; Bk[j][i] = 0.0; }
        Bk[i][i] = hf::kernel_inverse(pr.kernel, lam2[i]);
    }
    hf::mtprod<D>(Bk, R2, A);
    const double fA = 1.0, aa = 1.0, beta = pr.beta;
    const double xi = pr.ve_model == HF_LPTT ? pr.xi : 0.0;
#pragma unroll
    for (int i = 0; i < D; i++) {
        double Si[D];
#pragma unroll
        for (int j = 0; j < D; j++) Si[j] = (1.0 - beta) * (fA * A[i][j]) / (Re * De * (1.0 - xi)) - (1.0 - beta) * Du[i][j] / Re;
        Si[i] += -aa * (1.0 - beta) / (Re * De * (1.0 - xi));
#pragma unroll
        for (int j = 0; j < D; j++) F.S[i * D + j][cc] = Si[j];
    }
}

// ---------------------------------------------------------------------------
// Poisson: divergence rhs + first CG residual
// ---------------------------------------------------------------------------
struct CGVec {
    double *x;    // solution (dp or p)
    double *r, *z, *pa, *pb, *q;
    double *partials;
    Scal *sc;
};

template <int D>
__global__ void __launch_bounds__(kBlock) k_cg_init(DevProg P, DevFields F, DevMat M, CGVec V, double rtol, double atol)
{
    const int cc = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = P.ncell;
    double part[3] = {0.0, 0.0, 0.0};  // r.z, r.r, b.b
    if (cc < n) {
        const double pinv = P.pin >= 0
            ? (P.par.projtype == HF_INCREMENTAL ? P.pin_value - F.p[P.pin] : P.pin_value) : 0.0;
        double borig;
        if (cc == P.pin) {
            borig = pinv;
        } else {
            const double *cd = P.delta + (size_t)__ldg(P.cdelta + cc) * D;
            double sumdudx = 0.0;
#pragma unroll
            for (int dim = 0; dim < D; dim++) {
                const double ustarl = hf::query(P.rows, __ldg(P.dslots + (size_t)HF_P_UL(dim) * n + cc), F.us[dim]);
                const double ustarr = hf::query(P.rows, __ldg(P.dslots + (size_t)HF_P_UR(dim) * n + cc), F.us[dim]);
                sumdudx += (ustarr - ustarl) / (2.0 * 0.5 * cd[dim]);
            }
            borig = sumdudx / P.par.dt + M.brhs[cc];
        }
        const double bred = cc == P.pin ? pinv : -(borig - M.apin[cc] * pinv);
        double ax = 0.0;
        for (int k = M.ptr[cc]; k < M.ptr[cc + 1]; k++) ax += M.val[k] * V.x[M.col[k]];
        const double r = bred - ax;
        const double z = M.dinv[cc] * r;
        V.r[cc] = r;
        V.z[cc] = z;
        part[0] = r * z;
        part[1] = r * r;
        part[2] = borig * borig;
    }
    double tot[3];
    if (grid_sum<3>(part, V.partials, &V.sc->counter, tot) && threadIdx.x == 0) {
        Scal &s = *V.sc;
        s.rz = tot[0];
        s.rr = tot[1];
        s.bb = tot[2];
        const double t = fmax(rtol * sqrt(tot[2]), atol);
        s.tol2 = t * t;
        s.beta = 0.0;
        s.iters = 0;
        s.status = 0;
        s.done = !(tot[1] > s.tol2);
        if (!finite(tot[0]) || !finite(tot[1]) || !finite(tot[2])) { s.status = HF_ERR_NAN; s.done = 1; }
    }
}

// p_new = z + beta p_old ; q = M p_new ; alpha = rz / (p_new . q)
__global__ void __launch_bounds__(kBlock) k_cg_dir_spmv(DevMat M, CGVec V, const double *__restrict__ po, double *__restrict__ pn)
{
    if (V.sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double beta = V.sc->beta;
    const bool first = V.sc->iters == 0;
    double part[1] = {0.0};
    if (i < M.n) {
        double q = 0.0;
        if (first) {
            for (int k = M.ptr[i]; k < M.ptr[i + 1]; k++) q += M.val[k] * V.z[M.col[k]];
            pn[i] = V.z[i];
        } else {
            for (int k = M.ptr[i]; k < M.ptr[i + 1]; k++) {
                const int j = M.col[k];
                q += M.val[k] * (V.z[j] + beta * po[j]);
            }
            pn[i] = V.z[i] + beta * po[i];
        }
        V.q[i] = q;
        part[0] = pn[i] * q;
    }
    double tot[1];
    if (grid_sum<1>(part, V.partials, &V.sc->counter, tot) && threadIdx.x == 0) {
        Scal &s = *V.sc;
        s.pq = tot[0];
        if (!(tot[0] > 0.0) || !finite(tot[0])) {
            // p.q <= 0: the recurrence has reached rounding level.  Accept when
            // the residual is within 100x of the target, else report it.
            s.status = !finite(tot[0]) ? HF_ERR_NAN : (s.rr <= 1e4 * s.tol2 ? 0 : HF_ERR_NOT_CONVERGED);
            s.done = 1;
        } else {
            s.alpha = s.rz / tot[0];
        }
    }
}

// x += alpha p ; r -= alpha q ; z = D^-1 r ; beta = rz_new / rz
__global__ void __launch_bounds__(kBlock) k_cg_update(DevMat M, CGVec V, const double *__restrict__ pn)
{
    if (V.sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double alpha = V.sc->alpha;
    double part[2] = {0.0, 0.0};
    if (i < M.n) {
        V.x[i] += alpha * pn[i];
        const double r = V.r[i] - alpha * V.q[i];
        const double z = M.dinv[i] * r;
        V.r[i] = r;
        V.z[i] = z;
        part[0] = r * z;
        part[1] = r * r;
    }
    double tot[2];
    if (grid_sum<2>(part, V.partials, &V.sc->counter, tot) && threadIdx.x == 0) {
        Scal &s = *V.sc;
        s.beta = tot[0] / s.rz;
        s.rz = tot[0];
        s.rr = tot[1];
        s.iters += 1;
        if (!finite(tot[0]) || !finite(tot[1])) { s.status = HF_ERR_NAN; s.done = 1; }
        else if (!(tot[1] > s.tol2)) s.done = 1;
        else if (s.iters >= s.maxit) { s.status = HF_ERR_NOT_CONVERGED; s.done = 1; }
    }
}

// ---------------------------------------------------------------------------
// CG preconditioned by an AMG V-cycle (hf_amg.cuh): the residual update and the
// preconditioner are separate launches; the last V-cycle kernel on the finest
// level finishes r.z and the CG beta.
// ---------------------------------------------------------------------------
constexpr int kMaxLevels = 20;

struct DevCSR {
    int n;
    const int32_t *ptr;
    const int32_t *col;
    const double *val;
};

struct DevLevel {
    DevCSR A, P, R;
    const double *dinv;
    double *b, *x, *r, *out;
};

struct DevAMG {
    int nlev;        // levels with a smoother; the coarsest has a dense inverse
    DevLevel lev[kMaxLevels];
    int cn;
    const double *cinv;
    double *cb, *cx;
};

constexpr double kSmoothW = 2.0 / 3.0;

__device__ __forceinline__ double csr_row(const DevCSR &A, int i, const double *__restrict__ x)
{
    double s = 0.0;
    for (int k = A.ptr[i]; k < A.ptr[i + 1]; k++) s += A.val[k] * x[A.col[k]];
    return s;
}

__global__ void __launch_bounds__(kBlock) k_vc_smooth0(DevLevel L, const Scal *sc)
{
    if (sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.A.n) L.x[i] = kSmoothW * L.dinv[i] * L.b[i];
}

__global__ void __launch_bounds__(kBlock) k_vc_residual(DevLevel L, const Scal *sc)
{
    if (sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.A.n) L.r[i] = L.b[i] - csr_row(L.A, i, L.x);
}

// b_next = R r
__global__ void __launch_bounds__(kBlock) k_vc_restrict(DevCSR R, const double *__restrict__ r, double *bn, const Scal *sc)
{
    if (sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < R.n) bn[i] = csr_row(R, i, r);
}

// x = inv b on the coarsest level (dense, row-major)
__global__ void __launch_bounds__(kBlock) k_vc_coarse(int n, const double *__restrict__ inv, const double *__restrict__ b,
                                                    double *x, const Scal *sc)
{
    if (sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int k = 0; k < n; k++) s += inv[(size_t)i * n + k] * b[k];
    x[i] = s;
}

// x += P e
__global__ void __launch_bounds__(kBlock) k_vc_prolong(DevLevel L, const double *__restrict__ e, const Scal *sc)
{
    if (sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.P.n) L.x[i] += csr_row(L.P, i, e);
}

// out = x + w D^-1 (b - A x)
__global__ void __launch_bounds__(kBlock) k_vc_post(DevLevel L, const Scal *sc)
{
    if (sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.A.n) L.out[i] = L.x[i] + kSmoothW * L.dinv[i] * (L.b[i] - csr_row(L.A, i, L.x));
}

// finest-level post-smoothing writes z and finishes r.z -> beta
__global__ void __launch_bounds__(kBlock) k_vc_post_fine(DevLevel L, CGVec V)
{
    if (V.sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double part[1] = {0.0};
    if (i < L.A.n) {
        const double z = L.x[i] + kSmoothW * L.dinv[i] * (L.b[i] - csr_row(L.A, i, L.x));
        V.z[i] = z;
        part[0] = L.b[i] * z;   // b of the finest level is the CG residual
    }
    double tot[1];
    if (grid_sum<1>(part, V.partials, &V.sc->counter, tot) && threadIdx.x == 0) {
        Scal &s = *V.sc;
        if (s.iters == 0) s.beta = 0.0;
        else s.beta = tot[0] / s.rz;
        s.rz = tot[0];
        if (!finite(tot[0])) { s.status = HF_ERR_NAN; s.done = 1; }
    }
}

// first residual of the AMG-preconditioned solve (z comes from the V-cycle)
template <int D>
__global__ void __launch_bounds__(kBlock) k_pcg_init(DevProg P, DevFields F, DevMat M, CGVec V, double rtol, double atol)
{
    const int cc = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = P.ncell;
    double part[2] = {0.0, 0.0};  // r.r, b.b
    if (cc < n) {
        const double pinv = P.pin >= 0
            ? (P.par.projtype == HF_INCREMENTAL ? P.pin_value - F.p[P.pin] : P.pin_value) : 0.0;
        double borig;
        if (cc == P.pin) {
            borig = pinv;
        } else {
            const double *cd = P.delta + (size_t)__ldg(P.cdelta + cc) * D;
            double sumdudx = 0.0;
#pragma unroll
            for (int dim = 0; dim < D; dim++) {
                const double ustarl = hf::query(P.rows, __ldg(P.dslots + (size_t)HF_P_UL(dim) * n + cc), F.us[dim]);
                const double ustarr = hf::query(P.rows, __ldg(P.dslots + (size_t)HF_P_UR(dim) * n + cc), F.us[dim]);
                sumdudx += (ustarr - ustarl) / (2.0 * 0.5 * cd[dim]);
            }
            borig = sumdudx / P.par.dt + M.brhs[cc];
        }
        const double bred = cc == P.pin ? pinv : -(borig - M.apin[cc] * pinv);
        double ax = 0.0;
        for (int k = M.ptr[cc]; k < M.ptr[cc + 1]; k++) ax += M.val[k] * V.x[M.col[k]];
        const double r = bred - ax;
        V.r[cc] = r;
        part[0] = r * r;
        part[1] = borig * borig;
    }
    double tot[2];
    if (grid_sum<2>(part, V.partials, &V.sc->counter, tot) && threadIdx.x == 0) {
        Scal &s = *V.sc;
        s.rr = tot[0];
        s.bb = tot[1];
        const double t = fmax(rtol * sqrt(tot[1]), atol);
        s.tol2 = t * t;
        s.beta = 0.0;
        s.iters = 0;
        s.status = 0;
        s.done = !(tot[0] > s.tol2);
        if (!finite(tot[0]) || !finite(tot[1])) { s.status = HF_ERR_NAN; s.done = 1; }
    }
}

// x += alpha p ; r -= alpha q ; convergence on ||r||
__global__ void __launch_bounds__(kBlock) k_pcg_update(DevMat M, CGVec V, const double *__restrict__ pn)
{
    if (V.sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double alpha = V.sc->alpha;
    double part[1] = {0.0};
    if (i < M.n) {
        V.x[i] += alpha * pn[i];
        const double r = V.r[i] - alpha * V.q[i];
        V.r[i] = r;
        part[0] = r * r;
    }
    double tot[1];
    if (grid_sum<1>(part, V.partials, &V.sc->counter, tot) && threadIdx.x == 0) {
        Scal &s = *V.sc;
        s.rr = tot[0];
        s.iters += 1;
        if (!finite(tot[0])) { s.status = HF_ERR_NAN; s.done = 1; }
        else if (!(tot[0] > s.tol2)) s.done = 1;
        else if (s.iters >= s.maxit) { s.status = HF_ERR_NOT_CONVERGED; s.done = 1; }
    }
}

// ---------------------------------------------------------------------------
// BiCGStab on the same operator (non-symmetric rows, e.g. AMR interfaces)
// ---------------------------------------------------------------------------
struct BiVec {
    double *x, *b, *r, *rh, *p, *v, *s, *t, *ph, *sh;
    double *partials;
    Scal *sc;
};

template <int D>
__global__ void __launch_bounds__(kBlock) k_bi_init(DevProg P, DevFields F, DevMat M, BiVec V, double rtol, double atol, int from_step)
{
    const int cc = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = M.n;
    double part[3] = {0.0, 0.0, 0.0};  // r.r, b.b, rh.r
    if (cc < n) {
        double bred, borig;
        if (from_step) {
            const double pinv = P.pin >= 0
                ? (P.par.projtype == HF_INCREMENTAL ? P.pin_value - F.p[P.pin] : P.pin_value) : 0.0;
            if (cc == P.pin) {
                borig = pinv;
            } else {
                const double *cd = P.delta + (size_t)__ldg(P.cdelta + cc) * D;
                double sumdudx = 0.0;
#pragma unroll
                for (int dim = 0; dim < D; dim++) {
                    const double ustarl = hf::query(P.rows, __ldg(P.dslots + (size_t)HF_P_UL(dim) * n + cc), F.us[dim]);
                    const double ustarr = hf::query(P.rows, __ldg(P.dslots + (size_t)HF_P_UR(dim) * n + cc), F.us[dim]);
                    sumdudx += (ustarr - ustarl) / (2.0 * 0.5 * cd[dim]);
                }
                borig = sumdudx / P.par.dt + M.brhs[cc];
            }
            bred = cc == P.pin ? pinv : -(borig - M.apin[cc] * pinv);
            V.b[cc] = bred;  // kept for restarts
        } else {
            bred = V.b[cc];
            borig = bred;
        }
        double ax = 0.0;
        for (int k = M.ptr[cc]; k < M.ptr[cc + 1]; k++) ax += M.val[k] * V.x[M.col[k]];
        const double r = bred - ax;
        V.r[cc] = r;
        V.rh[cc] = r;
        V.p[cc] = 0.0;
        V.v[cc] = 0.0;
        part[0] = r * r;
        part[1] = borig * borig;
        part[2] = r * r;
    }
    double tot[3];
    if (grid_sum<3>(part, V.partials, &V.sc->counter, tot) && threadIdx.x == 0) {
        Scal &s = *V.sc;
        s.rr = tot[0];
        if (from_step) {
            s.bb = tot[1];
            const double t = fmax(rtol * sqrt(tot[1]), atol);
            s.tol2 = t * t;
            s.iters = 0;
        }
        s.rho = 1.0;
        s.alpha = 1.0;
        s.omega = 1.0;
        s.rho1 = tot[2];
        s.beta = 0.0;
        s.status = 0;
        s.done = !(tot[0] > s.tol2);
        if (!finite(tot[0])) { s.status = HF_ERR_NAN; s.done = 1; }
    }
}

__global__ void __launch_bounds__(kBlock) k_bi_p(DevMat M, BiVec V)
{
    if (V.sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M.n) return;
    const double beta = V.sc->beta, omega = V.sc->omega;
    const double p = V.r[i] + beta * (V.p[i] - omega * V.v[i]);
    V.p[i] = p;
    V.ph[i] = M.dinv[i] * p;
}

// y = A x ; partial dots -> scalars (which: 0 -> alpha, 1 -> omega)
__global__ void __launch_bounds__(kBlock) k_bi_spmv(DevMat M, BiVec V, const double *__restrict__ x, double *__restrict__ y, int which)
{
    if (V.sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double part[2] = {0.0, 0.0};
    if (i < M.n) {
        double acc = 0.0;
        for (int k = M.ptr[i]; k < M.ptr[i + 1]; k++) acc += M.val[k] * x[M.col[k]];
        y[i] = acc;
        if (which == 0) {
            part[0] = V.rh[i] * acc;
        } else {
            part[0] = acc * V.s[i];
            part[1] = acc * acc;
        }
    }
    double tot[2];
    if (grid_sum<2>(part, V.partials, &V.sc->counter, tot) && threadIdx.x == 0) {
        Scal &s = *V.sc;
        if (which == 0) {
            if (tot[0] == 0.0 || !finite(tot[0])) { s.status = finite(tot[0]) ? 1 : HF_ERR_NAN; s.done = 1; }
            else s.alpha = s.rho1 / tot[0];
        } else {
            s.omega = tot[1] > 0.0 ? tot[0] / tot[1] : 0.0;
            if (!finite(s.omega)) { s.status = HF_ERR_NAN; s.done = 1; }
        }
    }
}

__global__ void __launch_bounds__(kBlock) k_bi_s(DevMat M, BiVec V)
{
    if (V.sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M.n) return;
    const double s = V.r[i] - V.sc->alpha * V.v[i];
    V.s[i] = s;
    V.sh[i] = M.dinv[i] * s;
}

__global__ void __launch_bounds__(kBlock) k_bi_update(DevMat M, BiVec V)
{
    if (V.sc->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double alpha = V.sc->alpha, omega = V.sc->omega;
    double part[2] = {0.0, 0.0};
    if (i < M.n) {
        V.x[i] += alpha * V.ph[i] + omega * V.sh[i];
        const double r = V.s[i] - omega * V.t[i];
        V.r[i] = r;
        part[0] = r * r;
        part[1] = V.rh[i] * r;
    }
    double tot[2];
    if (grid_sum<2>(part, V.partials, &V.sc->counter, tot) && threadIdx.x == 0) {
        Scal &s = *V.sc;
        s.rr = tot[0];
        s.rho = s.rho1;
        s.rho1 = tot[1];
        s.iters += 1;
        if (!finite(tot[0])) { s.status = HF_ERR_NAN; s.done = 1; }
        else if (!(tot[0] > s.tol2)) s.done = 1;
        else if (s.iters >= s.maxit) { s.status = HF_ERR_NOT_CONVERGED; s.done = 1; }
        else if (s.rho1 == 0.0 || s.omega == 0.0) { s.status = 1; s.done = 1; }  // breakdown: restart
        else s.beta = (s.rho1 / s.rho) * (s.alpha / s.omega);
    }
}

// ---------------------------------------------------------------------------
// final velocity and pressure
// ---------------------------------------------------------------------------
template <int D>
__global__ void __launch_bounds__(kBlock) k_final(DevProg P, DevFields F)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < P.off[D]) {
        int d = 0;
#pragma unroll
        for (int k = 1; k < D; k++) d += (e >= P.off[k]);
        const int f = e - P.off[d];
        const int nf = P.nf[d];
        const hf_params &par = P.ipar[__ldg(P.finst[d] + f)];
        const double *pp = par.projtype == HF_INCREMENTAL ? F.dp : F.p;
        const double *fd = P.delta + (size_t)__ldg(P.vdelta[d] + f) * D;
        const double pl = hf::query(P.rows, __ldg(P.vslots[d] + (size_t)HF_V_PL * nf + f), pp);
        const double pr = hf::query(P.rows, __ldg(P.vslots[d] + (size_t)HF_V_PR * nf + f), pp);
        const double dpdx = (pr - pl) / (2.0 * 0.5 * fd[d]);
        F.u[d][f] = F.us[d][f] - par.dt * dpdx;
    } else {
        const int c = e - P.off[D];
        if (c < P.ncell && P.ipar[__ldg(P.cinst + c)].projtype == HF_INCREMENTAL) F.p[c] = F.p[c] + F.dp[c];
    }
}

#include "hf_batch.cuh"

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int blocks(long n) { return (int)((n + kBlock - 1) / kBlock); }

template <typename T>
int upload(std::vector<void *> &owned, T **dst, const T *src, size_t n, double &bytes)
{
    *dst = nullptr;
    size_t nb = sizeof(T) * (n ? n : 1);
    HF_CK(cudaMalloc((void **)dst, nb));
    owned.push_back(*dst);
    bytes += (double)nb;
    if (n && src) HF_CK(cudaMemcpy(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice));
    else HF_CK(cudaMemset(*dst, 0, nb));
    return HF_OK;
}

}  // namespace

struct hf_case {
    hf_options opt;
    hf_params par;
    int D;
    DevProg P;
    DevFields F;
    DevMat M;
    CGVec cg;
    BiVec bi;
    bool use_cg;
    bool use_amg = false;
    DevAMG amg{};
    int amg_levels = 0;
    // instances and the persistent per-instance Poisson solver (hf_batch.cuh)
    int ninst = 1;
    std::vector<int> coff;          // ninst + 1
    std::vector<int> foff[3];       // ninst + 1 per direction
    bool persistent = false;
    InstSolve *d_inst = nullptr;
    ILevel<double> *d_l64 = nullptr;
    ILevel<float> *d_l32 = nullptr;
    int *d_res_i = nullptr;         // iters, outer, status per instance (3 * ninst)
    double *d_res_d = nullptr;      // residual per instance
    int *h_res_i = nullptr;         // pinned mirrors
    double *h_res_d = nullptr;
    int64_t batch_levels = 0;
    std::vector<void *> owned;
    cudaStream_t stream = nullptr;
    Scal *h_scal = nullptr;   // pinned host mirror
    hf_stats stats;
    double bytes = 0;
    int nfacet_total = 0;
    // optional per-phase timing with CUDA events on the engine stream
    bool profile = false;
    cudaEvent_t ev[2 * HF_NPHASE] = {};
    double phase_ms[HF_NPHASE] = {};
    int64_t phase_launches[HF_NPHASE] = {};
};

namespace {

struct PhaseTimer {
    hf_case *C;
    int phase;
    int64_t launches0;
    PhaseTimer(hf_case *c, int p, int64_t l) : C(c), phase(p), launches0(l)
    {
        if (C->profile) cudaEventRecord(C->ev[2 * p], C->stream);
    }
    void stop(int64_t launches)
    {
        if (!C->profile) return;
        cudaEventRecord(C->ev[2 * phase + 1], C->stream);
        cudaEventSynchronize(C->ev[2 * phase + 1]);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, C->ev[2 * phase], C->ev[2 * phase + 1]);
        C->phase_ms[phase] += ms;
        C->phase_launches[phase] += launches - launches0;
    }
};

}  // namespace

namespace {

// Build the reduced, negated Poisson operator on the host.
int build_matrix(const hf_program *pg, const std::vector<int> &pins, std::vector<int32_t> &ptr, std::vector<int32_t> &col,
                 std::vector<double> &val, std::vector<double> &dinv, std::vector<double> &apin, bool &symmetric)
{
    const int n = pg->ncell;
    std::vector<char> pinned(n, 0);
    for (int p : pins)
        if (p >= 0) pinned[p] = 1;
    ptr.assign(n + 1, 0);
    col.clear();
    val.clear();
    dinv.assign(n, 1.0);
    apin.assign(n, 0.0);
    for (int r = 0; r < n; r++) {
        if (pinned[r]) {
            col.push_back(r);
            val.push_back(1.0);
        } else {
            double diag = 0.0;
            for (int64_t k = pg->p_ptr[r]; k < pg->p_ptr[r + 1]; k++) {
                int c = pg->p_col[k];
                if (c < 0 || c >= n) return fail(HF_ERR_INVALID, "Poisson column out of range");
                double v = pg->p_val[k];
                if (pinned[c]) { apin[r] += v; continue; }   // a row only reaches its own instance's pin
                col.push_back(c);
                val.push_back(-v);
                if (c == r) diag += -v;
            }
            if (!(diag > 0.0)) return fail(HF_ERR_INVALID, "Poisson row without a positive diagonal");
            dinv[r] = 1.0 / diag;
        }
        if (col.size() > (size_t)INT32_MAX) return fail(HF_ERR_UNSUPPORTED, "Poisson matrix too large for int32 indexing");
        ptr[r + 1] = (int32_t)col.size();
    }
    // symmetry check: every (r, c, v) must have a matching (c, r, v)
    symmetric = true;
    for (int r = 0; r < n && symmetric; r++) {
        for (int k = ptr[r]; k < ptr[r + 1]; k++) {
            int c = col[k];
            if (c == r) continue;
            bool found = false;
            for (int m = ptr[c]; m < ptr[c + 1]; m++)
                if (col[m] == r) {
                    found = fabs(val[m] - val[k]) <= 1e-13 * fabs(val[k]);
                    break;
                }
            if (!found) { symmetric = false; break; }
        }
    }
    return HF_OK;
}

int check_program(const hf_program *pg)
{
    if (!pg) return fail(HF_ERR_INVALID, "null program");
    const int D = pg->par.dim;
    if (D != 2 && D != 3) return fail(HF_ERR_INVALID, "dim must be 2 or 3");
    if (pg->par.flowtype != HF_NEWTONIAN && pg->par.flowtype != HF_VISCOELASTIC)
        return fail(HF_ERR_UNSUPPORTED, "flow type");
    const bool ve = pg->par.flowtype == HF_VISCOELASTIC;
    if (pg->vel_nslot != (ve ? HF_V_NSLOT_VE(D) : HF_V_NSLOT_NEWT(D))) return fail(HF_ERR_INVALID, "velocity slot count");
    if (ve && pg->cell_nslot != HF_C_NSLOT(D)) return fail(HF_ERR_INVALID, "cell slot count");
    if (pg->ncell <= 0) return fail(HF_ERR_INVALID, "empty mesh");
    if (pg->pin_row >= pg->ncell) return fail(HF_ERR_INVALID, "pin row out of range");
    // every code must address its field or a row
    auto okcode = [&](int32_t c, int64_t nfield) {
        return c >= 0 ? (int64_t)c < nfield : (-(int64_t)c - 1) < pg->nrows;
    };
    for (int64_t k = 0; k < pg->nnz; k++)
        if (pg->tmpl_col[k] < 0) return fail(HF_ERR_INVALID, "negative template column");
    for (int64_t r = 0; r < pg->nrows; r++)
        if (pg->row_tmpl[r] < 0 || pg->row_tmpl[r] >= pg->ntmpl || pg->row_base[r] < 0)
            return fail(HF_ERR_INVALID, "row template/base out of range");
    for (int64_t t = 0; t < pg->ntmpl; t++)
        if (pg->tmpl_ptr[t + 1] < pg->tmpl_ptr[t] || pg->tmpl_ptr[t + 1] > pg->nnz) return fail(HF_ERR_INVALID, "template pointer");
    for (int d = 0; d < D; d++) {
        const int64_t nf = pg->nfacet[d];
        for (int s = 0; s < pg->vel_nslot; s++) {
            // field of slot s: FU/V4/UL.../VC: facets of some direction, PL/PR/FL/FR and S: cells
            int64_t nfield;
            if (s == HF_V_FU) nfield = pg->nfacet[d];
            else if (s <= HF_V_FR) nfield = pg->ncell;
            else if (s < HF_V_NSLOT_NEWT(D)) {
                int d2 = (s - HF_V_BLK0) / HF_V_NB, k = (s - HF_V_BLK0) % HF_V_NB;
                nfield = (k < 4 || k >= 8) ? pg->nfacet[d2] : pg->nfacet[d];
            } else nfield = pg->ncell;
            for (int64_t f = 0; f < nf; f++)
                if (!okcode(pg->vel_slots[d][s * nf + f], nfield)) return fail(HF_ERR_INVALID, "velocity slot out of range");
        }
        for (int64_t f = 0; f < nf; f++)
            if (pg->vel_delta[d][f] >= pg->ndelta) return fail(HF_ERR_INVALID, "delta index out of range");
    }
    for (int dim = 0; dim < D; dim++)
        for (int s = 0; s < 2; s++)
            for (int64_t c = 0; c < pg->ncell; c++)
                if (!okcode(pg->div_slots[(size_t)(2 * dim + s) * pg->ncell + c], pg->nfacet[dim]))
                    return fail(HF_ERR_INVALID, "divergence slot out of range");
    for (int64_t c = 0; c < pg->ncell; c++)
        if (pg->cell_delta[c] >= pg->ndelta) return fail(HF_ERR_INVALID, "cell delta index out of range");
    if (ve) {
        for (int64_t c = 0; c < pg->ncell; c++)
            if (pg->cell_slots[c] != c) return fail(HF_ERR_UNSUPPORTED, "tensor self query is not a centre hit");
        for (int s = 1; s < pg->cell_nslot; s++) {
            int64_t nfield;
            if (s < HF_C_BLK0 + HF_C_NB * D) {
                int dim = (s - HF_C_BLK0) / HF_C_NB, k = (s - HF_C_BLK0) % HF_C_NB;
                nfield = k < 2 ? pg->nfacet[dim] : pg->ncell;
            } else {
                int pair = (s - HF_C_BLK0 - HF_C_NB * D) / HF_C_NQ;
                int dim = pair / (D - 1);
                nfield = pg->nfacet[dim];
            }
            for (int64_t c = 0; c < pg->ncell; c++)
                if (!okcode(pg->cell_slots[(size_t)s * pg->ncell + c], nfield)) return fail(HF_ERR_INVALID, "cell slot out of range");
        }
    }
    for (int64_t k = 0; k < pg->nnz; k++) (void)k;
    return HF_OK;
}

// general rows may read any field: their columns must fit the smallest field
// they can be applied to; the engine checks against the largest field and the
// slot checks above bound the row index, so check columns against the field
// sizes per referencing slot instead.
int check_rows(const hf_program *pg)
{
    const int D = pg->par.dim;
    std::vector<int64_t> limit((size_t)pg->nrows, INT64_MAX);
    auto note = [&](int32_t code, int64_t nfield) {
        if (code < 0) {
            int64_t r = -(int64_t)code - 1;
            limit[r] = std::min(limit[r], nfield);
        }
    };
    for (int d = 0; d < D; d++) {
        const int64_t nf = pg->nfacet[d];
        for (int s = 0; s < pg->vel_nslot; s++) {
            int64_t nfield;
            if (s == HF_V_FU) nfield = pg->nfacet[d];
            else if (s <= HF_V_FR) nfield = pg->ncell;
            else if (s < HF_V_NSLOT_NEWT(D)) {
                int d2 = (s - HF_V_BLK0) / HF_V_NB, k = (s - HF_V_BLK0) % HF_V_NB;
                nfield = (k < 4 || k >= 8) ? pg->nfacet[d2] : pg->nfacet[d];
            } else nfield = pg->ncell;
            for (int64_t f = 0; f < nf; f++) note(pg->vel_slots[d][s * nf + f], nfield);
        }
    }
    for (int dim = 0; dim < D; dim++)
        for (int s = 0; s < 2; s++)
            for (int64_t c = 0; c < pg->ncell; c++) note(pg->div_slots[(size_t)(2 * dim + s) * pg->ncell + c], pg->nfacet[dim]);
    if (pg->par.flowtype == HF_VISCOELASTIC) {
        for (int s = 1; s < pg->cell_nslot; s++) {
            int64_t nfield;
            if (s < HF_C_BLK0 + HF_C_NB * D) {
                int dim = (s - HF_C_BLK0) / HF_C_NB, k = (s - HF_C_BLK0) % HF_C_NB;
                nfield = k < 2 ? pg->nfacet[dim] : pg->ncell;
            } else {
                int pair = (s - HF_C_BLK0 - HF_C_NB * D) / HF_C_NQ;
                nfield = pg->nfacet[pair / (D - 1)];
            }
            for (int64_t c = 0; c < pg->ncell; c++) note(pg->cell_slots[(size_t)s * pg->ncell + c], nfield);
        }
    }
    // largest column of each template, then base + max column < field size for every row
    std::vector<int64_t> tmax((size_t)pg->ntmpl, -1);
    for (int64_t t = 0; t < pg->ntmpl; t++)
        for (int64_t k = pg->tmpl_ptr[t]; k < pg->tmpl_ptr[t + 1]; k++) tmax[t] = std::max(tmax[t], (int64_t)pg->tmpl_col[k]);
    for (int64_t r = 0; r < pg->nrows; r++)
        if ((int64_t)pg->row_base[r] + tmax[pg->row_tmpl[r]] >= limit[r]) return fail(HF_ERR_INVALID, "row column out of its field");
    return HF_OK;
}

// Host staging for many small device arrays: one allocation, one copy.
struct Arena {
    std::vector<char> host;
    size_t add(const void *src, size_t bytes)
    {
        const size_t off = (host.size() + 255) & ~size_t(255);
        host.resize(off + (bytes ? bytes : 8), 0);
        if (src && bytes) memcpy(host.data() + off, src, bytes);
        return off;
    }
    template <typename T>
    size_t vec(const std::vector<T> &v) { return add(v.data(), v.size() * sizeof(T)); }
    template <typename T>
    size_t zeros(size_t n) { return add(nullptr, n * sizeof(T)); }
};

template <typename T>
std::vector<T> cast_vec(const std::vector<double> &v)
{
    return std::vector<T>(v.begin(), v.end());
}

// Per-instance AMG hierarchies and work vectors for the persistent solver.
int build_batch_solver(hf_case *C, const std::vector<int32_t> &mptr, const std::vector<int32_t> &mcol,
                       const std::vector<double> &mval, const double *apin_dev, const double *brhs_dev,
                       const std::vector<int> &pins, bool mixed)
{
    const int ni = C->ninst;
    struct LvlOff { int n; size_t Ap, Ac, Av, Av32, Pp, Pc, Pv, Pv32, Rp, Rc, Rv, Rv32, d, d32, x, b, r, out, x32, b32, r32, out32; };
    struct InstOff {
        int n, coff, nlev, cn, pin;
        size_t cinv, cinv32, cb, cx, cb32, cx32, b, r, z, p, q, r32a, e32, t32, z32, p32, q32;
        std::vector<LvlOff> lv;
    };
    Arena ar;
    std::vector<InstOff> io(ni);
    for (int i = 0; i < ni; i++) {
        InstOff &o = io[i];
        const int c0 = C->coff[i], n = C->coff[i + 1] - C->coff[i];
        o.n = n;
        o.coff = c0;
        o.pin = pins[i] >= 0 ? pins[i] - c0 : -1;
        hf::HostCSR A;
        A.n = A.m = n;
        A.ptr.assign(n + 1, 0);
        for (int r = 0; r < n; r++) {
            for (int k = mptr[c0 + r]; k < mptr[c0 + r + 1]; k++) {
                const int c = mcol[k] - c0;
                if (c < 0 || c >= n) return fail(HF_ERR_INVALID, "Poisson row reaches another instance");
                A.col.push_back(c);
                A.val.push_back(mval[k]);
            }
            A.ptr[r + 1] = (int)A.col.size();
        }
        std::vector<hf::HostLevel> H = hf::build_hierarchy(A, 64);
        const hf::HostCSR &Cc = H.back().A;
        if (Cc.n > 2048) return fail(HF_ERR_UNSUPPORTED, "AMG coarsening stalled above 2048 rows");
        std::vector<double> inv;
        if (!hf::dense_inverse(Cc, inv)) return fail(HF_ERR_INVALID, "singular coarsest AMG level");
        o.nlev = (int)H.size() - 1;
        o.cn = Cc.n;
        o.cinv = ar.vec(inv);
        o.cinv32 = mixed ? ar.vec(cast_vec<float>(inv)) : 0;
        o.cb = ar.zeros<double>(o.cn);
        o.cx = ar.zeros<double>(o.cn);
        o.cb32 = mixed ? ar.zeros<float>(o.cn) : 0;
        o.cx32 = mixed ? ar.zeros<float>(o.cn) : 0;
        const int nl = std::max(o.nlev, 1);
        for (int l = 0; l < nl; l++) {
            const hf::HostLevel &h = H[l];
            LvlOff L{};
            L.n = h.A.n;
            L.Ap = ar.vec(h.A.ptr);
            L.Ac = ar.vec(h.A.col);
            L.Av = ar.vec(h.A.val);
            L.d = ar.vec(h.dinv);
            if (l < o.nlev) {
                L.Pp = ar.vec(h.P.ptr); L.Pc = ar.vec(h.P.col); L.Pv = ar.vec(h.P.val);
                L.Rp = ar.vec(h.R.ptr); L.Rc = ar.vec(h.R.col); L.Rv = ar.vec(h.R.val);
            }
            L.x = ar.zeros<double>(L.n); L.b = ar.zeros<double>(L.n);
            L.r = ar.zeros<double>(L.n); L.out = ar.zeros<double>(L.n);
            if (mixed) {
                L.Av32 = ar.vec(cast_vec<float>(h.A.val));
                L.d32 = ar.vec(cast_vec<float>(h.dinv));
                if (l < o.nlev) { L.Pv32 = ar.vec(cast_vec<float>(h.P.val)); L.Rv32 = ar.vec(cast_vec<float>(h.R.val)); }
                L.x32 = ar.zeros<float>(L.n); L.b32 = ar.zeros<float>(L.n);
                L.r32 = ar.zeros<float>(L.n); L.out32 = ar.zeros<float>(L.n);
            }
            o.lv.push_back(L);
        }
        o.b = ar.zeros<double>(n); o.r = ar.zeros<double>(n); o.z = ar.zeros<double>(n);
        o.p = ar.zeros<double>(n); o.q = ar.zeros<double>(n);
        if (mixed) {
            o.r32a = ar.zeros<float>(n); o.e32 = ar.zeros<float>(n); o.t32 = ar.zeros<float>(n);
            o.z32 = ar.zeros<float>(n); o.p32 = ar.zeros<float>(n); o.q32 = ar.zeros<float>(n);
        }
        C->batch_levels += nl;
    }
    char *base = nullptr;
    HF_CK(cudaMalloc((void **)&base, ar.host.size()));
    C->owned.push_back(base);
    C->bytes += (double)ar.host.size();
    HF_CK(cudaMemcpy(base, ar.host.data(), ar.host.size(), cudaMemcpyHostToDevice));
    auto I = [&](size_t off) { return (int32_t *)(base + off); };
    auto Dp = [&](size_t off) { return (double *)(base + off); };
    auto Fp = [&](size_t off) { return mixed ? (float *)(base + off) : (float *)nullptr; };
    std::vector<ILevel<double>> l64;
    std::vector<ILevel<float>> l32;
    std::vector<InstSolve> is(ni);
    // largest instance first, so the longest solves start in the first wave
    std::vector<int> order(ni);
    for (int i = 0; i < ni; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return io[a].n > io[b].n; });
    for (int k = 0; k < ni; k++) {
        const int i = order[k];
        const InstOff &o = io[i];
        InstSolve &s = is[k];
        s.inst = i;
        s.n = o.n;
        s.coff = o.coff;
        s.nlev = o.nlev;
        s.lev = (int)l64.size();
        s.cn = o.cn;
        s.cinv64 = Dp(o.cinv);
        s.cinv32 = mixed ? (const float *)(base + o.cinv32) : nullptr;
        s.cb64 = Dp(o.cb); s.cx64 = Dp(o.cx);
        s.cb32 = Fp(o.cb32); s.cx32 = Fp(o.cx32);
        s.Mp = I(o.lv[0].Ap); s.Mc = I(o.lv[0].Ac); s.Mv = Dp(o.lv[0].Av);
        s.apin = apin_dev + o.coff;
        s.brhs = brhs_dev + o.coff;
        s.pin = o.pin;
        s.b = Dp(o.b); s.r = Dp(o.r); s.z = Dp(o.z); s.p = Dp(o.p); s.q = Dp(o.q);
        s.r32 = Fp(o.r32a); s.e32 = Fp(o.e32); s.t32 = Fp(o.t32);
        s.z32 = Fp(o.z32); s.p32 = Fp(o.p32); s.q32 = Fp(o.q32);
        s.iters = C->d_res_i + 3 * i;
        s.outer = C->d_res_i + 3 * i + 1;
        s.status = C->d_res_i + 3 * i + 2;
        s.res = C->d_res_d + i;
        for (const LvlOff &L : o.lv) {
            ILevel<double> a{};
            a.n = L.n;
            a.Ap = I(L.Ap); a.Ac = I(L.Ac); a.Av = Dp(L.Av);
            a.Pp = L.Pp ? I(L.Pp) : nullptr; a.Pc = L.Pc ? I(L.Pc) : nullptr; a.Pv = L.Pv ? Dp(L.Pv) : nullptr;
            a.Rp = L.Rp ? I(L.Rp) : nullptr; a.Rc = L.Rc ? I(L.Rc) : nullptr; a.Rv = L.Rv ? Dp(L.Rv) : nullptr;
            a.dinv = Dp(L.d);
            a.x = Dp(L.x); a.b = Dp(L.b); a.r = Dp(L.r); a.out = Dp(L.out);
            l64.push_back(a);
            ILevel<float> f{};
            if (mixed) {
                f.n = L.n;
                f.Ap = a.Ap; f.Ac = a.Ac; f.Av = Fp(L.Av32);
                f.Pp = a.Pp; f.Pc = a.Pc; f.Pv = L.Pv32 ? Fp(L.Pv32) : nullptr;
                f.Rp = a.Rp; f.Rc = a.Rc; f.Rv = L.Rv32 ? Fp(L.Rv32) : nullptr;
                f.dinv = Fp(L.d32);
                f.x = Fp(L.x32); f.b = Fp(L.b32); f.r = Fp(L.r32); f.out = Fp(L.out32);
            }
            l32.push_back(f);
        }
    }
    double bytes = 0;
    int rc;
    if ((rc = upload(C->owned, &C->d_inst, is.data(), is.size(), bytes))) return rc;
    if ((rc = upload(C->owned, &C->d_l64, l64.data(), l64.size(), bytes))) return rc;
    if ((rc = upload(C->owned, &C->d_l32, l32.data(), l32.size(), bytes))) return rc;
    C->bytes += bytes;
    return HF_OK;
}

// one V-cycle z = V(r) on the case stream (hf_amg.cuh)
int64_t launch_vcycle(hf_case *C)
{
    const DevAMG &A = C->amg;
    cudaStream_t st = C->stream;
    const Scal *sc = C->cg.sc;
    int64_t launches = 0;
    for (int l = 0; l < A.nlev; l++) {
        const DevLevel &L = A.lev[l];
        k_vc_smooth0<<<blocks(L.A.n), kBlock, 0, st>>>(L, sc);
        k_vc_residual<<<blocks(L.A.n), kBlock, 0, st>>>(L, sc);
        double *bn = l + 1 < A.nlev ? A.lev[l + 1].b : A.cb;
        k_vc_restrict<<<blocks(L.R.n), kBlock, 0, st>>>(L.R, L.r, bn, sc);
        launches += 3;
    }
    k_vc_coarse<<<blocks(A.cn), kBlock, 0, st>>>(A.cn, A.cinv, A.cb, A.cx, sc);
    launches++;
    for (int l = A.nlev - 1; l >= 0; l--) {
        const DevLevel &L = A.lev[l];
        const double *e = l + 1 < A.nlev ? A.lev[l + 1].out : A.cx;
        k_vc_prolong<<<blocks(L.P.n), kBlock, 0, st>>>(L, e, sc);
        if (l == 0) k_vc_post_fine<<<blocks(L.A.n), kBlock, 0, st>>>(L, C->cg);
        else k_vc_post<<<blocks(L.A.n), kBlock, 0, st>>>(L, sc);
        launches += 2;
    }
    return launches;
}

template <int D>
int launch_step(hf_case *C)
{
    cudaStream_t st = C->stream;
    const bool ve = C->par.flowtype == HF_VISCOELASTIC;
    int64_t launches = 0;
    if (ve) {
        PhaseTimer t(C, HF_PHASE_VE_CELL, launches);
        k_ve_cell<D><<<blocks(C->P.ncell), kBlock, 0, st>>>(C->P, C->F);
        launches++;
        for (int k = 0; k < D * D; k++) std::swap(C->F.K[k], C->F.Knew[k]);
        t.stop(launches);
    }
    {
        PhaseTimer t(C, HF_PHASE_VELOCITY, launches);
        if (ve) k_velocity<D, true><<<blocks(C->nfacet_total), kBlock, 0, st>>>(C->P, C->F);
        else k_velocity<D, false><<<blocks(C->nfacet_total), kBlock, 0, st>>>(C->P, C->F);
        launches++;
        t.stop(launches);
    }
    HF_CK(cudaGetLastError());
    const double rtol = C->opt.poisson_rtol, atol = C->opt.poisson_atol;
    const int n = C->P.ncell;
    int rc = HF_OK;
    if (C->persistent) {
        {
            PhaseTimer t(C, HF_PHASE_POISSON_ITER, launches);
            k_batch_poisson<D><<<C->ninst, kPB, 0, st>>>(C->P, C->F, C->d_inst, C->d_l64, C->d_l32,
                                                          C->opt.precision == HF_PREC_MIXED, rtol, atol,
                                                          C->opt.poisson_maxit);
            launches++;
            t.stop(launches);
        }
        HF_CK(cudaGetLastError());
        HF_CK(cudaMemcpyAsync(C->h_res_i, C->d_res_i, sizeof(int) * 3 * C->ninst, cudaMemcpyDeviceToHost, st));
        HF_CK(cudaMemcpyAsync(C->h_res_d, C->d_res_d, sizeof(double) * C->ninst, cudaMemcpyDeviceToHost, st));
        HF_CK(cudaStreamSynchronize(st));
        int it_max = 0, out_max = 0;
        int64_t it_sum = 0;
        double res_max = 0.0;
        for (int i = 0; i < C->ninst; i++) {
            it_max = std::max(it_max, C->h_res_i[3 * i]);
            out_max = std::max(out_max, C->h_res_i[3 * i + 1]);
            it_sum += C->h_res_i[3 * i];
            res_max = std::max(res_max, C->h_res_d[i]);
            if (C->h_res_i[3 * i + 2] && rc == HF_OK)
                rc = fail(C->h_res_i[3 * i + 2], "Poisson solve failed in instance " + std::to_string(i));
        }
        C->h_scal->iters = it_max;
        C->h_scal->rr = res_max * res_max;
        C->h_scal->bb = 1.0;
        C->stats.last_outer = out_max;
        C->stats.total_iters += it_sum - it_max;   // the common update below adds it_max
    } else if (C->use_cg && C->use_amg) {
        {
            PhaseTimer t(C, HF_PHASE_POISSON_INIT, launches);
            k_pcg_init<D><<<blocks(n), kBlock, 0, st>>>(C->P, C->F, C->M, C->cg, rtol, atol);
            launches++;
            launches += launch_vcycle(C);
            t.stop(launches);
        }
        double *pa = C->cg.pa, *pb = C->cg.pb;
        int chunk = 4;
        for (;;) {
            PhaseTimer t(C, HF_PHASE_POISSON_ITER, launches);
            for (int k = 0; k < chunk; k++) {
                k_cg_dir_spmv<<<blocks(n), kBlock, 0, st>>>(C->M, C->cg, pa, pb);
                k_pcg_update<<<blocks(n), kBlock, 0, st>>>(C->M, C->cg, pb);
                launches += 2 + launch_vcycle(C);
                std::swap(pa, pb);
            }
            t.stop(launches);
            HF_CK(cudaMemcpyAsync(C->h_scal, C->cg.sc, sizeof(Scal), cudaMemcpyDeviceToHost, st));
            HF_CK(cudaStreamSynchronize(st));
            if (C->h_scal->done) break;
            chunk = std::min(chunk * 2, 16);
        }
        C->cg.pa = pa;
        C->cg.pb = pb;
        if (C->h_scal->status) rc = fail(C->h_scal->status, "Poisson AMG-CG failed");
    } else if (C->use_cg) {
        {
            PhaseTimer t(C, HF_PHASE_POISSON_INIT, launches);
            k_cg_init<D><<<blocks(n), kBlock, 0, st>>>(C->P, C->F, C->M, C->cg, rtol, atol);
            launches++;
            t.stop(launches);
        }
        double *pa = C->cg.pa, *pb = C->cg.pb;
        int chunk = 8;
        for (;;) {
            PhaseTimer t(C, HF_PHASE_POISSON_ITER, launches);
            for (int k = 0; k < chunk; k++) {
                k_cg_dir_spmv<<<blocks(n), kBlock, 0, st>>>(C->M, C->cg, pa, pb);
                k_cg_update<<<blocks(n), kBlock, 0, st>>>(C->M, C->cg, pb);
                std::swap(pa, pb);
                launches += 2;
            }
            t.stop(launches);
            HF_CK(cudaMemcpyAsync(C->h_scal, C->cg.sc, sizeof(Scal), cudaMemcpyDeviceToHost, st));
            HF_CK(cudaStreamSynchronize(st));
            if (C->h_scal->done) break;
            chunk = std::min(chunk * 2, 64);
        }
        C->cg.pa = pa;
        C->cg.pb = pb;
        if (C->h_scal->status) rc = fail(C->h_scal->status, "Poisson CG failed");
    } else {
        int restarts = 0;
        int from_step = 1;
        for (;;) {
            {
                PhaseTimer t(C, HF_PHASE_POISSON_INIT, launches);
                k_bi_init<D><<<blocks(n), kBlock, 0, st>>>(C->P, C->F, C->M, C->bi, rtol, atol, from_step);
                launches++;
                t.stop(launches);
            }
            int chunk = 4;
            for (;;) {
                PhaseTimer t(C, HF_PHASE_POISSON_ITER, launches);
                for (int k = 0; k < chunk; k++) {
                    k_bi_p<<<blocks(n), kBlock, 0, st>>>(C->M, C->bi);
                    k_bi_spmv<<<blocks(n), kBlock, 0, st>>>(C->M, C->bi, C->bi.ph, C->bi.v, 0);
                    k_bi_s<<<blocks(n), kBlock, 0, st>>>(C->M, C->bi);
                    k_bi_spmv<<<blocks(n), kBlock, 0, st>>>(C->M, C->bi, C->bi.sh, C->bi.t, 1);
                    k_bi_update<<<blocks(n), kBlock, 0, st>>>(C->M, C->bi);
                    launches += 5;
                }
                t.stop(launches);
                HF_CK(cudaMemcpyAsync(C->h_scal, C->bi.sc, sizeof(Scal), cudaMemcpyDeviceToHost, st));
                HF_CK(cudaStreamSynchronize(st));
                if (C->h_scal->done) break;
                chunk = std::min(chunk * 2, 32);
            }
            if (C->h_scal->status == 1 && restarts++ < 50) { from_step = 0; continue; }
            break;
        }
        if (C->h_scal->status) rc = fail(C->h_scal->status == 1 ? HF_ERR_NOT_CONVERGED : C->h_scal->status, "Poisson BiCGStab failed");
    }
    {
        PhaseTimer t(C, HF_PHASE_FINAL, launches);
        k_final<D><<<blocks(C->nfacet_total + n), kBlock, 0, st>>>(C->P, C->F);
        launches++;
        t.stop(launches);
    }
    HF_CK(cudaGetLastError());
    C->stats.last_iters = C->h_scal->iters;
    C->stats.total_iters += C->h_scal->iters;
    C->stats.last_residual = C->h_scal->bb > 0 ? sqrt(C->h_scal->rr / C->h_scal->bb) : sqrt(C->h_scal->rr);
    C->stats.kernel_launches += launches;
    C->stats.steps += 1;
    return rc;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" const char *hf_last_error(void) { return g_err.c_str(); }

extern "C" int hf_case_device_bytes(const hf_program *pg, const hf_options *opt, int64_t *bytes)
{
    (void)opt;
    if (!pg || !bytes) return fail(HF_ERR_INVALID, "null argument");
    const int D = pg->par.dim;
    int64_t nfac = 0;
    for (int d = 0; d < D; d++) nfac += pg->nfacet[d];
    int64_t b = 0;
    b += pg->nnz * 12 + pg->ntmpl * 8 + pg->nrows * 16 + 8;
    b += nfac * ((int64_t)pg->vel_nslot * 4 + 4 + 2);
    b += (int64_t)pg->ncell * (2 * D * 4 + 2);
    b += pg->pnnz * 12 + (int64_t)pg->ncell * 4 * 8;
    b += (int64_t)pg->cell_nslot * pg->ncell * 4 + pg->ncell * 4;
    b += nfac * 8 * 3 + (int64_t)pg->ncell * 8 * 3;                 // u, u*, FU; p, dp, F
    if (pg->par.flowtype == HF_VISCOELASTIC) b += (int64_t)pg->ncell * 8 * 4 * D * D;
    b += (int64_t)pg->ncell * 8 * 10;                                // solver vectors
    *bytes = b;
    return HF_OK;
}

extern "C" int hf_case_create(const hf_program *pg, const hf_options *opt_in, hf_case **out)
{
    if (!out) return fail(HF_ERR_INVALID, "null output");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(HF_ERR_NO_DEVICE, "no CUDA device");
    int rc = check_program(pg);
    if (rc) return rc;
    rc = check_rows(pg);
    if (rc) return rc;
    hf_options opt{};
    if (opt_in) opt = *opt_in;
    if (opt.poisson_rtol <= 0) opt.poisson_rtol = 1e-10;
    if (opt.poisson_atol <= 0) opt.poisson_atol = 1e-10;
    if (opt.poisson_maxit <= 0) opt.poisson_maxit = 20000;
    if (opt.precision != HF_PREC_FP64 && opt.precision != HF_PREC_MIXED) return fail(HF_ERR_INVALID, "precision");
    HF_CK(cudaSetDevice(opt.device));

    hf_case *C = new hf_case();
    C->opt = opt;
    C->par = pg->par;
    const int D = pg->par.dim;
    C->D = D;
    memset(&C->stats, 0, sizeof C->stats);
    auto cleanup = [&](int code) {
        hf_case_destroy(C);
        return code;
    };
    if (cudaStreamCreateWithFlags(&C->stream, cudaStreamNonBlocking) != cudaSuccess) return cleanup(fail(HF_ERR_CUDA, "stream"));
    if (cudaMallocHost((void **)&C->h_scal, sizeof(Scal)) != cudaSuccess) return cleanup(fail(HF_ERR_CUDA, "pinned scalars"));

    DevProg &P = C->P;
    memset(&P, 0, sizeof P);
    P.D = D;
    P.ncell = pg->ncell;
    P.par = pg->par;
    P.off[0] = 0;
    for (int d = 0; d < 3; d++) {
        P.nf[d] = d < D ? pg->nfacet[d] : 0;
        P.off[d + 1] = P.off[d] + P.nf[d];
    }
    C->nfacet_total = P.off[D];
    P.vns = pg->vel_nslot;
    P.cns = pg->cell_nslot;
    double &B = C->bytes;
    auto &own = C->owned;
#define UP(dst, src, n) do { if ((rc = upload(own, dst, src, (size_t)(n), B))) return cleanup(rc); } while (0)
    // instances: a plain program is a batch of one
    std::vector<hf_params> ipar;
    std::vector<int> pins;
    std::vector<double> pinv;
    if (pg->ninst > 0) {
        C->ninst = pg->ninst;
        for (int i = 0; i < pg->ninst; i++) {
            ipar.push_back(pg->inst_par[i]);
            pins.push_back(pg->inst_pin[i]);
            pinv.push_back(pg->inst_pin_value[i]);
            if (pg->inst_par[i].dim != D || pg->inst_par[i].flowtype != pg->par.flowtype)
                return cleanup(fail(HF_ERR_INVALID, "batch members differ in dim or flow type"));
        }
        C->coff.assign(pg->cell_off, pg->cell_off + pg->ninst + 1);
        for (int d = 0; d < D; d++) C->foff[d].assign(pg->facet_off[d], pg->facet_off[d] + pg->ninst + 1);
    } else {
        C->ninst = 1;
        ipar.push_back(pg->par);
        pins.push_back(pg->pin_row);
        pinv.push_back(pg->pin_value);
        C->coff = {0, pg->ncell};
        for (int d = 0; d < D; d++) C->foff[d] = {0, pg->nfacet[d]};
    }
    const int ni = C->ninst;
    if (C->coff[0] != 0 || C->coff[ni] != pg->ncell) return cleanup(fail(HF_ERR_INVALID, "cell offsets"));
    for (int d = 0; d < D; d++)
        if (C->foff[d][0] != 0 || C->foff[d][ni] != pg->nfacet[d]) return cleanup(fail(HF_ERR_INVALID, "facet offsets"));
    for (int i = 0; i < ni; i++) {
        if (C->coff[i + 1] <= C->coff[i]) return cleanup(fail(HF_ERR_INVALID, "empty instance"));
        if (pins[i] >= 0 && (pins[i] < C->coff[i] || pins[i] >= C->coff[i + 1]))
            return cleanup(fail(HF_ERR_INVALID, "pin outside its instance"));
    }
    P.par = ipar[0];
    P.pin = pins[0];
    P.pin_value = pinv[0];
    P.ninst = ni;
    {
        std::vector<int32_t> cinst(pg->ncell);
        for (int i = 0; i < ni; i++)
            for (int c = C->coff[i]; c < C->coff[i + 1]; c++) cinst[c] = i;
        UP((int32_t **)&P.cinst, cinst.data(), cinst.size());
        for (int d = 0; d < D; d++) {
            std::vector<int32_t> finst(pg->nfacet[d]);
            for (int i = 0; i < ni; i++)
                for (int f = C->foff[d][i]; f < C->foff[d][i + 1]; f++) finst[f] = i;
            UP((int32_t **)&P.finst[d], finst.data(), finst.size());
        }
        UP((hf_params **)&P.ipar, ipar.data(), ipar.size());
        UP((double **)&P.ipinv, pinv.data(), pinv.size());
    }
    UP((double **)&P.delta, pg->delta, (size_t)pg->ndelta * D);
    UP((int32_t **)&P.rows.tmpl, pg->row_tmpl, pg->nrows);
    UP((int32_t **)&P.rows.base, pg->row_base, pg->nrows);
    UP((double **)&P.rows.rhs, pg->row_rhs, pg->nrows);
    UP((int64_t **)&P.rows.tptr, pg->tmpl_ptr, pg->ntmpl + 1);
    UP((int32_t **)&P.rows.col, pg->tmpl_col, pg->nnz);
    UP((double **)&P.rows.w, pg->tmpl_w, pg->nnz);
    for (int d = 0; d < D; d++) {
        UP((int32_t **)&P.vslots[d], pg->vel_slots[d], (size_t)pg->vel_nslot * pg->nfacet[d]);
        UP((uint32_t **)&P.vflags[d], pg->vel_flags[d], pg->nfacet[d]);
        UP((uint16_t **)&P.vdelta[d], pg->vel_delta[d], pg->nfacet[d]);
    }
    UP((int32_t **)&P.dslots, pg->div_slots, (size_t)2 * D * pg->ncell);
    UP((uint16_t **)&P.cdelta, pg->cell_delta, pg->ncell);
    if (pg->par.flowtype == HF_VISCOELASTIC) {
        UP((int32_t **)&P.cslots, pg->cell_slots, (size_t)pg->cell_nslot * pg->ncell);
        UP((uint32_t **)&P.cflags, pg->cell_flags, pg->ncell);
    }
    // fields
    DevFields &F = C->F;
    memset(&F, 0, sizeof F);
    for (int d = 0; d < D; d++) {
        UP(&F.u[d], (const double *)nullptr, pg->nfacet[d]);
        UP(&F.us[d], (const double *)nullptr, pg->nfacet[d]);
        UP(&F.FU[d], (const double *)nullptr, pg->nfacet[d]);
    }
    UP(&F.p, (const double *)nullptr, pg->ncell);
    UP(&F.dp, (const double *)nullptr, pg->ncell);
    UP(&F.F, (const double *)nullptr, pg->ncell);
    if (pg->par.flowtype == HF_VISCOELASTIC) {
        for (int k = 0; k < D * D; k++) {
            UP(&F.K[k], (const double *)nullptr, pg->ncell);
            UP(&F.Knew[k], (const double *)nullptr, pg->ncell);
            UP(&F.S[k], (const double *)nullptr, pg->ncell);
            UP(&F.Du[k], (const double *)nullptr, pg->ncell);
        }
    }
    // Poisson operator
    std::vector<int32_t> mptr, mcol;
    std::vector<double> mval, dinv, apin;
    bool sym = false;
    if ((rc = build_matrix(pg, pins, mptr, mcol, mval, dinv, apin, sym))) return cleanup(rc);
    C->use_cg = opt.poisson == HF_POISSON_CG || (opt.poisson == HF_POISSON_AUTO && sym);
    if (opt.poisson == HF_POISSON_CG && !sym) return cleanup(fail(HF_ERR_UNSUPPORTED, "CG requested on a non-symmetric Poisson matrix"));
    // the persistent per-instance solver serves batches and small single cases;
    // one large case keeps the multi-kernel solver
    int maxn = 0;
    for (int i = 0; i < ni; i++) maxn = std::max(maxn, C->coff[i + 1] - C->coff[i]);
    C->persistent = C->use_cg && opt.precond != HF_PRECOND_JACOBI && (ni > 1 || maxn <= 131072);
    if (ni > 1 && !C->persistent) return cleanup(fail(HF_ERR_UNSUPPORTED, "batches need the AMG-CG Poisson solver"));
    if (opt.precision == HF_PREC_MIXED && !C->persistent)
        return cleanup(fail(HF_ERR_UNSUPPORTED, "the mixed form runs on the persistent per-instance solver"));
    DevMat &M = C->M;
    M.n = pg->ncell;
    UP((int32_t **)&M.ptr, mptr.data(), mptr.size());
    UP((int32_t **)&M.col, mcol.data(), mcol.size());
    UP((double **)&M.val, mval.data(), mval.size());
    UP((double **)&M.dinv, dinv.data(), dinv.size());
    UP((double **)&M.apin, apin.data(), apin.size());
    UP((double **)&M.brhs, pg->p_brhs, pg->ncell);
    const int nb = blocks(pg->ncell);
    Scal *sc = nullptr;
    UP(&sc, (const Scal *)nullptr, 1);
    {
        Scal h{};
        h.maxit = opt.poisson_maxit;
        if (cudaMemcpy(sc, &h, sizeof h, cudaMemcpyHostToDevice) != cudaSuccess) return cleanup(fail(HF_ERR_CUDA, "scalars"));
    }
    double *partials = nullptr;
    UP(&partials, (const double *)nullptr, (size_t)nb * 4);
    const int n = pg->ncell;
    if (C->use_cg) {
        C->cg.x = pg->par.projtype == HF_INCREMENTAL ? F.dp : F.p;
        UP(&C->cg.r, (const double *)nullptr, n);
        UP(&C->cg.z, (const double *)nullptr, n);
        UP(&C->cg.pa, (const double *)nullptr, n);
        UP(&C->cg.pb, (const double *)nullptr, n);
        UP(&C->cg.q, (const double *)nullptr, n);
        C->cg.partials = partials;
        C->cg.sc = sc;
        C->use_amg = opt.precond != HF_PRECOND_JACOBI && !C->persistent;
        if (C->persistent) {
            UP(&C->d_res_i, (const int *)nullptr, (size_t)3 * ni);
            UP(&C->d_res_d, (const double *)nullptr, (size_t)ni);
            if (cudaMallocHost((void **)&C->h_res_i, sizeof(int) * 3 * ni) != cudaSuccess ||
                cudaMallocHost((void **)&C->h_res_d, sizeof(double) * ni) != cudaSuccess)
                return cleanup(fail(HF_ERR_CUDA, "pinned results"));
            if ((rc = build_batch_solver(C, mptr, mcol, mval, M.apin, M.brhs, pins, opt.precision == HF_PREC_MIXED)))
                return cleanup(rc);
        }
        if (C->use_amg) {
            hf::HostCSR M0;
            M0.n = M0.m = n;
            M0.ptr.assign(mptr.begin(), mptr.end());
            M0.col.assign(mcol.begin(), mcol.end());
            M0.val = mval;
            std::vector<hf::HostLevel> H = hf::build_hierarchy(std::move(M0));
            if ((int)H.size() - 1 > kMaxLevels) return cleanup(fail(HF_ERR_UNSUPPORTED, "AMG hierarchy too deep"));
            DevAMG &A = C->amg;
            A.nlev = (int)H.size() - 1;
            C->amg_levels = (int)H.size();
            for (int l = 0; l < A.nlev; l++) {
                DevLevel &L = A.lev[l];
                const hf::HostLevel &h = H[l];
                auto up_csr = [&](DevCSR &d, const hf::HostCSR &s) {
                    d.n = s.n;
                    int r2;
                    if ((r2 = upload(own, (int32_t **)&d.ptr, s.ptr.data(), s.ptr.size(), B))) return r2;
                    if ((r2 = upload(own, (int32_t **)&d.col, s.col.data(), s.col.size(), B))) return r2;
                    return upload(own, (double **)&d.val, s.val.data(), s.val.size(), B);
                };
                if (l == 0) {
                    L.A = DevCSR{n, M.ptr, M.col, M.val};
                } else if ((rc = up_csr(L.A, h.A))) {
                    return cleanup(rc);
                }
                if ((rc = up_csr(L.P, h.P)) || (rc = up_csr(L.R, h.R))) return cleanup(rc);
                UP((double **)&L.dinv, h.dinv.data(), h.dinv.size());
                if (l == 0) {
                    L.b = C->cg.r;
                    L.out = C->cg.z;
                } else {
                    UP(&L.b, (const double *)nullptr, h.A.n);
                    UP(&L.out, (const double *)nullptr, h.A.n);
                }
                UP(&L.x, (const double *)nullptr, h.A.n);
                UP(&L.r, (const double *)nullptr, h.A.n);
            }
            std::vector<double> inv;
            if (!hf::dense_inverse(H.back().A, inv)) return cleanup(fail(HF_ERR_INVALID, "singular coarsest AMG level"));
            A.cn = H.back().A.n;
            UP((double **)&A.cinv, inv.data(), inv.size());
            UP(&A.cb, (const double *)nullptr, A.cn);
            UP(&A.cx, (const double *)nullptr, A.cn);
        }
    } else {
        BiVec &V = C->bi;
        V.x = pg->par.projtype == HF_INCREMENTAL ? F.dp : F.p;
        UP(&V.b, (const double *)nullptr, n);
        UP(&V.r, (const double *)nullptr, n);
        UP(&V.rh, (const double *)nullptr, n);
        UP(&V.p, (const double *)nullptr, n);
        UP(&V.v, (const double *)nullptr, n);
        UP(&V.s, (const double *)nullptr, n);
        UP(&V.t, (const double *)nullptr, n);
        UP(&V.ph, (const double *)nullptr, n);
        UP(&V.sh, (const double *)nullptr, n);
        V.partials = partials;
        V.sc = sc;
    }
#undef UP
    if (cudaDeviceSynchronize() != cudaSuccess) return cleanup(fail(HF_ERR_CUDA, "create sync"));
    C->stats.device_bytes = C->bytes;
    *out = C;
    return HF_OK;
}

static double *field_ptr(hf_case *C, int32_t field, int32_t comp, int64_t *n)
{
    const int D = C->D;
    const bool ve = C->par.flowtype == HF_VISCOELASTIC;
    auto facet = [&](double *const *arr) -> double * {
        if (comp < 0 || comp >= D) return nullptr;
        *n = C->P.nf[comp];
        return arr[comp];
    };
    auto cell = [&](double *p) -> double * { *n = C->P.ncell; return p; };
    auto tens = [&](double *const *arr) -> double * {
        if (!ve || comp < 0 || comp >= D * D) return nullptr;
        *n = C->P.ncell;
        return arr[comp];
    };
    switch (field) {
    case HF_FIELD_U: return facet(C->F.u);
    case HF_FIELD_USTAR: return facet(C->F.us);
    case HF_FIELD_P: return cell(C->F.p);
    case HF_FIELD_DP: return cell(C->F.dp);
    case HF_FIELD_F: return cell(C->F.F);
    case HF_FIELD_FU: return facet(C->F.FU);
    case HF_FIELD_KERNEL: return tens(C->F.K);
    case HF_FIELD_S: return tens(C->F.S);
    case HF_FIELD_DU: return tens(C->F.Du);
    }
    return nullptr;
}

extern "C" int hf_case_set_field(hf_case *C, int32_t field, int32_t comp, const double *host, int64_t n)
{
    if (!C || !host) return fail(HF_ERR_INVALID, "null argument");
    int64_t m = 0;
    double *p = field_ptr(C, field, comp, &m);
    if (!p || m != n) return fail(HF_ERR_INVALID, "field/component/size mismatch");
    HF_CK(cudaMemcpyAsync(p, host, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, C->stream));
    HF_CK(cudaStreamSynchronize(C->stream));
    return HF_OK;
}

extern "C" int hf_case_get_field(hf_case *C, int32_t field, int32_t comp, double *host, int64_t n)
{
    if (!C || !host) return fail(HF_ERR_INVALID, "null argument");
    int64_t m = 0;
    double *p = field_ptr(C, field, comp, &m);
    if (!p || m != n) return fail(HF_ERR_INVALID, "field/component/size mismatch");
    HF_CK(cudaMemcpyAsync(host, p, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, C->stream));
    HF_CK(cudaStreamSynchronize(C->stream));
    return HF_OK;
}

extern "C" int hf_case_step(hf_case *C, int32_t nsteps)
{
    if (!C) return fail(HF_ERR_INVALID, "null case");
    for (int s = 0; s < nsteps; s++) {
        int rc = C->D == 2 ? launch_step<2>(C) : launch_step<3>(C);
        if (rc) return rc;
    }
    return HF_OK;
}

extern "C" int hf_case_synchronize(hf_case *C)
{
    if (!C) return fail(HF_ERR_INVALID, "null case");
    HF_CK(cudaStreamSynchronize(C->stream));
    return HF_OK;
}

extern "C" int hf_case_stats(hf_case *C, hf_stats *out)
{
    if (!C || !out) return fail(HF_ERR_INVALID, "null argument");
    *out = C->stats;
    if (!C->persistent) out->last_outer = 1;
    return HF_OK;
}

extern "C" int hf_case_instances(hf_case *C, int32_t *ninst)
{
    if (!C || !ninst) return fail(HF_ERR_INVALID, "null argument");
    *ninst = C->ninst;
    return HF_OK;
}

extern "C" int hf_case_instance_result(hf_case *C, int32_t inst, int32_t *iters, int32_t *outer, int32_t *status,
                                       double *residual)
{
    if (!C || inst < 0 || inst >= C->ninst) return fail(HF_ERR_INVALID, "bad instance");
    if (!C->persistent) {
        if (iters) *iters = C->stats.last_iters;
        if (outer) *outer = 1;
        if (status) *status = 0;
        if (residual) *residual = C->stats.last_residual;
        return HF_OK;
    }
    if (iters) *iters = C->h_res_i[3 * inst];
    if (outer) *outer = C->h_res_i[3 * inst + 1];
    if (status) *status = C->h_res_i[3 * inst + 2];
    if (residual) *residual = C->h_res_d[inst];
    return HF_OK;
}

extern "C" int hf_case_solver_info(hf_case *C, int32_t *method, int32_t *nlev, int64_t *rows, int64_t *nnz_a,
                                   int64_t *nnz_p, int64_t *nnz_r, int32_t max_levels)
{
    if (!C || !method || !nlev) return fail(HF_ERR_INVALID, "null argument");
    *method = C->use_cg ? (C->use_amg ? HF_PRECOND_AMG : HF_PRECOND_JACOBI) : -1;
    *nlev = C->use_amg ? C->amg.nlev + 1 : 1;
    for (int l = 0; l < *nlev && l < max_levels; l++) {
        if (!C->use_amg) {
            if (rows) rows[l] = C->M.n;
            continue;
        }
        const bool coarse = l == C->amg.nlev;
        std::vector<int32_t> hp(2);
        auto nnz = [&](const DevCSR &d) -> int64_t {
            int32_t last = 0;
            if (d.ptr && cudaMemcpy(&last, d.ptr + d.n, sizeof last, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
            return last;
        };
        if (rows) rows[l] = coarse ? C->amg.cn : C->amg.lev[l].A.n;
        if (nnz_a) nnz_a[l] = coarse ? (int64_t)C->amg.cn * C->amg.cn : nnz(C->amg.lev[l].A);
        if (nnz_p) nnz_p[l] = coarse ? 0 : nnz(C->amg.lev[l].P);
        if (nnz_r) nnz_r[l] = coarse ? 0 : nnz(C->amg.lev[l].R);
    }
    return HF_OK;
}

extern "C" int hf_case_stream(hf_case *C, void **stream)
{
    if (!C || !stream) return fail(HF_ERR_INVALID, "null argument");
    *stream = (void *)C->stream;
    return HF_OK;
}

extern "C" int hf_case_profile(hf_case *C, int32_t enable)
{
    if (!C) return fail(HF_ERR_INVALID, "null case");
    if (enable && !C->ev[0])
        for (int k = 0; k < 2 * HF_NPHASE; k++) HF_CK(cudaEventCreate(&C->ev[k]));
    C->profile = enable != 0;
    for (int k = 0; k < HF_NPHASE; k++) { C->phase_ms[k] = 0.0; C->phase_launches[k] = 0; }
    return HF_OK;
}

extern "C" int hf_case_phase_times(hf_case *C, double *ms, int64_t *launches, int32_t n)
{
    if (!C || n < 0) return fail(HF_ERR_INVALID, "bad argument");
    for (int k = 0; k < n && k < HF_NPHASE; k++) {
        if (ms) ms[k] = C->phase_ms[k];
        if (launches) launches[k] = C->phase_launches[k];
    }
    return HF_OK;
}

extern "C" void hf_case_destroy(hf_case *C)
{
    if (!C) return;
    if (C->stream) cudaStreamSynchronize(C->stream);
    for (int k = 0; k < 2 * HF_NPHASE; k++)
        if (C->ev[k]) cudaEventDestroy(C->ev[k]);
    for (void *p : C->owned) cudaFree(p);
    if (C->h_scal) cudaFreeHost(C->h_scal);
    if (C->h_res_i) cudaFreeHost(C->h_res_i);
    if (C->h_res_d) cudaFreeHost(C->h_res_d);
    if (C->stream) cudaStreamDestroy(C->stream);
    delete C;
}

// ---------------------------------------------------------------------------
// linear-solver engine behind HigTree's _solver_vtable (solver.h:42-60):
// rows arrive one at a time on the host (set_Ai replaces a row, as PETSc's
// MatSetValues with INSERT_VALUES does for an unchanged pattern), the matrix is
// uploaded at assemble_matrix, and solve() runs Jacobi-preconditioned BiCGStab
// on the GPU from the current x (nonzero initial guess, solver-petsc.c:386-399)
// until ||b - A x|| <= max(rtol ||b||, atol).
// ---------------------------------------------------------------------------
namespace {

__global__ void __launch_bounds__(kBlock) k_slv_init(DevMat M, BiVec V, double rtol, double atol, int first)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double part[3] = {0.0, 0.0, 0.0};
    if (i < M.n) {
        double ax = 0.0;
        for (int k = M.ptr[i]; k < M.ptr[i + 1]; k++) ax += M.val[k] * V.x[M.col[k]];
        const double r = V.b[i] - ax;
        V.r[i] = r;
        V.rh[i] = r;
        V.p[i] = 0.0;
        V.v[i] = 0.0;
        part[0] = r * r;
        part[1] = V.b[i] * V.b[i];
    }
    double tot[3];
    if (grid_sum<3>(part, V.partials, &V.sc->counter, tot) && threadIdx.x == 0) {
        Scal &s = *V.sc;
        s.rr = tot[0];
        if (first) {
            s.bb = tot[1];
            const double t = fmax(rtol * sqrt(tot[1]), atol);
            s.tol2 = t * t;
            s.iters = 0;
        }
        s.rho = 1.0;
        s.alpha = 1.0;
        s.omega = 1.0;
        s.rho1 = tot[0];
        s.beta = 0.0;
        s.status = 0;
        s.done = !(tot[0] > s.tol2);
        if (!finite(tot[0])) { s.status = HF_ERR_NAN; s.done = 1; }
    }
}

}  // namespace

struct hf_slv {
    int first = 0, n = 0;
    std::vector<std::vector<std::pair<int, double>>> rows;
    std::vector<double> b, x;
    bool dirty_matrix = true;
    double rtol = 1e-10, atol = 1e-10;
    int maxit = 100000;
    int iters = 0;
    double residual = 0;
    int converged = 0;
    // device
    DevMat M{};
    BiVec V{};
    std::vector<void *> mat_owned, vec_owned;
    cudaStream_t stream = nullptr;
    Scal *h_scal = nullptr;
};

namespace {

void free_list(std::vector<void *> &v)
{
    for (void *p : v) cudaFree(p);
    v.clear();
}

int slv_upload_matrix(hf_slv *s)
{
    free_list(s->mat_owned);
    std::vector<int32_t> ptr(s->n + 1, 0), col;
    std::vector<double> val, dinv(s->n, 1.0);
    for (int r = 0; r < s->n; r++) {
        auto row = s->rows[r];
        std::sort(row.begin(), row.end());
        for (auto &e : row) {
            col.push_back(e.first);
            val.push_back(e.second);
            if (e.first == r && e.second != 0.0) dinv[r] = 1.0 / e.second;
        }
        ptr[r + 1] = (int32_t)col.size();
    }
    double bytes = 0;
    int rc;
    if ((rc = upload(s->mat_owned, (int32_t **)&s->M.ptr, ptr.data(), ptr.size(), bytes))) return rc;
    if ((rc = upload(s->mat_owned, (int32_t **)&s->M.col, col.data(), col.size(), bytes))) return rc;
    if ((rc = upload(s->mat_owned, (double **)&s->M.val, val.data(), val.size(), bytes))) return rc;
    if ((rc = upload(s->mat_owned, (double **)&s->M.dinv, dinv.data(), dinv.size(), bytes))) return rc;
    s->M.n = s->n;
    s->dirty_matrix = false;
    return HF_OK;
}

bool slv_row_ok(hf_slv *s, int32_t i) { return s && i >= s->first && i < s->first + s->n; }

}  // namespace

extern "C" int hf_slv_create(int32_t first_gid, int32_t size, hf_slv **out)
{
    if (!out || size <= 0) return fail(HF_ERR_INVALID, "bad size");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(HF_ERR_NO_DEVICE, "no CUDA device");
    hf_slv *s = new hf_slv();
    s->first = first_gid;
    s->n = size;
    s->rows.assign(size, {});
    s->b.assign(size, 0.0);
    s->x.assign(size, 0.0);
    double bytes = 0;
    int rc;
    auto bail = [&](int code) { hf_slv_destroy(s); return code; };
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(fail(HF_ERR_CUDA, "stream"));
    if (cudaMallocHost((void **)&s->h_scal, sizeof(Scal)) != cudaSuccess) return bail(fail(HF_ERR_CUDA, "pinned"));
    BiVec &V = s->V;
    double **vecs[] = {&V.x, &V.b, &V.r, &V.rh, &V.p, &V.v, &V.s, &V.t, &V.ph, &V.sh};
    for (double **v : vecs)
        if ((rc = upload(s->vec_owned, v, (const double *)nullptr, size, bytes))) return bail(rc);
    if ((rc = upload(s->vec_owned, &V.partials, (const double *)nullptr, (size_t)blocks(size) * 4, bytes))) return bail(rc);
    if ((rc = upload(s->vec_owned, &V.sc, (const Scal *)nullptr, 1, bytes))) return bail(rc);
    *out = s;
    return HF_OK;
}

extern "C" int hf_slv_set_maxnonzeros(hf_slv *s, int32_t maxnz)
{
    if (!s || maxnz < 0) return fail(HF_ERR_INVALID, "bad argument");
    return HF_OK;
}

extern "C" int hf_slv_set_Ai(hf_slv *s, int32_t i, int32_t numjs, const int32_t *j, const double *v)
{
    if (!slv_row_ok(s, i) || numjs < 0 || (numjs && (!j || !v))) return fail(HF_ERR_INVALID, "bad row");
    std::vector<std::pair<int, double>> row;
    for (int k = 0; k < numjs; k++) {
        if (!slv_row_ok(s, j[k])) return fail(HF_ERR_INVALID, "column out of range");
        int c = j[k] - s->first;
        bool merged = false;
        for (auto &e : row)
            if (e.first == c) { e.second += v[k]; merged = true; break; }
        if (!merged) row.push_back({c, v[k]});
    }
    auto &dst = s->rows[i - s->first];
    if (dst != row) {
        dst.swap(row);
        s->dirty_matrix = true;
    }
    return HF_OK;
}

extern "C" int hf_slv_set_bi(hf_slv *s, int32_t i, double v)
{
    if (!slv_row_ok(s, i)) return fail(HF_ERR_INVALID, "bad row");
    s->b[i - s->first] = v;
    return HF_OK;
}

extern "C" int hf_slv_add_bi(hf_slv *s, int32_t i, double v)
{
    if (!slv_row_ok(s, i)) return fail(HF_ERR_INVALID, "bad row");
    s->b[i - s->first] += v;
    return HF_OK;
}

extern "C" int hf_slv_set_xi(hf_slv *s, int32_t i, double v)
{
    if (!slv_row_ok(s, i)) return fail(HF_ERR_INVALID, "bad row");
    s->x[i - s->first] = v;
    return HF_OK;
}

extern "C" int hf_slv_set_x(hf_slv *s, const double *x)
{
    if (!s || !x) return fail(HF_ERR_INVALID, "null argument");
    std::copy(x, x + s->n, s->x.begin());
    return HF_OK;
}

extern "C" int hf_slv_get_xi(hf_slv *s, int32_t i, double *v)
{
    if (!slv_row_ok(s, i) || !v) return fail(HF_ERR_INVALID, "bad row");
    *v = s->x[i - s->first];
    return HF_OK;
}

extern "C" int hf_slv_get_x(hf_slv *s, double *x)
{
    if (!s || !x) return fail(HF_ERR_INVALID, "null argument");
    std::copy(s->x.begin(), s->x.end(), x);
    return HF_OK;
}

extern "C" int hf_slv_get_x_scatter(hf_slv *s, int32_t size, const int32_t *idx, double *x)
{
    if (!s || size < 0 || (size && (!idx || !x))) return fail(HF_ERR_INVALID, "bad argument");
    for (int k = 0; k < size; k++) {
        if (!slv_row_ok(s, idx[k])) return fail(HF_ERR_INVALID, "index out of range");
        x[k] = s->x[idx[k] - s->first];
    }
    return HF_OK;
}

extern "C" int hf_slv_assemble_matrix(hf_slv *s)
{
    if (!s) return fail(HF_ERR_INVALID, "null solver");
    return s->dirty_matrix ? slv_upload_matrix(s) : HF_OK;
}

extern "C" int hf_slv_assemble_rhs(hf_slv *s) { return s ? HF_OK : fail(HF_ERR_INVALID, "null solver"); }
extern "C" int hf_slv_assemble_output(hf_slv *s) { return s ? HF_OK : fail(HF_ERR_INVALID, "null solver"); }

extern "C" int hf_slv_set_tolerances(hf_slv *s, double rtol, double atol, int32_t maxit)
{
    if (!s || !(rtol > 0) || !(atol >= 0) || maxit <= 0) return fail(HF_ERR_INVALID, "bad tolerances");
    s->rtol = rtol;
    s->atol = atol;
    s->maxit = maxit;
    return HF_OK;
}

extern "C" int hf_slv_solve(hf_slv *s)
{
    if (!s) return fail(HF_ERR_INVALID, "null solver");
    if (s->dirty_matrix) {
        int rc = slv_upload_matrix(s);
        if (rc) return rc;
    }
    cudaStream_t st = s->stream;
    const int n = s->n;
    HF_CK(cudaMemcpyAsync(s->V.x, s->x.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
    HF_CK(cudaMemcpyAsync(s->V.b, s->b.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
    {
        Scal h{};
        h.maxit = s->maxit;
        *s->h_scal = h;
        HF_CK(cudaMemcpyAsync(s->V.sc, s->h_scal, sizeof(Scal), cudaMemcpyHostToDevice, st));
    }
    int restarts = 0, first = 1;
    for (;;) {
        k_slv_init<<<blocks(n), kBlock, 0, st>>>(s->M, s->V, s->rtol, s->atol, first);
        first = 0;
        int chunk = 4;
        for (;;) {
            for (int k = 0; k < chunk; k++) {
                k_bi_p<<<blocks(n), kBlock, 0, st>>>(s->M, s->V);
                k_bi_spmv<<<blocks(n), kBlock, 0, st>>>(s->M, s->V, s->V.ph, s->V.v, 0);
                k_bi_s<<<blocks(n), kBlock, 0, st>>>(s->M, s->V);
                k_bi_spmv<<<blocks(n), kBlock, 0, st>>>(s->M, s->V, s->V.sh, s->V.t, 1);
                k_bi_update<<<blocks(n), kBlock, 0, st>>>(s->M, s->V);
            }
            HF_CK(cudaMemcpyAsync(s->h_scal, s->V.sc, sizeof(Scal), cudaMemcpyDeviceToHost, st));
            HF_CK(cudaStreamSynchronize(st));
            if (s->h_scal->done) break;
            chunk = std::min(chunk * 2, 32);
        }
        if (s->h_scal->status == 1 && restarts++ < 50) continue;
        break;
    }
    HF_CK(cudaGetLastError());
    HF_CK(cudaMemcpyAsync(s->x.data(), s->V.x, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    HF_CK(cudaStreamSynchronize(st));
    const Scal &r = *s->h_scal;
    s->iters = r.iters;
    s->residual = r.bb > 0 ? sqrt(r.rr / r.bb) : sqrt(r.rr);
    s->converged = r.status == 0;
    if (r.status == HF_ERR_NAN) return fail(HF_ERR_NAN, "NaN in BiCGStab");
    if (r.status) return fail(HF_ERR_NOT_CONVERGED, "BiCGStab did not converge");
    return HF_OK;
}

extern "C" int hf_slv_result(hf_slv *s, int32_t *iterations, double *residual, int32_t *converged)
{
    if (!s) return fail(HF_ERR_INVALID, "null solver");
    if (iterations) *iterations = s->iters;
    if (residual) *residual = s->residual;
    if (converged) *converged = s->converged;
    return HF_OK;
}

extern "C" void hf_slv_destroy(hf_slv *s)
{
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    free_list(s->mat_owned);
    free_list(s->vec_owned);
    if (s->h_scal) cudaFreeHost(s->h_scal);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}
