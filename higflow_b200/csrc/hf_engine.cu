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
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
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
// A set of (general row, field read) pairs that k_vrows evaluates once per
// use into val: pair u's value is -rhs[u] + sum_k w_k * field(tag[u])[col_k]
// in stencil order (dp_interpolate_from_stencil, pdomain.c:1026-1053).  Slot
// codes of the kernels that read them index the pairs.  Sliced layout
// (SELL-32, entries in pairs): pair u is lane l = u % 32 of slice u / 32, and
// its entries 2j and 2j + 1 sit side by side at sptr[u / 32] + 64 j + 2 l, so
// a warp reads two entries of its 32 pairs with one coalesced 16-byte weight
// load and one 4-byte (or 8-byte) column load per thread; slices are padded
// to an even length; plen[u] is the pair's entry count.  Columns are absolute (row base
// added) in scol, or, when every pair's entries lie within +-32767 of its
// first column pcol0[u] (interpolation stencils are local: 2D meshes up to
// several thousand cells a side), 16-bit offsets in scol16 (scol null).
// Weights are FP64 (sw).
struct PairRows {
    int n;
    const uint8_t *tag;
    const double *rhs;
    const int64_t *sptr;
    const uint8_t *plen;
    const int32_t *scol;
    const int16_t *scol16;
    const int32_t *pcol0;
    const double *sw;
    double *val;
    // under step limits (null otherwise): a pair of a frozen instance is
    // skipped, its instance found from its first column's element
    const int64_t *ilim;
    const int32_t *finst[3];
    const int32_t *cinst;
};

// the instance of a pair whose first column is `col` in the field of `tag`
// (vtag_field's numbering: facet fields FU[d] 0-2 and u[d] 5-7, the rest cells)
__device__ __forceinline__ int pair_inst(const int32_t *const finst[3], const int32_t *cinst, int tag, int col)
{
    // (selects, not a dynamic index: that would copy the parameters to local memory)
    const int d = tag <= 2 ? tag : tag - 5;
    const int32_t *fi = d == 0 ? finst[0] : d == 1 ? finst[1] : finst[2];
    if (tag <= 2 || (tag >= 5 && tag <= 7)) return __ldg(fi + col);
    return __ldg(cinst + col);
}

// The mixed form's velocity-stage pairs by FP32 pattern.  The interpolation
// weights HigTree computes for each row differ from row to row in their last
// bits (each row is fitted at its own coordinates) and list the stencil's
// points in a row-dependent order; with the entries in column order and the
// weights in FP32, most rows share a few (column offsets, weights) patterns:
// on 16 of the batched Giesekus cavities 7,368 patterns cover 1.16 M rows
// (50.5 M entries).  The pairs keep their order (consecutive pairs are
// consecutive facets of one slot: a warp's field gathers touch about 9
// sectors per entry, and its 32 pairs use about 3.6 patterns), each reads its
// pattern's (offset, weight) entries from the small table that stays in L1/L2
// instead of streaming its own columns and weights from HBM.  The sum runs
// in column order: FP64 values times FP32 weights, summed in FP64.
struct PatEntry {
    int32_t off;            // column offset from the pair's first column
    float w;                // FP32 weight
};
struct PatRows {
    int n;                  // pairs (the velocity pair set's order)
    const int32_t *pid;     // per pair: its pattern
    const int32_t *col0;    // ... the absolute column of offset 0 (its row's smallest)
    const uint8_t *tag;     // ... the field it reads
    const double *rhs;      // ... its row's boundary term
    const int32_t *pstart;  // per pattern: first entry
    const uint8_t *plen;    // per pattern: entry count
    const PatEntry *ent;
    double *val;
    const int64_t *ilim;        // as in PairRows
    const int32_t *finst[3];
    const int32_t *cinst;
};

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
    // general rows of the velocity stage, one per (row, field read) pair: the
    // velocity slot codes index these pairs (vrow: the same rows for
    // hf::query), evaluated by k_vrows at the start of the stage
    hf::Rows<double> vrow;
    PairRows vr;
    // general rows of the viscoelastic cell stage (velocity at the cell's
    // faces and corners, the kernel's neighbours; FP64 weights in both
    // forms), evaluated by k_vrows ahead of k_ve_cell: negative cell slot
    // codes index cr.val (a kernel query's pair is the first of the upper
    // triangle's components, which follow it in row-major order)
    PairRows cr;
    // semi-implicit Euler: the velocity kernel writes each direction's
    // right-hand side, u + dt (sources - grad p [+ div S] - conv) plus the
    // system's boundary part sie_bc, into sie_b instead of u*
    int sie;
    double *sie_b[3];
    const double *sie_bc[3];
    // BDF2's second solve: its boundary part, and the source - grad p [+ div
    // S] - conv bracket of the velocity kernel, kept for its right-hand side
    const double *sie_bc2[3];
    double *sie_e[3];
    // GPTT: E_{alpha,beta}(eps Re De tr S / (1 - beta)) per cell, written by
    // k_gptt_ml ahead of k_ve_cell (null when no instance is GPTT)
    double *gptt_e;
    const int32_t *dslots;
    const uint16_t *cdelta;
    const int32_t *cslots;
    const uint32_t *cflags;
    int cns;
    int pin;               // single-instance path: instance 0's pin and parameters (par)
    int projtype_all;      // the projection type of every instance, or -1 when they differ
                           // (saves the per-element instance lookup before the field loads)
    double pin_value;
    // per-instance parameters and element -> instance maps (batches)
    int ninst;
    const hf_params *ipar;
    const int32_t *cinst;
    const int32_t *finst[3];
    const double *ipinv;
    // per-instance step limits (hf_case_set_step_limits): steps left, < 0 no
    // limit; an instance at 0 is frozen: no kernel changes its fields.  Null
    // until limits are set.
    const int64_t *ilim;
};

__device__ __forceinline__ bool frozen(const DevProg &P, int inst)
{
    return P.ilim && __ldg(P.ilim + inst) == 0;
}

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
// arr[d] for a small runtime d without indexing the parameter array
// (a dynamic index would copy the kernel parameters to local memory)
template <int N, typename T>
__device__ __forceinline__ T pick(T const (&arr)[N], int d)
{
    T v = arr[0];
#pragma unroll
    for (int k = 1; k < N; k++)
        if (d == k) v = arr[k];
    return v;
}

// field read by velocity slot s of a facet normal to d (slot table in
// include/higflow_b200.h)
template <int D>
__device__ __forceinline__ const double *vslot_field(const DevFields &F, int d, int s)
{
    if (s == HF_V_FU) return pick<3>(F.FU, d);
    if (s == HF_V_PL || s == HF_V_PR) return F.p;
    if (s == HF_V_FL || s == HF_V_FR) return F.F;
    if (s < HF_V_NSLOT_NEWT(D)) {
        const int d2 = (s - HF_V_BLK0) / HF_V_NB, k = (s - HF_V_BLK0) % HF_V_NB;
        return (k < 4 || k >= 8) ? F.u[d2] : pick<3>(F.u, d);
    }
    const int d2 = (s - HF_V_NSLOT_NEWT(D)) / HF_V_NS;
    return d == 0 ? F.S[d2] : d == 1 ? F.S[D + d2] : F.S[(D - 1) * D + d2];
}

// field of a general-row pair by tag: 0-2 FU[d], 3 p, 4 F, 5-7 u[d], 8-16
// S[d * D + d2], 17-25 K[d * D + d2] (switches: a dynamic index would copy
// the parameters)

__device__ __forceinline__ const double *vtag_field(const DevFields &F, int tag)
{
    switch (tag) {
    case 0: return F.FU[0];
    case 1: return F.FU[1];
    case 2: return F.FU[2];
    case 3: return F.p;
    case 4: return F.F;
    case 5: return F.u[0];
    case 6: return F.u[1];
    case 7: return F.u[2];
    case 8: return F.S[0];
    case 9: return F.S[1];
    case 10: return F.S[2];
    case 11: return F.S[3];
    case 12: return F.S[4];
    case 13: return F.S[5];
    case 14: return F.S[6];
    case 15: return F.S[7];
    case 16: return F.S[8];
    case 17: return F.K[0];
    case 18: return F.K[1];
    case 19: return F.K[2];
    case 20: return F.K[3];
    case 21: return F.K[4];
    case 22: return F.K[5];
    case 23: return F.K[6];
    case 24: return F.K[7];
    default: return F.K[8];
    }
}

// General-row pairs (PairRows), one thread per pair: the long interpolation
// stencils (tens of entries) run here, coalesced and without divergence,
// instead of inside the per-facet and per-cell kernels.  Entry k of the 32
// pairs of a warp is one 128-byte (or 64-byte, 16-bit) column load and one
// 256-byte weight load; the sum is dp_interpolate_from_stencil's
// (pdomain.c:1026-1053): -rhs, then the entries in stencil order, in FP64.
// (launch bounds of the largest block size the tuner tries)
template <bool C16>
__global__ void __launch_bounds__(512) k_vrows(PairRows R, DevFields F)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= R.n) return;
    const int tag = __ldg(R.tag + u);
    const double *__restrict__ fb = vtag_field(F, tag);
    if (C16) fb += __ldg(R.pcol0 + u);
    const int n = __ldg(R.plen + u);
    const int64_t e0 = __ldg(R.sptr + (u >> 5)) + 2 * (u & 31);
    if (R.ilim && n > 0) {
        const int c0 = C16 ? __ldg(R.pcol0 + u) + (int)__ldg(R.scol16 + e0) : __ldg(R.scol + e0);
        if (__ldg(R.ilim + pair_inst(R.finst, R.cinst, tag, c0)) == 0) return;
    }
    const double2 *__restrict__ w2 = reinterpret_cast<const double2 *>(R.sw + e0);
    double res = 0.0;
    res += -__ldg(R.rhs + u);
    // the entries stream through once (evict-first loads keep L1 for the
    // field gathers), two per load, eight entries' loads in flight per thread
#pragma unroll 4
    for (int j = 0; 2 * j < n; j++) {
        const double2 w = __ldcs(w2 + 32 * j);
        int ca, cb;
        if (C16) {
            const int c = __ldcs(reinterpret_cast<const int *>(R.scol16 + e0) + 32 * j);
            ca = (int)(short)(c & 0xffff);
            cb = c >> 16;
        } else {
            const int2 c = __ldcs(reinterpret_cast<const int2 *>(R.scol + e0) + 32 * j);
            ca = c.x;
            cb = c.y;
        }
        res += __ldg(fb + ca) * w.x;
        if (2 * j + 1 < n) res += __ldg(fb + cb) * w.y;
    }
    R.val[u] = res;
}

// PatRows: one thread per pair; -rhs, then the pattern's entries in column
// order, FP64 values times FP32 weights summed in FP64.  Rounding the values
// or the sum to FP32 as well puts noise of about 1e-7 of the velocity into
// every step's Poisson right-hand side that the extrapolated initial guess
// cannot follow (measured on the batched Giesekus cavities at Poisson rtol
// 1e-6: 7.2 CG iterations per instance-step against 4.4 with FP64 sums, 4.0
// for the plain form).
__global__ void __launch_bounds__(512) k_vrows_pat(PatRows R, DevFields F)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= R.n) return;
    const int p = __ldg(R.pid + u);
    const int tag = __ldg(R.tag + u), c0 = __ldg(R.col0 + u);
    if (R.ilim && __ldg(R.ilim + pair_inst(R.finst, R.cinst, tag, c0)) == 0) return;
    const double *__restrict__ fb = vtag_field(F, tag) + c0;
    const int e0 = __ldg(R.pstart + p), n = __ldg(R.plen + p);
    const int2 *__restrict__ ent = reinterpret_cast<const int2 *>(R.ent) + e0;
    double res = 0.0;
    res += -__ldg(R.rhs + u);
#pragma unroll 4
    for (int k = 0; k < n; k++) {
        const int2 e = __ldg(ent + k);
        res += __ldg(fb + e.x) * (double)__int_as_float(e.y);
    }
    R.val[u] = res;
}

// CUBISTA convective flux of the facet velocity along one direction
// (higflow_computational_cell, hig-flow-discret.c:157-260), out of line: k_velocity
// would otherwise carry one inlined copy of these branches per direction.
// conv1 / conv2 come in with the previous direction's values, as in the
// reference, where a NaN ratio leaves them unassigned.
template <typename T>
__device__ __noinline__ void cubista_facet_t(T ufacet, T ul, T ur, T ull, T urr, int infll, int infrr, T vcr, T vcl,
                                             T &conv1, T &conv2)
{
    const T a = T(1.7500), b = T(0.3750), c = T(0.7500), dd = T(0.1250), ee = T(0.2500);
    if (vcr > T(0)) {
        if (hf::flt_eq(ur, ul)) {
            conv1 = vcr * ufacet;
        } else {
            const T fi = (ufacet - ul) / (ur - ul);
            if ((fi <= T(0)) || (fi >= T(1))) {
                conv1 = vcr * ufacet;
            } else {
                if (fi < b) conv1 = vcr * (a * ufacet - c * ul);
                if ((fi >= b) && (fi <= c)) conv1 = vcr * (c * ufacet + b * ur - dd * ul);
                if (fi > c) conv1 = vcr * (ee * ufacet + c * ur);
            }
        }
    } else {
        if (hf::flt_eq(ufacet, urr)) {
            conv1 = vcr * ur;
        } else {
            const T fi = (ur - urr) / (ufacet - urr);
            if ((fi <= T(0)) || (fi >= T(1))) {
                conv1 = vcr * ur;
            } else {
                if (fi < b) conv1 = infrr == 1 ? vcr * (a * ur - c * urr) : vcr * ur;
                if ((fi >= b) && (fi <= c)) conv1 = infrr == 1 ? vcr * (c * ur + b * ufacet - dd * urr) : vcr * ur;
                if (fi > c) conv1 = vcr * (c * ufacet + ee * ur);
            }
        }
    }
    if (vcl > T(0)) {
        if (hf::flt_eq(ufacet, ull)) {
            conv2 = vcl * ul;
        } else {
            const T fi = (ul - ull) / (ufacet - ull);
            if ((fi <= T(0)) || (fi >= T(1))) {
                conv2 = vcl * ul;
            } else {
                if (fi < b) conv2 = infll == 1 ? vcl * (a * ul - c * ull) : vcl * ul;
                if ((fi >= b) && (fi <= c)) conv2 = infll == 1 ? vcl * (b * ufacet + c * ul - dd * ull) : vcl * ul;
                if (fi > c) conv2 = vcl * (c * ufacet + ee * ul);
            }
        }
    } else {
        if (hf::flt_eq(ul, ur)) {
            conv2 = vcl * ufacet;
        } else {
            const T fi = (ufacet - ur) / (ul - ur);
            if ((fi <= T(0)) || (fi >= T(1))) {
                conv2 = vcl * ufacet;
            } else {
                if (fi < b) conv2 = vcl * (a * ufacet - c * ur);
                if ((fi >= b) && (fi <= c)) conv2 = vcl * (b * ul + c * ufacet - dd * ur);
                if (fi > c) conv2 = vcl * (c * ul + ee * ufacet);
            }
        }
    }
}

// (FP64: the reference's arithmetic; the mixed form takes the FP32 instantiation)
template <typename T>
__device__ __forceinline__ double2 cubista_facet(double ufacet, double ul, double ur, double ull, double urr, int infll,
                                                 int infrr, double vcr, double vcl, double conv1, double conv2)
{
    T c1 = (T)conv1, c2 = (T)conv2;
    cubista_facet_t<T>((T)ufacet, (T)ul, (T)ur, (T)ull, (T)urr, infll, infrr, (T)vcr, (T)vcl, c1, c2);
    return make_double2((double)c1, (double)c2);
}

// 128-thread blocks by default: the prefetched slots take ~170 registers per
// thread, and three such blocks fit an SM where one 256-thread block would
// (the tuner also tries 64 and 256)
constexpr int kVelBlock = 128;

// MIX: the mixed form, whose CUBISTA fluxes are evaluated in FP32 (the time
// update and everything else stay FP64)
template <int D, bool VE, bool MIX>
__global__ void __launch_bounds__(256) k_velocity(DevProg P, DevFields F)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= P.off[D]) return;
    int d = 0;
#pragma unroll
    for (int k = 1; k < D; k++) d += (e >= P.off[k]);
    const int f = e - pick<4>(P.off, d);
    const int nf = pick<3>(P.nf, d);
    const int32_t *__restrict__ sl = pick<3>(P.vslots, d);
    int inst = -1;
    if (P.ilim) {
        // under step limits a frozen instance's facets skip their loads
        inst = __ldg(pick<3>(P.finst, d) + f);
        if (frozen(P, inst)) return;
    }
    // every slot code, then every slot value (a centre hit's field entry or a
    // general row's value from k_vrows), as independent loads issued together
    constexpr int NS = VE ? HF_V_NSLOT_VE(D) : HF_V_NSLOT_NEWT(D);
    int32_t code[NS];
    double val[NS];
    // (the u[d] corner slots of the facet's own direction are not read)
    auto unused = [&](int s) {
        return s >= HF_V_BLK0 && s < HF_V_NSLOT_NEWT(D) && (s - HF_V_BLK0) % HF_V_NB < 4 && (s - HF_V_BLK0) / HF_V_NB == d;
    };
#pragma unroll
    for (int s = 0; s < NS; s++) code[s] = unused(s) ? 0 : __ldg(sl + (size_t)s * nf + f);
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const double *src = code[s] >= 0 ? vslot_field<D>(F, d, s) + code[s] : P.vr.val + (-code[s] - 1);
        val[s] = unused(s) ? 0.0 : __ldg(src);
    }
#define SLQ(s, fld) (val[s])
    const double *fd = P.delta + (size_t)__ldg(pick<3>(P.vdelta, d) + f) * D;
    const uint32_t fl = __ldg(pick<3>(P.vflags, d) + f);
    if (inst < 0) inst = __ldg(pick<3>(P.finst, d) + f);
    const hf_params &par = P.ipar[inst];
    int convec = par.convecdiscrtype;
    const int second = par.secondconvecdiscrtype;
    double conv1 = 0.0, conv2 = 0.0;
    const double *ud = pick<3>(F.u, d);
    const double ufacet = __ldg(ud + f);
    double Fs = SLQ(HF_V_FU, pick<3>(F.FU, d));
    // the mixed form divides by each direction's spacing once and multiplies
    // (a quotient within one rounding of the plain form's)
    double ifd[D], ifd2[D];
#pragma unroll
    for (int d2 = 0; d2 < D; d2++) {
        ifd[d2] = MIX ? 1.0 / fd[d2] : 0.0;
        ifd2[d2] = MIX ? 1.0 / (fd[d2] * fd[d2]) : 0.0;
    }
#define HF_QUOT(a, b, inv) (MIX ? (a) * (inv) : (a) / (b))
    const double pl = SLQ(HF_V_PL, F.p);
    const double pr = SLQ(HF_V_PR, F.p);
    const double dpdx = HF_QUOT(pr - pl, 2.0 * 0.5 * fd[d], ifd[d]);
    const double Fl = SLQ(HF_V_FL, F.F);
    const double Fr = SLQ(HF_V_FR, F.F);
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
            const double vrr = SLQ(B + HF_V_V4 + 0, F.u[d2]);
            const double vlr = SLQ(B + HF_V_V4 + 1, F.u[d2]);
            const double vrl = SLQ(B + HF_V_V4 + 2, F.u[d2]);
            const double vll = SLQ(B + HF_V_V4 + 3, F.u[d2]);
            v[d2] = 0.25 * (vll + vlr + vrl + vrr);
        }
        const double ul = SLQ(B + HF_V_UL, ud);
        const int infl = (fl >> (4 * d2 + 0)) & 1;
        if (infl == 0 && convec == HF_SECOND_ORDER) convec = HF_FIRST_ORDER;
        const double ur = SLQ(B + HF_V_UR, ud);
        const int infr = (fl >> (4 * d2 + 1)) & 1;
        if (infr == 0 && convec == HF_SECOND_ORDER) convec = HF_FIRST_ORDER;
        dudxc[d2] = HF_QUOT(ur - ul, 2.0 * 1.0 * fd[d2], 0.5 * ifd[d2]);
        dudxr[d2] = HF_QUOT(ur - ufacet, 1.0 * fd[d2], ifd[d2]);
        dudxl[d2] = HF_QUOT(ufacet - ul, 1.0 * fd[d2], ifd[d2]);
        const double urr = SLQ(B + HF_V_URR, ud);
        const int infrr = (fl >> (4 * d2 + 3)) & 1;
        const double ull = SLQ(B + HF_V_ULL, ud);
        const int infll = (fl >> (4 * d2 + 2)) & 1;
        if (convec == HF_SECOND_ORDER) {
            if (second == HF_QUICK) {
                dudxrr[d2] = HF_QUOT(urr - ur, 1.0 * fd[d2], ifd[d2]);
                dudxll[d2] = HF_QUOT(ul - ull, 1.0 * fd[d2], ifd[d2]);
            } else if (second == HF_CUBISTA) {
                const double vcr = SLQ(B + HF_V_VCR, F.u[d2]);
                const double vcl = SLQ(B + HF_V_VCL, F.u[d2]);
                const double2 cv = cubista_facet<typename std::conditional<MIX, float, double>::type>(
                    ufacet, ul, ur, ull, urr, infll, infrr, vcr, vcl, conv1, conv2);
                conv1 = cv.x;
                conv2 = cv.y;
                vc[d2] = HF_QUOT(conv1 - conv2, fd[d], ifd[d]);
            }
        }
        du2dx2[d2] = HF_QUOT(ul - 2.0 * ufacet + ur, fd[d2] * fd[d2] * 1.0 * 1.0, ifd2[d2]);
    }
    double tens = 0.0;
    if (VE) {
        double dSdx[D];
#pragma unroll
        for (int d2 = 0; d2 < D; d2++) {
            const int B = HF_V_NSLOT_NEWT(D) + HF_V_NS * d2;
            const double *Sf = vslot_field<D>(F, d, HF_V_NSLOT_NEWT(D) + HF_V_NS * d2);
            if (d2 == d) {
                const double Sl = SLQ(B + 0, Sf);
                const double Sr = SLQ(B + 2, Sf);
                dSdx[d2] = HF_QUOT(Sr - Sl, 2.0 * 0.5 * fd[d2], ifd[d2]);
            } else {
                const double l1 = SLQ(B + 0, Sf);
                const double l2 = SLQ(B + 1, Sf);
                const double Sl = 0.5 * (l1 + l2);
                const double r1 = SLQ(B + 2, Sf);
                const double r2 = SLQ(B + 3, Sf);
                const double Sr = 0.5 * (r1 + r2);
                dSdx[d2] = HF_QUOT(Sr - Sl, 2.0 * 1.0 * fd[d2], 0.5 * ifd[d2]);
            }
        }
#pragma unroll
        for (int d2 = 0; d2 < D; d2++) tens += dSdx[d2];
    }
#undef SLQ
#undef HF_QUOT
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
    if (P.sie) {
        // semi-implicit Euler (hig-flow-step.c:812-829; viscoelastic
        // hig-flow-step-viscoelastic.c:1136-1147): diffusion moves to the
        // system matrix; its boundary part is added to the right-hand side.
        // Crank-Nicolson (hig-flow-step.c:908-917, viscoelastic :1243-1257)
        // keeps half of the diffusion here.
        if (par.tempdiscrtype == HF_SEMI_IMPLICIT_BDF2) {
            // hig-flow-step.c:1020-1033 (viscoelastic :1349-1363): the bracket
            // is kept for the second solve's right-hand side (k_bdf2_rhs)
            double e = 0.0;
            e += Fs;
            e -= pterm;
            if (VE) e += tens;
            e -= conv;
            pick<3>(P.sie_e, d)[f] = e;
            double rhs = e;
            rhs *= 0.5 * par.dt;
            rhs += 0.25 * par.dt * diff;
            rhs += ufacet;
            pick<3>(P.sie_b, d)[f] = rhs + __ldg(pick<3>(P.sie_bc, d) + f);
            return;
        }
        double rhs = 0.0;
        if (par.tempdiscrtype == HF_SEMI_IMPLICIT_CN) rhs += 0.5 * diff;
        rhs += Fs;
        rhs -= pterm;
        if (VE) rhs += tens;
        rhs -= conv;
        rhs *= par.dt;
        rhs += ufacet;
        pick<3>(P.sie_b, d)[f] = rhs + __ldg(pick<3>(P.sie_bc, d) + f);
        return;
    }
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
    pick<3>(F.us, d)[f] = ufacet + par.dt * rhs;
}

// ---------------------------------------------------------------------------
// viscoelastic cell stage (Du, constitutive update, polymeric tensor)
// ---------------------------------------------------------------------------
// 128-thread blocks capped at 64 registers in 2D (8 blocks, 32 warps per SM):
// the kernel is latency bound, and occupancy beats the spills it costs
// (measured on 4.29 M cells: 4 blocks 1.60 ms, 5: 1.38, 6: 1.31, 7: 1.24,
// 8: 1.22, 16 at 32 registers: 1.19 with far more spill traffic)
constexpr int kVeBlock = 128;

// The GPTT model's Mittag-Leffler factor of every GPTT cell, from the stress
// that k_ve_cell then reads (trace summed in its order).  A kernel of its own:
// the out-of-line evaluation inside k_ve_cell would spill that kernel's
// registers for every model.
template <int D>
__global__ void __launch_bounds__(kBlock) k_gptt_ml(DevProg P, DevFields F)
{
    const int cc = blockIdx.x * blockDim.x + threadIdx.x;
    if (cc >= P.ncell) return;
    const int inst = __ldg(P.cinst + cc);
    if (frozen(P, inst)) return;
    const hf_params &pr = P.ipar[inst];
    if (pr.ve_model != HF_GPTT) return;
    double trS = 0.0;
#pragma unroll
    for (int i = 0; i < D; i++) trS += F.S[i * D + i][cc];
    P.gptt_e[cc] = hf::gptt_ml(pr.alpha_gptt, pr.beta_gptt, pr.epsilon * pr.Re * pr.De * trS / (1.0 - pr.beta));
}

// IMPL: the implicit constitutive step (hf_params.ve_discrtype, the same for
// every instance of a case), a separate instantiation so that the explicit
// kernel carries none of its code
// MIX: the mixed form, whose CUBISTA cell convection is evaluated in FP32 and
// whose velocity derivatives and M/De term multiply by reciprocals (within one
// rounding of the quotients; the eigensystem, kernel transform and time
// update stay FP64 and as the reference computes them)
template <int D, bool IMPL, bool MIX>
__global__ void __launch_bounds__(kVeBlock, D == 2 ? 8 : 4) k_ve_cell(DevProg P, DevFields F)
{
    const int cc = blockIdx.x * blockDim.x + threadIdx.x;
    if (cc >= P.ncell) return;
    const int n = P.ncell;
#define CS(s) __ldg(P.cslots + (size_t)(s) * n + cc)
    const double *cd = P.delta + (size_t)__ldg(P.cdelta + cc) * D;
    const uint32_t fl = __ldg(P.cflags + cc);
    const int inst = __ldg(P.cinst + cc);
    if (frozen(P, inst)) {
        // the stage's output replaces K after it (pointer swap): carry K over
#pragma unroll
        for (int k = 0; k < D * D; k++) F.Knew[k][cc] = F.K[k][cc];
        return;
    }
    const hf_params &pr = P.ipar[inst];
    // The velocity values this cell reads: its face velocities (u[dim] at
    // -/+ half a cell, UVL/UVR) and the Du corner queries (HF_C_NQ per ordered
    // pair dim != dim2, on u[dim]).  All slot codes, then all values as
    // independent loads: a centre hit from the field, a general row (cells at
    // boundaries) from its cell-stage pair, which k_vrows evaluated.
    constexpr int NU = 2 * D, NQ = HF_C_NQ * D * (D - 1);
    int32_t cu[NU + NQ];
    double vu[NU + NQ];
    auto uslot = [](int k) { return k < NU ? HF_C_BLK0 + HF_C_NB * (k >> 1) + (k & 1) : HF_C_BLK0 + HF_C_NB * D + (k - NU); };
    auto ufield = [&](int k) { return F.u[k < NU ? (k >> 1) : (k - NU) / (HF_C_NQ * (D - 1))]; };
#pragma unroll
    for (int k = 0; k < NU + NQ; k++) cu[k] = CS(uslot(k));
#pragma unroll
    for (int k = 0; k < NU + NQ; k++) vu[k] = cu[k] >= 0 ? __ldg(ufield(k) + cu[k]) : __ldg(P.cr.val + (-cu[k] - 1));
    // velocity at the faces of this cell, shared by Du, u_c and the CUBISTA flux
    double vl[D], vr[D];
#pragma unroll
    for (int dim = 0; dim < D; dim++) {
        vl[dim] = vu[2 * dim + 0];
        vr[dim] = vu[2 * dim + 1];
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
                    const int Q = NU + HF_C_NQ * pair;
                    pair++;
                    double vrr = vu[Q + 0];
                    double vll = vu[Q + 1];
                    ul = 0.25 * (vll + vl[dim] + vr[dim] + vrr);
                    vrr = vu[Q + 2];
                    vll = vu[Q + 3];
                    ur = 0.25 * (vll + vl[dim] + vr[dim] + vrr);
                }
                // (mixed form: times the reciprocal spacing, within one rounding)
                Du[dim][dim2] = MIX ? (ur - ul) * (1.0 / cd[dim2]) : (ur - ul) / (2.0 * 0.5 * cd[dim2]);
                F.Du[dim * D + dim2][cc] = Du[dim][dim2];
            }
        }
    }
    // constitutive step (hig-flow-step-viscoelastic.c:384-521); the self slot
    // is the cell's own index (checked at create)
    const double Re = pr.Re, De = pr.De, tol = pr.kernel_tol, small = HF_EPSMACH;
    const double iDe = MIX ? 1.0 / De : 0.0;
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
            if (pr.ve_model == HF_LPTT || pr.ve_model == HF_GPTT) Mt[i][j] -= pr.xi * 0.5 * (Du[i][j] + Du[j][i]);
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
    // e-FENE (hig_flow_calculate_m_e_fene, hig-flow-step-viscoelastic.c:1855-1876)
    double fA = 0.0;
    if (pr.ve_model == HF_E_FENE) {
        double trA = 0.0;
#pragma unroll
        for (int i = 0; i < D; i++) trA += lam[i];
        const double b = pr.L2_fene, lf = pr.lambda_fene, E = pr.E_fene;
        fA = b / (b - trA) - E * sqrt(b) * exp(-sqrt(trA) / lf) * (1.0 / (trA * lf) + 1 / (trA * sqrt(trA)));
    }
    // GPTT (hig_flow_calculate_m_gptt, :1771-1830): Gamma(beta_g) times the
    // Mittag-Leffler E_{alpha_g,beta_g}(eps Re De tr S / (1 - beta)) in place of
    // LPTT's linear factor
    double mlv = 0.0;
    if (pr.ve_model == HF_GPTT) mlv = P.gptt_e[cc];
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
        } else if (pr.ve_model == HF_GPTT) {
            Ma[i][i] = (1.0 - lam[i]) * pr.gamma_gptt * mlv * jl[i];
        } else if (pr.ve_model == HF_E_FENE) {
            Ma[i][i] = (1.0 - fA * lam[i]) * jl[i];
        } else {
            Ma[i][i] = (1.0 - lam[i]) * jl[i];
        }
    }
    hf::mtprod<D>(Ba, Rm, BB);
    hf::mtprod<D>(Ma, Rm, MM);
    // explicit: RHS = Omega K - K Omega + 2B + M/De (hig_flow_kernel_rhs);
    // implicit: RHS = 2B + M/De (hig_flow_implicit_kernel_rhs, :1956-1963), the
    // Omega terms being in the per-cell system
    constexpr bool implicit = IMPL;
    double RHS[D][D];
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) {
            if (implicit) {
                RHS[i][j] = 2.0 * BB[i][j] + (MIX ? MM[i][j] * iDe : MM[i][j] / De);
                continue;
            }
            double ok = 0.0, ko = 0.0;
#pragma unroll
            for (int k = 0; k < D; k++) {
                ok += Om[i][k] * K[k][j];
                ko += K[i][k] * Om[k][j];
            }
            RHS[i][j] = ok - ko + 2.0 * BB[i][j] + (MIX ? MM[i][j] * iDe : MM[i][j] / De);
        }
    // the kernel's neighbour values: per direction KL, KR, KLL, KRR (the same
    // codes for every component; a general row's pairs are the upper
    // triangle's components in row-major order), loaded component by
    // component, all directions at once
    // (KLL/KRR are loaded for every cell, so that no load waits for the
    // instance's parameters; without CUBISTA their values go unused)
    const bool cub = pr.ve_convecdiscrtype == HF_CELL_CUBISTA;
    int32_t ck[4 * D];
#pragma unroll
    for (int k = 0; k < 4 * D; k++) ck[k] = CS(HF_C_BLK0 + HF_C_NB * (k >> 2) + HF_C_KL + (k & 3));
    double Knew[D][D];
    double bsys[D * D];   // implicit form: the per-cell system's right-hand side
#pragma unroll
    for (int i = 0; i < D; i++) {
#pragma unroll
        for (int j = i; j < D; j++) {
            const double *Kf = F.K[i * D + j];
            const int m = i * D - i * (i - 1) / 2 + (j - i);   // upper-triangle index of (i, j)
            double kv[4 * D];
#pragma unroll
            for (int k = 0; k < 4 * D; k++) kv[k] = ck[k] >= 0 ? __ldg(Kf + ck[k]) : __ldg(P.cr.val + (-ck[k] - 1) + m);
            double rhs = 0.0;
#pragma unroll
            for (int dim = 0; dim < D; dim++) {
                const int il = (fl >> (4 * dim + 0)) & 1, ir = (fl >> (4 * dim + 1)) & 1;
                const int ill = (fl >> (4 * dim + 2)) & 1, irr = (fl >> (4 * dim + 3)) & 1;
                const double kl = kv[4 * dim + 0];
                const double kr = kv[4 * dim + 1];
                if (cub) {
                    const double kll = kv[4 * dim + 2];
                    const double krr = kv[4 * dim + 3];
                    if (MIX)
                        rhs -= (double)hf::cubista_cell_t<float>((float)kl, (float)kr, (float)kll, (float)krr, il, ir,
                                                                 ill, irr, (float)vl[dim], (float)vr[dim],
                                                                 (float)K[i][j], (float)cd[dim]);
                    else
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
            if (implicit) {
                // hig-flow-step-viscoelastic.c:861-864 for (i, j) and (j, i);
                // their convective parts are equal (K is stored symmetric)
                double r1 = rhs;
                r1 += RHS[i][j];
                r1 *= pr.dt;
                r1 += K[i][j];
                bsys[i * D + j] = r1;
                if (j != i) {
                    double r2 = rhs;
                    r2 += RHS[j][i];
                    r2 *= pr.dt;
                    r2 += K[j][i];
                    bsys[j * D + i] = r2;
                }
                continue;
            }
            rhs += RHS[i][j];
            const double kernel = K[i][j] + pr.dt * rhs;
            Knew[i][j] = kernel;
            Knew[j][i] = kernel;
        }
    }
    if (implicit) {
        double om[D * D];
#pragma unroll
        for (int i = 0; i < D; i++)
#pragma unroll
            for (int j = 0; j < D; j++) om[i * D + j] = Om[i][j];
        hf::implicit_kernel_solve<D>(om, pr.dt, bsys);
        // the upper triangle of the solution, mirrored (:868-877)
#pragma unroll
        for (int i = 0; i < D; i++)
#pragma unroll
            for (int j = i; j < D; j++) {
                Knew[i][j] = bsys[i * D + j];
                Knew[j][i] = bsys[i * D + j];
            }
    }
#undef CS
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) F.Knew[i * D + j][cc] = Knew[i][j];
}

// Polymeric tensor from the new kernel (hig-flow-step-viscoelastic.c:244-318),
// one thread per cell, after k_ve_cell (F as k_ve_cell saw it: K_new holds
// the new kernel).  Kept apart from k_ve_cell so that neither kernel carries
// both eigensolves: fewer registers per thread and less code per launch.
template <int D>
__global__ void __launch_bounds__(kBlock) k_ve_stress(DevProg P, DevFields F)
{
    const int cc = blockIdx.x * blockDim.x + threadIdx.x;
    if (cc >= P.ncell) return;
    const int inst = __ldg(P.cinst + cc);
    if (frozen(P, inst)) return;
    const hf_params &pr = P.ipar[inst];
    const double Re = pr.Re, De = pr.De;
    double Knew[D][D], Du[D][D];
#pragma unroll
    for (int i = 0; i < D; i++)
#pragma unroll
        for (int j = 0; j < D; j++) {
            Knew[i][j] = F.Knew[i * D + j][cc];
            Du[i][j] = F.Du[i * D + j][cc];
        }
    double lam2[D], R2[D][D], Bk[D][D], A[D][D];
    hf::jacobi<D>(Knew, lam2, R2);
#pragma unroll
    for (int i = 0; i < D; i++) {
#pragma unroll
        for (int j = i + 1; j < D; j++) { Bk[i][j] = 0.0; Bk[j][i] = 0.0; }
        Bk[i][i] = hf::kernel_inverse(pr.kernel, lam2[i]);
    }
    hf::mtprod<D>(Bk, R2, A);
    // the model switch of hig-flow-step-viscoelastic.c:274-309: LPTT and GPTT set xi;
    // e-FENE computes its fA there but falls through to the default, so its
    // stress is formed with fA = a = 1, xi = 0 like Oldroyd-B and Giesekus
    const double fA = 1.0, aa = 1.0, beta = pr.beta;
    const double xi = pr.ve_model == HF_LPTT || pr.ve_model == HF_GPTT ? pr.xi : 0.0;
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
#include "hf_pcg.cuh"

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

// Runge-Kutta combinations of the intermediate velocity on every facet
// (hig-flow-step.c:697, :772): which 0: u* = 0.5 (u + u*); 2: u* = u/3 + 2 u*/3
template <int D>
__global__ void __launch_bounds__(kBlock) k_rk_combine(DevProg P, DevFields F, int which)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= P.off[D]) return;
    int d = 0;
#pragma unroll
    for (int k = 1; k < D; k++) d += (e >= P.off[k]);
    const int f = e - pick<4>(P.off, d);
    if (frozen(P, __ldg(pick<3>(P.finst, d) + f))) return;
    const double u = pick<3>(F.u, d)[f], ustar = pick<3>(F.us, d)[f];
    if (which == 0) pick<3>(F.us, d)[f] = 0.5 * (u + ustar);
    else pick<3>(F.us, d)[f] = u / 3.0 + 2.0 * ustar / 3.0;
}

// BDF2's second right-hand side (hig-flow-step.c:1119-1120, viscoelastic
// hig-flow-step-viscoelastic.c:1452-1453): bracket * (dt/3)
// + (4 uaux - u)/3, plus the second system's boundary part; facets of one
// direction
__global__ void __launch_bounds__(kBlock) k_bdf2_rhs(int n, double dt, const double *__restrict__ e,
                                                   const double *__restrict__ ua, const double *__restrict__ u,
                                                   const double *__restrict__ bc2, double *__restrict__ b)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
    double rhs = e[f];
    rhs *= 1.0 / 3.0 * dt;
    rhs += (4.0 * ua[f] - u[f]) / 3.0;
    b[f] = rhs + bc2[f];
}

// CFL number of every instance (higflow_compute_CFL, hig-flow-timestep.c:7-40):
// per cell, sum over d of |(u_l + u_r) / 2| / (the cell's face area normal to d),
// u_l and u_r the face velocities (the divergence's own queries, on u); the
// instance's maximum by an atomic max on the bit patterns (non-negative doubles
// order as their bits, so the result does not depend on the order).
template <int D>
__global__ void __launch_bounds__(kBlock) k_cfl(DevProg P, DevFields F, unsigned long long *imax)
{
    const int cc = blockIdx.x * blockDim.x + threadIdx.x;
    if (cc >= P.ncell) return;
    const int n = P.ncell;
    const double *cd = P.delta + (size_t)__ldg(P.cdelta + cc) * D;
    double u_dx_norm = 0.0;
#pragma unroll
    for (int dim = 0; dim < D; dim++) {
        const double ul = hf::query(P.rows, __ldg(P.dslots + (size_t)HF_P_UL(dim) * n + cc), F.u[dim]);
        const double ur = hf::query(P.rows, __ldg(P.dslots + (size_t)HF_P_UR(dim) * n + cc), F.u[dim]);
        const double u = (ul + ur) / 2.0;
        double facet_area = 1.0;
#pragma unroll
        for (int dim2 = 0; dim2 < D; dim2++)
            if (dim2 != dim) facet_area *= cd[dim2];
        u_dx_norm += fabs(u) / facet_area;
    }
    if (u_dx_norm > 0.0)
        atomicMax(imax + __ldg(P.cinst + cc), (unsigned long long)__double_as_longlong(u_dx_norm));
}

// BiCGStab start on a given system: r = b - A x, scalars reset; first: the
// tolerance from ||b|| (hf_slv_solve, the semi-implicit velocity systems)
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
        const int f = e - pick<4>(P.off, d);
        const int nf = pick<3>(P.nf, d);
        const int inst = __ldg(pick<3>(P.finst, d) + f);
        if (frozen(P, inst)) return;
        const hf_params &par = P.ipar[inst];
        const int pt = P.projtype_all >= 0 ? P.projtype_all : par.projtype;
        const double *pp = pt == HF_INCREMENTAL ? F.dp : F.p;
        const double *fd = P.delta + (size_t)__ldg(pick<3>(P.vdelta, d) + f) * D;
        const int32_t *sl = pick<3>(P.vslots, d);
        const int32_t cl = __ldg(sl + (size_t)HF_V_PL * nf + f), cr = __ldg(sl + (size_t)HF_V_PR * nf + f);
        const double pl = hf::query(P.vrow, cl, pp);
        const double pr = hf::query(P.vrow, cr, pp);
        const double dpdx = (pr - pl) / (2.0 * 0.5 * fd[d]);
        pick<3>(F.u, d)[f] = __ldg(pick<3>(F.us, d) + f) - par.dt * dpdx;
    } else {
        const int c = e - P.off[D];
        if (c < P.ncell && !frozen(P, __ldg(P.cinst + c)) &&
            (P.projtype_all >= 0 ? P.projtype_all : P.ipar[__ldg(P.cinst + c)].projtype) == HF_INCREMENTAL)
            F.p[c] = F.p[c] + F.dp[c];
    }
}


// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int blocks(long n) { return (int)((n + kBlock - 1) / kBlock); }

template <typename T>
int upload(std::vector<void *> &owned, T **dst, const T *src, size_t n, double &bytes, cudaStream_t st = nullptr)
{
    *dst = nullptr;
    size_t nb = sizeof(T) * (n ? n : 1);
    if (st) {
        // stream-ordered: no device-wide synchronisation, so cases can be
        // created and freed while others are stepping (or being captured)
        HF_CK(cudaMallocAsync((void **)dst, nb, st));
        owned.push_back(*dst);
        bytes += (double)nb;
        if (n && src) HF_CK(cudaMemcpyAsync(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice, st));
        else HF_CK(cudaMemsetAsync(*dst, 0, nb, st));
        return HF_OK;
    }
    HF_CK(cudaMalloc((void **)dst, nb));
    owned.push_back(*dst);
    bytes += (double)nb;
    if (n && src) HF_CK(cudaMemcpy(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice));
    else HF_CK(cudaMemset(*dst, 0, nb));
    return HF_OK;
}

// Freed stream-ordered memory stays in the device's default pool for the next
// case instead of going back to the driver at every synchronisation.
void keep_pool_memory(int dev)
{
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lk(mu);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    done.push_back(dev);
}

}  // namespace

struct hf_case {
    hf_options opt;
    hf_params par;
    int D;
    DevProg P;
    DevFields F;
    DevMat M;
    BiVec bi;
    bool use_cg;
    // semi-implicit Euler: per direction (I - dt/Re Lap_h) as CSR, solved by
    // BiCGStab into u* (scratch Vu shared by the directions)
    bool sie = false;
    bool bdf2 = false;
    bool gptt = false;              // some instance uses the GPTT model
    DevMat Mu[3] = {};
    DevMat Mu2[3] = {};             // BDF2: the second solve's systems
    double *ua[3] = {};             // BDF2: the first solve's velocity (dpuaux)
    BiVec Vu{};
    int64_t vel_iters = 0;          // their BiCGStab iterations, all steps
    int64_t sie_launches = 0;       // their kernels, all steps
    int sie_rc = 0;                 // status of the last step's solves
    std::vector<hf_params> h_ipar;  // per-instance parameters as last uploaded
    std::vector<double> dt0;        // per-instance dt at create (adaptive time step)
    unsigned long long *cfl_max = nullptr;   // per-instance CFL scratch
    // instances
    int ninst = 1;
    std::vector<int> coff;          // ninst + 1
    std::vector<int> foff[3];       // ninst + 1 per direction
    // batched AMG-PCG (hf_pcg.cuh) and the graphs that run one step each
    bool amg = false;
    bool bi_amg = false;            // BiCGStab path preconditioned by the AMG V-cycle
    bool mixed = false;
    PcgFine G{};
    double *pa = nullptr, *pb = nullptr;   // CG directions (alternating)
    float *pa32 = nullptr, *pb32 = nullptr;   // the mixed form's inner directions
    int nlev = 1;                   // multigrid levels including the finest
    VLev<double> L64[kMaxLevels] = {};
    VLev<float> L32[kMaxLevels] = {};
    int nreg = 0;                   // levels run by level-synchronous kernels (above every tail)
    VLev<double> *h64 = nullptr;    // the level tables in device memory (tail kernel)
    VLev<float> *h32 = nullptr;
    TailInst<double> *t64 = nullptr;
    TailInst<float> *t32 = nullptr;
    int64_t coarse_rows = 0, coarse_dense = 0;
    std::vector<int64_t> lrows, lnnz_a, lnnz_p, lnnz_r;
    int body_kernels = 0;           // kernels of one loop body (two iterations)
    int fixed_kernels = 0;          // kernels of a step outside the loop
    IScal *h_S = nullptr;           // pinned mirrors
    Ctl *h_ctl = nullptr;
    cudaStream_t body_stream = nullptr;
    cudaGraph_t graph[2] = {};
    cudaGraphExec_t exec[2] = {};
    int64_t ntemplates = 0;         // row templates of the finest Poisson operator
    int64_t vel_entries = 0;        // stored entries of the velocity-stage rows (padded slices; patterns)
    bool vmix = false;              // mixed form's velocity and cell stages (FP32 weights, FP32 CUBISTA)
    PatRows vp = {};                // mixed form: the velocity-stage pairs by FP32 pattern
    int64_t cell_entries = 0;       // ... and of the cell-stage rows
    int64_t *ilim = nullptr;        // per-instance step limits on the device (null: none)
    // launch shapes of the tuned kernels (hf_options.tuning): k_vrows,
    // k_velocity, k_ve_cell block sizes; tuned before the first step
    int blk_vrows = kBlock, blk_vel = kVelBlock, blk_ve = kVeBlock;
    bool tuned = false;
    bool graph_profile = false;     // graphs were captured with phase events
    bool phase_pending = false;     // a profiled step's events are not read yet
    bool capturing = false;         // a step graph is being captured
    int64_t bodies0 = 0;            // loop bodies before that step
    int parity = 0;
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
    // symmetry check: every (r, c, v) must have a matching (c, r, v) up to
    // the rounding of HigTree's weights, which grows with the mesh (up to
    // 1.4e-13 relative measured on 512^2 cavities and 640 x 160 channels);
    // rows that are structurally non-symmetric differ at O(1)
    symmetric = true;
    for (int r = 0; r < n && symmetric; r++) {
        for (int k = ptr[r]; k < ptr[r + 1]; k++) {
            int c = col[k];
            if (c == r) continue;
            bool found = false;
            for (int m = ptr[c]; m < ptr[c + 1]; m++)
                if (col[m] == r) {
                    found = fabs(val[m] - val[k]) <= 1e-10 * fabs(val[k]);
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

// A CSR matrix as row templates: rows whose entries have the same column
// offsets from the row's anchor and the same values, in entry order, share one
// template.  The anchor is the row index (square operators, rd only) or the
// row's first column (transfer operators, kept in base).
struct TemplateForm {
    std::vector<uint32_t> rd;    // per row: (first entry << kTLenBits) | entry count
    std::vector<int32_t> base;   // per row: anchor column (first-column anchors)
    std::vector<int32_t> toff;
    std::vector<double> tval;
    bool ok = false;             // false: a row too long or too many entries
};

TemplateForm make_templates(const std::vector<int32_t> &ptr, const std::vector<int32_t> &col,
                            const std::vector<double> &val, bool anchor_is_row)
{
    TemplateForm t;
    const int n = (int)ptr.size() - 1;
    t.rd.resize(n);
    if (!anchor_is_row) t.base.resize(n);
    // 64-bit content hash -> descriptor; a hash shared by different contents
    // moves to the next hash value (open addressing over the key space)
    std::unordered_map<uint64_t, uint32_t> seen;
    seen.reserve(1024);
    for (int i = 0; i < n; i++) {
        const int a = ptr[i], len = ptr[i + 1] - a;
        if (len >= (1 << kTLenBits)) return t;
        const int32_t anchor = anchor_is_row ? i : (len ? col[a] : 0);
        if (!anchor_is_row) t.base[i] = anchor;
        uint64_t h = 0x9e3779b97f4a7c15ull ^ (uint64_t)len;
        for (int k = a; k < a + len; k++) {
            uint64_t v;
            memcpy(&v, &val[k], sizeof v);
            h = (h ^ (uint64_t)(uint32_t)(col[k] - anchor)) * 0x100000001b3ull;
            h = (h ^ v) * 0x100000001b3ull;
            h ^= h >> 29;
        }
        for (;; h++) {
            auto it = seen.find(h);
            if (it == seen.end()) {
                if (t.toff.size() + len >= ((size_t)1 << (32 - kTLenBits))) return t;
                const uint32_t d = ((uint32_t)t.toff.size() << kTLenBits) | (uint32_t)len;
                for (int k = a; k < a + len; k++) {
                    t.toff.push_back(col[k] - anchor);
                    t.tval.push_back(val[k]);
                }
                seen.emplace(h, d);
                t.rd[i] = d;
                break;
            }
            const uint32_t d = it->second;
            const int k0 = (int)(d >> kTLenBits);
            bool same = (int)(d & ((1u << kTLenBits) - 1)) == len;
            for (int k = 0; same && k < len; k++)
                same = t.toff[k0 + k] == col[a + k] - anchor && memcmp(&t.tval[k0 + k], &val[a + k], sizeof(double)) == 0;
            if (same) {
                t.rd[i] = d;
                break;
            }
        }
    }
    t.ok = true;
    return t;
}

// Host copy of one concatenated level of the batched hierarchy.
struct LevelHost {
    int n = 0;
    std::vector<int32_t> Ap, Ac, Pp, Pc, Rp, Rc;
    std::vector<double> Av, dinv, Pv, Rv;
    std::vector<Blk> sblk, ablk;
    TemplateForm At, Pt, Rt;   // the same operators as templates (coarse A; P, R)
};

struct LevelOff {
    size_t Ap, Ac, Av, dinv, Pp, Pc, Pv, Rp, Rc, Rv, b, x, r, out, sblk, ablk;
    size_t Ard, Atoff, Atval, Prb, Ptoff, Ptval, Rrb, Rtoff, Rtval;
};

std::vector<uint2> pack_rb(const TemplateForm &t)
{
    std::vector<uint2> rb(t.rd.size());
    for (size_t i = 0; i < rb.size(); i++) rb[i] = make_uint2(t.rd[i], (uint32_t)t.base[i]);
    return rb;
}

// Blocks of kBlock rows over the instances a level-synchronous kernel of level
// l covers: smooth_only, the instances smoothed there by those kernels (l below
// the instance's tail level s); otherwise every instance on the finest level
// and, on a coarser level, those whose rows the regular restriction fills
// (l up to s).
// Blocks hold kBlockRows rows (kRPT per thread) on levels large enough to
// fill the device several times over, kBlock rows (one per thread) below that.
std::vector<Blk> block_table(const std::vector<std::vector<int>> &off, const std::vector<int> &tail, int l,
                             bool smooth_only)
{
    std::vector<Blk> t;
    const int ni = (int)tail.size();
    const int chunk = off[l][ni] >= (1 << 19) ? kBlockRows : kBlock;
    for (int i = 0; i < ni; i++) {
        if (smooth_only ? l >= tail[i] : (l > 0 && l > tail[i])) continue;
        const int r0 = off[l][i], rows = off[l][i + 1] - r0;
        const int nb = (rows + chunk - 1) / chunk, first = (int)t.size();
        for (int b = 0; b < nb; b++)
            t.push_back(Blk{r0 + b * chunk, std::min(chunk, rows - b * chunk), i, first, nb, 0, 0, 0});
    }
    return t;
}

template <typename T>
LevelOff place_level(Arena &ar, const LevelHost &h, bool fine)
{
    LevelOff o{};
    if (!fine) {
        o.Ap = ar.vec(h.Ap);
        o.Ac = ar.vec(h.Ac);
        o.b = ar.zeros<T>(h.n);
    }
    if (!fine) o.Av = ar.vec(cast_vec<T>(h.Av));   // the finest level's operator is the row templates
    o.dinv = ar.vec(cast_vec<T>(h.dinv));   // omega D^-1 (the finest level's too)
    if (!h.Pp.empty()) {
        o.Pp = ar.vec(h.Pp); o.Pc = ar.vec(h.Pc); o.Pv = ar.vec(cast_vec<T>(h.Pv));
        o.Rp = ar.vec(h.Rp); o.Rc = ar.vec(h.Rc); o.Rv = ar.vec(cast_vec<T>(h.Rv));
    }
    if (h.At.ok) {
        o.Ard = ar.vec(h.At.rd); o.Atoff = ar.vec(h.At.toff); o.Atval = ar.vec(cast_vec<T>(h.At.tval));
    }
    if (h.Pt.ok) {
        o.Prb = ar.vec(pack_rb(h.Pt)); o.Ptoff = ar.vec(h.Pt.toff); o.Ptval = ar.vec(cast_vec<T>(h.Pt.tval));
    }
    if (h.Rt.ok) {
        o.Rrb = ar.vec(pack_rb(h.Rt)); o.Rtoff = ar.vec(h.Rt.toff); o.Rtval = ar.vec(cast_vec<T>(h.Rt.tval));
    }
    o.x = ar.zeros<T>(h.n);
    o.r = ar.zeros<T>(h.n);
    o.out = ar.zeros<T>(h.n);
    o.sblk = ar.vec(h.sblk);
    o.ablk = ar.vec(h.ablk);
    return o;
}

template <typename T>
VLev<T> make_level(char *base, const LevelOff &o, const LevelHost &h, const TRows<T> &At, bool fine)
{
    VLev<T> v{};
    v.n = h.n;
    if (fine) {
        v.At = At;
    } else {
        v.Ap = (const int32_t *)(base + o.Ap);
        v.Ac = (const int32_t *)(base + o.Ac);
        v.b = (T *)(base + o.b);
    }
    if (o.Av) v.Av = (const T *)(base + o.Av);
    if (o.dinv) v.dinv = (const T *)(base + o.dinv);
    if (o.Pp) {
        v.Pp = (const int32_t *)(base + o.Pp); v.Pc = (const int32_t *)(base + o.Pc); v.Pv = (const T *)(base + o.Pv);
        v.Rp = (const int32_t *)(base + o.Rp); v.Rc = (const int32_t *)(base + o.Rc); v.Rv = (const T *)(base + o.Rv);
    }
    if (o.Ard) v.At = TRows<T>{(const uint32_t *)(base + o.Ard), (const int32_t *)(base + o.Atoff), (const T *)(base + o.Atval)};
    if (o.Prb) v.Pt = BRows<T>{(const uint2 *)(base + o.Prb), (const int32_t *)(base + o.Ptoff), (const T *)(base + o.Ptval)};
    if (o.Rrb) v.Rt = BRows<T>{(const uint2 *)(base + o.Rrb), (const int32_t *)(base + o.Rtoff), (const T *)(base + o.Rtval)};
    v.x = (T *)(base + o.x);
    v.r = (T *)(base + o.r);
    v.out = (T *)(base + o.out);
    v.sblk = (const Blk *)(base + o.sblk);
    v.ablk = (const Blk *)(base + o.ablk);
    v.nsblk = (int)h.sblk.size();
    v.nablk = (int)h.ablk.size();
    return v;
}

// Per-instance smoothed-aggregation hierarchies (hf_amg.cuh), concatenated
// level by level, the finest-level CG state and the loop control.
int build_pcg(hf_case *C, const std::vector<int32_t> &mptr, const std::vector<int32_t> &mcol,
              const std::vector<double> &mval, const std::vector<int> &pins)
{
    const int ni = C->ninst;
    const bool amg = C->amg, mixed = C->mixed;
    struct InstHier {
        std::vector<hf::HostLevel> H;
        std::vector<double> inv;   // row-major
        std::string err;
    };
    std::vector<InstHier> IH(ni);
    std::vector<int> clev(ni, 0);
    if (amg) {
        std::atomic<int> next{0};
        auto work = [&]() {
            for (int i; (i = next++) < ni;) {
                InstHier &ih = IH[i];
                const int c0 = C->coff[i], n = C->coff[i + 1] - c0;
                hf::HostCSR A;
                A.n = A.m = n;
                A.ptr.assign(n + 1, 0);
                for (int r = 0; r < n && ih.err.empty(); r++) {
                    for (int k = mptr[c0 + r]; k < mptr[c0 + r + 1]; k++) {
                        const int c = mcol[k] - c0;
                        if (c < 0 || c >= n) { ih.err = "Poisson row reaches another instance"; break; }
                        A.col.push_back(c);
                        A.val.push_back(mval[k]);
                    }
                    A.ptr[r + 1] = (int)A.col.size();
                }
                if (!ih.err.empty()) continue;
                ih.H = hf::build_hierarchy(std::move(A), kMaxCoarse, kMaxLevels);
                const hf::HostLevel &last = ih.H.back();
                if (!last.P.ptr.empty()) { ih.err = "AMG hierarchy deeper than the level limit"; continue; }
                const int cn = last.A.n;
                if (cn > kCoarseCap) { ih.err = "AMG coarsening stalled above the dense-solve limit"; continue; }
                std::vector<double> inv;
                if (!hf::dense_inverse(last.A, inv)) { ih.err = "singular coarsest AMG level"; continue; }
                ih.inv = std::move(inv);
            }
        };
        const unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
        std::vector<std::thread> th;
        for (unsigned t = 0; t + 1 < nt && (int)t < ni; t++) th.emplace_back(work);
        work();
        for (auto &t : th) t.join();
        for (int i = 0; i < ni; i++) {
            if (!IH[i].err.empty()) return fail(HF_ERR_UNSUPPORTED, IH[i].err + " (instance " + std::to_string(i) + ")");
            clev[i] = (int)IH[i].H.size() - 1;
        }
    }
    int nlev = 1;
    for (int i = 0; i < ni; i++) nlev = std::max(nlev, clev[i] + 1);
    C->nlev = nlev;
    // row offsets of every instance on every level
    std::vector<std::vector<int>> off(nlev, std::vector<int>(ni + 1, 0));
    for (int l = 0; l < nlev; l++)
        for (int i = 0; i < ni; i++) {
            const int rows = l == 0 ? C->coff[i + 1] - C->coff[i] : (clev[i] >= l ? IH[i].H[l].A.n : 0);
            off[l][i + 1] = off[l][i] + rows;
        }
    // tail level of every instance: its first level with at most kTailRows rows
    // (the coarsest level always qualifies); the levels above it are run by the
    // level-synchronous kernels
    std::vector<int> tail(ni, 0);
    C->nreg = 0;
    for (int i = 0; i < ni && amg; i++) {
        int s = 0;
        while (s < clev[i] && off[s][i + 1] - off[s][i] > kTailRows) s++;
        tail[i] = s;
        C->nreg = std::max(C->nreg, s);
    }
    std::vector<LevelHost> LH(nlev);
    C->lrows.assign(nlev, 0);
    C->lnnz_a.assign(nlev, 0);
    C->lnnz_p.assign(nlev, 0);
    C->lnnz_r.assign(nlev, 0);
    for (int l = 0; l < nlev; l++) {
        LevelHost &h = LH[l];
        h.n = off[l][ni];
        C->lrows[l] = h.n;
        if (l == 0) {
            C->lnnz_a[0] = (int64_t)mcol.size();
            if (amg) {
                // the smoothing sweeps' omega D^-1, with each instance's own weight
                h.dinv.resize(h.n);
                for (int i = 0; i < ni; i++) {
                    const hf::HostLevel &hl = IH[i].H[0];
                    for (size_t r = 0; r < hl.dinv.size(); r++) h.dinv[off[0][i] + r] = hl.omega * hl.dinv[r];
                }
            }
        } else {
            h.Ap.assign(1, 0);
            for (int i = 0; i < ni; i++) {
                if (clev[i] < l) continue;
                const hf::HostLevel &hl = IH[i].H[l];
                for (int r = 0; r < hl.A.n; r++) {
                    for (int k = hl.A.ptr[r]; k < hl.A.ptr[r + 1]; k++) {
                        h.Ac.push_back(hl.A.col[k] + off[l][i]);
                        h.Av.push_back(hl.A.val[k]);
                    }
                    h.Ap.push_back((int32_t)h.Ac.size());
                }
                for (double d : hl.dinv) h.dinv.push_back(hl.omega * d);
            }
            C->lnnz_a[l] = (int64_t)h.Ac.size();
        }
        if (l + 1 < nlev) {
            // P: rows of this level -> next level; R: rows of the next level -> this level
            h.Pp.assign(1, 0);
            h.Rp.assign(1, 0);
            for (int i = 0; i < ni; i++) {
                if (clev[i] < l) continue;
                const int rows = off[l][i + 1] - off[l][i];
                if (clev[i] == l) {   // coarsest here: no transfer rows
                    for (int r = 0; r < rows; r++) h.Pp.push_back((int32_t)h.Pc.size());
                    continue;
                }
                const hf::HostLevel &hl = IH[i].H[l];
                for (int r = 0; r < hl.P.n; r++) {
                    for (int k = hl.P.ptr[r]; k < hl.P.ptr[r + 1]; k++) {
                        h.Pc.push_back(hl.P.col[k] + off[l + 1][i]);
                        h.Pv.push_back(hl.P.val[k]);
                    }
                    h.Pp.push_back((int32_t)h.Pc.size());
                }
                for (int r = 0; r < hl.R.n; r++) {
                    for (int k = hl.R.ptr[r]; k < hl.R.ptr[r + 1]; k++) {
                        h.Rc.push_back(hl.R.col[k] + off[l][i]);
                        h.Rv.push_back(hl.R.val[k]);
                    }
                    h.Rp.push_back((int32_t)h.Rc.size());
                }
            }
            C->lnnz_p[l] = (int64_t)h.Pc.size();
            C->lnnz_r[l] = (int64_t)h.Rc.size();
        }
        h.sblk = block_table(off, tail, l, true);
        h.ablk = block_table(off, tail, l, false);
    }
    // the finest level's blocks carry their halo, for the kernels that stage a
    // vector over the block's rows and halo in shared memory: every column the
    // block's rows reach lies in [row0 + pad0, row0 + cnt + pad1), pad0 <= 0 <=
    // pad1, and that range lies inside the level (columns are valid indices)
    {
        const int n0 = LH[0].n;
        std::vector<int32_t> cmin(n0), cmax(n0);
        for (int i = 0; i < n0; i++) {
            cmin[i] = cmax[i] = i;
            for (int k = mptr[i]; k < mptr[i + 1]; k++) {
                cmin[i] = std::min(cmin[i], mcol[k]);
                cmax[i] = std::max(cmax[i], mcol[k]);
            }
        }
        for (std::vector<Blk> *t : {&LH[0].sblk, &LH[0].ablk})
            for (Blk &b : *t) {
                int lo = b.row0, hi = b.row0 + b.cnt - 1;
                for (int i = b.row0; i < b.row0 + b.cnt; i++) {
                    lo = std::min(lo, cmin[i]);
                    hi = std::max(hi, cmax[i]);
                }
                b.pad0 = lo - b.row0;
                b.pad1 = hi - (b.row0 + b.cnt - 1);
            }
    }

    // every index the kernels follow must stay inside its array
    for (int l = 0; l < nlev; l++) {
        const LevelHost &h = LH[l];
        const int nn = l + 1 < nlev ? LH[l + 1].n : 0;
        auto cols_ok = [](const std::vector<int32_t> &p, const std::vector<int32_t> &c, size_t rows, int ncol) {
            if (p.size() != rows + 1 || p.back() != (int32_t)c.size()) return false;
            for (int32_t v : c)
                if (v < 0 || v >= ncol) return false;
            return true;
        };
        bool ok = l == 0 || cols_ok(h.Ap, h.Ac, h.n, h.n);
        if (ok && l + 1 < nlev) ok = cols_ok(h.Pp, h.Pc, h.n, nn) && cols_ok(h.Rp, h.Rc, nn, h.n);
        for (const std::vector<Blk> *t : {&h.sblk, &h.ablk})
            for (const Blk &b : *t) {
                if (b.row0 < 0 || b.cnt <= 0 || b.cnt > kBlockRows || b.row0 + b.cnt > h.n) ok = false;
                if (l == 0 && (b.pad0 > 0 || b.pad1 < 0 || b.row0 + b.pad0 < 0 || b.row0 + b.cnt + b.pad1 > h.n)) ok = false;
            }
        if (!ok) return fail(HF_ERR_INVALID, "inconsistent multigrid level " + std::to_string(l));
    }
    for (int i = 0; i < ni && amg; i++) {
        if (off[clev[i]][i + 1] > LH[clev[i]].n || off[clev[i]][i + 1] - off[clev[i]][i] > kCoarseCap)
            return fail(HF_ERR_INVALID, "inconsistent coarsest level");
        if (tail[i] > clev[i] || clev[i] >= kMaxLevels) return fail(HF_ERR_INVALID, "inconsistent tail level");
    }

    // the finest operator as row templates: rows with the same column offsets
    // and values (in entry order) share one template
    const int nf = C->P.ncell;
    std::vector<uint32_t> rd(nf);
    std::vector<int32_t> tp(1, 0), toff;
    std::vector<double> tval;
    {
        std::unordered_map<std::string, uint32_t> seen;
        std::string key;
        for (int i = 0; i < nf; i++) {
            key.clear();
            const int len = mptr[i + 1] - mptr[i];
            if (len >= (1 << kTLenBits)) return fail(HF_ERR_UNSUPPORTED, "Poisson row with more than 127 entries");
            for (int k = mptr[i]; k < mptr[i + 1]; k++) {
                const int32_t o = mcol[k] - i;
                key.append((const char *)&o, sizeof o);
                key.append((const char *)&mval[k], sizeof(double));
            }
            auto it = seen.find(key);
            if (it != seen.end()) {
                rd[i] = it->second;
                continue;
            }
            if (toff.size() + len >= ((size_t)1 << (32 - kTLenBits)))
                return fail(HF_ERR_UNSUPPORTED, "too many distinct Poisson rows for the template table");
            const uint32_t d = ((uint32_t)toff.size() << kTLenBits) | (uint32_t)len;
            seen.emplace(key, d);
            for (int k = mptr[i]; k < mptr[i + 1]; k++) {
                toff.push_back(mcol[k] - i);
                tval.push_back(mval[k]);
            }
            tp.push_back((int32_t)toff.size());
            rd[i] = d;
        }
    }
    // template forms of the operators and transfers the level-synchronous
    // kernels read (levels above the last tail start); the tails keep CSR
    if (amg) {
        std::vector<std::thread> th;
        for (int l = 0; l < C->nreg && l + 1 < nlev; l++) {
            LevelHost &h = LH[l];
            if (l > 0) th.emplace_back([&h]() { h.At = make_templates(h.Ap, h.Ac, h.Av, true); });
            th.emplace_back([&h]() { h.Pt = make_templates(h.Pp, h.Pc, h.Pv, false); });
            th.emplace_back([&h]() { h.Rt = make_templates(h.Rp, h.Rc, h.Rv, false); });
        }
        for (auto &t : th) t.join();
    }

    // device arena: hierarchy (in the V-cycle's precision), dense inverses,
    // CG vectors, partial sums, instance scalars and loop control
    Arena ar;
    ar.add(nullptr, 8);   // offset 0 stays unused: a zero offset means "absent"
    std::vector<LevelOff> LO(nlev);
    if (amg)
        for (int l = 0; l < nlev; l++)
            LO[l] = mixed ? place_level<float>(ar, LH[l], l == 0) : place_level<double>(ar, LH[l], l == 0);
    std::vector<size_t> inv_off(ni, 0);
    if (amg)
        for (int i = 0; i < ni; i++)
            inv_off[i] = mixed ? ar.vec(cast_vec<float>(IH[i].inv)) : ar.vec(IH[i].inv);
    const int n = C->P.ncell;
    const size_t o_r = ar.zeros<double>(n), o_z = ar.zeros<double>(n), o_q = ar.zeros<double>(n);
    const size_t o_pa = ar.zeros<double>(n), o_pb = ar.zeros<double>(n), o_xprev = ar.zeros<double>(n),
                 o_xprev2 = ar.zeros<double>(n);
    const size_t o_part = ar.zeros<double>((size_t)LH[0].ablk.size() * 2);
    // mixed form: the inner solve's FP32 vectors
    size_t o_r32 = 0, o_z32 = 0, o_q32 = 0, o_e32 = 0, o_pa32 = 0, o_pb32 = 0;
    if (mixed) {
        o_r32 = ar.zeros<float>(n);
        o_z32 = ar.zeros<float>(n);
        o_q32 = ar.zeros<float>(n);
        o_e32 = ar.zeros<float>(n);
        o_pa32 = ar.zeros<float>(n);
        o_pb32 = ar.zeros<float>(n);
    }
    std::vector<IScal> S(ni);
    for (int i = 0; i < ni; i++) {
        memset(&S[i], 0, sizeof(IScal));
        S[i].tail0 = amg && tail[i] == 0;
        S[i].done = 1;
    }
    const size_t o_S = ar.vec(S);
    Ctl ctl{};
    ctl.maxbodies = C->opt.poisson_maxit / 2 + 2;
    const size_t o_ctl = ar.add(&ctl, sizeof ctl);
    std::vector<int32_t> ipin(pins.begin(), pins.end());
    const size_t o_pin = ar.vec(ipin);
    const size_t o_fblk = ar.vec(LH[0].ablk);
    const size_t o_rd = ar.vec(rd), o_toff = ar.vec(toff), o_tval = ar.vec(tval);
    const size_t o_tval32 = mixed ? ar.vec(cast_vec<float>(tval)) : 0;
    C->ntemplates = (int64_t)tp.size() - 1;

    char *base = nullptr;
    HF_CK(cudaMallocAsync((void **)&base, ar.host.size(), C->stream));
    C->owned.push_back(base);
    C->bytes += (double)ar.host.size();
    HF_CK(cudaMemcpyAsync(base, ar.host.data(), ar.host.size(), cudaMemcpyHostToDevice, C->stream));
    HF_CK(cudaStreamSynchronize(C->stream));   // the host arena goes away with this function

    PcgFine &G = C->G;
    G.n = n;
    G.A.rd = (const uint32_t *)(base + o_rd);
    G.A.toff = (const int32_t *)(base + o_toff);
    G.A.tval = (const double *)(base + o_tval);
    G.dinv = C->M.dinv;
    G.apin = C->M.apin;
    G.brhs = C->M.brhs;
    G.ipin = (const int32_t *)(base + o_pin);
    G.ipar = C->P.ipar;
    G.p = C->F.p;
    G.dp = C->F.dp;
    G.xprev = (double *)(base + o_xprev);
    G.xprev2 = (double *)(base + o_xprev2);
    G.cinst = C->P.cinst;
    G.r = (double *)(base + o_r);
    G.z = (double *)(base + o_z);
    G.q = (double *)(base + o_q);
    G.partials = (double *)(base + o_part);
    G.S = (IScal *)(base + o_S);
    G.ctl = (Ctl *)(base + o_ctl);
    G.blk = (const Blk *)(base + o_fblk);
    G.nblk = (int)LH[0].ablk.size();
    G.ninst = ni;
    G.projtype_all = C->P.projtype_all;
    G.rtol = C->opt.poisson_rtol;
    G.atol = C->opt.poisson_atol;
    G.maxit = C->opt.poisson_maxit;
    C->pa = (double *)(base + o_pa);
    C->pb = (double *)(base + o_pb);
    if (mixed) {
        G.A32 = TRows<float>{G.A.rd, G.A.toff, (const float *)(base + o_tval32)};
        G.r32 = (float *)(base + o_r32);
        G.z32 = (float *)(base + o_z32);
        G.q32 = (float *)(base + o_q32);
        G.e32 = (float *)(base + o_e32);
        G.eta = kInnerEta;
        G.inner_maxit = kInnerMaxit;
        C->pa32 = (float *)(base + o_pa32);
        C->pb32 = (float *)(base + o_pb32);
    }
    if (amg) {
        for (int l = 0; l < nlev; l++) {
            if (mixed) {
                const TRows<float> At32{G.A.rd, G.A.toff, (const float *)(base + o_tval32)};
                C->L32[l] = make_level<float>(base, LO[l], LH[l], At32, l == 0);
            } else {
                C->L64[l] = make_level<double>(base, LO[l], LH[l], G.A, l == 0);
            }
        }
        // the per-instance tails: level table and row ranges
        std::vector<TailInst<double>> t64(ni);
        std::vector<TailInst<float>> t32(ni);
        C->coarse_rows = 0;
        C->coarse_dense = 0;
        for (int i = 0; i < ni; i++) {
            TailInst<double> &a = t64[i];
            TailInst<float> &b = t32[i];
            memset(&a, 0, sizeof a);
            memset(&b, 0, sizeof b);
            a.inst = b.inst = i;
            a.s = b.s = tail[i];
            a.clev = b.clev = clev[i];
            for (int l = 0; l <= clev[i]; l++) {
                a.row0[l] = b.row0[l] = off[l][i];
                a.nrow[l] = b.nrow[l] = off[l][i + 1] - off[l][i];
            }
            a.inv = mixed ? nullptr : (const double *)(base + inv_off[i]);
            b.inv = mixed ? (const float *)(base + inv_off[i]) : nullptr;
            const int64_t cn = a.nrow[clev[i]];
            C->coarse_rows += cn;
            C->coarse_dense += cn * cn;
        }
        double bytes = 0;
        int rc;
        if (mixed) {
            if ((rc = upload(C->owned, &C->t32, t32.data(), t32.size(), bytes, C->stream)) ||
                (rc = upload(C->owned, &C->h32, C->L32, (size_t)nlev, bytes, C->stream)))
                return rc;
        } else if ((rc = upload(C->owned, &C->t64, t64.data(), t64.size(), bytes, C->stream)) ||
                   (rc = upload(C->owned, &C->h64, C->L64, (size_t)nlev, bytes, C->stream))) {
            return rc;
        }
        C->bytes += bytes;
    }
    C->h_S = new IScal[ni]();
    C->h_ctl = new Ctl();
    return HF_OK;
}

// ---------------------------------------------------------------------------
// one time step as a CUDA graph
// ---------------------------------------------------------------------------
// A kernel of the CG loop body, launched with programmatic stream
// serialization (the kernel starts with pdl_wait, hf_pcg.cuh)
template <typename... KArgs, typename... Args>
void launch_pdl(void (*kern)(KArgs...), int grid, int block, cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

template <typename T, typename R>
void enqueue_vcycle(hf_case *C, cudaStream_t st, const VLev<T> *L, const VLev<T> *H, const TailInst<T> *ti,
                    const R *r0, int &kernels)
{
    const IScal *S = C->G.S;
    // the large levels, every instance at once, down to each instance's tail
    for (int l = 0; l < C->nreg; l++) {
        if (L[l].nsblk) {
            if (l == 0) launch_pdl(k_vc_down<T, true, R>, L[l].nsblk, kBlock, st, L[l], r0, S);
            else launch_pdl(k_vc_down<T, false, R>, L[l].nsblk, kBlock, st, L[l], r0, S);
            kernels++;
        }
        if (L[l + 1].nablk) {
            launch_pdl(k_vc_restrict<T>, L[l + 1].nablk, kBlock, st, L[l], L[l + 1], S);
            kernels++;
        }
    }
    // the small levels: one CTA per instance
    launch_pdl(k_vc_tail<T, R>, C->ninst, kTailThreads, st, H, ti, r0, S);
    kernels++;
    for (int l = C->nreg - 1; l >= 0; l--) {
        if (!L[l].nsblk) continue;
        launch_pdl(k_vc_prolong<T>, L[l].nsblk, kBlock, st, L[l], (const T *)L[l + 1].out, S);
        kernels++;
        if (l > 0) {
            launch_pdl(k_vc_post<T>, L[l].nsblk, kBlock, st, L[l], S);
            kernels++;
        }
    }
    kernels++;
}

// two CG iterations (the direction vectors alternate, so two keep the graph
// static); cond == 0: eager launches, the body is only counted on the device
void enqueue_body(hf_case *C, cudaStream_t st, cudaGraphConditionalHandle cond, int &kernels)
{
    for (int it = 0; it < 2; it++) {
        const int set = it == 1 ? (cond ? 1 : 2) : 0;
        if (C->mixed) {
            // the inner FP32 iteration of the mixed form
            enqueue_vcycle<float, float>(C, st, C->L32, C->h32, C->t32, C->G.r32, kernels);
            launch_pdl(k_pcg_z32, C->G.nblk, kBlock, st, C->G, C->L32[0]);
            float *po = it == 0 ? C->pa32 : C->pb32, *pn = it == 0 ? C->pb32 : C->pa32;
            launch_pdl(k_pcg_dir32, C->G.nblk, kBlock, st, C->G, (const float *)po, pn);
            launch_pdl(k_pcg_update32, C->G.nblk, kBlock, st, C->G, (const float *)pn, cond, set);
            kernels += 3;
            continue;
        }
        if (!C->amg) {
            launch_pdl(k_pcg_z<double, true>, C->G.nblk, kBlock, st, C->G, VLev<double>{});
        } else {
            enqueue_vcycle<double, double>(C, st, C->L64, C->h64, C->t64, C->G.r, kernels);
            launch_pdl(k_pcg_z<double, false>, C->G.nblk, kBlock, st, C->G, C->L64[0]);
        }
        kernels++;
        double *po = it == 0 ? C->pa : C->pb, *pn = it == 0 ? C->pb : C->pa;
        launch_pdl(k_pcg_dir, C->G.nblk, kBlock, st, C->G, (const double *)po, pn);
        launch_pdl(k_pcg_update, C->G.nblk, kBlock, st, C->G, (const double *)pn, cond, set);
        kernels += 2;
    }
}

// One semi-implicit velocity system: BiCGStab with Jacobi scaling on Mu from
// x0 into x, right-hand side b
int sie_solve_dir(hf_case *C, const DevMat &Mu, double *x, const double *x0, double *b, int d, int64_t &launches)
{
    cudaStream_t st = C->stream;
    const double rtol = C->opt.poisson_rtol, atol = C->opt.poisson_atol;
    const int n = Mu.n;
    BiVec V = C->Vu;
    V.x = x;
    V.b = b;
    HF_CK(cudaMemcpyAsync(V.x, x0, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, st));
    Scal h{};
    h.maxit = C->opt.poisson_maxit;
    *C->h_scal = h;
    HF_CK(cudaMemcpyAsync(V.sc, C->h_scal, sizeof(Scal), cudaMemcpyHostToDevice, st));
    int restarts = 0, first = 1;
    for (;;) {
        k_slv_init<<<blocks(n), kBlock, 0, st>>>(Mu, V, rtol, atol, first);
        launches++;
        first = 0;
        int chunk = 4;
        for (;;) {
            for (int k = 0; k < chunk; k++) {
                k_bi_p<<<blocks(n), kBlock, 0, st>>>(Mu, V);
                k_bi_spmv<<<blocks(n), kBlock, 0, st>>>(Mu, V, V.ph, V.v, 0);
                k_bi_s<<<blocks(n), kBlock, 0, st>>>(Mu, V);
                k_bi_spmv<<<blocks(n), kBlock, 0, st>>>(Mu, V, V.sh, V.t, 1);
                k_bi_update<<<blocks(n), kBlock, 0, st>>>(Mu, V);
                launches += 5;
            }
            HF_CK(cudaMemcpyAsync(C->h_scal, V.sc, sizeof(Scal), cudaMemcpyDeviceToHost, st));
            HF_CK(cudaStreamSynchronize(st));
            if (C->h_scal->done) break;
            chunk = std::min(chunk * 2, 32);
        }
        if (C->h_scal->status == 1 && restarts++ < 50) continue;   // breakdown: restart from x
        break;
    }
    HF_CK(cudaGetLastError());
    const int status = C->h_scal->status;
    if (status)
        return fail(status == 1 ? HF_ERR_NOT_CONVERGED : status,
                    "semi-implicit velocity BiCGStab failed in direction " + std::to_string(d));
    C->vel_iters += C->h_scal->iters;
    return HF_OK;
}

// The semi-implicit velocity systems of one step (after the velocity kernel
// wrote their right-hand sides): per direction BiCGStab with Jacobi scaling,
// from u as the initial guess, into u*, to the Poisson solve's tolerances (the
// reference hands both systems to the same solver engine).  BDF2 solves twice:
// into uaux, then (right-hand sides from k_bdf2_rhs) into u*.  Host-driven:
// the host reads the scalars between chunks of iterations.
int sie_solves(hf_case *C, int64_t &launches)
{
    const int D = C->D;
    for (int d = 0; d < D; d++) {
        double *x = C->bdf2 ? C->ua[d] : C->F.us[d];
        int rc = sie_solve_dir(C, C->Mu[d], x, C->F.u[d], C->P.sie_b[d], d, launches);
        if (rc) return rc;
    }
    if (!C->bdf2) return HF_OK;
    for (int d = 0; d < D; d++) {
        const int n = C->Mu2[d].n;
        k_bdf2_rhs<<<blocks(n), kBlock, 0, C->stream>>>(n, C->par.dt, C->P.sie_e[d], C->ua[d], C->F.u[d],
                                                         C->P.sie_bc2[d], C->P.sie_b[d]);
        launches++;
        int rc = sie_solve_dir(C, C->Mu2[d], C->F.us[d], C->ua[d], C->P.sie_b[d], d, launches);
        if (rc) return rc;
    }
    return HF_OK;
}

// a phase timing event; while a step graph is captured it becomes an
// event-record node of the graph
void record(hf_case *C, int phase, int end)
{
    if (!C->profile) return;
    if (C->capturing) cudaEventRecordWithFlags(C->ev[2 * phase + end], C->stream, cudaEventRecordExternal);
    else cudaEventRecord(C->ev[2 * phase + end], C->stream);
}

// k_vrows over one pair set at the case's block size for it
void enqueue_pairs(hf_case *C, const PairRows &R, const DevFields &F, cudaStream_t st)
{
    const int bs = C->blk_vrows, nb = (R.n + bs - 1) / bs;
    if (R.scol16) k_vrows<true><<<nb, bs, 0, st>>>(R, F);
    else k_vrows<false><<<nb, bs, 0, st>>>(R, F);
}

// the velocity stage's general rows: by pattern (mixed form) or sliced
void enqueue_vrows(hf_case *C, const DevFields &F, cudaStream_t st)
{
    if (C->vp.n) {
        const int bs = C->blk_vrows, nb = (C->vp.n + bs - 1) / bs;
        k_vrows_pat<<<nb, bs, 0, st>>>(C->vp, F);
    } else {
        enqueue_pairs(C, C->P.vr, F, st);
    }
}

// The viscoelastic cell stage's main kernel at the case's block size
template <int D>
void enqueue_ve_cell(hf_case *C, const DevFields &F, cudaStream_t st)
{
    const int vb = C->blk_ve, nb = (C->P.ncell + vb - 1) / vb;
    const bool mix = C->vmix;
    if (C->par.ve_discrtype == HF_VE_IMPLICIT) {
        if (mix) k_ve_cell<D, true, true><<<nb, vb, 0, st>>>(C->P, F);
        else k_ve_cell<D, true, false><<<nb, vb, 0, st>>>(C->P, F);
    } else {
        if (mix) k_ve_cell<D, false, true><<<nb, vb, 0, st>>>(C->P, F);
        else k_ve_cell<D, false, false><<<nb, vb, 0, st>>>(C->P, F);
    }
}

template <int D>
int enqueue_velocity(hf_case *C, const DevFields &F, cudaStream_t st);

// The launch-shape tuner (hf_options.tuning == 0): before the first step, each
// tuned kernel runs a few times at each candidate block size on this case's
// own data, timed with CUDA events on the case stream, and the fastest size is
// kept.  The kernels tried write only what the step itself rewrites before
// reading it (row values, u*, the new kernel tensor and Du), and every size
// gives the same bits (each thread's work and order do not depend on the
// block size), so tuning changes no result.
template <int D>
int autotune(hf_case *C)
{
    C->tuned = true;
    if (C->opt.tuning != 0) return HF_OK;
    cudaStream_t st = C->stream;
    cudaEvent_t a, b;
    HF_CK(cudaEventCreate(&a));
    HF_CK(cudaEventCreate(&b));
    auto time_it = [&](auto launch) -> float {
        launch();   // warm
        cudaEventRecord(a, st);
        for (int r = 0; r < 3; r++) launch();
        cudaEventRecord(b, st);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    };
    auto pick = [&](int &slot, std::initializer_list<int> sizes, auto launch) {
        float best = 1e30f;
        int keep = slot;
        for (int bs : sizes) {
            slot = bs;
            const float ms = time_it(launch);
            if (cudaGetLastError() != cudaSuccess) continue;
            if (ms < best) {
                best = ms;
                keep = bs;
            }
        }
        slot = keep;
    };
    const DevFields F = C->F;
    // k_vrows alone on the velocity-stage pairs (the facet kernel reads its
    // output); the cell-stage pairs are evaluated once for k_ve_cell's trials
    if (C->P.vr.n) pick(C->blk_vrows, {128, 256, 512}, [&]() { enqueue_vrows(C, F, st); });
    if (!C->sie) pick(C->blk_vel, {64, 128, 256}, [&]() { enqueue_velocity<D>(C, F, st); });
    if (C->par.flowtype == HF_VISCOELASTIC) {
        if (C->P.cr.n) enqueue_pairs(C, C->P.cr, F, st);
        pick(C->blk_ve, {64, 128}, [&]() { enqueue_ve_cell<D>(C, F, st); });
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    HF_CK(cudaStreamSynchronize(st));
    HF_CK(cudaGetLastError());
    return HF_OK;
}

// The velocity stage of one step: explicit Euler (k_vrows + k_velocity), and
// for the explicit Runge-Kutta forms its combination with u.  The reference's
// Runge-Kutta stages call higflow_explicit_euler_intermediate_velocity(ns, in,
// out), whose computational cell reads ns->dpu whatever `in` is
// (hig-flow-step.c:639; viscoelastic hig-flow-step-viscoelastic.c:957), so
// every stage evaluates the same E(u) and the schemes reduce to RK2: u* =
// 0.5 (u + E(u)); RK3: u* = u/3 + 2 E(u)/3 (the auxiliary velocity feeds no
// later stage).  E(u) is evaluated once here: a repeat would give the same bits.
// Returns the kernels launched.
template <int D>
int enqueue_velocity(hf_case *C, const DevFields &F, cudaStream_t st)
{
    const bool ve = C->par.flowtype == HF_VISCOELASTIC;
    int n = 0;
    if (C->P.vr.n) {
        record(C, HF_PHASE_VELOCITY_ROWS, 0);
        enqueue_vrows(C, F, st);
        record(C, HF_PHASE_VELOCITY_ROWS, 1);
        n++;
    }
    const int vb = C->blk_vel, nb = (C->nfacet_total + vb - 1) / vb;
    const bool mix = C->vmix;
    if (ve) {
        if (mix) k_velocity<D, true, true><<<nb, vb, 0, st>>>(C->P, F);
        else k_velocity<D, true, false><<<nb, vb, 0, st>>>(C->P, F);
    } else {
        if (mix) k_velocity<D, false, true><<<nb, vb, 0, st>>>(C->P, F);
        else k_velocity<D, false, false><<<nb, vb, 0, st>>>(C->P, F);
    }
    n++;
    const int scheme = C->par.tempdiscrtype;
    if (scheme == HF_EXPLICIT_RK2 || scheme == HF_EXPLICIT_RK3) {
        k_rk_combine<D><<<blocks(C->nfacet_total), kBlock, 0, st>>>(C->P, F, scheme == HF_EXPLICIT_RK2 ? 0 : 2);
        n++;
    }
    return n;
}

// The kernels of a step before the Poisson iterations: viscoelastic cell stage
// (F's K/Knew swap after it), intermediate velocity, Poisson right-hand side.
template <int D>
void enqueue_pre(hf_case *C, DevFields &F, int &fixed)
{
    cudaStream_t st = C->stream;
    const bool ve = C->par.flowtype == HF_VISCOELASTIC;
    if (ve) {
        record(C, HF_PHASE_VE_CELL, 0);
        if (C->gptt) {
            k_gptt_ml<D><<<blocks(C->P.ncell), kBlock, 0, st>>>(C->P, F);
            fixed++;
        }
        if (C->P.cr.n) {
            enqueue_pairs(C, C->P.cr, F, st);
            fixed++;
        }
        record(C, HF_PHASE_VE_CELL_MAIN, 0);
        enqueue_ve_cell<D>(C, F, st);
        record(C, HF_PHASE_VE_CELL_MAIN, 1);
        k_ve_stress<D><<<blocks(C->P.ncell), kBlock, 0, st>>>(C->P, F);
        record(C, HF_PHASE_VE_CELL, 1);
        for (int k = 0; k < D * D; k++) std::swap(F.K[k], F.Knew[k]);
        fixed += 2;
    }
    record(C, HF_PHASE_VELOCITY, 0);
    fixed += enqueue_velocity<D>(C, F, st);
    if (C->sie) C->sie_rc = sie_solves(C, C->sie_launches);   // eager steps only (no graph for this form)
    record(C, HF_PHASE_VELOCITY, 1);
    record(C, HF_PHASE_POISSON_INIT, 0);
    k_pcg_extrapolate<<<blocks(C->P.ncell), kBlock, 0, st>>>(C->G);
    k_pcg_init<D><<<C->G.nblk, kBlock, 0, st>>>(C->P, F, C->G);
    record(C, HF_PHASE_POISSON_INIT, 1);
    record(C, HF_PHASE_POISSON_ITER, 0);
    fixed += 3;
}

// ... and after them: per-instance totals, final velocity and pressure
template <int D>
void enqueue_post(hf_case *C, const DevFields &F, int &fixed)
{
    cudaStream_t st = C->stream;
    record(C, HF_PHASE_POISSON_ITER, 1);
    record(C, HF_PHASE_FINAL, 0);
    // (k_final first: k_step_end counts the instances' step limits down)
    k_final<D><<<blocks(C->nfacet_total + C->P.ncell), kBlock, 0, st>>>(C->P, F);
    k_step_end<<<1, kBlock, 0, st>>>(C->G);
    record(C, HF_PHASE_FINAL, 1);
    fixed += 2;
}

// One step with eager launches: the host reads the loop control after each body.
template <int D>
int eager_step(hf_case *C)
{
    DevFields F = C->F;
    int fixed = 0, body = 0;
    enqueue_pre<D>(C, F, fixed);
    if (C->sie_rc) return C->sie_rc;
    // the mixed form: up to kMaxSweeps inner solves, each followed by the FP64
    // correction; the plain form: one solve
    const int sweeps = C->mixed ? kMaxSweeps : 1;
    for (int sw = 0; sw < sweeps; sw++) {
        for (;;) {
            body = 0;
            enqueue_body(C, C->stream, 0, body);
            HF_CK(cudaGetLastError());
            HF_CK(cudaMemcpyAsync(C->h_ctl, C->G.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, C->stream));
            HF_CK(cudaStreamSynchronize(C->stream));
            if (!(C->h_ctl->active > 0 && C->h_ctl->bodies < C->h_ctl->maxbodies)) break;
        }
        if (!C->mixed) break;
        k_ir_correct<<<C->G.nblk, kBlock, 0, C->stream>>>(C->G, 0, 0, sw == sweeps - 1);
        fixed++;
        HF_CK(cudaGetLastError());
        HF_CK(cudaMemcpyAsync(C->h_ctl, C->G.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, C->stream));
        HF_CK(cudaStreamSynchronize(C->stream));
        if (C->h_ctl->active == 0) break;
    }
    enqueue_post<D>(C, F, fixed);
    HF_CK(cudaGetLastError());
    C->fixed_kernels = fixed;
    C->body_kernels = body;
    return HF_OK;
}

// Capture one step with the fields F (K/Knew as they are before the step).
template <int D>
int capture_step(hf_case *C, DevFields F, cudaGraph_t *gout)
{
    cudaStream_t st = C->stream;
    int fixed = 0, body = 0;
    HF_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    C->capturing = true;
    enqueue_pre<D>(C, F, fixed);

    // the iterations: a conditional WHILE node after everything captured so far;
    // the mixed form has kMaxSweeps of them, each followed by its FP64
    // correction, which sets the next one's condition
    const int sweeps = C->mixed ? kMaxSweeps : 1;
    cudaError_t e = cudaSuccess;
    cudaGraphConditionalHandle cond[kMaxSweeps] = {};
    bool have[kMaxSweeps] = {};
    cudaGraph_t g = nullptr;
    for (int sw = 0; sw < sweeps && e == cudaSuccess; sw++) {
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps);
        if (e == cudaSuccess && !have[sw]) e = cudaGraphConditionalHandleCreate(&cond[sw], g, 1, cudaGraphCondAssignDefault);
        have[sw] = true;
        cudaGraphNodeParams cp{};
        cudaGraphNode_t node = nullptr;
        if (e == cudaSuccess) {
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = cond[sw];
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            e = cudaGraphAddNode(&node, g, deps, ndeps, &cp);
        }
        if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
        if (e == cudaSuccess) {
            cudaGraph_t bg = cp.conditional.phGraph_out[0];
            e = cudaStreamBeginCaptureToGraph(C->body_stream, bg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                body = 0;
                enqueue_body(C, C->body_stream, cond[sw], body);
                e = cudaStreamEndCapture(C->body_stream, &bg);
            }
        }
        if (e == cudaSuccess && C->mixed) {
            // the correction sets the condition of the next sweep (created with
            // the next node; a handle is a value, so it is created first here)
            cudaGraphConditionalHandle next = 0;
            const bool last = sw == sweeps - 1;
            if (!last) e = cudaGraphConditionalHandleCreate(&next, g, 1, cudaGraphCondAssignDefault);
            if (e == cudaSuccess) {
                k_ir_correct<<<C->G.nblk, kBlock, 0, st>>>(C->G, next, last ? 0 : 1, last ? 1 : 0);
                fixed++;
                if (!last) {
                    cond[sw + 1] = next;
                    have[sw + 1] = true;
                }
            }
        }
    }
    enqueue_post<D>(C, F, fixed);
    cudaGraph_t done = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(st, &done);
    C->capturing = false;
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (done) cudaGraphDestroy(done);
        cudaGetLastError();
        return fail(HF_ERR_CUDA, std::string("step graph capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    HF_CK(cudaGetLastError());
    *gout = done;
    C->fixed_kernels = fixed;
    C->body_kernels = body;
    return HF_OK;
}

void destroy_graphs(hf_case *C)
{
    for (int q = 0; q < 2; q++) {
        if (C->exec[q]) cudaGraphExecDestroy(C->exec[q]);
        if (C->graph[q]) cudaGraphDestroy(C->graph[q]);
        C->exec[q] = nullptr;
        C->graph[q] = nullptr;
    }
}

// graph q runs a step that starts at parity q (K/Knew swapped for odd parity)
template <int D>
int ensure_graphs(hf_case *C)
{
    if (C->exec[0] && C->graph_profile == C->profile) return HF_OK;
    destroy_graphs(C);
    const bool ve = C->par.flowtype == HF_VISCOELASTIC;
    for (int q = 0; q < (ve ? 2 : 1); q++) {
        DevFields F = C->F;
        if (ve && q != C->parity)
            for (int k = 0; k < D * D; k++) std::swap(F.K[k], F.Knew[k]);
        int rc = capture_step<D>(C, F, &C->graph[q]);
        if (rc) return rc;
        HF_CK(cudaGraphInstantiate(&C->exec[q], C->graph[q], 0));
    }
    C->graph_profile = C->profile;
    return HF_OK;
}

// device -> host copies of the instance scalars and the loop control
int pull_state(hf_case *C)
{
    HF_CK(cudaMemcpyAsync(C->h_S, C->G.S, sizeof(IScal) * C->ninst, cudaMemcpyDeviceToHost, C->stream));
    HF_CK(cudaMemcpyAsync(C->h_ctl, C->G.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, C->stream));
    HF_CK(cudaStreamSynchronize(C->stream));
    return HF_OK;
}

// the first failed solve since the last check, as a status (then cleared)
int take_error(hf_case *C)
{
    const Ctl &c = *C->h_ctl;
    if (!c.err_status) return HF_OK;
    const int code = c.err_status;
    std::string msg = "Poisson solve failed (" + std::to_string(code) + ") in instance " + std::to_string(c.err_inst) +
                      " at step " + std::to_string(c.err_step);
    HF_CK(cudaMemsetAsync(&C->G.ctl->err_status, 0, sizeof(int32_t), C->stream));
    HF_CK(cudaStreamSynchronize(C->stream));
    return fail(code, msg);
}

// Phase times of the last profiled step (its graph recorded the phase events);
// waits for it.
int collect_phases(hf_case *C)
{
    if (!C->phase_pending) return HF_OK;
    C->phase_pending = false;
    int rc = pull_state(C);
    if (rc) return rc;
    const bool ve = C->par.flowtype == HF_VISCOELASTIC;
    for (int p = 0; p < HF_NPHASE; p++) {
        if ((p == HF_PHASE_VE_CELL || p == HF_PHASE_VE_CELL_MAIN) && !ve) continue;
        if (p == HF_PHASE_VELOCITY_ROWS && !C->P.vr.n) continue;
        float ms = 0.f;
        HF_CK(cudaEventElapsedTime(&ms, C->ev[2 * p], C->ev[2 * p + 1]));
        C->phase_ms[p] += ms;
    }
    const bool rk = C->par.tempdiscrtype == HF_EXPLICIT_RK2 || C->par.tempdiscrtype == HF_EXPLICIT_RK3;
    if (ve) C->phase_launches[HF_PHASE_VE_CELL] += 2 + (C->gptt ? 1 : 0) + (C->P.cr.n ? 1 : 0);
    if (ve) C->phase_launches[HF_PHASE_VE_CELL_MAIN] += 1;
    C->phase_launches[HF_PHASE_VELOCITY] += 1 + (C->P.vr.n ? 1 : 0) + (rk ? 1 : 0);
    if (C->P.vr.n) C->phase_launches[HF_PHASE_VELOCITY_ROWS] += 1;
    C->phase_launches[HF_PHASE_POISSON_INIT] += 2;
    C->phase_launches[HF_PHASE_POISSON_ITER] += (C->h_ctl->total_bodies - C->bodies0) * C->body_kernels;
    C->phase_launches[HF_PHASE_FINAL] += 2;
    return HF_OK;
}

template <int D>
int graph_steps(hf_case *C, int nsteps, bool sync)
{
    // the semi-implicit form solves its velocity systems with a host-driven
    // loop, so its steps run eagerly
    const bool eager = C->opt.eager != 0 || C->sie;
    int rc = C->tuned ? HF_OK : autotune<D>(C);
    if (rc) return rc;
    rc = eager ? HF_OK : ensure_graphs<D>(C);
    if (rc) return rc;
    const bool ve = C->par.flowtype == HF_VISCOELASTIC;
    auto one = [&]() -> int {
        if (eager) return eager_step<D>(C);
        HF_CK(cudaGraphLaunch(C->exec[ve ? C->parity : 0], C->stream));
        return HF_OK;
    };
    for (int s = 0; s < nsteps; s++) {
        if (C->profile) {
            // one profiled step in flight at a time: its events are reused
            if ((rc = C->phase_pending ? collect_phases(C) : pull_state(C))) return rc;
            C->bodies0 = C->h_ctl->total_bodies;
            if ((rc = one())) return rc;
            C->phase_pending = true;
        } else if ((rc = one())) {
            return rc;
        }
        if (ve) {
            for (int k = 0; k < D * D; k++) std::swap(C->F.K[k], C->F.Knew[k]);
            C->parity ^= 1;
        }
        C->stats.steps += 1;
    }
    if (!sync) return HF_OK;
    if ((rc = collect_phases(C)) || (rc = pull_state(C))) return rc;
    return take_error(C);
}

// w = M^-1 v with the instance's AMG V-cycle (the BiCGStab path with AMG:
// right preconditioning, k_bi_p / k_bi_s's Jacobi values overwritten);
// returns the kernels launched
int bi_precondition(hf_case *C, const double *v, double *w, cudaStream_t st)
{
    int kernels = 0;
    enqueue_vcycle<double, double>(C, st, C->L64, C->h64, C->t64, v, kernels);
    launch_pdl(k_bi_amg_post, C->G.nblk, kBlock, st, C->G, C->L64[0], v, w);
    return kernels;   // (enqueue_vcycle counts one more than it launches: the post kernel)
}

// BiCGStab (non-symmetric Poisson rows): one instance, host-driven loop
template <int D>
int bicg_step(hf_case *C)
{
    cudaStream_t st = C->stream;
    const bool ve = C->par.flowtype == HF_VISCOELASTIC;
    int64_t launches = 0;
    if (ve) {
        PhaseTimer t(C, HF_PHASE_VE_CELL, launches);
        if (C->gptt) {
            k_gptt_ml<D><<<blocks(C->P.ncell), kBlock, 0, st>>>(C->P, C->F);
            launches++;
        }
        if (C->P.cr.n) {
            enqueue_pairs(C, C->P.cr, C->F, st);
            launches++;
        }
        // (the BiCGStab path is plain FP64: the mixed form needs the CG solver)
        if (C->par.ve_discrtype == HF_VE_IMPLICIT)
            k_ve_cell<D, true, false><<<(C->P.ncell + kVeBlock - 1) / kVeBlock, kVeBlock, 0, st>>>(C->P, C->F);
        else
            k_ve_cell<D, false, false><<<(C->P.ncell + kVeBlock - 1) / kVeBlock, kVeBlock, 0, st>>>(C->P, C->F);
        k_ve_stress<D><<<blocks(C->P.ncell), kBlock, 0, st>>>(C->P, C->F);
        launches += 2;
        for (int k = 0; k < D * D; k++) std::swap(C->F.K[k], C->F.Knew[k]);
        t.stop(launches);
    }
    {
        PhaseTimer t(C, HF_PHASE_VELOCITY, launches);
        launches += enqueue_velocity<D>(C, C->F, st);
        if (C->sie) {
            int rc = sie_solves(C, launches);
            if (rc) return rc;
        }
        t.stop(launches);
    }
    HF_CK(cudaGetLastError());
    const double rtol = C->opt.poisson_rtol, atol = C->opt.poisson_atol;
    const int n = C->P.ncell;
    int rc = HF_OK;
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
                if (C->bi_amg) launches += bi_precondition(C, C->bi.p, C->bi.ph, st);
                k_bi_spmv<<<blocks(n), kBlock, 0, st>>>(C->M, C->bi, C->bi.ph, C->bi.v, 0);
                k_bi_s<<<blocks(n), kBlock, 0, st>>>(C->M, C->bi);
                if (C->bi_amg) launches += bi_precondition(C, C->bi.s, C->bi.sh, st);
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
    if (C->h_scal->status)
        rc = fail(C->h_scal->status == 1 ? HF_ERR_NOT_CONVERGED : C->h_scal->status, "Poisson BiCGStab failed");
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

int run_steps(hf_case *C, int nsteps, bool sync)
{
    if (!C->use_cg) {
        for (int s = 0; s < nsteps; s++) {
            int rc = C->D == 2 ? bicg_step<2>(C) : bicg_step<3>(C);
            if (rc) return rc;
        }
        return HF_OK;
    }
    return C->D == 2 ? graph_steps<2>(C, nsteps, sync) : graph_steps<3>(C, nsteps, sync);
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

// A pair set's sliced layout (PairRows) from its rows, uploaded on the case
// stream into device memory the case owns: fills R except rhs; entries = the
// stored (padded) entry count.  A slice holds 32 consecutive pairs padded to
// its longest; consecutive pairs are consecutive elements of one slot, so
// lengths within a slice rarely differ.
int build_pairs(hf_case *C, std::vector<void *> &own, double &B, const hf_program *pg,
                const std::vector<int32_t> &ptmpl, const std::vector<int32_t> &pbase,
                const std::vector<double> &prhs, const std::vector<uint8_t> &ptag, PairRows &R,
                int64_t &entries, const char *what)
{
    (void)prhs;
    int rc;
    const size_t np = ptmpl.size(), nsl = (np + 31) / 32;
    R.n = (int)np;
    std::vector<int64_t> sptr(nsl + 1, 0);
    std::vector<uint8_t> plen(np);
    for (size_t sl = 0; sl < nsl; sl++) {
        int64_t mx = 0;
        for (size_t u = sl * 32; u < std::min(np, sl * 32 + 32); u++) {
            const int64_t len = pg->tmpl_ptr[ptmpl[u] + 1] - pg->tmpl_ptr[ptmpl[u]];
            if (len > 255) return fail(HF_ERR_UNSUPPORTED, std::string(what) + " stencil longer than 255 entries");
            plen[u] = (uint8_t)len;
            mx = std::max(mx, len);
        }
        sptr[sl + 1] = sptr[sl] + 32 * ((mx + 1) & ~(int64_t)1);   // entries in pairs (see PairRows)
    }
    const size_t ne = (size_t)sptr[nsl];
    // the columns: 16-bit offsets from the pair's first column when every
    // pair's entries stay within +-32767 of it, else 32-bit
    bool c16 = true;
    std::vector<int32_t> pcol0(np, 0);
    for (size_t u = 0; u < np && c16; u++) {
        const int64_t a0 = pg->tmpl_ptr[ptmpl[u]];
        pcol0[u] = plen[u] ? pbase[u] + pg->tmpl_col[a0] : 0;
        for (int k = 0; k < plen[u]; k++) {
            const int64_t d = (int64_t)pbase[u] + pg->tmpl_col[a0 + k] - pcol0[u];
            if (d < -32767 || d > 32767) { c16 = false; break; }
        }
    }
    std::vector<int32_t> scol(c16 ? 0 : ne, 0);
    std::vector<int16_t> scol16(c16 ? ne : 0, 0);
    std::vector<double> sw(ne, 0.0);
    for (size_t u = 0; u < np; u++) {
        const int64_t a0 = pg->tmpl_ptr[ptmpl[u]];
        for (int k = 0; k < plen[u]; k++) {
            const int64_t at = sptr[u / 32] + 64 * (k / 2) + 2 * (int64_t)(u % 32) + (k % 2);
            const int64_t c = (int64_t)pbase[u] + pg->tmpl_col[a0 + k];
            if (c < 0 || c > INT32_MAX) return fail(HF_ERR_INVALID, std::string(what) + " column out of range");
            if (c16) scol16[at] = (int16_t)(c - pcol0[u]);
            else scol[at] = (int32_t)c;
            sw[at] = pg->tmpl_w[a0 + k];
        }
    }
    R.scol = nullptr;
    R.scol16 = nullptr;
    R.pcol0 = nullptr;
    R.sw = nullptr;
    if ((rc = upload(own, (int64_t **)&R.sptr, sptr.data(), sptr.size(), B, C->stream))) return rc;
    if ((rc = upload(own, (uint8_t **)&R.plen, plen.data(), plen.size(), B, C->stream))) return rc;
    if (c16) {
        if ((rc = upload(own, (int16_t **)&R.scol16, scol16.data(), scol16.size(), B, C->stream))) return rc;
        if ((rc = upload(own, (int32_t **)&R.pcol0, pcol0.data(), pcol0.size(), B, C->stream))) return rc;
    } else {
        if ((rc = upload(own, (int32_t **)&R.scol, scol.data(), scol.size(), B, C->stream))) return rc;
    }
    if ((rc = upload(own, (double **)&R.sw, sw.data(), sw.size(), B, C->stream))) return rc;
    if ((rc = upload(own, (uint8_t **)&R.tag, ptag.data(), ptag.size(), B, C->stream))) return rc;
    if ((rc = upload(own, &R.val, (const double *)nullptr, np, B, C->stream))) return rc;
    entries = (int64_t)ne;
    // wait for the uploads before the host staging vectors go away
    if (cudaStreamSynchronize(C->stream) != cudaSuccess) return fail(HF_ERR_CUDA, std::string(what) + " rows");
    return HF_OK;
}

// The mixed form's velocity pairs by FP32 pattern (PatRows), uploaded on the
// case stream: R (the velocity pair set) gets its count and result array
// only; entries = the patterns' entry count.
int build_patterns(hf_case *C, std::vector<void *> &own, double &B, const hf_program *pg,
                   const std::vector<int32_t> &ptmpl, const std::vector<int32_t> &pbase,
                   const std::vector<double> &prhs, const std::vector<uint8_t> &ptag, PairRows &R, PatRows &V,
                   int64_t &entries)
{
    int rc;
    const size_t np = ptmpl.size();
    R.n = V.n = (int)np;
    // the pattern of every template the pairs use: its entries in column
    // order (weight bits breaking ties), offsets from its smallest column,
    // FP32 weights, byte for byte
    std::vector<int32_t> tpat(pg->ntmpl, -1), tmin(pg->ntmpl, 0), pstart;
    std::vector<uint8_t> plen;
    std::vector<PatEntry> ent;
    std::unordered_map<std::string, int32_t> known;
    std::string key;
    std::vector<PatEntry> row;
    for (size_t u = 0; u < np; u++) {
        const int32_t t = ptmpl[u];
        if (tpat[t] >= 0) continue;
        const int64_t a = pg->tmpl_ptr[t], e = pg->tmpl_ptr[t + 1];
        if (e - a > 255) return fail(HF_ERR_UNSUPPORTED, "velocity-stage stencil longer than 255 entries");
        int32_t m = 0;
        for (int64_t k = a; k < e; k++) m = k == a ? pg->tmpl_col[k] : std::min(m, pg->tmpl_col[k]);
        row.clear();
        for (int64_t k = a; k < e; k++) row.push_back({pg->tmpl_col[k] - m, (float)pg->tmpl_w[k]});
        std::sort(row.begin(), row.end(), [](const PatEntry &x, const PatEntry &y) {
            if (x.off != y.off) return x.off < y.off;
            uint32_t bx, by;
            memcpy(&bx, &x.w, 4);
            memcpy(&by, &y.w, 4);
            return bx < by;
        });
        key.assign((const char *)row.data(), row.size() * sizeof(PatEntry));
        auto it = known.find(key);
        if (it == known.end()) {
            if (ent.size() + row.size() > (size_t)INT32_MAX) return fail(HF_ERR_UNSUPPORTED, "too many velocity-stage patterns");
            it = known.emplace(key, (int32_t)pstart.size()).first;
            pstart.push_back((int32_t)ent.size());
            plen.push_back((uint8_t)row.size());
            ent.insert(ent.end(), row.begin(), row.end());
        }
        tpat[t] = it->second;
        tmin[t] = m;
    }
    std::vector<int32_t> pid(np), col0(np);
    for (size_t u = 0; u < np; u++) {
        const int64_t c = (int64_t)pbase[u] + tmin[ptmpl[u]];
        if (c < 0 || c > INT32_MAX) return fail(HF_ERR_INVALID, "velocity-stage column out of range");
        pid[u] = tpat[ptmpl[u]];
        col0[u] = (int32_t)c;
    }
    if ((rc = upload(own, (int32_t **)&V.pid, pid.data(), np, B, C->stream))) return rc;
    if ((rc = upload(own, (int32_t **)&V.col0, col0.data(), np, B, C->stream))) return rc;
    if ((rc = upload(own, (uint8_t **)&V.tag, ptag.data(), np, B, C->stream))) return rc;
    if ((rc = upload(own, (double **)&V.rhs, prhs.data(), np, B, C->stream))) return rc;
    if ((rc = upload(own, (int32_t **)&V.pstart, pstart.data(), pstart.size(), B, C->stream))) return rc;
    if ((rc = upload(own, (uint8_t **)&V.plen, plen.data(), plen.size(), B, C->stream))) return rc;
    if ((rc = upload(own, (PatEntry **)&V.ent, ent.data(), ent.size(), B, C->stream))) return rc;
    if ((rc = upload(own, &R.val, (const double *)nullptr, np, B, C->stream))) return rc;
    V.val = R.val;
    entries = (int64_t)ent.size();
    // wait for the uploads before the host staging vectors go away
    if (cudaStreamSynchronize(C->stream) != cudaSuccess) return fail(HF_ERR_CUDA, "velocity-stage patterns");
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
    if (cudaStreamCreateWithFlags(&C->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&C->body_stream, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(HF_ERR_CUDA, "stream"));
    C->h_scal = new Scal();
    keep_pool_memory(opt.device);

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
#define UP(dst, src, n) do { if ((rc = upload(own, dst, src, (size_t)(n), B, C->stream))) return cleanup(rc); } while (0)
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
            if (pg->inst_par[i].tempdiscrtype != pg->par.tempdiscrtype)
                return cleanup(fail(HF_ERR_UNSUPPORTED, "batch members differ in intermediate-velocity scheme"));
            if (pg->inst_par[i].ve_discrtype != pg->par.ve_discrtype)
                return cleanup(fail(HF_ERR_UNSUPPORTED, "batch members differ in constitutive scheme"));
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
    for (const hf_params &q : ipar) {
        if (q.flowtype != HF_VISCOELASTIC) continue;
        if (q.ve_model != HF_OLDROYD_B && q.ve_model != HF_GIESEKUS && q.ve_model != HF_LPTT && q.ve_model != HF_GPTT &&
            q.ve_model != HF_E_FENE)
            return cleanup(fail(HF_ERR_UNSUPPORTED, "viscoelastic model other than Oldroyd-B, Giesekus, LPTT, GPTT, e-FENE"));
        // the reference's Mittag-Leffler evaluation takes 0 < alpha <= 5 and
        // beta <= 5 (hig-flow-mittag-leffler.c:143-153)
        if (q.ve_model == HF_GPTT && !(q.alpha_gptt > 0.0 && q.alpha_gptt <= 5.0 && q.beta_gptt <= 5.0))
            return cleanup(fail(HF_ERR_INVALID, "GPTT needs 0 < alpha_gptt <= 5 and beta_gptt <= 5"));
    }
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
    P.projtype_all = ipar[0].projtype;
    for (int i = 1; i < ni; i++)
        if (ipar[i].projtype != P.projtype_all) P.projtype_all = -1;
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
        C->h_ipar = ipar;
        C->dt0.resize(ni);
        for (int i = 0; i < ni; i++) C->dt0[i] = ipar[i].dt;
        UP(&C->cfl_max, (const unsigned long long *)nullptr, ni);
        UP((double **)&P.ipinv, pinv.data(), pinv.size());
        for (const hf_params &q : ipar) C->gptt |= q.flowtype == HF_VISCOELASTIC && q.ve_model == HF_GPTT;
        if (C->gptt) UP(&P.gptt_e, (const double *)nullptr, pg->ncell);
    }
    UP((double **)&P.delta, pg->delta, (size_t)pg->ndelta * D);
    UP((int32_t **)&P.rows.tmpl, pg->row_tmpl, pg->nrows);
    UP((int32_t **)&P.rows.base, pg->row_base, pg->nrows);
    UP((double **)&P.rows.rhs, pg->row_rhs, pg->nrows);
    UP((int64_t **)&P.rows.tptr, pg->tmpl_ptr, pg->ntmpl + 1);
    UP((int32_t **)&P.rows.col, pg->tmpl_col, pg->nnz);
    UP((double **)&P.rows.w, pg->tmpl_w, pg->nnz);
    {
        // velocity slots: general codes renumbered to (row, field read) pairs,
        // so that k_vrows can evaluate each pair once per step on its field
        std::vector<int32_t> pair_first(pg->nrows, -1);
        std::vector<uint8_t> tag_first(pg->nrows, 0);
        std::unordered_map<uint64_t, int32_t> extra;   // pairs of rows read on a second field
        std::vector<int32_t> ptmpl, pbase;
        std::vector<double> prhs;
        std::vector<uint8_t> ptag;
        bool overflow = false;
        auto pair_index = [&](int64_t r, int tag) -> int32_t {
            auto add = [&]() {
                if (ptmpl.size() >= (size_t)INT32_MAX) overflow = true;
                ptmpl.push_back(pg->row_tmpl[r]);
                pbase.push_back(pg->row_base[r]);
                prhs.push_back(pg->row_rhs[r]);
                ptag.push_back((uint8_t)tag);
                return (int32_t)(ptmpl.size() - 1);
            };
            if (pair_first[r] < 0) {
                tag_first[r] = (uint8_t)tag;
                return pair_first[r] = add();
            }
            if (tag_first[r] == tag) return pair_first[r];
            const uint64_t key = (uint64_t)r * 32 + (uint64_t)tag;
            auto it = extra.find(key);
            if (it != extra.end()) return it->second;
            const int32_t u = add();
            extra.emplace(key, u);
            return u;
        };
        std::vector<int32_t> row;
        for (int d = 0; d < D; d++) {
            const int64_t nf = pg->nfacet[d];
            UP((int32_t **)&P.vslots[d], (const int32_t *)nullptr, (size_t)pg->vel_nslot * nf);
            for (int s = 0; s < pg->vel_nslot; s++) {
                int tag;
                if (s == HF_V_FU) tag = d;
                else if (s == HF_V_PL || s == HF_V_PR) tag = 3;
                else if (s == HF_V_FL || s == HF_V_FR) tag = 4;
                else if (s < HF_V_NSLOT_NEWT(D)) {
                    const int d2 = (s - HF_V_BLK0) / HF_V_NB, k = (s - HF_V_BLK0) % HF_V_NB;
                    tag = 5 + ((k < 4 || k >= 8) ? d2 : d);
                } else {
                    tag = 8 + d * D + (s - HF_V_NSLOT_NEWT(D)) / HF_V_NS;
                }
                const int32_t *sl = pg->vel_slots[d] + (size_t)s * nf;
                row.assign(sl, sl + nf);
                for (int64_t f = 0; f < nf; f++)
                    if (row[f] < 0) row[f] = -pair_index(-(int64_t)row[f] - 1, tag) - 1;
                if (overflow) return cleanup(fail(HF_ERR_UNSUPPORTED, "too many velocity-stage rows"));
                if (cudaMemcpyAsync((int32_t *)P.vslots[d] + (size_t)s * nf, row.data(), sizeof(int32_t) * nf,
                                    cudaMemcpyHostToDevice, C->stream) != cudaSuccess)
                    return cleanup(fail(HF_ERR_CUDA, "velocity slots"));
            }
            UP((uint32_t **)&P.vflags[d], pg->vel_flags[d], pg->nfacet[d]);
            UP((uint16_t **)&P.vdelta[d], pg->vel_delta[d], pg->nfacet[d]);
        }
        C->vmix = opt.precision == HF_PREC_MIXED;
        if (C->vmix) rc = build_patterns(C, own, B, pg, ptmpl, pbase, prhs, ptag, P.vr, C->vp, C->vel_entries);
        else rc = build_pairs(C, own, B, pg, ptmpl, pbase, prhs, ptag, P.vr, C->vel_entries, "velocity-stage");
        if (rc) return cleanup(rc);
        P.vrow.tptr = P.rows.tptr;
        P.vrow.col = P.rows.col;
        P.vrow.w = P.rows.w;
        UP((int32_t **)&P.vrow.tmpl, ptmpl.data(), ptmpl.size());
        UP((int32_t **)&P.vrow.base, pbase.data(), pbase.size());
        UP((double **)&P.vrow.rhs, prhs.data(), prhs.size());
        P.vr.rhs = P.vrow.rhs;
    }
    UP((int32_t **)&P.dslots, pg->div_slots, (size_t)2 * D * pg->ncell);
    UP((uint16_t **)&P.cdelta, pg->cell_delta, pg->ncell);
    if (pg->par.flowtype == HF_VISCOELASTIC) {
        // cell slots: the general codes k_ve_cell reads renumbered to cell-stage
        // pairs (velocity at the faces and corners on u[d]; the kernel's
        // neighbours on each upper-triangle component, consecutive pairs)
        const int64_t nc = pg->ncell;
        std::vector<int32_t> cs(pg->cell_slots, pg->cell_slots + (size_t)pg->cell_nslot * nc);
        std::vector<int32_t> ptmpl, pbase;
        std::vector<double> prhs;
        std::vector<uint8_t> ptag;
        std::unordered_map<uint64_t, int32_t> seen;   // (row, first tag) -> first pair
        bool overflow = false;
        auto pairs_of = [&](int64_t r, const int *tags, int ntag) -> int32_t {
            const uint64_t key = (uint64_t)r * 32 + (uint64_t)tags[0];
            auto it = seen.find(key);
            if (it != seen.end()) return it->second;
            if (ptmpl.size() + ntag >= (size_t)INT32_MAX) overflow = true;
            const int32_t first = (int32_t)ptmpl.size();
            for (int m = 0; m < ntag; m++) {
                ptmpl.push_back(pg->row_tmpl[r]);
                pbase.push_back(pg->row_base[r]);
                prhs.push_back(pg->row_rhs[r]);
                ptag.push_back((uint8_t)tags[m]);
            }
            seen.emplace(key, first);
            return first;
        };
        int ktags[6], nk = 0;
        for (int i = 0; i < D; i++)
            for (int j = i; j < D; j++) ktags[nk++] = 17 + i * D + j;
        const int NU = 2 * D, NQ = HF_C_NQ * D * (D - 1);
        for (int k = 0; k < NU + NQ; k++) {
            const int slot = k < NU ? HF_C_BLK0 + HF_C_NB * (k >> 1) + (k & 1) : HF_C_BLK0 + HF_C_NB * D + (k - NU);
            const int tag = 5 + (k < NU ? (k >> 1) : (k - NU) / (HF_C_NQ * (D - 1)));
            int32_t *sl = cs.data() + (size_t)slot * nc;
            for (int64_t c = 0; c < nc; c++)
                if (sl[c] < 0) sl[c] = -pairs_of(-(int64_t)sl[c] - 1, &tag, 1) - 1;
        }
        for (int k = 0; k < 4 * D; k++) {
            int32_t *sl = cs.data() + (size_t)(HF_C_BLK0 + HF_C_NB * (k >> 2) + HF_C_KL + (k & 3)) * nc;
            for (int64_t c = 0; c < nc; c++)
                if (sl[c] < 0) sl[c] = -pairs_of(-(int64_t)sl[c] - 1, ktags, nk) - 1;
        }
        if (overflow) return cleanup(fail(HF_ERR_UNSUPPORTED, "too many cell-stage rows"));
        UP((int32_t **)&P.cslots, cs.data(), cs.size());
        UP((uint32_t **)&P.cflags, pg->cell_flags, pg->ncell);
        if ((rc = build_pairs(C, own, B, pg, ptmpl, pbase, prhs, ptag, P.cr, C->cell_entries, "cell-stage")))
            return cleanup(rc);
        UP((double **)&P.cr.rhs, prhs.data(), prhs.size());
        // wait for the uploads before the host staging vectors go away
        if (cudaStreamSynchronize(C->stream) != cudaSuccess) return cleanup(fail(HF_ERR_CUDA, "cell slots"));
    }
    // fields
    DevFields &F = C->F;
    memset(&F, 0, sizeof F);
    const bool rk = pg->par.tempdiscrtype == HF_EXPLICIT_RK2 || pg->par.tempdiscrtype == HF_EXPLICIT_RK3;
    if (pg->par.tempdiscrtype != HF_EXPLICIT_EULER && !rk && pg->par.tempdiscrtype != HF_SEMI_IMPLICIT_EULER &&
        pg->par.tempdiscrtype != HF_SEMI_IMPLICIT_CN && pg->par.tempdiscrtype != HF_SEMI_IMPLICIT_BDF2)
        return cleanup(fail(HF_ERR_UNSUPPORTED, "unknown intermediate-velocity scheme"));
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
    // semi-implicit Euler (higflow_semi_implicit_euler_intermediate_velocity,
    // hig-flow-step.c:788-883): the row of facet f of direction d is
    //   alpha u_f + sum_d2 w_d2 (S(f + delta_d2) + S(f - delta_d2)),
    //   w_d2 = -dt / (Re delta_d2^2),  alpha = 1 - 2 sum_d2 w_d2,
    // where S(point) is the point's interpolation stencil: the recorded UR / UL
    // slots of block d2 (the same sfd_get_stencil queries, made there with
    // weight 1); entries on one facet are added in stencil order, and each
    // stencil's boundary term (w times the row's rhs) goes to the right-hand
    // side, as sfd_get_stencil does with stn_add_to_rhs.
    const int scheme = pg->par.tempdiscrtype;
    if (scheme == HF_SEMI_IMPLICIT_EULER || scheme == HF_SEMI_IMPLICIT_CN || scheme == HF_SEMI_IMPLICIT_BDF2) {
        if (ni > 1) return cleanup(fail(HF_ERR_UNSUPPORTED, "semi-implicit velocity in a batch"));
        C->sie = true;
        C->bdf2 = scheme == HF_SEMI_IMPLICIT_BDF2;
        P.sie = 1;
        const double dt = pg->par.dt, Re = pg->par.Re;
        // the weights as the reference writes them: -dt/(Re d^2) (Euler,
        // hig-flow-step.c:837), - 0.5*dt/(..) (Crank-Nicolson, :939), - 0.25*dt/(..)
        // then - 1.0/3.0*dt/(..) (BDF2, :1042, :1129)
        auto weight = [&](int stage, double fd) {
            if (scheme == HF_SEMI_IMPLICIT_CN) return -0.5 * dt / (Re * fd * fd);
            if (scheme == HF_SEMI_IMPLICIT_BDF2) return stage == 0 ? -0.25 * dt / (Re * fd * fd) : -1.0 / 3.0 * dt / (Re * fd * fd);
            return -dt / (Re * fd * fd);
        };
        int maxnf = 0;
        for (int stage = 0; stage < (C->bdf2 ? 2 : 1); stage++)
        for (int d = 0; d < D; d++) {
            const int nf = pg->nfacet[d];
            maxnf = std::max(maxnf, nf);
            std::vector<int32_t> ptr(1, 0), col;
            std::vector<double> val, dg(nf, 0.0), bc(nf, 0.0);
            std::vector<std::pair<int32_t, double>> row;
            auto add = [&](int32_t c, double v) {
                for (auto &e : row)
                    if (e.first == c) { e.second += v; return; }
                row.emplace_back(c, v);
            };
            for (int f = 0; f < nf; f++) {
                row.clear();
                const double *fd = pg->delta + (size_t)pg->vel_delta[d][f] * D;
                double alpha = 0.0, b = 0.0;
                for (int d2 = 0; d2 < D; d2++) {
                    const double w = weight(stage, fd[d2]);
                    alpha -= 2.0 * w;
                    for (int side : {HF_V_UR, HF_V_UL}) {
                        const int32_t code = pg->vel_slots[d][(size_t)(HF_V_BLK0 + HF_V_NB * d2 + side) * nf + f];
                        if (code >= 0) {
                            if (code >= nf) return cleanup(fail(HF_ERR_INVALID, "velocity slot outside its field"));
                            add(code, w);
                            continue;
                        }
                        const int64_t r = -(int64_t)code - 1;
                        if (r >= pg->nrows) return cleanup(fail(HF_ERR_INVALID, "velocity slot outside the rows"));
                        const int64_t t = pg->row_tmpl[r];
                        for (int64_t k = pg->tmpl_ptr[t]; k < pg->tmpl_ptr[t + 1]; k++) {
                            const int64_t c = (int64_t)pg->row_base[r] + pg->tmpl_col[k];
                            if (c < 0 || c >= nf) return cleanup(fail(HF_ERR_INVALID, "stencil column outside its field"));
                            add((int32_t)c, w * pg->tmpl_w[k]);
                        }
                        b += w * pg->row_rhs[r];
                    }
                }
                alpha = 1.0 + alpha;
                add(f, alpha);
                for (auto &e : row) {
                    col.push_back(e.first);
                    val.push_back(e.second);
                    if (e.first == f) dg[f] = e.second;
                }
                ptr.push_back((int32_t)col.size());
                bc[f] = b;
            }
            for (int f = 0; f < nf; f++) dg[f] = dg[f] != 0.0 ? 1.0 / dg[f] : 1.0;
            DevMat &Mu = stage == 0 ? C->Mu[d] : C->Mu2[d];
            Mu.n = nf;
            UP((int32_t **)&Mu.ptr, ptr.data(), ptr.size());
            UP((int32_t **)&Mu.col, col.data(), col.size());
            UP((double **)&Mu.val, val.data(), val.size());
            UP((double **)&Mu.dinv, dg.data(), dg.size());
            if (stage == 0) {
                UP((double **)&P.sie_bc[d], bc.data(), bc.size());
                UP(&P.sie_b[d], (const double *)nullptr, nf);
                if (C->bdf2) {
                    UP(&P.sie_e[d], (const double *)nullptr, nf);
                    UP(&C->ua[d], (const double *)nullptr, nf);
                }
            } else {
                UP((double **)&P.sie_bc2[d], bc.data(), bc.size());
            }
        }
        BiVec &V = C->Vu;
        UP(&V.r, (const double *)nullptr, maxnf);
        UP(&V.rh, (const double *)nullptr, maxnf);
        UP(&V.p, (const double *)nullptr, maxnf);
        UP(&V.v, (const double *)nullptr, maxnf);
        UP(&V.s, (const double *)nullptr, maxnf);
        UP(&V.t, (const double *)nullptr, maxnf);
        UP(&V.ph, (const double *)nullptr, maxnf);
        UP(&V.sh, (const double *)nullptr, maxnf);
        UP(&V.partials, (const double *)nullptr, (size_t)blocks(maxnf) * 4);
        UP(&V.sc, (const Scal *)nullptr, 1);
    }
    // Poisson operator
    std::vector<int32_t> mptr, mcol;
    std::vector<double> mval, dinv, apin;
    bool sym = false;
    if ((rc = build_matrix(pg, pins, mptr, mcol, mval, dinv, apin, sym))) return cleanup(rc);
    C->use_cg = opt.poisson == HF_POISSON_CG || (opt.poisson == HF_POISSON_AUTO && sym);
    if (opt.poisson == HF_POISSON_CG && !sym) return cleanup(fail(HF_ERR_UNSUPPORTED, "CG requested on a non-symmetric Poisson matrix"));
    if (ni > 1 && !C->use_cg) return cleanup(fail(HF_ERR_UNSUPPORTED, "batches need symmetric Poisson rows (CG)"));
    if (opt.precision == HF_PREC_MIXED && !C->use_cg)
        return cleanup(fail(HF_ERR_UNSUPPORTED, "the mixed form needs the CG solver"));
    C->amg = opt.precond != HF_PRECOND_JACOBI;   // BiCGStab too: the V-cycle preconditions it
    C->bi_amg = !C->use_cg && C->amg;
    C->mixed = C->use_cg && C->amg && opt.precision == HF_PREC_MIXED;
    DevMat &M = C->M;
    M.n = pg->ncell;
    if (!C->use_cg) {   // BiCGStab reads CSR; the CG path keeps the row templates
        UP((int32_t **)&M.ptr, mptr.data(), mptr.size());
        UP((int32_t **)&M.col, mcol.data(), mcol.size());
        UP((double **)&M.val, mval.data(), mval.size());
    }
    UP((double **)&M.dinv, dinv.data(), dinv.size());
    UP((double **)&M.apin, apin.data(), apin.size());
    UP((double **)&M.brhs, pg->p_brhs, pg->ncell);
    const int nb = blocks(pg->ncell);
    Scal *sc = nullptr;
    UP(&sc, (const Scal *)nullptr, 1);
    {
        Scal h{};
        h.maxit = opt.poisson_maxit;
        if (cudaMemcpyAsync(sc, &h, sizeof h, cudaMemcpyHostToDevice, C->stream) != cudaSuccess)
            return cleanup(fail(HF_ERR_CUDA, "scalars"));
    }
    double *partials = nullptr;
    UP(&partials, (const double *)nullptr, (size_t)nb * 4);
    const int n = pg->ncell;
    if (C->use_cg) {
        if ((rc = build_pcg(C, mptr, mcol, mval, pins))) return cleanup(rc);
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
        if (C->bi_amg) {
            // the instance's hierarchy for the preconditioner; its CG state
            // stays idle (the instance is marked not done, so that the
            // V-cycle kernels run on it).  An operator the hierarchy's row
            // encoding cannot hold keeps the Jacobi scaling.
            rc = build_pcg(C, mptr, mcol, mval, pins);
            if (rc == HF_ERR_UNSUPPORTED) {
                C->bi_amg = false;
                C->amg = false;
                rc = HF_OK;
            } else if (rc) {
                return cleanup(rc);
            } else if (cudaMemsetAsync(&C->G.S[0].done, 0, sizeof(int32_t), C->stream) != cudaSuccess) {
                return cleanup(fail(HF_ERR_CUDA, "preconditioner state"));
            }
        }
    }
#undef UP
    if (cudaStreamSynchronize(C->stream) != cudaSuccess) return cleanup(fail(HF_ERR_CUDA, "create sync"));
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
    // a new value of the solve's unknown restarts its time history (the next
    // initial guess is the value itself, not an extrapolation)
    if (C->G.xprev && (field == HF_FIELD_DP || field == HF_FIELD_P)) {
        k_pcg_restart<<<blocks(C->P.ncell), kBlock, 0, C->stream>>>(C->G);
        HF_CK(cudaGetLastError());
    }
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
    if (!C || nsteps < 0) return fail(HF_ERR_INVALID, "bad argument");
    return run_steps(C, nsteps, true);
}

extern "C" int hf_case_step_async(hf_case *C, int32_t nsteps)
{
    if (!C || nsteps < 0) return fail(HF_ERR_INVALID, "bad argument");
    return run_steps(C, nsteps, false);
}

extern "C" int hf_case_synchronize(hf_case *C)
{
    if (!C) return fail(HF_ERR_INVALID, "null case");
    HF_CK(cudaStreamSynchronize(C->stream));
    if (!C->use_cg) return HF_OK;
    int rc = collect_phases(C);
    if (!rc) rc = pull_state(C);
    return rc ? rc : take_error(C);
}

extern "C" int hf_case_stats(hf_case *C, hf_stats *out)
{
    if (!C || !out) return fail(HF_ERR_INVALID, "null argument");
    if (C->use_cg) {
        int rc = pull_state(C);
        if (rc) return rc;
        hf_stats &s = C->stats;
        s.last_iters = 0;
        s.last_residual = 0.0;
        s.total_iters = 0;
        s.last_outer = 1;
        for (int i = 0; i < C->ninst; i++) {
            const IScal &q = C->h_S[i];
            s.last_iters = std::max(s.last_iters, q.iters + q.iters_prev);
            s.last_outer = std::max(s.last_outer, C->mixed ? q.outer + 1 : 1);
            s.last_residual = std::max(s.last_residual, q.bb > 0 ? sqrt(q.rr / q.bb) : sqrt(q.rr));
            s.total_iters += q.total_iters;
        }
        s.kernel_launches = s.steps * C->fixed_kernels + C->h_ctl->total_bodies * C->body_kernels + C->sie_launches;
    }
    *out = C->stats;
    if (!C->use_cg) out->last_outer = 1;
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
    if (outer) *outer = 1;
    if (!C->use_cg) {
        if (iters) *iters = C->stats.last_iters;
        if (status) *status = C->h_scal->status == 1 ? HF_ERR_NOT_CONVERGED : C->h_scal->status;
        if (residual) *residual = C->stats.last_residual;
        return HF_OK;
    }
    int rc = pull_state(C);
    if (rc) return rc;
    const IScal &q = C->h_S[inst];
    if (iters) *iters = q.iters + q.iters_prev;
    if (outer) *outer = C->mixed ? q.outer + 1 : 1;
    if (status) *status = q.status;
    if (residual) *residual = q.bb > 0 ? sqrt(q.rr / q.bb) : sqrt(q.rr);
    return HF_OK;
}

// Adaptive time step (higflow_adjust_timestep, hig-flow-timestep.c:115-139),
// every instance on its own CFL number.  Waits for the case's stream.
extern "C" int hf_case_adjust_timestep(hf_case *C, double *cfl, double *dt, int32_t n)
{
    if (!C) return fail(HF_ERR_INVALID, "null case");
    if ((cfl || dt) && n != C->ninst) return fail(HF_ERR_INVALID, "array size is not the instance count");
    if (C->sie) return fail(HF_ERR_UNSUPPORTED, "adaptive time step with the semi-implicit velocity (its matrix holds dt)");
    const int ni = C->ninst;
    cudaStream_t st = C->stream;
    if (C->D == 2 || C->D == 3) {
        HF_CK(cudaMemsetAsync(C->cfl_max, 0, sizeof(unsigned long long) * ni, st));
        if (C->D == 2) k_cfl<2><<<blocks(C->P.ncell), kBlock, 0, st>>>(C->P, C->F, C->cfl_max);
        else k_cfl<3><<<blocks(C->P.ncell), kBlock, 0, st>>>(C->P, C->F, C->cfl_max);
        HF_CK(cudaGetLastError());
    }
    std::vector<unsigned long long> bits(ni);
    HF_CK(cudaMemcpyAsync(bits.data(), C->cfl_max, sizeof(unsigned long long) * ni, cudaMemcpyDeviceToHost, st));
    HF_CK(cudaStreamSynchronize(st));
    const double max_cfl = 0.1, max_dt_factor = 1.1;   // MAX_CFL, MAX_DT_FACTOR (hig-flow-timestep.h:13-14)
    for (int i = 0; i < ni; i++) {
        double norm;
        memcpy(&norm, &bits[i], sizeof norm);
        hf_params &par = C->h_ipar[i];
        const double c = norm * par.dt;
        const double dtmax = C->dt0[i] * 32.0;
        const double dt_factor = std::min(max_cfl / (c + 1.0e-12), max_dt_factor);
        const double newdt = dt_factor * par.dt;
        par.dt = std::min(newdt, dtmax);
        if (cfl) cfl[i] = c;
        if (dt) dt[i] = par.dt;
    }
    // the kernels read dt from the device parameter array (captured step
    // graphs included), so the next step uses the new values
    HF_CK(cudaMemcpyAsync((void *)C->P.ipar, C->h_ipar.data(), sizeof(hf_params) * ni, cudaMemcpyHostToDevice, st));
    HF_CK(cudaStreamSynchronize(st));
    C->par.dt = C->h_ipar[0].dt;
    C->P.par.dt = C->h_ipar[0].dt;
    return HF_OK;
}

extern "C" int hf_case_set_timestep(hf_case *C, const double *dt, int32_t n)
{
    if (!C || !dt) return fail(HF_ERR_INVALID, "null argument");
    if (n != C->ninst) return fail(HF_ERR_INVALID, "array size is not the instance count");
    bool same = true;
    for (int i = 0; i < n; i++) {
        if (!(dt[i] > 0.0) || !std::isfinite(dt[i])) return fail(HF_ERR_INVALID, "time step must be positive and finite");
        same = same && dt[i] == C->h_ipar[i].dt;
    }
    if (C->sie) {
        if (same) return HF_OK;
        return fail(HF_ERR_UNSUPPORTED, "new time step with the semi-implicit velocity (its matrix holds dt)");
    }
    // (the parameters go to the device on every call, as the host's dt of
    // each step; no step of this case is in flight past the synchronisation)
    for (int i = 0; i < n; i++) C->h_ipar[i].dt = dt[i];
    HF_CK(cudaMemcpyAsync((void *)C->P.ipar, C->h_ipar.data(), sizeof(hf_params) * n, cudaMemcpyHostToDevice,
                          C->stream));
    HF_CK(cudaStreamSynchronize(C->stream));
    C->par.dt = C->h_ipar[0].dt;
    C->P.par.dt = C->h_ipar[0].dt;
    return HF_OK;
}

extern "C" int hf_case_launch_shapes(hf_case *C, int32_t *blocks, int32_t n)
{
    if (!C || !blocks || n < 3) return fail(HF_ERR_INVALID, "bad argument");
    blocks[0] = C->blk_vrows;
    blocks[1] = C->blk_vel;
    blocks[2] = C->blk_ve;
    return HF_OK;
}

extern "C" int hf_case_set_step_limits(hf_case *C, const int64_t *steps, int32_t n)
{
    if (!C || !steps) return fail(HF_ERR_INVALID, "null argument");
    if (n != C->ninst) return fail(HF_ERR_INVALID, "array size is not the instance count");
    if (!C->use_cg || C->sie) return fail(HF_ERR_UNSUPPORTED, "step limits need the CG Poisson path and an explicit velocity");
    std::vector<int64_t> h(steps, steps + n);
    for (int64_t &v : h)
        if (v < 0) v = -1;
    HF_CK(cudaStreamSynchronize(C->stream));   // no step of this case in flight
    if (!C->ilim) {
        double bytes = 0;
        int rc = upload(C->owned, &C->ilim, h.data(), h.size(), bytes, C->stream);
        if (rc) return rc;
        C->bytes += bytes;
        C->P.ilim = C->ilim;
        C->G.ilim = C->ilim;
        // the row-pair kernels skip frozen instances' pairs too
        for (PairRows *R : {&C->P.vr, &C->P.cr}) {
            R->ilim = C->ilim;
            for (int d = 0; d < 3; d++) R->finst[d] = C->P.finst[d];
            R->cinst = C->P.cinst;
        }
        C->vp.ilim = C->ilim;
        for (int d = 0; d < 3; d++) C->vp.finst[d] = C->P.finst[d];
        C->vp.cinst = C->P.cinst;
        destroy_graphs(C);   // the captured kernels hold the parameters without limits
    } else {
        HF_CK(cudaMemcpyAsync(C->ilim, h.data(), sizeof(int64_t) * h.size(), cudaMemcpyHostToDevice, C->stream));
    }
    HF_CK(cudaStreamSynchronize(C->stream));
    return HF_OK;
}

extern "C" int hf_case_instance_failures(hf_case *C, int32_t *status, int32_t n)
{
    if (!C || !status) return fail(HF_ERR_INVALID, "null argument");
    if (n != C->ninst) return fail(HF_ERR_INVALID, "array size is not the instance count");
    if (!C->use_cg) {
        for (int i = 0; i < n; i++) status[i] = 0;
        return HF_OK;
    }
    int rc = pull_state(C);
    if (rc) return rc;
    for (int i = 0; i < n; i++) status[i] = C->h_S[i].failed;
    return HF_OK;
}

extern "C" int hf_case_instance_iters(hf_case *C, int64_t *total_iters, int32_t n)
{
    if (!C || !total_iters || n != C->ninst) return fail(HF_ERR_INVALID, "bad argument");
    if (!C->use_cg) {
        total_iters[0] = C->stats.total_iters;
        return HF_OK;
    }
    int rc = pull_state(C);
    if (rc) return rc;
    for (int i = 0; i < n; i++) total_iters[i] = C->h_S[i].total_iters;
    return HF_OK;
}

extern "C" int hf_case_solver_info(hf_case *C, int32_t *method, int32_t *nlev, int64_t *rows, int64_t *nnz_a,
                                   int64_t *nnz_p, int64_t *nnz_r, int32_t max_levels)
{
    if (!C || !method || !nlev) return fail(HF_ERR_INVALID, "null argument");
    *method = C->use_cg ? (C->amg ? HF_PRECOND_AMG : HF_PRECOND_JACOBI) : -1;
    if (!C->amg) {
        *nlev = 1;
        if (max_levels > 0) {
            if (rows) rows[0] = C->M.n;
            if (nnz_a) nnz_a[0] = C->use_cg ? C->lnnz_a[0] : 0;
            if (nnz_p) nnz_p[0] = 0;
            if (nnz_r) nnz_r[0] = 0;
        }
        return HF_OK;
    }
    // the concatenated levels, then one entry for the dense coarsest solves
    *nlev = C->nlev + 1;
    const int64_t crows = C->coarse_rows, cdense = C->coarse_dense;
    for (int l = 0; l < *nlev && l < max_levels; l++) {
        const bool dense = l == C->nlev;
        if (rows) rows[l] = dense ? crows : C->lrows[l];
        if (nnz_a) nnz_a[l] = dense ? cdense : C->lnnz_a[l];
        if (nnz_p) nnz_p[l] = dense ? 0 : C->lnnz_p[l];
        if (nnz_r) nnz_r[l] = dense ? 0 : C->lnnz_r[l];
    }
    return HF_OK;
}

extern "C" int hf_case_launch_counts(hf_case *C, int32_t *per_step, int32_t *per_body)
{
    if (!C || !per_step || !per_body) return fail(HF_ERR_INVALID, "null argument");
    *per_step = C->fixed_kernels;
    *per_body = C->body_kernels;
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
    int rc = collect_phases(C);
    if (rc) return rc;
    if (enable && !C->ev[0])
        for (int k = 0; k < 2 * HF_NPHASE; k++) HF_CK(cudaEventCreate(&C->ev[k]));
    C->profile = enable != 0;
    for (int k = 0; k < HF_NPHASE; k++) { C->phase_ms[k] = 0.0; C->phase_launches[k] = 0; }
    return HF_OK;
}

extern "C" int hf_case_phase_times(hf_case *C, double *ms, int64_t *launches, int32_t n)
{
    if (!C || n < 0) return fail(HF_ERR_INVALID, "bad argument");
    int rc = collect_phases(C);
    if (rc) return rc;
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
    destroy_graphs(C);
    for (int k = 0; k < 2 * HF_NPHASE; k++)
        if (C->ev[k]) cudaEventDestroy(C->ev[k]);
    for (void *p : C->owned) cudaFreeAsync(p, C->stream);
    delete C->h_scal;
    delete[] C->h_S;
    delete C->h_ctl;
    if (C->body_stream) cudaStreamDestroy(C->body_stream);
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

// ---------------------------------------------------------------------------
// BiCGStab without allocation: the hf_slv_solve iteration on a CSR system the
// caller already holds in device memory, with every work vector in one static
// device buffer.  For callers that cannot allocate once they run: a host code
// that sizes its whole HBM budget at start-up, or one that solves on a stream
// while other streams of the same device are busy, where cudaMalloc/cudaFree
// would synchronise the device and stall them.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNaMaxRows = 1 << 16;                            // 65536 rows
constexpr int kNaMaxBlocks = (kNaMaxRows + kBlock - 1) / kBlock;
constexpr size_t kNaScalDoubles = (sizeof(Scal) + 7) / 8;
// dinv, r, rh, p, v, s, t, ph, sh; partial sums; scalars (about 4.7 MB)
constexpr size_t kNaDoubles = 9 * (size_t)kNaMaxRows + 4 * (size_t)kNaMaxBlocks + kNaScalDoubles;
static __device__ __align__(256) double g_noalloc_scratch[kNaDoubles];

constexpr int kNaMaxDevices = 64;
std::mutex g_na_mutex;
double *g_na_ptr[kNaMaxDevices] = {};

// dinv = 1 / a_ii (1 where the diagonal is missing or zero), as slv_upload_matrix
__global__ void __launch_bounds__(kBlock) k_na_dinv(DevMat M, double *dinv)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M.n) return;
    double d = 1.0;
    for (int k = M.ptr[i]; k < M.ptr[i + 1]; k++)
        if (M.col[k] == i && M.val[k] != 0.0) d = 1.0 / M.val[k];
    dinv[i] = d;
}

// fresh scalars: zero (the reduction counter too, so a call that stopped on an
// error leaves nothing behind for the next one), iteration cap set
__global__ void k_na_begin(Scal *sc, int maxit)
{
    Scal z{};
    z.maxit = maxit;
    *sc = z;
}

// An error inside the no-alloc solve: wait for the kernels already queued (they
// use the shared scratch) when the stream still answers, forget the kept scratch
// address of the device (the next call looks it up again), then report.
int na_fail(cudaStream_t st, int dev, const std::string &msg)
{
    cudaStreamSynchronize(st);
    cudaGetLastError();
    {
        std::lock_guard<std::mutex> lock(g_na_mutex);
        g_na_ptr[dev] = nullptr;
    }
    return fail(HF_ERR_CUDA, msg);
}

}  // namespace

namespace {

__global__ void __launch_bounds__(kBlock) k_mittag_leffler(int n, double a, double b, int fi,
                                                           const double *__restrict__ z, double *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const hf::Cx e = hf::mittag_leffler<2>(a, b, hf::cx_make(z[2 * i], z[2 * i + 1]), fi);
    out[2 * i] = e.re;
    out[2 * i + 1] = e.im;
}

}  // namespace

extern "C" int hf_mittag_leffler(double alpha, double beta, const double *z, int64_t n, int32_t fi, double *out)
{
    if (n < 0 || n > (int64_t)1 << 30 || (n > 0 && (!z || !out))) return fail(HF_ERR_INVALID, "bad argument");
    if (!(alpha > 0.0 && alpha <= 5.0) || !(beta <= 5.0))
        return fail(HF_ERR_INVALID, "Mittag-Leffler needs 0 < alpha <= 5 and beta <= 5");
    if (fi < 1 || fi > 8) return fail(HF_ERR_INVALID, "Mittag-Leffler accuracy digits fi must be 1..8");
    if (n == 0) return HF_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(HF_ERR_NO_DEVICE, "no CUDA device");
    double *d = nullptr;
    const size_t bytes = sizeof(double) * 2 * (size_t)n;
    HF_CK(cudaMalloc(&d, 2 * bytes));
    cudaError_t e = cudaMemcpy(d, z, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_mittag_leffler<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock>>>((int)n, alpha, beta, fi, d, d + 2 * n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(HF_ERR_CUDA, std::string("Mittag-Leffler evaluation: ") + cudaGetErrorString(e));
    return HF_OK;
}

extern "C" int hf_slv_solve_device_noalloc(int32_t n, const int32_t *ptr, const int32_t *col, const double *val,
                                           const double *b, double *x, double rtol, double atol, int32_t maxit,
                                           void *stream, int32_t *iterations, double *residual)
{
    if (n <= 0 || !ptr || !col || !val || !b || !x || maxit <= 0) return fail(HF_ERR_INVALID, "bad argument");
    if (n > kNaMaxRows)
        return fail(HF_ERR_INVALID, "system of " + std::to_string(n) + " rows exceeds the static scratch of " +
                                        std::to_string(kNaMaxRows) + " rows");
    int dev = 0;
    HF_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNaMaxDevices) return fail(HF_ERR_INVALID, "device ordinal beyond the scratch table");
    double *base;
    {
        // once per device, with that device current: the scratch's address
        std::lock_guard<std::mutex> lock(g_na_mutex);
        if (!g_na_ptr[dev]) {
            double *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return fail(HF_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            g_na_ptr[dev] = p;
        }
        base = g_na_ptr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    DevMat M{};
    M.n = n;
    M.ptr = ptr;
    M.col = col;
    M.val = val;
    double *dinv = base;
    M.dinv = dinv;
    BiVec V{};
    double *v = base + kNaMaxRows;
    V.x = x;
    V.b = const_cast<double *>(b);   // k_slv_init and k_bi_* only read b
    V.r = v; v += kNaMaxRows;
    V.rh = v; v += kNaMaxRows;
    V.p = v; v += kNaMaxRows;
    V.v = v; v += kNaMaxRows;
    V.s = v; v += kNaMaxRows;
    V.t = v; v += kNaMaxRows;
    V.ph = v; v += kNaMaxRows;
    V.sh = v; v += kNaMaxRows;
    V.partials = v; v += 4 * (size_t)kNaMaxBlocks;
    V.sc = (Scal *)v;
    k_na_dinv<<<blocks(n), kBlock, 0, st>>>(M, dinv);
    k_na_begin<<<1, 1, 0, st>>>(V.sc, maxit);
    Scal h{};
    int restarts = 0, first = 1;
    for (;;) {
        k_slv_init<<<blocks(n), kBlock, 0, st>>>(M, V, rtol, atol, first);
        first = 0;
        int chunk = 4;
        for (;;) {
            for (int k = 0; k < chunk; k++) {
                k_bi_p<<<blocks(n), kBlock, 0, st>>>(M, V);
                k_bi_spmv<<<blocks(n), kBlock, 0, st>>>(M, V, V.ph, V.v, 0);
                k_bi_s<<<blocks(n), kBlock, 0, st>>>(M, V);
                k_bi_spmv<<<blocks(n), kBlock, 0, st>>>(M, V, V.sh, V.t, 1);
                k_bi_update<<<blocks(n), kBlock, 0, st>>>(M, V);
            }
            cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaMemcpyAsync(&h, V.sc, sizeof(Scal), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return na_fail(st, dev, std::string("no-alloc BiCGStab: ") + cudaGetErrorString(e));
            if (h.done) break;
            chunk = std::min(chunk * 2, 32);
        }
        if (h.status == 1 && restarts++ < 50) continue;
        break;
    }
    if (iterations) *iterations = h.iters;
    if (residual) *residual = h.bb > 0 ? sqrt(h.rr / h.bb) : sqrt(h.rr);
    if (h.status == HF_ERR_NAN) return fail(HF_ERR_NAN, "NaN in BiCGStab");
    if (h.status) return fail(HF_ERR_NOT_CONVERGED, "BiCGStab did not converge");
    return HF_OK;
}
