// Batched, level-synchronous AMG-PCG for the Poisson projection.
//
// A program may hold many independent instances (a batch); each one keeps its
// own Krylov scalars and convergence test, so its result does not depend on the
// other instances it shares the launches with.  Every kernel covers all
// instances of one multigrid level at once: rows are concatenated instance by
// instance per level, and a table of blocks (Blk) maps each CTA to a row range
// of exactly one instance.  That gives
//   - full-device launches even when single instances are small, and
//   - per-instance reductions without atomics on data: each CTA writes its
//     partial sums, the last CTA of an instance to arrive adds the instance's
//     partials in block order (the same order on every run) and updates the
//     instance's scalars.
// Converged instances are skipped block by block.
//
// One CG iteration (hig-flow-step.c:48-131 solves the same system with PETSc's
// KSP; the operator here is the reduced, negated SPD form built on the host):
//   V-cycle  down: x = w D^-1 b, r = b - A x, b_next = R r     (per level)
//            coarsest: x = inv b per instance (dense)
//            up:   x += P e, out = x + w D^-1 (b - A x)         (per level)
//   z        finest post-smoothing writes z, r.z -> beta
//   dir      p = z + beta p_old, q = A p, p.q -> alpha
//   update   x += alpha p, r -= alpha q, r.r -> convergence
// Precision: the CG recurrences and the finest operator are always FP64; the
// mixed form runs the V-cycle (a preconditioner only needs a few digits) on
// FP32 copies of the hierarchy, halving its bytes.
//
// The iterations of a step run inside a CUDA graph as a conditional WHILE node;
// the last CTA of the second update kernel of each loop body sets the condition
// (any instance still active and the body cap not reached), so a whole time
// step is one graph launch with no host round trip.
#pragma once

#include <cstdint>

constexpr int kMaxLevels = 16;       // multigrid levels including the finest
constexpr int kMaxCoarse = 128;      // rows of the coarsest level (dense inverse)
constexpr int kCoarseCap = 1024;     // largest coarsest level accepted (stalled coarsening)
constexpr int kCoarseThreads = 128;

// rows [row0, row0 + cnt) of instance inst at one level; first/nblk: the
// instance's block range in the same table (for reductions)
struct Blk {
    int32_t row0, cnt, inst, first, nblk, pad0, pad1, pad2;
};

// Krylov state of one instance
struct IScal {
    double rz, alpha, beta, rr, bb, tol2;
    int32_t iters, status, done, clev;   // clev: the instance's coarsest level
    uint32_t counter, pad;
    int64_t total_iters;
};

// loop control and error record of the whole case
struct Ctl {
    int32_t active;       // instances not converged in the running step
    int32_t bodies;       // loop bodies run in the running step
    uint32_t gcount;      // blocks arrived at the last update kernel of a body
    int32_t maxbodies;
    int32_t err_status, err_inst;
    int64_t err_step;
    int64_t step;         // steps completed
    int64_t total_bodies;
};

// The finest operator as row templates: row i applies template rt[i], whose
// entries k in [tp[t], tp[t+1]) are (column offset toff[k], value tval[k]).
// On a uniform grid a handful of templates per instance cover every row, so a
// row costs one 4-byte index instead of its CSR columns and values.
template <typename T>
struct TRows {
    const int32_t *rt, *tp, *toff;
    const T *tval;
};

// sum over row i of val_k * f(i + off_k), in the row's entry order
template <typename T, typename Fn>
__device__ __forceinline__ T trow(const TRows<T> &A, int i, Fn f)
{
    const int t = __ldg(A.rt + i);
    const int e = __ldg(A.tp + t + 1);
    T s = T(0);
    for (int k = __ldg(A.tp + t); k < e; k++) s += __ldg(A.tval + k) * f(i + __ldg(A.toff + k));
    return s;
}

template <typename T>
struct VLev {
    int n;
    const int32_t *Ap, *Ac;   // CSR on the coarse levels; the finest level uses At
    const T *Av, *dinv;
    TRows<T> At;
    const int32_t *Pp, *Pc;   // rows: this level, columns: next level
    const T *Pv;
    const int32_t *Rp, *Rc;   // rows: next level, columns: this level
    const T *Rv;
    T *b, *x, *r, *out;       // b unused on the finest level (the CG residual is)
    const Blk *sblk, *ablk;   // smoothed instances' rows / all rows of the level
    int nsblk, nablk;
};

template <typename T>
struct CoarseInst {
    const T *b;               // level b (nullptr on the finest level)
    const double *b64;        // the CG residual when the coarsest level is the finest
    T *out;
    const T *inv;             // row-major cn x cn
    int32_t inst, cn;
};

struct PcgFine {
    int n;
    TRows<double> A;
    const double *dinv, *apin, *brhs;
    const int32_t *ipin;      // per instance: pinned global row or -1
    const hf_params *ipar;
    double *p, *dp;           // unknown: dp (incremental projection) or p
    double *r, *z, *q;
    double *partials;
    IScal *S;
    Ctl *ctl;
    const Blk *blk;
    int nblk, ninst;
    double rtol, atol;
    int maxit;
};

constexpr double kSmoothW = 2.0 / 3.0;

namespace pcg {

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
        v[k] = x;   // valid in thread 0
    }
    __syncthreads();
}

// Per-instance sums: true in every thread of the instance's last block, with
// tot[] the instance totals (partials added in block order).
template <int NV>
__device__ bool inst_sum(double (&v)[NV], const Blk &B, double *partials, IScal *S, double (&tot)[NV])
{
    __shared__ double sh[NV][kBlock / 32];
    __shared__ bool last;
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) partials[(size_t)blockIdx.x * NV + k] = v[k];
        __threadfence();
        const unsigned t = atomicAdd(&S[B.inst].counter, 1u);
        last = (t == (unsigned)B.nblk - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) acc[k] = 0.0;
    for (int b = threadIdx.x; b < B.nblk; b += kBlock) {
#pragma unroll
        for (int k = 0; k < NV; k++) acc[k] += ((volatile double *)partials)[(size_t)(B.first + b) * NV + k];
    }
    block_sum<NV>(acc, sh);
    __shared__ double bc[NV];
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) bc[k] = acc[k];
        S[B.inst].counter = 0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) tot[k] = bc[k];
    return true;
}

// block descriptor and the instance's done flag, shared by the block
__device__ __forceinline__ bool load_blk(const Blk *tab, const IScal *S, Blk &B)
{
    __shared__ Blk sb;
    __shared__ int sd;
    if (threadIdx.x == 0) {
        sb = tab[blockIdx.x];
        sd = ((volatile const IScal *)S)[sb.inst].done;
    }
    __syncthreads();
    B = sb;
    return sd != 0;
}

__device__ __forceinline__ void finish_instance(IScal &s, Ctl *ctl)
{
    s.done = 1;
    atomicSub(&ctl->active, 1);
}

}  // namespace pcg

// divergence right-hand side of every instance and the first residual
// (higflow_pressure, hig-flow-step.c:58-120, with the instance's own dt and pin)
template <int D>
__global__ void __launch_bounds__(kBlock) k_pcg_init(DevProg P, DevFields F, PcgFine G)
{
    Blk B;
    pcg::load_blk(G.blk, G.S, B);   // a new solve: the done flags are reset here
    const hf_params &par = G.ipar[B.inst];
    const bool incr = par.projtype == HF_INCREMENTAL;
    const double *x = incr ? G.dp : G.p;
    const int pin = G.ipin[B.inst];
    const double pinv = pin >= 0 ? (incr ? P.ipinv[B.inst] - F.p[pin] : P.ipinv[B.inst]) : 0.0;
    const int n = P.ncell;
    double part[2] = {0.0, 0.0};   // r.r, b.b
    if ((int)threadIdx.x < B.cnt) {
        const int cc = B.row0 + threadIdx.x;
        double borig;
        if (cc == pin) {
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
            borig = sumdudx / par.dt + G.brhs[cc];
        }
        const double bred = cc == pin ? pinv : -(borig - G.apin[cc] * pinv);
        const double ax = trow(G.A, cc, [&](int j) { return x[j]; });
        const double r = bred - ax;
        G.r[cc] = r;
        part[0] = r * r;
        part[1] = borig * borig;
    }
    double tot[2];
    if (pcg::inst_sum<2>(part, B, G.partials, G.S, tot) && threadIdx.x == 0) {
        IScal &s = G.S[B.inst];
        s.rr = tot[0];
        s.bb = tot[1];
        const double t = fmax(G.rtol * sqrt(tot[1]), G.atol);
        s.tol2 = t * t;
        s.beta = 0.0;
        s.iters = 0;
        s.status = 0;
        s.done = !(tot[0] > s.tol2);
        if (!isfinite(tot[0]) || !isfinite(tot[1])) { s.status = HF_ERR_NAN; s.done = 1; }
        if (!s.done) atomicAdd(&G.ctl->active, 1);
    }
}

// x = w D^-1 b ; r = b - A x on the smoothed rows of one level
template <typename T, bool FINE>
__global__ void __launch_bounds__(kBlock) k_vc_down(VLev<T> L, const double *__restrict__ r0, const IScal *S)
{
    Blk B;
    if (pcg::load_blk(L.sblk, S, B) || (int)threadIdx.x >= B.cnt) return;
    const int i = B.row0 + threadIdx.x;
    const T w = T(kSmoothW);
    const T bi = FINE ? T(r0[i]) : L.b[i];
    T s = T(0);
    if (FINE) {
        s = trow(L.At, i, [&](int j) { return w * __ldg(L.dinv + j) * T(__ldg(r0 + j)); });
    } else {
        for (int k = L.Ap[i]; k < L.Ap[i + 1]; k++) {
            const int j = L.Ac[k];
            s += L.Av[k] * (w * L.dinv[j] * L.b[j]);
        }
    }
    L.x[i] = w * L.dinv[i] * bi;
    L.r[i] = bi - s;
}

// b_next = R r on every row of the next level
template <typename T>
__global__ void __launch_bounds__(kBlock) k_vc_restrict(VLev<T> L, VLev<T> Ln, const IScal *S)
{
    Blk B;
    if (pcg::load_blk(Ln.ablk, S, B) || (int)threadIdx.x >= B.cnt) return;
    const int i = B.row0 + threadIdx.x;
    T s = T(0);
    for (int k = L.Rp[i]; k < L.Rp[i + 1]; k++) s += L.Rv[k] * L.r[L.Rc[k]];
    Ln.b[i] = s;
}

// out = inv b on each instance's coarsest level; one block per instance, one
// warp per row at a time: the lanes split the row (row-major, coalesced) and
// add their partial sums in a fixed shuffle order
template <typename T>
__global__ void __launch_bounds__(kCoarseThreads) k_vc_coarse(const CoarseInst<T> *ci, const IScal *S)
{
    __shared__ T sb[kCoarseCap];
    __shared__ CoarseInst<T> c;
    __shared__ int done;
    if (threadIdx.x == 0) {
        c = ci[blockIdx.x];
        done = ((volatile const IScal *)S)[c.inst].done;
    }
    __syncthreads();
    if (done) return;
    for (int i = threadIdx.x; i < c.cn; i += kCoarseThreads) sb[i] = c.b64 ? T(c.b64[i]) : c.b[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = warp; i < c.cn; i += kCoarseThreads / 32) {
        const T *row = c.inv + (size_t)i * c.cn;
        T s = T(0);
        for (int k = lane; k < c.cn; k += 32) s += row[k] * sb[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) c.out[i] = s;
    }
}

// x += P e on the smoothed rows (e: the next level's correction)
template <typename T>
__global__ void __launch_bounds__(kBlock) k_vc_prolong(VLev<T> L, const T *__restrict__ e, const IScal *S)
{
    Blk B;
    if (pcg::load_blk(L.sblk, S, B) || (int)threadIdx.x >= B.cnt) return;
    const int i = B.row0 + threadIdx.x;
    T s = T(0);
    for (int k = L.Pp[i]; k < L.Pp[i + 1]; k++) s += L.Pv[k] * e[L.Pc[k]];
    L.x[i] += s;
}

// out = x + w D^-1 (b - A x) on the smoothed rows of a coarse level
template <typename T>
__global__ void __launch_bounds__(kBlock) k_vc_post(VLev<T> L, const IScal *S)
{
    Blk B;
    if (pcg::load_blk(L.sblk, S, B) || (int)threadIdx.x >= B.cnt) return;
    const int i = B.row0 + threadIdx.x;
    T s = T(0);
    for (int k = L.Ap[i]; k < L.Ap[i + 1]; k++) s += L.Av[k] * L.x[L.Ac[k]];
    L.out[i] = L.x[i] + T(kSmoothW) * L.dinv[i] * (L.b[i] - s);
}

// z on the finest level (post-smoothing, the dense solve's output, or D^-1 r),
// then r.z -> beta per instance
template <typename T, bool JACOBI>
__global__ void __launch_bounds__(kBlock) k_pcg_z(PcgFine G, VLev<T> L0)
{
    Blk B;
    if (pcg::load_blk(G.blk, G.S, B)) return;
    double part[1] = {0.0};
    if ((int)threadIdx.x < B.cnt) {
        const int i = B.row0 + threadIdx.x;
        const double ri = G.r[i];
        double z;
        if (JACOBI) {
            z = G.dinv[i] * ri;
        } else if (G.S[B.inst].clev == 0) {
            z = double(L0.out[i]);
        } else {
            const T s = trow(L0.At, i, [&](int j) { return L0.x[j]; });
            z = double(L0.x[i] + T(kSmoothW) * L0.dinv[i] * (T(ri) - s));
        }
        G.z[i] = z;
        part[0] = ri * z;
    }
    double tot[1];
    if (pcg::inst_sum<1>(part, B, G.partials, G.S, tot) && threadIdx.x == 0) {
        IScal &s = G.S[B.inst];
        s.beta = s.iters == 0 ? 0.0 : tot[0] / s.rz;
        s.rz = tot[0];
        if (!isfinite(tot[0])) { s.status = HF_ERR_NAN; pcg::finish_instance(s, G.ctl); }
    }
}

// p_new = z + beta p_old ; q = A p_new ; alpha = r.z / p.q
__global__ void __launch_bounds__(kBlock) k_pcg_dir(PcgFine G, const double *__restrict__ po, double *__restrict__ pn)
{
    Blk B;
    if (pcg::load_blk(G.blk, G.S, B)) return;
    const IScal &sc = G.S[B.inst];
    const bool first = sc.iters == 0;
    const double beta = sc.beta;
    double part[1] = {0.0};
    if ((int)threadIdx.x < B.cnt) {
        const int i = B.row0 + threadIdx.x;
        double q, p;
        if (first) {
            q = trow(G.A, i, [&](int j) { return G.z[j]; });
            p = G.z[i];
        } else {
            q = trow(G.A, i, [&](int j) { return G.z[j] + beta * po[j]; });
            p = G.z[i] + beta * po[i];
        }
        pn[i] = p;
        G.q[i] = q;
        part[0] = p * q;
    }
    double tot[1];
    if (pcg::inst_sum<1>(part, B, G.partials, G.S, tot) && threadIdx.x == 0) {
        IScal &s = G.S[B.inst];
        if (!(tot[0] > 0.0) || !isfinite(tot[0])) {
            // p.q <= 0: the recurrence has reached rounding level.  Accept when
            // the residual is within 100x of the target, else report it.
            s.status = !isfinite(tot[0]) ? HF_ERR_NAN : (s.rr <= 1e4 * s.tol2 ? 0 : HF_ERR_NOT_CONVERGED);
            pcg::finish_instance(s, G.ctl);
        } else {
            s.alpha = s.rz / tot[0];
        }
    }
}

// x += alpha p ; r -= alpha q ; convergence on ||r||.  set_cond != 0: the last
// block of the grid counts the loop body and (set_cond == 1, inside the step
// graph) sets the loop condition for the next body; with eager launches the
// host reads the count and the active instances instead.
__global__ void __launch_bounds__(kBlock) k_pcg_update(PcgFine G, const double *__restrict__ pn,
                                                       cudaGraphConditionalHandle cond, int set_cond)
{
    Blk B;
    const bool skip = pcg::load_blk(G.blk, G.S, B);
    if (!skip) {
        const bool incr = G.ipar[B.inst].projtype == HF_INCREMENTAL;
        double *x = incr ? G.dp : G.p;
        const double alpha = G.S[B.inst].alpha;
        double part[1] = {0.0};
        if ((int)threadIdx.x < B.cnt) {
            const int i = B.row0 + threadIdx.x;
            x[i] += alpha * pn[i];
            const double r = G.r[i] - alpha * G.q[i];
            G.r[i] = r;
            part[0] = r * r;
        }
        double tot[1];
        if (pcg::inst_sum<1>(part, B, G.partials, G.S, tot) && threadIdx.x == 0) {
            IScal &s = G.S[B.inst];
            s.rr = tot[0];
            s.iters += 1;
            if (!isfinite(tot[0])) { s.status = HF_ERR_NAN; pcg::finish_instance(s, G.ctl); }
            else if (!(tot[0] > s.tol2)) pcg::finish_instance(s, G.ctl);
            else if (s.iters >= G.maxit) { s.status = HF_ERR_NOT_CONVERGED; pcg::finish_instance(s, G.ctl); }
        }
    }
    if (!set_cond) return;
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned t = atomicAdd(&G.ctl->gcount, 1u);
        if (t == gridDim.x - 1) {
            __threadfence();
            Ctl &c = *G.ctl;
            c.gcount = 0;
            c.bodies += 1;
            const int active = ((volatile Ctl *)G.ctl)->active;
            if (set_cond == 1) cudaGraphSetConditional(cond, (active > 0 && c.bodies < c.maxbodies) ? 1u : 0u);
        }
    }
}

// end of a step: per-instance totals, the first failure, loop counters reset
__global__ void __launch_bounds__(kBlock) k_step_end(PcgFine G)
{
    Ctl *c = G.ctl;
    for (int i = threadIdx.x; i < G.ninst; i += kBlock) {
        IScal &s = G.S[i];
        if (!s.done) {   // stopped by the body cap: count as not converged
            s.status = HF_ERR_NOT_CONVERGED;
            s.done = 1;
        }
        s.total_iters += s.iters;
        if (s.status && atomicCAS(&c->err_status, 0, s.status) == 0) {
            c->err_inst = i;
            c->err_step = c->step;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        c->total_bodies += c->bodies;
        c->step += 1;
        c->active = 0;
        c->bodies = 0;
    }
}
