// Shared-memory-staged, step-synchronous sweeps: the production triangular sweeps.
//
// Each CTA owns a set of rows (part_kernels.cuh explains the partition and why it is
// deadlock-free). Its slice of the plan is copied into shared memory once per sweep, laid out
// so that a thread finds its next row by arithmetic instead of a chain of dependent loads:
//
//   The CTA walks the schedule's group levels in the global order. A level whose groups hold
//   up to m rows is split into m steps; step j holds the j-th row of every group of the level,
//   so the rows of a group (a tree coarsened by the reference, merge/Coarsen.cpp:73-403) still
//   run in their order, separated by a CTA barrier. Inside a step, row k belongs to thread
//   k (k, k+blockDim, ... when a step is wider than the CTA), and its entries sit at a fixed
//   stride, so a row is found by arithmetic.
//
// Measured on B200 (ncu, C1): with the plan read from global memory a level cost ~2500 cycles,
// ~60 dependent instructions of ~40 cycles each.
//
// Slots (shared-memory solution cells) are the rows' positions in the lower sweep's order; the
// upper sweep carries an explicit slot per position, so a row's upper-sweep right-hand side
// (its lower-sweep result) is read from, and its result written to, the same slot.
//
// Per CTA and direction, int block: [E | step_row (S+1) | ne (nl) | rowid (nl) | slot (nl) |
// dep (nl*E)] and value block: [diag (nl) | val (nl*E)], both 16-byte padded. Every row of the
// CTA has the same entry stride E (its widest row), so row `pos`'s entries sit at pos*E + j and
// the hot path is fully unrolled. dep >= 0: local slot (final after the barrier); dep < 0:
// -(row+1) of a row owned by another CTA (value-as-flag wait on its global slot).
#pragma once

#include "device_common.cuh"
#include "part_kernels.cuh"

namespace baas {

constexpr int kStageBlock = 512;

struct StagedDir {
    const int *ioff, *voff;   // P + 1 element offsets of each CTA's int / value block
    const int *ns, *nl, *ne;  // P: steps, rows, padded entries of each CTA
    const int *ints;          // packed int blocks
    const int *vsrcT;         // laid out like the value blocks: position in the caller's CSR
    const int *vsrcA;         // same, position in A's value array (the IC0 factor)
};

struct StagedPlan {
    int P;
    StagedDir dir[2];
};

__host__ __device__ constexpr int pad4(int x) { return (x + 3) & ~3; }

// Shared-memory carve-up, identical on host and device.
struct StageLayout {
    int S, nl, ent;
    int nint;                              // ints of the block (padded)
    int off_x, off_ints, off_vals, total;  // byte offsets
    template <typename T>
    __host__ __device__ void make(int S_, int nl_, int ent_) {
        S = S_;
        nl = nl_;
        ent = ent_;
        nint = pad4(1 + (S + 1) + 3 * nl + ent);
        off_x = 0;
        off_ints = ((nl * (int)sizeof(T)) + 15) & ~15;
        off_vals = off_ints + nint * 4;
        total = off_vals + ((((nl + ent) * (int)sizeof(T)) + 15) & ~15);
    }
};

template <typename T>
struct StageView {
    T *xs;
    const int *step_row, *ne, *rowid, *slot, *dep;
    const T *diag, *val;
    int S, E;
};

template <typename T>
__device__ __forceinline__ StageView<T> stage_view(unsigned char *smem, const StageLayout &L) {
    StageView<T> v;
    v.xs = reinterpret_cast<T *>(smem + L.off_x);
    const int *I = reinterpret_cast<const int *>(smem + L.off_ints);
    v.E = I[0];
    v.step_row = I + 1;
    v.ne = v.step_row + (L.S + 1);
    v.rowid = v.ne + L.nl;
    v.slot = v.rowid + L.nl;
    v.dep = v.slot + L.nl;
    const T *V = reinterpret_cast<const T *>(smem + L.off_vals);
    v.diag = V;
    v.val = V + L.nl;
    v.S = L.S;
    return v;
}

template <typename T>
__device__ __forceinline__ StageLayout stage_layout(const StagedPlan &pl, int d, int c) {
    StageLayout L;
    const StagedDir &D = pl.dir[d];
    L.make<T>(__ldg(D.ns + c), __ldg(D.nl + c), __ldg(D.ne + c));
    return L;
}

// 16-byte copy of n4 int4 words by all threads of the CTA.
__device__ __forceinline__ void copy16(void *dst, const void *src, int n4) {
    int4 *d = reinterpret_cast<int4 *>(dst);
    const int4 *s = reinterpret_cast<const int4 *>(src);
    for (int i = threadIdx.x; i < n4; i += blockDim.x) d[i] = s[i];
}

__device__ __forceinline__ void stage_ints(const StagedPlan &pl, int d, int c, const StageLayout &L, unsigned char *smem) {
    const StagedDir &D = pl.dir[d];
    copy16(smem + L.off_ints, D.ints + __ldg(D.ioff + c), L.nint / 4);
}

// Value of dependency d (see the block layout): local slot or a wait on another CTA's row.
template <typename T>
__device__ __forceinline__ bool dep_value(const StageView<T> &v, int d, const T *xg, Waiter &w, T &xv) {
    if (d >= 0) {
        xv = v.xs[d];
        return true;
    }
    return wait_value<T>(xg + (-d - 1), xv, w, -d - 1);
}

// One row, entry stride E known at compile time (EK > 0) or read from the view (EK == 0).
// pf holds values of remote dependencies loaded one step earlier (sentinel: wait for it now).
template <typename T, bool EXACT, int EK>
__device__ __forceinline__ bool stage_row(const StageView<T> &v, int pos, int slot, const T *xg, Waiter &w, const T *pf,
                                          T &out) {
    const int E = EK > 0 ? EK : v.E;
    const int ne = v.ne[pos];
    const int *dp = v.dep + pos * E;
    const T *vp = v.val + pos * E;
    T sum = T(0);
    if constexpr (EK > 0) {
        int d[EK];
        T a[EK], xv[EK];
#pragma unroll
        for (int j = 0; j < EK; j++) {
            d[j] = dp[j];
            a[j] = vp[j];
        }
        bool ok = true;
#pragma unroll
        for (int j = 0; j < EK; j++)
            if (j < ne) {
                if (d[j] >= 0) {
                    xv[j] = v.xs[d[j]];
                } else {
                    xv[j] = pf ? pf[j] : Sent<T>::value();
                    if (Sent<T>::is(xv[j]) && !wait_value<T>(xg + (-d[j] - 1), xv[j], w, -d[j] - 1)) ok = false;
                }
            }
        if (!ok) return false;
#pragma unroll
        for (int j = 0; j < EK; j++)
            if (j < ne) {
                if constexpr (EXACT)
                    sum = __dadd_rn(sum, __dmul_rn(xv[j], a[j]));
                else
                    sum = fmaf(xv[j], a[j], sum);
            }
    } else {
        for (int j = 0; j < ne; j++) {
            T xv;
            const int d = dp[j];
            if (d >= 0)
                xv = v.xs[d];
            else if (!wait_value<T>(xg + (-d - 1), xv, w, -d - 1))
                return false;
            if constexpr (EXACT)
                sum = __dadd_rn(sum, __dmul_rn(xv, vp[j]));
            else
                sum = fmaf(xv, vp[j], sum);
        }
    }
    if constexpr (EXACT)
        out = __ddiv_rn(__dsub_rn(v.xs[slot], sum), v.diag[pos]);
    else
        out = (v.xs[slot] - sum) * v.diag[pos];  // FP32 mode stores 1/diag
    return true;
}

// Issue the loads of row pos's remote dependencies (their values, or the sentinel if not yet
// written); they complete while the CTA waits at the barrier.
template <typename T, int EK>
__device__ __forceinline__ void prefetch_remote(const StageView<T> &v, int pos, const T *xg, T *pf) {
#pragma unroll
    for (int j = 0; j < EK; j++) pf[j] = Sent<T>::value();
    if (pos < 0) return;
    const int ne = v.ne[pos];
    const int *dp = v.dep + pos * EK;
#pragma unroll
    for (int j = 0; j < EK; j++) {
        const int d = dp[j];
        if (j < ne && d < 0) pf[j] = Sent<T>::load(xg + (-d - 1));
    }
}

// Step-synchronous walk: at step s thread t runs rows step_row[s] + t, + blockDim, ... UPPER
// selects the explicit slot map. Writes x to its slot and to the global slot of its row
// (value-as-flag) and calls on_row(row, x). Before each barrier a thread issues the loads of
// its next row's remote dependencies, so their L2 latency overlaps the barrier. Every thread
// passes every barrier, also after a failed wait, so the CTA never splits.
template <typename T, bool EXACT, bool UPPER, int EK, typename OnRow>
__device__ __forceinline__ bool staged_walk_e(const StageView<T> &v, T *xg, Waiter &w, OnRow on_row) {
    constexpr int NP = EK > 0 ? EK : 1;
    bool alive = true;
    T pf[NP];
    int rb = v.step_row[0];
    if constexpr (EK > 0) prefetch_remote<T, EK>(v, rb + (int)threadIdx.x < v.step_row[1] ? rb + (int)threadIdx.x : -1, xg, pf);
    for (int s = 0; s < v.S; s++) {
        const int re = v.step_row[s + 1];
        for (int pos = rb + (int)threadIdx.x; pos < re && alive; pos += blockDim.x) {
            const int slot = UPPER ? v.slot[pos] : pos;
            T out;
            const T *use_pf = (EK > 0 && pos == rb + (int)threadIdx.x) ? pf : nullptr;
            if (!stage_row<T, EXACT, EK>(v, pos, slot, xg, w, use_pf, out)) {
                alive = false;
                break;
            }
            v.xs[slot] = out;
            const int row = v.rowid[pos];
            Sent<T>::store(xg + row, out);
            on_row(row, out);
        }
        if constexpr (EK > 0) {
            const int nb = re + (int)threadIdx.x;
            const int ne_ = s + 1 < v.S ? v.step_row[s + 2] : re;
            prefetch_remote<T, EK>(v, nb < ne_ ? nb : -1, xg, pf);
        }
        rb = re;
        __syncthreads();
    }
    return alive;
}

// Dispatch on the CTA's entry stride (the 5- and 7-point stencils' lower triangles have 2 and
// 3 off-diagonal entries per row).
template <typename T, bool EXACT, bool UPPER, typename OnRow>
__device__ __forceinline__ bool staged_walk(const StageView<T> &v, T *xg, Waiter &w, OnRow on_row) {
    switch (v.E) {
        case 0:
        case 1: return staged_walk_e<T, EXACT, UPPER, 1>(v, xg, w, on_row);
        case 2: return staged_walk_e<T, EXACT, UPPER, 2>(v, xg, w, on_row);
        case 3: return staged_walk_e<T, EXACT, UPPER, 3>(v, xg, w, on_row);
        case 4: return staged_walk_e<T, EXACT, UPPER, 4>(v, xg, w, on_row);
        default: return staged_walk_e<T, EXACT, UPPER, 0>(v, xg, w, on_row);
    }
}

// Standalone FP64 sweep of the caller's CSR T (values gathered through vsrcT), nrhs right-hand
// sides one after another.
template <bool UPPER>
__global__ void __launch_bounds__(kStageBlock, 1) k_sweep_staged(StagedPlan pl, const double *__restrict__ tval,
                                                                const double *__restrict__ b, int ldb, double *x, int ldx,
                                                                int nrhs, DevStatus *st, unsigned int spin_limit,
                                                                unsigned long long *trace) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int d = UPPER ? 1 : 0;
    const int c = blockIdx.x;
    Waiter w(spin_limit, st);
    trace_mark(trace, 0);
    const StageLayout L = stage_layout<double>(pl, d, c);
    stage_ints(pl, d, c, L, smem);
    {
        double *V = reinterpret_cast<double *>(smem + L.off_vals);
        const int *src = pl.dir[d].vsrcT + __ldg(pl.dir[d].voff + c);
        for (int i = threadIdx.x; i < L.nl + L.ent; i += blockDim.x) {
            const int si = __ldg(src + i);
            V[i] = si >= 0 ? __ldg(tval + si) : 0.0;
        }
    }
    __syncthreads();
    trace_mark(trace, 1);
    const StageView<double> v = stage_view<double>(smem, L);
    for (int r = 0; r < nrhs; r++) {
        const double *br = b + (size_t)r * ldb;
        double *xr = x + (size_t)r * ldx;
        for (int p = threadIdx.x; p < L.nl; p += blockDim.x) v.xs[UPPER ? v.slot[p] : p] = __ldg(br + v.rowid[p]);
        __syncthreads();
        trace_mark(trace, 2 + 2 * r);
        staged_walk<double, true, UPPER>(v, xr, w, [](int, double) {});
        trace_mark(trace, 3 + 2 * r);
        __shared__ int s_bad;
        if (threadIdx.x == 0) s_bad = ld_relaxed_u32(&st->code) != 0u;
        __syncthreads();
        if (s_bad) return;
    }
}

// ---------------------------------------------------------------------------------------
// Persistent ICCG with staged sweeps: IC0 (level-synchronous, part_kernels.cuh), packing of
// L and U = L^T into the staged value blocks, and the pcg_opt loop
// (test/iccg_level_merge.cpp:380-533, break at tol) in one cooperative launch of P CTAs.
// ---------------------------------------------------------------------------------------
struct StagedIccgArgs {
    int n;
    const int *a_rowptr, *a_colidx, *a_diag;
    const double *a_val;
    const double *b;
    double *x;
    PartView fac;     // level plan of the factorisation
    StagedPlan pl;    // staged sweep plan (dir 0: L, dir 1: U = L^T)
    int nv[2];        // lengths of the packed value arrays (per direction)
    double *gv64[2];  // packed FP64 value blocks (diag | val), per direction
    float *gv32[2];   // packed FP32 value blocks (1/diag | val), per direction
    double *lu;
    int *gflag;
    int epoch;
    double *r, *y, *z, *p, *Ap;
    float *y32, *z32;
    double *part_a, *part_b, *part_c;
    unsigned int *bar;
    DevStatus *st;
    int maxiter;
    double tol;
    int *out_iters;
    double *out_relres;
    unsigned int spin_limit;
    unsigned long long *trace;
};

// z = U^-1 L^-1 r on this CTA's rows; p = z if set_p; adds this thread's r.z to rz.
template <typename T>
__device__ void staged_precond(const StagedIccgArgs &A, unsigned char *smem, bool set_p, double &rz, Waiter &w) {
    const int c = blockIdx.x;
    T *yg = sizeof(T) == 8 ? (T *)A.y : (T *)A.y32;
    T *zg = sizeof(T) == 8 ? (T *)A.z : (T *)A.z32;
    {
        const StageLayout L = stage_layout<T>(A.pl, 0, c);
        __syncthreads();
        stage_ints(A.pl, 0, c, L, smem);
        const T *gv = sizeof(T) == 8 ? (const T *)A.gv64[0] : (const T *)A.gv32[0];
        copy16(smem + L.off_vals, gv + __ldg(A.pl.dir[0].voff + c), (((L.nl + L.ent) * (int)sizeof(T)) + 15) / 16);
        __syncthreads();
        const StageView<T> v = stage_view<T>(smem, L);
        for (int p = threadIdx.x; p < L.nl; p += blockDim.x) v.xs[p] = (T)A.r[v.rowid[p]];
        __syncthreads();
        trace_mark(A.trace, 56);
        staged_walk<T, sizeof(T) == 8, false>(v, yg, w, [](int, T) {});
        trace_mark(A.trace, 57);
    }
    {
        const StageLayout L = stage_layout<T>(A.pl, 1, c);
        __syncthreads();
        stage_ints(A.pl, 1, c, L, smem);
        const T *gv = sizeof(T) == 8 ? (const T *)A.gv64[1] : (const T *)A.gv32[1];
        copy16(smem + L.off_vals, gv + __ldg(A.pl.dir[1].voff + c), (((L.nl + L.ent) * (int)sizeof(T)) + 15) / 16);
        __syncthreads();
        const StageView<T> v = stage_view<T>(smem, L);
        // xs already holds y in every slot of this CTA
        trace_mark(A.trace, 58);
        staged_walk<T, sizeof(T) == 8, true>(v, zg, w, [&](int row, T out) {
            const double zd = (double)out;
            rz = __dadd_rn(rz, __dmul_rn(A.r[row], zd));
            if (set_p) A.p[row] = zd;
        });
        trace_mark(A.trace, 59);
    }
}

// T = double: FP64 factors; T = float: FP32 factors (one instantiation each keeps the register
// budget of each variant to one precision).
template <typename T>
__global__ void __launch_bounds__(kStageBlock, 1) k_iccg_staged(StagedIccgArgs A) {
    constexpr bool kMixed = sizeof(T) == 4;
    extern __shared__ __align__(16) unsigned char smem[];
    const int n = A.n;
    const int W = gridDim.x * blockDim.x;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned int nb = 0;
    Waiter w(A.spin_limit, A.st);
#define BAAS_BARRIER()                                            \
    do {                                                          \
        if (!grid_barrier(A.bar, nb, A.st, A.spin_limit)) return; \
    } while (0)

    trace_mark(A.trace, 0);
    const int nnz = __ldg(A.a_rowptr + n);
    for (int e = gt; e < nnz; e += W) A.lu[e] = A.a_val[e];
    BAAS_BARRIER();
    trace_mark(A.trace, 1);

    factor_part<false>(A.fac, A.a_rowptr, A.a_colidx, A.a_diag, A.lu, A.gflag, A.epoch, w, A.st);
    BAAS_BARRIER();
    trace_mark(A.trace, 2);

    // pack L and U = L^T into the staged value blocks (IC0_preconditioner split, :874-891);
    // r = b - A x; sentinels
    for (int d = 0; d < 2; d++) {
        const int *src = A.pl.dir[d].vsrcA;
        for (int i = gt; i < A.nv[d]; i += W) {
            const int si = __ldg(src + i);
            const double v = si >= 0 ? ld_l2(A.lu + si) : 0.0;
            A.gv64[d][i] = v;
            A.gv32[d][i] = __double2float_rn(v);
        }
    }
    double acc = 0.0;
    for (int i = gt; i < n; i += W) {
        double s = 0.0;
        for (int e = __ldg(A.a_rowptr + i); e < __ldg(A.a_rowptr + i + 1); e++)
            s = __dadd_rn(s, __dmul_rn(A.a_val[e], A.x[__ldg(A.a_colidx + e)]));
        const double ri = __dadd_rn(-s, A.b[i]);
        A.r[i] = ri;
        acc = __dadd_rn(acc, __dmul_rn(ri, ri));
        if constexpr (kMixed) {
            A.y32[i] = Sent<float>::value();
            A.z32[i] = Sent<float>::value();
        } else {
            A.y[i] = Sent<double>::value();
            A.z[i] = Sent<double>::value();
        }
    }
    put_partial<kStageBlock>(A.part_b, acc);
    BAAS_BARRIER();
    if constexpr (kMixed) {
        // FP32 value blocks hold the reciprocal diagonal (each CTA converts its own rows)
        for (int d = 0; d < 2; d++) {
            const int c = blockIdx.x;
            const int vo = __ldg(A.pl.dir[d].voff + c), nl = __ldg(A.pl.dir[d].nl + c);
            for (int p = threadIdx.x; p < nl; p += blockDim.x) A.gv32[d][vo + p] = __frcp_rn(__double2float_rn(A.gv64[d][vo + p]));
        }
        __threadfence_block();
    }
    const double norm0 = sqrt(grid_total<kStageBlock>(A.part_b, gridDim.x));
    trace_mark(A.trace, 3);

    double rzl = 0.0;
    staged_precond<T>(A, smem, true, rzl, w);
    trace_mark(A.trace, 4);
    put_partial<kStageBlock>(A.part_c, rzl);
    BAAS_BARRIER();
    double rz = grid_total<kStageBlock>(A.part_c, gridDim.x);
    trace_mark(A.trace, 5);

    int iters = 0;
    double rel = 1.0;
    for (int k = 1; k <= A.maxiter; ++k) {
        const double old_rz = rz;
        acc = 0.0;
        for (int i = gt; i < n; i += W) {
            double s = 0.0;
            for (int e = __ldg(A.a_rowptr + i); e < __ldg(A.a_rowptr + i + 1); e++)
                s = __dadd_rn(s, __dmul_rn(A.a_val[e], A.p[__ldg(A.a_colidx + e)]));
            A.Ap[i] = s;
            acc = __dadd_rn(acc, __dmul_rn(A.p[i], s));
            if constexpr (kMixed)
                A.y32[i] = Sent<float>::value();
            else
                A.y[i] = Sent<double>::value();
        }
        put_partial<kStageBlock>(A.part_a, acc);
        BAAS_BARRIER();
        const double alpha = old_rz / grid_total<kStageBlock>(A.part_a, gridDim.x);
        if (k <= 8) trace_mark(A.trace, 6 + 5 * (k - 1));

        acc = 0.0;
        for (int i = gt; i < n; i += W) {
            A.x[i] = __dadd_rn(A.x[i], __dmul_rn(alpha, A.p[i]));
            const double ri = __dadd_rn(A.r[i], __dmul_rn(-alpha, A.Ap[i]));
            A.r[i] = ri;
            acc = __dadd_rn(acc, __dmul_rn(ri, ri));
            if constexpr (kMixed)
                A.z32[i] = Sent<float>::value();
            else
                A.z[i] = Sent<double>::value();
        }
        put_partial<kStageBlock>(A.part_b, acc);
        BAAS_BARRIER();
        rel = sqrt(grid_total<kStageBlock>(A.part_b, gridDim.x)) / norm0;
        if (k <= 8) trace_mark(A.trace, 7 + 5 * (k - 1));
        iters = k;
        if (rel < A.tol) break;

        rzl = 0.0;
        staged_precond<T>(A, smem, false, rzl, w);
        if (k <= 8) trace_mark(A.trace, 8 + 5 * (k - 1));
        put_partial<kStageBlock>(A.part_c, rzl);
        BAAS_BARRIER();
        rz = grid_total<kStageBlock>(A.part_c, gridDim.x);
        const double beta = rz / old_rz;
        if (k <= 8) trace_mark(A.trace, 9 + 5 * (k - 1));

        for (int i = gt; i < n; i += W) {
            const double zi = kMixed ? (double)A.z32[i] : A.z[i];
            A.p[i] = __dadd_rn(zi, __dmul_rn(beta, A.p[i]));
        }
        BAAS_BARRIER();
        if (k <= 8) trace_mark(A.trace, 10 + 5 * (k - 1));
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *A.out_iters = iters;
        *A.out_relres = rel;
    }
#undef BAAS_BARRIER
}

}  // namespace baas
