// Single-CTA walks for systems whose vectors fit in one SM's shared memory (BAAS_WALK_SMALL).
//
// A shallow row DAG (the k-NN stiffness matrices: 12,000 rows in 23 row levels) spends almost all
// of a multi-CTA walk's time in grid barriers and in L2 round trips for the solution vector. Here
// one CTA of kSmallBlock threads owns the whole system: the sweep's solution lives in shared
// memory, a level ends at __syncthreads, and the matrix entries of the next level are loaded into
// registers while the current level computes, so their latency overlaps the level's work.
//
// Levels are row levels (a row waits only for the rows its entries name), rows ascending inside a
// level; every row is computed by one thread in the reference's order: forward sums ascending
// (merge/SpTRSV.cpp:24-39), backward sums descending (:642-652), IC0 column-match dot products in
// ascending column order (merge/IC.cpp:6-29, :32-89). Sweeps and factors are therefore bit-identical
// to the other walks'. ICCG's dot products are one block reduction in a fixed order.
#pragma once

#include "device_common.cuh"

namespace baas {

constexpr int kSmallBlock = 512;
constexpr int kSmallPF = 6;          // entries of a row carried across a level barrier
constexpr int kSmallLevShared = 2048;  // level offsets staged in shared memory up to this many levels

struct SmallDir {
    int nlev;
    const int *lev;   // nlev + 1 offsets into rec
    const int4 *rec;  // rows by level: {row, first entry, off-diagonal entries, diagonal position}
};

struct SmallArgs {
    int n;
    SmallDir dir[2];                        // 0: forward (L), 1: backward (U = L^T)
    const int *a_rowptr, *a_colidx, *a_diag;
    const double *a_val;
    const int *ic_ptr;                      // nnz + 1: IC0 column-match pairs of each lower entry
    const int2 *ic_pair;                    // (position in row i, position in row j), ascending column
    const int *ub_col, *ub_pos;             // U's off-diagonal entries (rows ascending, columns
                                            // ascending): column, and the lu position of L(col, row)
    int nub;
    double *lu;                             // the IC0 factor in A's layout
    double *ut;                             // U's off-diagonal values gathered from lu
    float *lf32, *ut32, *rcp32;             // FP32 factors: L (A's layout), U, reciprocal diagonal
    const double *b;
    double *x, *r, *Ap;
    DevStatus *st;
    int maxiter;
    double tol;
    int reuse;                              // the factor in lu is current: skip IC0
    int *out_iters;
    double *out_relres;
    const double *xf;                       // adjoint: the forward solution (grad_a = -lambda x^T)
    double *grad_a;
};

// One row of a level, its entries in registers (the first kSmallPF in summation order), its
// diagonal (FP32: the reciprocal) and, unless it lives in shared memory, its right-hand side.
template <typename V>
struct SmallRow {
    int i, e, cnt;
    V dv, rhs;
    int col[kSmallPF];
    V val[kSmallPF];
};

// Where a sweep reads a row's diagonal and right-hand side.
template <typename V>
struct SmallSrc {
    const int *col;
    const V *val;
    const V *diag;       // indexed by the diagonal position (by_row = 0) or by the row (1)
    int by_row;
    const double *rhs;   // global right-hand side, or nullptr: the row's own slot of xs
};

template <bool DESC>
__device__ __forceinline__ int small_pos(int e, int cnt, int q) {
    return DESC ? e + cnt - 1 - q : e + q;
}

template <typename V, bool DESC>
__device__ __forceinline__ void small_load(const int4 *rec, int q, const SmallSrc<V> &S, SmallRow<V> &r) {
    const int4 c = __ldg(rec + q);
    r.i = c.x;
    r.e = c.y;
    r.cnt = c.z;
    r.dv = S.diag[S.by_row ? c.x : c.w];
    if (S.rhs) r.rhs = (V)S.rhs[c.x];
#pragma unroll
    for (int k = 0; k < kSmallPF; k++)
        if (k < r.cnt) {
            const int p = small_pos<DESC>(r.e, r.cnt, k);
            r.col[k] = __ldg(S.col + p);
            r.val[k] = S.val[p];
        }
}

// Entries k0.. of a row (summation order), four at a time: the four entries' loads are issued
// together, then added in order.
template <typename V, bool DESC>
__device__ __forceinline__ void small_tail(int e, int cnt, int k0, const V *xs, const SmallSrc<V> &S, V &sum) {
    int k = k0;
    for (; k + 4 <= cnt; k += 4) {
        int c[4];
        V v[4];
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const int p = small_pos<DESC>(e, cnt, k + t);
            c[t] = __ldg(S.col + p);
            v[t] = S.val[p];
        }
#pragma unroll
        for (int t = 0; t < 4; t++) {
            if constexpr (sizeof(V) == 8)
                sum = __dadd_rn(sum, __dmul_rn(v[t], xs[c[t]]));
            else
                sum = fmaf(xs[c[t]], v[t], sum);
        }
    }
    for (; k < cnt; k++) {
        const int p = small_pos<DESC>(e, cnt, k);
        const V v = S.val[p];
        if constexpr (sizeof(V) == 8)
            sum = __dadd_rn(sum, __dmul_rn(v, xs[__ldg(S.col + p)]));
        else
            sum = fmaf(xs[__ldg(S.col + p)], v, sum);
    }
}

// (rhs - sum) / d in the reference's order; FP32: fused sum and the reciprocal diagonal.
template <typename V, bool DESC>
__device__ __forceinline__ V small_finish(const SmallRow<V> &r, const V *xs, const SmallSrc<V> &S) {
    V sum = (V)0;
    const int np = min(r.cnt, kSmallPF);
#pragma unroll
    for (int k = 0; k < kSmallPF; k++)
        if (k < np) {
            if constexpr (sizeof(V) == 8)
                sum = __dadd_rn(sum, __dmul_rn(r.val[k], xs[r.col[k]]));
            else
                sum = fmaf(xs[r.col[k]], r.val[k], sum);
        }
    small_tail<V, DESC>(r.e, r.cnt, kSmallPF, xs, S, sum);
    const V rhs = S.rhs ? r.rhs : xs[r.i];
    if constexpr (sizeof(V) == 8)
        return __ddiv_rn(__dsub_rn(rhs, sum), r.dv);
    else
        return (rhs - sum) * r.dv;
}

// A row of a level with more rows than threads: the same arithmetic, entries loaded as it goes.
template <typename V, bool DESC>
__device__ __forceinline__ void small_direct(const int4 *rec, int q, V *xs, const SmallSrc<V> &S) {
    const int4 c = __ldg(rec + q);
    const V dv = S.diag[S.by_row ? c.x : c.w];
    const V rhs = S.rhs ? (V)S.rhs[c.x] : xs[c.x];
    V sum = (V)0;
    small_tail<V, DESC>(c.y, c.z, 0, xs, S, sum);
    if constexpr (sizeof(V) == 8)
        xs[c.x] = __ddiv_rn(__dsub_rn(rhs, sum), dv);
    else
        xs[c.x] = (rhs - sum) * dv;
}

// One sweep over the levels of D into xs (shared memory). With S.rhs == nullptr the right-hand
// side is the row's own slot of xs (the backward sweep runs in place on the forward result). lev:
// the level offsets, staged in shared memory by the caller when they fit.
template <typename V, bool DESC>
__device__ __forceinline__ void small_sweep(const SmallDir &D, const int *lev, V *xs, const SmallSrc<V> &S) {
    const int tid = threadIdx.x;
    SmallRow<V> cur, nxt;
    cur.cnt = -1;
    if (D.nlev > 0 && lev[0] + tid < lev[1]) small_load<V, DESC>(D.rec, lev[0] + tid, S, cur);
    for (int l = 0; l < D.nlev; l++) {
        const int lb = lev[l], le = lev[l + 1];
        nxt.cnt = -1;
        if (l + 1 < D.nlev && le + tid < lev[l + 2]) small_load<V, DESC>(D.rec, le + tid, S, nxt);
        if (cur.cnt >= 0) xs[cur.i] = small_finish<V, DESC>(cur, xs, S);
        for (int q = lb + tid + kSmallBlock; q < le; q += kSmallBlock) small_direct<V, DESC>(D.rec, q, xs, S);
        __syncthreads();
        cur = nxt;
    }
}

// Fixed-order block sum: each thread's partial, then warps by shuffles, then warp 0 over the warps.
__device__ __forceinline__ double small_block_sum(double v, double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();  // red is reused by consecutive sums
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double t = 0.0;
    if (wid == 0) {
        t = lane < kSmallBlock / 32 ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t = __dadd_rn(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (lane == 0) red[32] = t;
    }
    __syncthreads();
    return red[32];
}

// IC0 of the rows of the forward levels, in place on lu (A's layout; lu already holds A's values).
// Row i's lower entry k (column j): lu[k] = (lu[k] - sum of the column-match products) / lu[diag j];
// then lu[diag i] = sqrt(a_ii - sum of squares) when positive, else counted and left unchanged.
// lu is read with plain loads: rows of earlier levels were written by other threads of this CTA
// before the level barrier.
__device__ __forceinline__ void small_ic0(const SmallArgs &A, const int *lev) {
    const SmallDir &D = A.dir[0];
    int bad = 0;
    for (int l = 0; l < D.nlev; l++) {
        for (int q = lev[l] + (int)threadIdx.x; q < lev[l + 1]; q += kSmallBlock) {
            const int4 c = __ldg(D.rec + q);  // {row, first entry, lower entries, diagonal}
            for (int k = c.y; k < c.y + c.z; k++) {
                const int j = __ldg(A.a_colidx + k);
                const int pb = __ldg(A.ic_ptr + k), pe = __ldg(A.ic_ptr + k + 1);
                double dp = 0.0;
                int p = pb;
                for (; p + 4 <= pe; p += 4) {  // four pairs' loads in flight
                    int2 pr[4];
                    double u[4], v[4];
#pragma unroll
                    for (int t = 0; t < 4; t++) pr[t] = __ldg(A.ic_pair + p + t);
#pragma unroll
                    for (int t = 0; t < 4; t++) {
                        u[t] = A.lu[pr[t].x];
                        v[t] = A.lu[pr[t].y];
                    }
#pragma unroll
                    for (int t = 0; t < 4; t++) dp = __dadd_rn(dp, __dmul_rn(u[t], v[t]));
                }
                for (; p < pe; p++) {
                    const int2 pr = __ldg(A.ic_pair + p);
                    dp = __dadd_rn(dp, __dmul_rn(A.lu[pr.x], A.lu[pr.y]));
                }
                A.lu[k] = __ddiv_rn(__dsub_rn(A.lu[k], dp), A.lu[__ldg(A.a_diag + j)]);
            }
            double dv = 0.0;
            for (int k = c.y; k < c.y + c.z; k++) {
                const double v = A.lu[k];
                dv = __dadd_rn(dv, __dmul_rn(v, v));
            }
            const double aii = A.lu[c.w];
            const double t = __dsub_rn(aii, dv);
            if (t > 0.0)
                A.lu[c.w] = __dsqrt_rn(t);
            else
                bad++;
        }
        __syncthreads();
    }
    if (bad) atomicAdd(&A.st->zero_pivots, bad);
}

// Level offsets of both directions in shared memory when they fit (else read from global).
__device__ __forceinline__ void small_stage_levels(const SmallArgs &A, int *sl, const int *(&lev)[2]) {
    int off = 0;
    for (int d = 0; d < 2; d++) {
        const int m = A.dir[d].nlev + 1;
        if (m <= kSmallLevShared) {
            for (int k = threadIdx.x; k < m; k += kSmallBlock) sl[off + k] = __ldg(A.dir[d].lev + k);
            lev[d] = sl + off;
            off += m;
        } else {
            lev[d] = A.dir[d].lev;
        }
    }
    __syncthreads();
}

// Standalone IC0 (baas_ic0 with BAAS_WALK_SMALL): lu holds A's values on entry.
__global__ void __launch_bounds__(kSmallBlock, 1) k_ic0_small(SmallArgs A) {
    __shared__ int sl[2 * kSmallLevShared];
    const int *lev[2];
    small_stage_levels(A, sl, lev);
    small_ic0(A, lev[0]);
}

// Standalone sweep of the caller's triangular CSR (baas_sptrsv, one right-hand side): UPPER = the
// transposed factor, diagonal first, summed descending. x = T^-1 b.
template <bool UPPER>
__global__ void __launch_bounds__(kSmallBlock, 1) k_sweep_small(SmallArgs A, const int *tcol, const double *tval) {
    extern __shared__ __align__(16) unsigned char smem_small[];
    __shared__ int sl[2 * kSmallLevShared];
    const int *lev[2];
    small_stage_levels(A, sl, lev);
    double *xs = reinterpret_cast<double *>(smem_small);
    const SmallSrc<double> S{tcol, tval, tval, 0, A.b};
    small_sweep<double, UPPER>(A.dir[UPPER ? 1 : 0], lev[UPPER ? 1 : 0], xs, S);
    for (int i = threadIdx.x; i < A.n; i += kSmallBlock) A.x[i] = xs[i];
}

// ICCG in one CTA: IC0 (unless reuse), then pcg_opt's loop (test/iccg_level_merge.cpp:458-503)
// with the vector updates of the reference's order. T = double: FP64 factors; float: FP32 factors
// (sweeps in FP32, the reciprocal diagonal, vectors and dot products in FP64).
template <typename T>
__global__ void __launch_bounds__(kSmallBlock, 1) k_iccg_small(SmallArgs A) {
    extern __shared__ __align__(16) unsigned char smem_small[];
    __shared__ int sl[2 * kSmallLevShared];
    __shared__ double red[33];
    const int n = A.n, tid = threadIdx.x;
    const int *lev[2];
    small_stage_levels(A, sl, lev);
    double *ps = reinterpret_cast<double *>(smem_small);   // p
    T *zs = reinterpret_cast<T *>(smem_small + 8 * (size_t)n);  // y, then z in place

    if (!A.reuse) {
        for (int e = tid; e < __ldg(A.a_rowptr + n); e += kSmallBlock) A.lu[e] = __ldg(A.a_val + e);
        __syncthreads();
        small_ic0(A, lev[0]);
    }
    // U's values from lu (IC0_preconditioner's split, test/iccg_level_merge.cpp:874-891); FP32
    // copies of L, U and the reciprocal diagonal
    for (int e = tid; e < A.nub; e += kSmallBlock) {
        const double v = A.lu[__ldg(A.ub_pos + e)];
        if constexpr (sizeof(T) == 8)
            A.ut[e] = v;
        else
            A.ut32[e] = __double2float_rn(v);
    }
    if constexpr (sizeof(T) == 4) {
        for (int i = tid; i < n; i += kSmallBlock) {
            A.rcp32[i] = __frcp_rn(__double2float_rn(A.lu[__ldg(A.a_diag + i)]));
            for (int e = __ldg(A.a_rowptr + i); e < __ldg(A.a_diag + i); e++) A.lf32[e] = __double2float_rn(A.lu[e]);
        }
    }
    __syncthreads();

    const T *lval = sizeof(T) == 8 ? (const T *)A.lu : (const T *)A.lf32;
    const T *uval = sizeof(T) == 8 ? (const T *)A.ut : (const T *)A.ut32;
    const T *dg = sizeof(T) == 8 ? (const T *)A.lu : (const T *)A.rcp32;
    const SmallSrc<T> SL{A.a_colidx, lval, dg, sizeof(T) == 4, A.r};
    const SmallSrc<T> SU{A.ub_col, uval, dg, sizeof(T) == 4, nullptr};
    // z = U^-1 L^-1 r, in place in zs; returns r.z
    auto precond = [&]() -> double {
        small_sweep<T, false>(A.dir[0], lev[0], zs, SL);
        small_sweep<T, true>(A.dir[1], lev[1], zs, SU);
        double acc = 0.0;
        for (int i = tid; i < n; i += kSmallBlock) acc = __dadd_rn(acc, __dmul_rn(A.r[i], (double)zs[i]));
        return small_block_sum(acc, red);
    };

    // r = b - A x
    double acc = 0.0;
    for (int i = tid; i < n; i += kSmallBlock) {
        double s = 0.0;
        for (int e = __ldg(A.a_rowptr + i); e < __ldg(A.a_rowptr + i + 1); e++)
            s = __dadd_rn(s, __dmul_rn(__ldg(A.a_val + e), A.x[__ldg(A.a_colidx + e)]));
        const double ri = __dadd_rn(-s, __ldg(A.b + i));
        A.r[i] = ri;
        acc = __dadd_rn(acc, __dmul_rn(ri, ri));
    }
    const double norm0 = sqrt(small_block_sum(acc, red));
    double rz = precond();
    for (int i = tid; i < n; i += kSmallBlock) ps[i] = (double)zs[i];
    __syncthreads();

    int iters = 0;
    double rel = 1.0;
    for (int k = 1; k <= A.maxiter; ++k) {
        const double old_rz = rz;
        acc = 0.0;
        for (int i = tid; i < n; i += kSmallBlock) {
            double s = 0.0;
            for (int e = __ldg(A.a_rowptr + i); e < __ldg(A.a_rowptr + i + 1); e++)
                s = __dadd_rn(s, __dmul_rn(__ldg(A.a_val + e), ps[__ldg(A.a_colidx + e)]));
            A.Ap[i] = s;
            acc = __dadd_rn(acc, __dmul_rn(ps[i], s));
        }
        const double alpha = old_rz / small_block_sum(acc, red);
        acc = 0.0;
        for (int i = tid; i < n; i += kSmallBlock) {
            A.x[i] = __dadd_rn(A.x[i], __dmul_rn(alpha, ps[i]));
            const double ri = __dadd_rn(A.r[i], __dmul_rn(-alpha, A.Ap[i]));
            A.r[i] = ri;
            acc = __dadd_rn(acc, __dmul_rn(ri, ri));
        }
        rel = sqrt(small_block_sum(acc, red)) / norm0;
        iters = k;
        if (rel < A.tol) break;
        rz = precond();
        const double beta = rz / old_rz;
        for (int i = tid; i < n; i += kSmallBlock) ps[i] = __dadd_rn((double)zs[i], __dmul_rn(beta, ps[i]));
        __syncthreads();
    }
    __syncthreads();
    if (A.grad_a) {
        // gradient on the pattern: dL/dA_ij = -lambda_i x_j (this launch solved for lambda)
        for (int i = tid; i < n; i += kSmallBlock) {
            const double li = -A.x[i];
            for (int e = __ldg(A.a_rowptr + i); e < __ldg(A.a_rowptr + i + 1); e++)
                A.grad_a[e] = __dmul_rn(li, __ldg(A.xf + __ldg(A.a_colidx + e)));
        }
    }
    if (tid == 0) {
        *A.out_iters = iters;
        *A.out_relres = rel;
    }
}

}  // namespace baas
