// The single-CTA walk (BAAS_WALK_SMALL): systems whose vectors fit in one SM's shared memory.
//
// A shallow row DAG (the k-NN stiffness matrices: 12,000 rows in 23 row levels) spends almost all
// of a grid-wide walk's time in grid barriers and in L2 round trips for the solution vector. Here
// one CTA, or one thread-block cluster of CS CTAs, owns the whole system: every CTA keeps the
// sweep's full solution in its shared memory, a row's result is stored into every copy (distributed
// shared memory), a level ends at the CTA or cluster barrier, and the matrix entries of the next
// level are loaded into registers while the current level computes. The cluster multiplies the
// loads in flight (one SM alone is bound by L2 latency) at the cost of a cluster barrier per level.
//
// Levels are row levels (a row waits only for the rows its entries name), rows ascending inside a
// level; every row is computed by one thread in the reference's order: forward sums ascending
// (merge/SpTRSV.cpp:24-39), backward sums descending (:642-652), IC0 column-match dot products in
// ascending column order (merge/IC.cpp:6-29, :32-89). Sweeps and factors are therefore bit-identical
// to the other walks'. ICCG's dot products are sums in a fixed order (threads, warps, CTAs).
#pragma once

#include <cooperative_groups.h>

#include "device_common.cuh"

namespace baas {

constexpr int kSmallBlock = 256;
constexpr int kSmallPF = 12;         // entries of a row carried across a level barrier
constexpr int kSmallLevShared = 2048;  // level offsets staged in shared memory up to this many levels

struct SmallDir {
    int nlev;
    const int *lev;   // nlev + 1 offsets into rec
    const int4 *rec;  // rows by level: {row, first entry, off-diagonal entries, diagonal position}
};

struct SmallArgs {
    int n;
    int nnz_a, nnz_t, npair;                // sizes for the bounds-checked build: A, the caller's T, IC0 pairs
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
    int n, nval, ndiag;  // rows, entries of col / val, entries of diag (bounds-checked build)
    DevStatus *st;
};

template <bool DESC>
__device__ __forceinline__ int small_pos(int e, int cnt, int q) {
    return DESC ? e + cnt - 1 - q : e + q;
}

template <typename V, bool DESC>
__device__ __forceinline__ void small_load(const int4 *rec, int q, const SmallSrc<V> &S, SmallRow<V> &r) {
    const int4 c = __ldg(rec + bounded(q, S.n, S.st, 101));
    r.i = bounded(c.x, S.n, S.st, 102);
    r.e = c.y;
    r.cnt = c.z;
    r.dv = S.diag[S.by_row ? r.i : bounded(c.w, S.ndiag, S.st, 103)];
    if (S.rhs) r.rhs = (V)S.rhs[r.i];
#pragma unroll
    for (int k = 0; k < kSmallPF; k++)
        if (k < r.cnt) {
            const int p = bounded(small_pos<DESC>(r.e, r.cnt, k), S.nval, S.st, 104);
            r.col[k] = bounded(__ldg(S.col + p), S.n, S.st, 105);
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
            const int p = bounded(small_pos<DESC>(e, cnt, k + t), S.nval, S.st, 106);
            c[t] = bounded(__ldg(S.col + p), S.n, S.st, 107);
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
        const int p = bounded(small_pos<DESC>(e, cnt, k), S.nval, S.st, 108);
        const V v = S.val[p];
        const int c = bounded(__ldg(S.col + p), S.n, S.st, 109);
        if constexpr (sizeof(V) == 8)
            sum = __dadd_rn(sum, __dmul_rn(v, xs[c]));
        else
            sum = fmaf(xs[c], v, sum);
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

// The CTAs that share the walk: one CTA (CS = 1), or a thread-block cluster of CS CTAs whose
// shared memories each hold a full copy of the sweep's solution. A row's result is stored into
// every copy (distributed shared memory), and a level ends at the cluster barrier, whose
// release/acquire order covers those stores and global memory alike.
template <int CS>
struct SmallGrp {
    static __device__ __forceinline__ int rank() {
        if constexpr (CS == 1)
            return 0;
        else
            return (int)cooperative_groups::this_cluster().block_rank();
    }
    static __device__ __forceinline__ void sync() {
        if constexpr (CS == 1)
            __syncthreads();
        else
            cooperative_groups::this_cluster().sync();
    }
    template <typename V>
    static __device__ __forceinline__ void put(V *xs, int i, V v) {
        if constexpr (CS == 1) {
            xs[i] = v;
        } else {
            cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
#pragma unroll
            for (int r = 0; r < CS; r++) cl.map_shared_rank(xs, (unsigned int)r)[i] = v;
        }
    }
};

// A row of a level with more rows than threads: the same arithmetic, entries loaded as it goes.
template <typename V, bool DESC, int CS>
__device__ __forceinline__ void small_direct(const int4 *rec, int q, V *xs, const SmallSrc<V> &S) {
    int4 c = __ldg(rec + bounded(q, S.n, S.st, 110));
    c.x = bounded(c.x, S.n, S.st, 111);
    const V dv = S.diag[S.by_row ? c.x : bounded(c.w, S.ndiag, S.st, 112)];
    const V rhs = S.rhs ? (V)S.rhs[c.x] : xs[c.x];
    V sum = (V)0;
    small_tail<V, DESC>(c.y, c.z, 0, xs, S, sum);
    V o;
    if constexpr (sizeof(V) == 8)
        o = __ddiv_rn(__dsub_rn(rhs, sum), dv);
    else
        o = (rhs - sum) * dv;
    SmallGrp<CS>::put(xs, c.x, o);
}

// One sweep over the levels of D into xs (shared memory). With S.rhs == nullptr the right-hand
// side is the row's own slot of xs (the backward sweep runs in place on the forward result). lev:
// the level offsets, staged in shared memory by the caller when they fit. A level's rows go to the
// cluster's threads with the CTA rank minor, so every SM of the cluster takes a share.
template <typename V, bool DESC, int CS>
__device__ __forceinline__ void small_sweep(const SmallDir &D, const int *lev, V *xs, const SmallSrc<V> &S) {
    const int gt = (int)threadIdx.x * CS + SmallGrp<CS>::rank();
    constexpr int G = CS * kSmallBlock;
    SmallRow<V> cur, nxt;
    cur.cnt = -1;
    if (D.nlev > 0 && lev[0] + gt < lev[1]) small_load<V, DESC>(D.rec, lev[0] + gt, S, cur);
    for (int l = 0; l < D.nlev; l++) {
        const int lb = lev[l], le = lev[l + 1];
        nxt.cnt = -1;
        if (l + 1 < D.nlev && le + gt < lev[l + 2]) small_load<V, DESC>(D.rec, le + gt, S, nxt);
        if (cur.cnt >= 0) SmallGrp<CS>::put(xs, cur.i, small_finish<V, DESC>(cur, xs, S));
        for (int q = lb + gt + G; q < le; q += G) small_direct<V, DESC, CS>(D.rec, q, xs, S);
        SmallGrp<CS>::sync();
        cur = nxt;
    }
}

// Fixed-order sum over the CTA (each thread's partial, warps by shuffles, warp 0 over the warps)
// and then over the cluster: every CTA stores its sum into every CTA's slot for it (two buffers,
// alternating, so a slot is rewritten only after every CTA has read it) and adds the slots in
// rank order, so all CTAs hold the same total.
template <int CS>
struct SmallSum {
    double red[33];
    double cred[2][CS];
    int parity;
};

template <int CS>
__device__ __forceinline__ double small_sum(double v, SmallSum<CS> &sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();  // red is reused by consecutive sums
    if (lane == 0) sh.red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        double t = lane < kSmallBlock / 32 ? sh.red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t = __dadd_rn(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (lane == 0) sh.red[32] = t;
    }
    if constexpr (CS == 1) {
        __syncthreads();
        return sh.red[32];
    } else {
        const int par = sh.parity;
        __syncthreads();
        if (threadIdx.x < CS) {
            cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
            cl.map_shared_rank(&sh.cred[par][0], threadIdx.x)[cl.block_rank()] = sh.red[32];
        }
        SmallGrp<CS>::sync();
        double t = 0.0;
#pragma unroll
        for (int r = 0; r < CS; r++) t = __dadd_rn(t, sh.cred[par][r]);
        __syncthreads();
        if (threadIdx.x == 0) sh.parity = par ^ 1;
        __syncthreads();
        return t;
    }
}

// IC0 scratch in shared memory, per thread (slot-major so that a warp's accesses fall in
// different banks): a row's lower values and pivots and the values of its column-match partners
// (doubles), and the pairs' positions in the row and each entry's first pair (bytes).
constexpr int kIcRow = 16;    // lower entries of a row that use the scratch
constexpr int kIcPairs = 48;  // column-match pairs of a row that use the scratch
constexpr int kIcDoubles = 2 * kIcRow + kIcPairs;
constexpr int kIcBytes = kIcPairs + kIcRow + 1;
constexpr size_t kIcScratch = (size_t)kSmallBlock * (8 * kIcDoubles + kIcBytes);

// IC0 of the rows of the forward levels, in place on lu (A's layout; lu already holds A's values).
// Row i's lower entry k (column j): lu[k] = (lu[k] - sum of the column-match products) / lu[diag j];
// then lu[diag i] = sqrt(a_ii - sum of squares) when positive, else counted and left unchanged.
// lu is read with plain loads: rows of earlier levels were written before the level barrier.
// With scratch (kIcScratch bytes of shared memory), a row within its limits first loads
// everything that does not depend on its own results -- its values, its pivots, its partners'
// values, all issued together -- and then runs the products from shared memory; other rows take
// the entry-by-entry path. Both perform the same operations in the same order.
template <int CS>
__device__ __forceinline__ void small_ic0(const SmallArgs &A, const int *lev, unsigned char *scratch) {
    const SmallDir &D = A.dir[0];
    const int gt = (int)threadIdx.x * CS + SmallGrp<CS>::rank();
    constexpr int G = CS * kSmallBlock;
    double *sd = reinterpret_cast<double *>(scratch) + threadIdx.x;
    unsigned char *sb = scratch + (size_t)8 * kIcDoubles * kSmallBlock + threadIdx.x;
#define IC_D(k) sd[(k) * kSmallBlock]
#define IC_B(k) sb[(k) * kSmallBlock]
    int bad = 0;
    for (int l = 0; l < D.nlev; l++) {
        for (int q = lev[l] + gt; q < lev[l + 1]; q += G) {
            int4 c = __ldg(D.rec + bounded(q, A.n, A.st, 120));  // {row, first entry, lower entries, diagonal}
            c.w = bounded(c.w, A.nnz_a, A.st, 121);
            const int rb = c.y, m = c.z;
            bounded(rb + m, A.nnz_a + 1, A.st, 122);
            const int pb0 = __ldg(A.ic_ptr + rb);
            const int np = __ldg(A.ic_ptr + rb + m) - pb0;
            bounded(pb0 + np, A.npair + 1, A.st, 123);
            if (scratch && m <= kIcRow && np <= kIcPairs) {
#pragma unroll 4
                for (int k = 0; k < m; k++) {
                    IC_D(k) = A.lu[rb + k];
                    IC_D(kIcRow + k) = A.lu[bounded(__ldg(A.a_diag + bounded(__ldg(A.a_colidx + rb + k), A.n, A.st, 126)),
                                                    A.nnz_a, A.st, 127)];
                }
#pragma unroll 4
                for (int k = 0; k <= m; k++) IC_B(kIcPairs + k) = (unsigned char)(__ldg(A.ic_ptr + rb + k) - pb0);
#pragma unroll 4
                for (int p = 0; p < np; p++) {
                    const int2 pr = __ldg(A.ic_pair + pb0 + p);
                    IC_B(p) = (unsigned char)bounded(pr.x - rb, m, A.st, 124);
                    IC_D(2 * kIcRow + p) = A.lu[bounded(pr.y, A.nnz_a, A.st, 125)];
                }
                for (int k = 0; k < m; k++) {
                    double dp = 0.0;
                    for (int p = IC_B(kIcPairs + k); p < IC_B(kIcPairs + k + 1); p++)
                        dp = __dadd_rn(dp, __dmul_rn(IC_D(IC_B(p)), IC_D(2 * kIcRow + p)));
                    const double v = __ddiv_rn(__dsub_rn(IC_D(k), dp), IC_D(kIcRow + k));
                    IC_D(k) = v;
                    A.lu[rb + k] = v;
                }
            } else {
                for (int k = rb; k < rb + m; k++) {
                    const int j = __ldg(A.a_colidx + k);
                    const int pb = __ldg(A.ic_ptr + k), pe = __ldg(A.ic_ptr + k + 1);
                    const double djj = A.lu[__ldg(A.a_diag + j)];
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
                    A.lu[k] = __ddiv_rn(__dsub_rn(A.lu[k], dp), djj);
                }
            }
            double dv = 0.0;
            for (int k = rb; k < rb + m; k++) {
                const double v = A.lu[k];
                dv = __dadd_rn(dv, __dmul_rn(v, v));
            }
            const double t = __dsub_rn(A.lu[c.w], dv);
            if (t > 0.0)
                A.lu[c.w] = __dsqrt_rn(t);
            else
                bad++;
        }
        SmallGrp<CS>::sync();
    }
#undef IC_D
#undef IC_B
    if (bad) atomicAdd(&A.st->zero_pivots, bad);
}

// Level offsets of both directions in shared memory when they fit (else read from global). Ends
// with the group barrier, which also guarantees every CTA of a cluster has started before any
// stores into its shared memory.
template <int CS>
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
    SmallGrp<CS>::sync();
}

// Standalone IC0 (baas_ic0 with BAAS_WALK_SMALL): lu holds A's values on entry.
template <int CS>
__global__ void __launch_bounds__(kSmallBlock, 1) k_ic0_small(SmallArgs A) {
    extern __shared__ __align__(16) unsigned char smem_small[];  // kIcScratch bytes
    __shared__ int sl[2 * kSmallLevShared];
    const int *lev[2];
    small_stage_levels<CS>(A, sl, lev);
    small_ic0<CS>(A, lev[0], smem_small);
    SmallGrp<CS>::sync();
}

// Standalone sweep of the caller's triangular CSR (baas_sptrsv, one right-hand side): UPPER = the
// transposed factor, diagonal first, summed descending. x = T^-1 b.
template <bool UPPER, int CS>
__global__ void __launch_bounds__(kSmallBlock, 1) k_sweep_small(SmallArgs A, const int *tcol, const double *tval) {
    extern __shared__ __align__(16) unsigned char smem_small[];
    __shared__ int sl[2 * kSmallLevShared];
    const int *lev[2];
    small_stage_levels<CS>(A, sl, lev);
    double *xs = reinterpret_cast<double *>(smem_small);
    const SmallSrc<double> S{tcol, tval, tval, 0, A.b, A.n, A.nnz_t, A.nnz_t, A.st};
    small_sweep<double, UPPER, CS>(A.dir[UPPER ? 1 : 0], lev[UPPER ? 1 : 0], xs, S);
    const int gt = (int)threadIdx.x * CS + SmallGrp<CS>::rank();
    for (int i = gt; i < A.n; i += CS * kSmallBlock) A.x[i] = xs[i];
    SmallGrp<CS>::sync();  // no CTA leaves while others may still store into its shared memory
}

// ICCG on one CTA or one cluster: IC0 (unless reuse), then pcg_opt's loop
// (test/iccg_level_merge.cpp:458-503) with the vector updates in the reference's order. T =
// double: FP64 factors; float: FP32 factors (sweeps in FP32 with the reciprocal diagonal; vectors
// and dot products in FP64). Rows of the vector phases are split across the cluster's threads;
// every CTA keeps full copies of z (from the sweeps' stores) and of p (each CTA updates all of p
// from its own copies, identically).
template <typename T, int CS>
__global__ void __launch_bounds__(kSmallBlock, 1) k_iccg_small(SmallArgs A) {
    extern __shared__ __align__(16) unsigned char smem_small[];
    __shared__ int sl[2 * kSmallLevShared];
    __shared__ SmallSum<CS> sh;
    const int n = A.n, tid = threadIdx.x;
    const int gt = tid * CS + SmallGrp<CS>::rank();
    constexpr int G = CS * kSmallBlock;
    if (tid == 0) sh.parity = 0;
    const int *lev[2];
    small_stage_levels<CS>(A, sl, lev);
    double *ps = reinterpret_cast<double *>(smem_small);       // p
    T *zs = reinterpret_cast<T *>(smem_small + 8 * (size_t)n);  // y, then z in place

    if (!A.reuse) {
        const int nnz = __ldg(A.a_rowptr + n);
        for (int e = gt; e < nnz; e += G) A.lu[e] = __ldg(A.a_val + e);
        SmallGrp<CS>::sync();
        small_ic0<CS>(A, lev[0], smem_small);  // p and z are not in use yet: their space is the scratch
    }
    // U's values from lu (IC0_preconditioner's split, test/iccg_level_merge.cpp:874-891); FP32
    // copies of L, U and the reciprocal diagonal
    for (int e = gt; e < A.nub; e += G) {
        const double v = A.lu[__ldg(A.ub_pos + e)];
        if constexpr (sizeof(T) == 8)
            A.ut[e] = v;
        else
            A.ut32[e] = __double2float_rn(v);
    }
    if constexpr (sizeof(T) == 4) {
        for (int i = gt; i < n; i += G) {
            A.rcp32[i] = __frcp_rn(__double2float_rn(A.lu[__ldg(A.a_diag + i)]));
            for (int e = __ldg(A.a_rowptr + i); e < __ldg(A.a_diag + i); e++) A.lf32[e] = __double2float_rn(A.lu[e]);
        }
    }
    SmallGrp<CS>::sync();

    const T *lval = sizeof(T) == 8 ? (const T *)A.lu : (const T *)A.lf32;
    const T *uval = sizeof(T) == 8 ? (const T *)A.ut : (const T *)A.ut32;
    const T *dg = sizeof(T) == 8 ? (const T *)A.lu : (const T *)A.rcp32;
    const int nd = sizeof(T) == 4 ? n : A.nnz_a;
    const SmallSrc<T> SL{A.a_colidx, lval, dg, sizeof(T) == 4, A.r, n, A.nnz_a, nd, A.st};
    const SmallSrc<T> SU{A.ub_col, uval, dg, sizeof(T) == 4, nullptr, n, A.nub, nd, A.st};
    // z = U^-1 L^-1 r, in place in zs (every CTA's copy); returns r.z
    auto precond = [&]() -> double {
        small_sweep<T, false, CS>(A.dir[0], lev[0], zs, SL);
        small_sweep<T, true, CS>(A.dir[1], lev[1], zs, SU);
        double acc = 0.0;
        for (int i = gt; i < n; i += G) acc = __dadd_rn(acc, __dmul_rn(A.r[i], (double)zs[i]));
        return small_sum<CS>(acc, sh);
    };

    // r = b - A x
    double acc = 0.0;
    for (int i = gt; i < n; i += G) {
        double s = 0.0;
        for (int e = __ldg(A.a_rowptr + i); e < __ldg(A.a_rowptr + i + 1); e++)
            s = __dadd_rn(s, __dmul_rn(__ldg(A.a_val + e), A.x[__ldg(A.a_colidx + e)]));
        const double ri = __dadd_rn(-s, __ldg(A.b + i));
        A.r[i] = ri;
        acc = __dadd_rn(acc, __dmul_rn(ri, ri));
    }
    const double norm0 = sqrt(small_sum<CS>(acc, sh));
    double rz = precond();
    for (int i = tid; i < n; i += kSmallBlock) ps[i] = (double)zs[i];
    __syncthreads();

    int iters = 0;
    double rel = 1.0;
    for (int k = 1; k <= A.maxiter; ++k) {
        const double old_rz = rz;
        acc = 0.0;
        for (int i = gt; i < n; i += G) {
            double s = 0.0;
            for (int e = __ldg(A.a_rowptr + i); e < __ldg(A.a_rowptr + i + 1); e++)
                s = __dadd_rn(s, __dmul_rn(__ldg(A.a_val + e), ps[__ldg(A.a_colidx + e)]));
            A.Ap[i] = s;
            acc = __dadd_rn(acc, __dmul_rn(ps[i], s));
        }
        const double alpha = old_rz / small_sum<CS>(acc, sh);
        acc = 0.0;
        for (int i = gt; i < n; i += G) {
            A.x[i] = __dadd_rn(A.x[i], __dmul_rn(alpha, ps[i]));
            const double ri = __dadd_rn(A.r[i], __dmul_rn(-alpha, A.Ap[i]));
            A.r[i] = ri;
            acc = __dadd_rn(acc, __dmul_rn(ri, ri));
        }
        rel = sqrt(small_sum<CS>(acc, sh)) / norm0;
        iters = k;
        if (rel < A.tol) break;
        rz = precond();
        const double beta = rz / old_rz;
        for (int i = tid; i < n; i += kSmallBlock) ps[i] = __dadd_rn((double)zs[i], __dmul_rn(beta, ps[i]));
        __syncthreads();
    }
    SmallGrp<CS>::sync();
    if (A.grad_a) {
        // gradient on the pattern: dL/dA_ij = -lambda_i x_j (this launch solved for lambda)
        for (int i = gt; i < n; i += G) {
            const double li = -A.x[i];
            for (int e = __ldg(A.a_rowptr + i); e < __ldg(A.a_rowptr + i + 1); e++)
                A.grad_a[e] = __dmul_rn(li, __ldg(A.xf + __ldg(A.a_colidx + e)));
        }
    }
    if (gt == 0) {
        *A.out_iters = iters;
        *A.out_relres = rel;
    }
    SmallGrp<CS>::sync();  // no CTA leaves while others may still store into its shared memory
}

}  // namespace baas
