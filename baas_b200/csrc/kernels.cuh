// Sparse kernels of the BAAS hot path on sm_100a.
//
// Execution model (all kernels here): a persistent, co-resident grid (cooperative launch).
// The schedule's coarsened groups, listed level by level (the BAAS LevelSet order), are the
// work items; item q goes to worker q mod W (worker = one thread), and a worker processes a
// group's rows in ascending order, exactly as one reference thread processes a group
// (merge/SpTRSV.cpp:458-471). Dependencies are point-to-point:
//   - sweeps: the solution slot itself is the ready flag (a signalling-NaN sentinel until
//     written), so one relaxed L2 load both waits for and fetches a dependency;
//   - factorisations: an epoch-stamped per-row flag published with st.release after the
//     row's values, read with ld.acquire before the parent row's values.
// Items are assigned in a topological order and every worker walks its items in that order,
// so the smallest unfinished item always has all its inputs: no deadlock while all workers
// are resident, which the cooperative launch guarantees. Every wait is bounded (Waiter).
//
// FP64 arithmetic uses the _rn intrinsics in the reference's operation order (no FMA
// contraction, sequential sums), so factors and sweeps are bit-identical to the reference's
// serial and p2p routines (merge/SpTRSV.cpp:24-39, :601-660, merge/IC.cpp:6-89, :296-393,
// merge/ILU.cpp:350-386).
#pragma once

#include "device_common.cuh"

namespace baas {

constexpr int kBlock = 256;

// ---------------------------------------------------------------------------------------
// Forward / backward row of a sweep over a caller CSR (values read in place).
//   forward : x_i = (b_i - sum_{j<i} T_ij x_j) / T_ii, diagonal last, sum ascending
//             (merge/SpTRSV.cpp:464-470)
//   backward: x_i = (b_i - sum_{j>i} T_ij x_j) / T_ii, diagonal first, sum DESCENDING
//             (merge/SpTRSV.cpp:642-652, the p2p routine Scheduler uses)
// ---------------------------------------------------------------------------------------
template <bool UPPER>
__device__ __forceinline__ bool sweep_row_csr(int row, const int *__restrict__ rowptr, const int *__restrict__ colidx,
                                              const double *__restrict__ val, const double *__restrict__ b, int ldb,
                                              double *x, int ldx, int nrhs, Waiter &w) {
    const int beg = __ldg(rowptr + row), end = __ldg(rowptr + row + 1);
    const double d = __ldg(val + (UPPER ? beg : end - 1));
    const int ob = UPPER ? beg + 1 : beg, oe = UPPER ? end : end - 1;
    for (int r = 0; r < nrhs; r++) {
        const double *xr = x + (size_t)r * ldx;
        double sum = 0.0;
        int done = 0;
        const int cnt = oe - ob;
        while (done < cnt) {
            const int m = min(4, cnt - done);
            int c[4];
            double a[4], v[4];
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (k < m) {
                    const int e = UPPER ? (oe - 1 - done - k) : (ob + done + k);
                    c[k] = __ldg(colidx + e);
                    a[k] = __ldg(val + e);
                }
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (k < m) v[k] = Sent<double>::load(xr + c[k]);
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (k < m) {
                    while (Sent<double>::is(v[k])) {
                        if (!w.tick(row)) return false;
                        v[k] = Sent<double>::load(xr + c[k]);
                    }
                    sum = __dadd_rn(sum, __dmul_rn(v[k], a[k]));
                }
            done += m;
        }
        const double xv = __ddiv_rn(__dsub_rn(__ldg(b + (size_t)r * ldb + row), sum), d);
        Sent<double>::store(x + (size_t)r * ldx + row, xv);
    }
    return true;
}

template <bool UPPER>
__global__ void __launch_bounds__(kBlock) k_sweep_csr(int nitems, const int *__restrict__ item_ptr, const int *__restrict__ ord,
                                                      const int *__restrict__ rowptr, const int *__restrict__ colidx,
                                                      const double *__restrict__ val, const double *__restrict__ b, int ldb,
                                                      double *x, int ldx, int nrhs, DevStatus *st, unsigned int spin_limit) {
    Waiter w(spin_limit, st);
    const int W = gridDim.x * blockDim.x;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nitems; q += W) {
        const int pb = __ldg(item_ptr + q), pe = __ldg(item_ptr + q + 1);
        for (int p = pb; p < pe; p++)
            if (!sweep_row_csr<UPPER>(__ldg(ord + p), rowptr, colidx, val, b, ldb, x, ldx, nrhs, w)) return;
    }
}

template <typename T>
__global__ void k_fill_sentinel(T *x, int n, int nrhs, int ldx) {
    const long long total = (long long)n * nrhs;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / n, row = i - r * n;
        x[r * ldx + row] = Sent<T>::value();
    }
}

// ---------------------------------------------------------------------------------------
// IC0, up-looking, one row: merge/IC.cpp:296-393 with sparse_dot_product :6-29.
// lu holds A's values on entry (full pattern); only the lower part is updated.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ bool ic0_row(int i, const int *__restrict__ rowptr, const int *__restrict__ colidx,
                                        const int *__restrict__ diagptr, double *lu, int *flags, int epoch, Waiter &w,
                                        DevStatus *st) {
    const int rb = __ldg(rowptr + i), di = __ldg(diagptr + i);
    for (int k = rb; k < di; k++) {
        const int j = __ldg(colidx + k);
        if (!wait_flag(flags + j, epoch, w, i)) return false;
        double dp = 0.0;
        int l1 = rb, l2 = __ldg(rowptr + j);
        const int u1 = di, u2 = __ldg(diagptr + j);
        while (l1 < u1 && l2 < u2) {
            const int c1 = __ldg(colidx + l1), c2 = __ldg(colidx + l2);
            if (c1 == c2) {
                const double pj = Sent<double>::load(lu + l2);
                dp = __dadd_rn(dp, __dmul_rn(lu[l1], pj));
                l1++;
                l2++;
            } else if (c1 < c2) {
                l1++;
            } else {
                l2++;
            }
        }
        const double ljj = Sent<double>::load(lu + u2);
        lu[k] = __ddiv_rn(__dsub_rn(lu[k], dp), ljj);
    }
    double dv = 0.0;
    for (int k = rb; k < di; k++) dv = __dadd_rn(dv, __dmul_rn(lu[k], lu[k]));
    const double t = __dsub_rn(lu[di], dv);
    if (t > 0.0)
        lu[di] = __dsqrt_rn(t);
    else
        atomicAdd(&st->zero_pivots, 1);
    st_release_s32(flags + i, epoch);
    return true;
}

// ILU0, up-looking, one row: merge/ILU.cpp:638-720 (= ilu0csr_uplooking_ref :350-386).
__device__ __forceinline__ bool ilu0_row(int i, const int *__restrict__ rowptr, const int *__restrict__ colidx,
                                         const int *__restrict__ diagptr, double *lu, int *flags, int epoch, Waiter &w,
                                         DevStatus *st) {
    const int rb = __ldg(rowptr + i), di = __ldg(diagptr + i), re = __ldg(rowptr + i + 1);
    for (int j = rb; j < di; j++) {
        const int c = __ldg(colidx + j);
        if (!wait_flag(flags + c, epoch, w, i)) return false;
        const int dc = __ldg(diagptr + c), ec = __ldg(rowptr + c + 1);
        const double pivot = Sent<double>::load(lu + dc);
        if (pivot == 0.0) atomicAdd(&st->zero_pivots, 1);
        const double tmp = __ddiv_rn(lu[j], pivot);
        lu[j] = tmp;
        int k1 = j + 1, k2 = dc + 1;
        while (k1 < re && k2 < ec) {
            const int c1 = __ldg(colidx + k1), c2 = __ldg(colidx + k2);
            if (c1 < c2) {
                k1++;
            } else if (c1 > c2) {
                k2++;
            } else {
                lu[k1] = __dsub_rn(lu[k1], __dmul_rn(tmp, Sent<double>::load(lu + k2)));
                k1++;
                k2++;
            }
        }
    }
    st_release_s32(flags + i, epoch);
    return true;
}

template <bool ILU>
__global__ void __launch_bounds__(kBlock) k_factor(int nitems, const int *__restrict__ item_ptr, const int *__restrict__ ord,
                                                   const int *__restrict__ rowptr, const int *__restrict__ colidx,
                                                   const int *__restrict__ diagptr, double *lu, int *flags, int epoch,
                                                   DevStatus *st, unsigned int spin_limit) {
    Waiter w(spin_limit, st);
    const int W = gridDim.x * blockDim.x;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nitems; q += W) {
        const int pb = __ldg(item_ptr + q), pe = __ldg(item_ptr + q + 1);
        for (int p = pb; p < pe; p++) {
            const int row = __ldg(ord + p);
            const bool ok = ILU ? ilu0_row(row, rowptr, colidx, diagptr, lu, flags, epoch, w, st)
                                : ic0_row(row, rowptr, colidx, diagptr, lu, flags, epoch, w, st);
            if (!ok) return;
        }
    }
}

// ---------------------------------------------------------------------------------------
// Persistent ICCG: IC0, factor packing, and the whole PCG loop of pcg_opt
// (test/iccg_level_merge.cpp:380-533, break at tol) in one cooperative launch.
// ---------------------------------------------------------------------------------------
struct IccgArgs {
    int n;
    const int *a_rowptr, *a_colidx, *a_diag;
    const double *a_val;
    const double *b;
    double *x;
    // work items in forward / backward order
    int nitems;
    const int *f_item_ptr, *f_ord, *b_item_ptr, *b_ord;
    // packed factors in processing order: forward L (off-diagonals ascending), backward
    // U = L^T (off-diagonals descending); *_src are positions in A's value array
    const int *fp_ptr, *fp_col, *fp_src, *fp_dsrc;
    const int *bp_ptr, *bp_col, *bp_src, *bp_dsrc;
    double *fp_val, *fp_diag, *bp_val, *bp_diag;
    float *fp_val32, *fp_diag32, *bp_val32, *bp_diag32;
    int nnzf, nnzb;
    double *lu;
    int *flags;
    int epoch;
    double *r, *y, *z, *p, *Ap;
    float *y32, *z32;
    double *part_a, *part_b, *part_c;  // per-CTA partial sums
    unsigned int *bar;
    DevStatus *st;
    int maxiter;
    double tol;
    int mixed;
    int *out_iters;
    double *out_relres;
    unsigned int spin_limit;
};

template <typename T>
__device__ __forceinline__ T to_t(double v);
template <>
__device__ __forceinline__ double to_t<double>(double v) { return v; }
template <>
__device__ __forceinline__ float to_t<float>(double v) { return __double2float_rn(v); }

// One packed sweep row. FP64: reference order and rounding. FP32: fused multiply-add.
template <typename T, bool UPPER>
__device__ __forceinline__ bool packed_row(int p, int row, const int *__restrict__ ptr, const int *__restrict__ col,
                                           const T *__restrict__ val, const T *__restrict__ diag, T bval, T *out,
                                           Waiter &w, T &res) {
    const int eb = __ldg(ptr + p), ee = __ldg(ptr + p + 1);
    T sum = T(0);
    int e = eb;
    while (e < ee) {
        const int m = min(4, ee - e);
        int c[4];
        T a[4], v[4];
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (k < m) {
                c[k] = __ldg(col + e + k);
                a[k] = val[e + k];
            }
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (k < m) v[k] = Sent<T>::load(out + c[k]);
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (k < m) {
                while (Sent<T>::is(v[k])) {
                    if (!w.tick(row)) return false;
                    v[k] = Sent<T>::load(out + c[k]);
                }
                if constexpr (sizeof(T) == 8)
                    sum = __dadd_rn(sum, __dmul_rn(v[k], a[k]));
                else
                    sum = fmaf(v[k], a[k], sum);
            }
        e += m;
    }
    T xv;
    if constexpr (sizeof(T) == 8)
        xv = __ddiv_rn(__dsub_rn(bval, sum), diag[p]);
    else
        xv = __fdiv_rn(bval - sum, diag[p]);
    Sent<T>::store(out + row, xv);
    res = xv;
    return true;
}

// z = U^-1 L^-1 r on packed factors; also p = z (if set_p) and the r.z partial.
template <typename T>
__device__ bool precond_apply(const IccgArgs &A, T *y, T *z, bool set_p, double &rz_local, Waiter &w) {
    const int W = gridDim.x * blockDim.x;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const T *fval = sizeof(T) == 8 ? (const T *)A.fp_val : (const T *)A.fp_val32;
    const T *fdiag = sizeof(T) == 8 ? (const T *)A.fp_diag : (const T *)A.fp_diag32;
    const T *bval = sizeof(T) == 8 ? (const T *)A.bp_val : (const T *)A.bp_val32;
    const T *bdiag = sizeof(T) == 8 ? (const T *)A.bp_diag : (const T *)A.bp_diag32;
    for (int q = gt; q < A.nitems; q += W) {
        const int pb = __ldg(A.f_item_ptr + q), pe = __ldg(A.f_item_ptr + q + 1);
        for (int p = pb; p < pe; p++) {
            const int row = __ldg(A.f_ord + p);
            T res;
            if (!packed_row<T, false>(p, row, A.fp_ptr, A.fp_col, fval, fdiag, to_t<T>(A.r[row]), y, w, res)) return false;
        }
    }
    for (int q = gt; q < A.nitems; q += W) {
        const int pb = __ldg(A.b_item_ptr + q), pe = __ldg(A.b_item_ptr + q + 1);
        for (int p = pb; p < pe; p++) {
            const int row = __ldg(A.b_ord + p);
            T yv;
            if (!wait_value<T>(y + row, yv, w, row)) return false;
            T res;
            if (!packed_row<T, true>(p, row, A.bp_ptr, A.bp_col, bval, bdiag, yv, z, w, res)) return false;
            const double zd = (double)res;
            rz_local = __dadd_rn(rz_local, __dmul_rn(A.r[row], zd));
            if (set_p) A.p[row] = zd;
        }
    }
    return true;
}

__global__ void __launch_bounds__(kBlock) k_iccg(IccgArgs A) {
    const int n = A.n;
    const int W = gridDim.x * blockDim.x;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned int nb = 0;  // barriers passed
    Waiter w(A.spin_limit, A.st);
    bool alive = true;
#define BAAS_BARRIER()                                                    \
    do {                                                                  \
        if (!grid_barrier(A.bar, nb, A.st, A.spin_limit)) return;         \
    } while (0)

    // lu = A.values
    const int nnz = __ldg(A.a_rowptr + n);
    for (int e = gt; e < nnz; e += W) A.lu[e] = A.a_val[e];
    BAAS_BARRIER();

    // IC0 over the schedule's items (Scheduler::runIC0, test/Schedule.hpp:316-322)
    for (int q = gt; q < A.nitems && alive; q += W) {
        const int pb = __ldg(A.f_item_ptr + q), pe = __ldg(A.f_item_ptr + q + 1);
        for (int p = pb; p < pe; p++)
            if (!ic0_row(__ldg(A.f_ord + p), A.a_rowptr, A.a_colidx, A.a_diag, A.lu, A.flags, A.epoch, w, A.st)) {
                alive = false;
                break;
            }
    }
    // a failed thread still joins the barrier; the barrier then sees the status and every CTA
    // returns
    BAAS_BARRIER();

    // pack L and U = L^T in processing order (IC0_preconditioner split, :874-891);
    // r = b - A x (dcsrmv(-1, 1), blas/spmv.cpp:29-45); sentinel y, z
    for (int e = gt; e < A.nnzf; e += W) {
        const double v = A.lu[__ldg(A.fp_src + e)];
        A.fp_val[e] = v;
        A.fp_val32[e] = __double2float_rn(v);
    }
    for (int e = gt; e < A.nnzb; e += W) {
        const double v = A.lu[__ldg(A.bp_src + e)];
        A.bp_val[e] = v;
        A.bp_val32[e] = __double2float_rn(v);
    }
    double acc = 0.0;
    for (int i = gt; i < n; i += W) {
        const double fd = A.lu[__ldg(A.fp_dsrc + i)], bd = A.lu[__ldg(A.bp_dsrc + i)];
        A.fp_diag[i] = fd;
        A.bp_diag[i] = bd;
        A.fp_diag32[i] = __double2float_rn(fd);
        A.bp_diag32[i] = __double2float_rn(bd);
        double s = 0.0;
        for (int e = __ldg(A.a_rowptr + i); e < __ldg(A.a_rowptr + i + 1); e++)
            s = __dadd_rn(s, __dmul_rn(A.a_val[e], A.x[__ldg(A.a_colidx + e)]));
        const double ri = __dadd_rn(-s, A.b[i]);
        A.r[i] = ri;
        acc = __dadd_rn(acc, __dmul_rn(ri, ri));
        if (A.mixed) {
            A.y32[i] = Sent<float>::value();
            A.z32[i] = Sent<float>::value();
        } else {
            A.y[i] = Sent<double>::value();
            A.z[i] = Sent<double>::value();
        }
    }
    double bs = block_sum<kBlock>(acc);
    if (threadIdx.x == 0) A.part_b[blockIdx.x] = bs;
    BAAS_BARRIER();
    const double norm0 = sqrt(grid_total<kBlock>(A.part_b, gridDim.x));

    // z = M^-1 r, p = z, rz = r.z
    double rzl = 0.0;
    bool ok = A.mixed ? precond_apply<float>(A, A.y32, A.z32, true, rzl, w) : precond_apply<double>(A, A.y, A.z, true, rzl, w);
    (void)ok;  // a failed wait set the status; the barrier below stops every CTA
    bs = block_sum<kBlock>(rzl);
    if (threadIdx.x == 0) A.part_c[blockIdx.x] = bs;
    BAAS_BARRIER();
    double rz = grid_total<kBlock>(A.part_c, gridDim.x);

    int iters = 0;
    double rel = 1.0;
    for (int k = 1; k <= A.maxiter; ++k) {
        const double old_rz = rz;
        // Ap = A p, p.Ap; reset y
        acc = 0.0;
        for (int i = gt; i < n; i += W) {
            double s = 0.0;
            for (int e = __ldg(A.a_rowptr + i); e < __ldg(A.a_rowptr + i + 1); e++)
                s = __dadd_rn(s, __dmul_rn(A.a_val[e], A.p[__ldg(A.a_colidx + e)]));
            A.Ap[i] = s;
            acc = __dadd_rn(acc, __dmul_rn(A.p[i], s));
            if (A.mixed)
                A.y32[i] = Sent<float>::value();
            else
                A.y[i] = Sent<double>::value();
        }
        bs = block_sum<kBlock>(acc);
        if (threadIdx.x == 0) A.part_a[blockIdx.x] = bs;
        BAAS_BARRIER();
        const double alpha = old_rz / grid_total<kBlock>(A.part_a, gridDim.x);

        // x += alpha p; r -= alpha Ap; r.r; reset z
        acc = 0.0;
        for (int i = gt; i < n; i += W) {
            A.x[i] = __dadd_rn(A.x[i], __dmul_rn(alpha, A.p[i]));
            const double ri = __dadd_rn(A.r[i], __dmul_rn(-alpha, A.Ap[i]));
            A.r[i] = ri;
            acc = __dadd_rn(acc, __dmul_rn(ri, ri));
            if (A.mixed)
                A.z32[i] = Sent<float>::value();
            else
                A.z[i] = Sent<double>::value();
        }
        bs = block_sum<kBlock>(acc);
        if (threadIdx.x == 0) A.part_b[blockIdx.x] = bs;
        BAAS_BARRIER();
        rel = sqrt(grid_total<kBlock>(A.part_b, gridDim.x)) / norm0;
        iters = k;
        if (rel < A.tol) break;

        // z = M^-1 r; rz = r.z
        rzl = 0.0;
        ok = A.mixed ? precond_apply<float>(A, A.y32, A.z32, false, rzl, w) : precond_apply<double>(A, A.y, A.z, false, rzl, w);
        bs = block_sum<kBlock>(rzl);
        if (threadIdx.x == 0) A.part_c[blockIdx.x] = bs;
        BAAS_BARRIER();
        rz = grid_total<kBlock>(A.part_c, gridDim.x);
        const double beta = rz / old_rz;

        // p = z + beta p
        for (int i = gt; i < n; i += W) {
            const double zi = A.mixed ? (double)A.z32[i] : A.z[i];
            A.p[i] = __dadd_rn(zi, __dmul_rn(beta, A.p[i]));
        }
        BAAS_BARRIER();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *A.out_iters = iters;
        *A.out_relres = rel;
    }
#undef BAAS_BARRIER
}

}  // namespace baas
