// Batched ICCG: many independent SPD systems, each with R right-hand sides, in one persistent
// cooperative launch.
//
// The systems are concatenated into one block-diagonal matrix, so one BAAS schedule covers them
// all: their level sets merge, IC0 and both triangular sweeps run on the combined matrix exactly
// as for one system (there are no dependencies between systems), and the sweeps walk all R
// right-hand sides together. Each (system, right-hand side) pair is its own CG instance with its
// own alpha, beta, residual norm and convergence; the reference has no batched solver, so the
// per-instance recurrence is pcg_opt's (test/iccg_level_merge.cpp:380-533) with a break at tol.
//
// Vector phases (SpMV, updates, dot products) give each CTA a contiguous row range. A CTA
// reduces its rows of each system it touches with a fixed-order block reduction and writes one
// partial per (system, right-hand side); after the grid barrier every CTA sums, for each system
// it touches, the partials of the CTAs covering that system in CTA order. So every CTA derives
// the same scalars, bit for bit, without another barrier. Instances that have converged stop
// updating; the launch ends when a global count of active instances reaches zero (read after a
// barrier, so every CTA sees the same count).
#pragma once

#include "staged.cuh"

namespace baas {

struct BatchPlan {
    int nsys, R, maxls;
    const int *sys_off;  // nsys + 1 row offsets
    const int *vlo;      // P + 1: row range of each CTA in the vector phases
    const int *sys_lo;   // P: first system of each CTA's row range
    const int *nls;      // P: systems in each CTA's row range
    const int *cta_lo;   // nsys: first CTA whose row range holds rows of the system
    const int *cta_hi;   // nsys: last such CTA
};

struct BatchArgs {
    int n, ldb;
    const int *a_rowptr, *a_colidx, *a_diag;
    const double *a_val;
    const double *B;
    double *X;
    PartView fac;
    ChunkPlan pl;
    BatchPlan bp;
    double *gv64[2];
    float *gv32[2];
    double *lu;
    int *gflag;
    int epoch;
    double *r, *p, *Ap;   // n * R each, column-major (ld = n)
    double *y, *z;        // FP64 factors
    float *y32, *z32;     // FP32 factors
    double *part;         // 2 * P * maxls * R partials (two buffers, alternating per reduction)
    unsigned int *bar;
    unsigned int *active; // instances still iterating
    DevStatus *st;
    int maxiter;
    double tol;
    int *out_iters;       // nsys * R (instance = s * R + r)
    double *out_relres;
    unsigned int spin_limit;
    int scal_off;         // byte offset of the scalar table in dynamic shared memory
};

// Scalar table of one CTA (dynamic shared memory): per local system and right-hand side.
struct BatchScal {
    double *rz, *norm0, *t;  // t: the last reduction's totals
    int *act, *its;
    __device__ void carve(unsigned char *base, int maxls) {
        const int m = maxls * kMaxRhs;
        rz = reinterpret_cast<double *>(base);
        norm0 = rz + m;
        t = norm0 + m;
        act = reinterpret_cast<int *>(t + m);
        its = act + m;
    }
};
__host__ __device__ constexpr int batch_scal_bytes(int maxls) { return maxls * kMaxRhs * (3 * 8 + 2 * 4); }

// Deterministic sum of R per-thread values over the block (fixed shuffle tree, fixed warp order);
// every thread receives the totals in v.
template <int BLOCK>
__device__ __forceinline__ void block_sum_rhs(double (&v)[kMaxRhs], int R) {
    __shared__ double s_part[BLOCK / 32][kMaxRhs];
    __shared__ double s_tot[kMaxRhs];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < kMaxRhs; r++)
        if (r < R) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[r] += __shfl_xor_sync(0xffffffffu, v[r], o);
            if (lane == 0) s_part[wid][r] = v[r];
        }
    __syncthreads();
    if ((int)threadIdx.x < R) {
        double t = 0.0;
        for (int w = 0; w < BLOCK / 32; w++) t += s_part[w][threadIdx.x];
        s_tot[threadIdx.x] = t;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kMaxRhs; r++)
        if (r < R) v[r] = s_tot[r];
    __syncthreads();
}

// Per local system ls of this CTA: f(row range [a, b), system ls, acc[R]) adds the thread's
// share; the block totals go to the CTA's partials in buffer `buf` (reductions alternate
// buffers: a CTA may write reduction k+1's partials while another still reads reduction k's,
// but never before every CTA has passed the barrier that follows those reads).
template <typename F>
__device__ __forceinline__ void batch_partials(const BatchArgs &A, int buf, F f) {
    const int c = blockIdx.x, R = A.bp.R;
    const int lo = __ldg(A.bp.vlo + c), hi = __ldg(A.bp.vlo + c + 1);
    const int s0 = __ldg(A.bp.sys_lo + c), nl = __ldg(A.bp.nls + c);
    for (int ls = 0; ls < nl; ls++) {
        const int s = s0 + ls;
        const int a = max(lo, __ldg(A.bp.sys_off + s)), b = min(hi, __ldg(A.bp.sys_off + s + 1));
        double acc[kMaxRhs];
#pragma unroll
        for (int r = 0; r < kMaxRhs; r++) acc[r] = 0.0;
        f(a, b, ls, acc);
        block_sum_rhs<kStageBlock>(acc, R);
        if ((int)threadIdx.x < R)
            A.part[(((size_t)buf * gridDim.x + c) * A.bp.maxls + ls) * R + threadIdx.x] = acc[threadIdx.x];
    }
}

// After the grid barrier: totals of the last partials, for this CTA's systems, into sc.t.
__device__ __forceinline__ void batch_totals(const BatchArgs &A, int buf, const BatchScal &sc) {
    const int c = blockIdx.x, R = A.bp.R;
    const int s0 = __ldg(A.bp.sys_lo + c), nl = __ldg(A.bp.nls + c);
    for (int k = threadIdx.x; k < nl * R; k += blockDim.x) {
        const int ls = k / R, r = k - ls * R, s = s0 + ls;
        double t = 0.0;
        for (int cc = __ldg(A.bp.cta_lo + s); cc <= __ldg(A.bp.cta_hi + s); cc++) {
            const int l2 = s - __ldg(A.bp.sys_lo + cc);
            t += Sent<double>::load(A.part + (((size_t)buf * gridDim.x + cc) * A.bp.maxls + l2) * R + r);
        }
        sc.t[ls * kMaxRhs + r] = t;
    }
    __syncthreads();
}

// Element-wise row loops of the vector phases. Each thread issues the loads of several rows
// before the stores of any of them (a row loop that stores between its loads keeps one row's
// loads in flight at a time), and adds its rows to its sums in the order of a row-at-a-time loop,
// so every sum keeps its bits. The arrays a loop reads are written by other phases of the launch,
// so they are read through plain pointers (never the read-only path).
constexpr int kVecRows = 4;  // rows in flight per thread

// Right-hand side r on rows [a, b): x += alpha p, r -= alpha Ap (act), acc += r.r, z sentinel.
template <typename T>
__device__ __forceinline__ double batch_update_rows(double *__restrict__ x, double *__restrict__ rr,
                                                    const double *p, const double *Ap, T *__restrict__ zg, int a,
                                                    int b, bool act, double alpha, double acc) {
    const int bd = blockDim.x;
    for (int i0 = a + (int)threadIdx.x; i0 < b; i0 += kVecRows * bd) {
        double xv[kVecRows], rv[kVecRows], pv[kVecRows], av[kVecRows];
#pragma unroll
        for (int u = 0; u < kVecRows; u++) {
            const int i = i0 + u * bd;
            if (i < b) {
                rv[u] = rr[i];
                if (act) {
                    xv[u] = x[i];
                    pv[u] = p[i];
                    av[u] = Ap[i];
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kVecRows; u++) {
            const int i = i0 + u * bd;
            if (i < b) {
                if (act) {
                    x[i] = __dadd_rn(xv[u], __dmul_rn(alpha, pv[u]));
                    rv[u] = __dadd_rn(rv[u], __dmul_rn(-alpha, av[u]));
                    rr[i] = rv[u];
                }
                acc = __dadd_rn(acc, __dmul_rn(rv[u], rv[u]));
                zg[i] = Sent<T>::value();
            }
        }
    }
    return acc;
}

// Right-hand side r on rows [a, b): acc += r.z.
template <typename T>
__device__ __forceinline__ double batch_rz_rows(const double *rr, const T *zg, int a, int b, double acc) {
    const int bd = blockDim.x;
    for (int i0 = a + (int)threadIdx.x; i0 < b; i0 += kVecRows * bd) {
        double rv[kVecRows], zv[kVecRows];
#pragma unroll
        for (int u = 0; u < kVecRows; u++) {
            const int i = i0 + u * bd;
            if (i < b) {
                rv[u] = rr[i];
                zv[u] = (double)Sent<T>::load(zg + i);
            }
        }
#pragma unroll
        for (int u = 0; u < kVecRows; u++)
            if (i0 + u * bd < b) acc = __dadd_rn(acc, __dmul_rn(rv[u], zv[u]));
    }
    return acc;
}

// Right-hand side r on rows [a, b): p = z + beta p.
template <typename T>
__device__ __forceinline__ void batch_p_rows(double *__restrict__ p, const T *zg, int a, int b, double beta) {
    const int bd = blockDim.x;
    for (int i0 = a + (int)threadIdx.x; i0 < b; i0 += kVecRows * bd) {
        double pv[kVecRows], zv[kVecRows];
#pragma unroll
        for (int u = 0; u < kVecRows; u++) {
            const int i = i0 + u * bd;
            if (i < b) {
                pv[u] = p[i];
                zv[u] = (double)Sent<T>::load(zg + i);
            }
        }
#pragma unroll
        for (int u = 0; u < kVecRows; u++) {
            const int i = i0 + u * bd;
            if (i < b) p[i] = __dadd_rn(zv[u], __dmul_rn(beta, pv[u]));
        }
    }
}

template <typename T, bool MR, bool IEEE, int RW>
__device__ __forceinline__ bool batch_precond(const BatchArgs &A, WinStream<T> &ws, unsigned char *smem, Waiter &w) {
    T *yg = sizeof(T) == 8 ? (T *)A.y : (T *)A.y32;
    T *zg = sizeof(T) == 8 ? (T *)A.z : (T *)A.z32;
    T *xs = reinterpret_cast<T *>(smem);
    const int n0 = ws.ctl->n0;
    {
        const WalkIO<T, double, MR, false> lo{xs, yg, A.r, nullptr, A.n, A.n, A.bp.R};
        if (!walk_dir<T, double, false, MR, false, kDiv<T, IEEE>, RW>(ws, 0, n0, lo, w, A.spin_limit, A.st)) return false;
    }
    const WalkIO<T, T, MR, false> up{xs, zg, yg, nullptr, A.n, A.n, A.bp.R};
    return walk_dir<T, T, true, MR, false, kDiv<T, IEEE>, RW>(ws, n0, ws.total(), up, w, A.spin_limit, A.st);
}

// IEEE (FP64 factors only): sweep divisions by __ddiv_rn, for the repeat of a launch whose
// div_fast divisions left their range. RW = 2 or 4 (FP32 factors, that many right-hand sides):
// the sweeps take the row-wide walk.
template <typename T, bool MR, bool IEEE, int RW>
__global__ void __launch_bounds__(kStageBlock, 1) k_iccg_batched(BatchArgs A) {
    constexpr bool kMixed = sizeof(T) == 4;
    extern __shared__ __align__(128) unsigned char smem[];
    const int n = A.n, R = A.bp.R, c = blockIdx.x;
    const int W = gridDim.x * blockDim.x;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned int nb = 0;
    Waiter w(A.spin_limit, A.st);
    WinStream<T> ws;
    ws.init(A.pl, 0, true, kMixed ? (const T *)A.gv32[0] : (const T *)A.gv64[0],
            kMixed ? (const T *)A.gv32[1] : (const T *)A.gv64[1], smem, 0xFFFFFFFFu);
    BatchScal sc;
    sc.carve(smem + A.scal_off, A.bp.maxls);
    T *yg = kMixed ? (T *)A.y32 : (T *)A.y;
    T *zg = kMixed ? (T *)A.z32 : (T *)A.z;
    const int s0 = __ldg(A.bp.sys_lo + c), nls = __ldg(A.bp.nls + c);
    int red = 0;  // reductions so far (partial buffer = red & 1)
#define BAAS_BARRIER()                                            \
    do {                                                          \
        if (!grid_barrier(A.bar, nb, A.st, A.spin_limit)) {       \
            ws.drain(A.spin_limit);                               \
            return;                                               \
        }                                                         \
    } while (0)

    // IC0 of the block-diagonal matrix and the packing of its factors
    const int nnz = __ldg(A.a_rowptr + n);
    for (int e = gt; e < nnz; e += W) A.lu[e] = A.a_val[e];
    BAAS_BARRIER();
    factor_part<false>(A.fac, A.a_rowptr, A.a_colidx, A.a_diag, A.lu, A.gflag, A.epoch, w, A.st);
    BAAS_BARRIER();
    pack_factor<T>(A.pl.dir[0], A.lu, A.gv64[0], A.gv32[0]);
    pack_factor<T>(A.pl.dir[1], A.lu, A.gv64[1], A.gv32[1]);
    fence_async_global();

    // r = B - A X, sentinels, |r0|^2 per instance
    batch_partials(A, red & 1, [&](int a, int b, int, double (&acc)[kMaxRhs]) {
        for (int i = a + (int)threadIdx.x; i < b; i += blockDim.x) {
            const int e0 = __ldg(A.a_rowptr + i), e1 = __ldg(A.a_rowptr + i + 1);
#pragma unroll
            for (int r = 0; r < kMaxRhs; r++)
                if (r < R) {
                    const double *x = A.X + (size_t)r * A.ldb;
                    double s = 0.0;
                    for (int e = e0; e < e1; e++) s = __dadd_rn(s, __dmul_rn(A.a_val[e], x[__ldg(A.a_colidx + e)]));
                    const double ri = __dadd_rn(-s, A.B[(size_t)r * A.ldb + i]);
                    A.r[(size_t)r * n + i] = ri;
                    acc[r] = __dadd_rn(acc[r], __dmul_rn(ri, ri));
                    yg[(size_t)r * n + i] = Sent<T>::value();
                    zg[(size_t)r * n + i] = Sent<T>::value();
                }
        }
    });
    BAAS_BARRIER();
    batch_totals(A, red++ & 1, sc);
    for (int q = threadIdx.x; q < nls * kMaxRhs; q += blockDim.x) {
        const int ls = q / kMaxRhs, r = q - ls * kMaxRhs;
        sc.norm0[q] = r < R ? sqrt(sc.t[q]) : 0.0;
        sc.act[q] = r < R && sc.norm0[q] > 0.0;
        sc.its[q] = 0;
        // an instance whose right-hand side is already solved (zero residual) never iterates
        if (r < R && !sc.act[q] && c == __ldg(A.bp.cta_lo + s0 + ls)) {
            atomicSub(A.active, 1u);
            A.out_iters[(s0 + ls) * R + r] = 0;
            A.out_relres[(s0 + ls) * R + r] = 0.0;
        }
    }
    __syncthreads();

    if (!batch_precond<T, MR, IEEE, RW>(A, ws, smem, w)) {
        ws.drain(A.spin_limit);
        return;
    }
    // the vector phases read z of rows other CTAs' walks computed
    BAAS_BARRIER();
    batch_partials(A, red & 1, [&](int a, int b, int, double (&acc)[kMaxRhs]) {
        for (int i = a + (int)threadIdx.x; i < b; i += blockDim.x)
#pragma unroll
            for (int r = 0; r < kMaxRhs; r++)
                if (r < R) {
                    const double zd = (double)Sent<T>::load(zg + (size_t)r * n + i);
                    A.p[(size_t)r * n + i] = zd;
                    acc[r] = __dadd_rn(acc[r], __dmul_rn(A.r[(size_t)r * n + i], zd));
                }
    });
    BAAS_BARRIER();
    batch_totals(A, red++ & 1, sc);
    for (int k = threadIdx.x; k < nls * kMaxRhs; k += blockDim.x) sc.rz[k] = sc.t[k];
    __syncthreads();

    int k = 1;
    for (; k <= A.maxiter; ++k) {
        // Ap = A p, p.Ap; y sentinels
        batch_partials(A, red & 1, [&](int a, int b, int, double (&acc)[kMaxRhs]) {
            for (int i = a + (int)threadIdx.x; i < b; i += blockDim.x) {
                const int e0 = __ldg(A.a_rowptr + i), e1 = __ldg(A.a_rowptr + i + 1);
                // each entry of A read once for all right-hand sides
                double s[kMaxRhs];
#pragma unroll
                for (int r = 0; r < kMaxRhs; r++) s[r] = 0.0;
                for (int e = e0; e < e1; e++) {
                    const double v = __ldg(A.a_val + e);
                    const int j = __ldg(A.a_colidx + e);
#pragma unroll
                    for (int r = 0; r < kMaxRhs; r++)
                        if (r < R) s[r] = __dadd_rn(s[r], __dmul_rn(v, A.p[(size_t)r * n + j]));
                }
#pragma unroll
                for (int r = 0; r < kMaxRhs; r++)
                    if (r < R) {
                        A.Ap[(size_t)r * n + i] = s[r];
                        acc[r] = __dadd_rn(acc[r], __dmul_rn(A.p[(size_t)r * n + i], s[r]));
                        yg[(size_t)r * n + i] = Sent<T>::value();
                    }
            }
        });
        BAAS_BARRIER();
        batch_totals(A, red++ & 1, sc);
        // x += alpha p, r -= alpha Ap (active instances), |r|^2; z sentinels
        batch_partials(A, red & 1, [&](int a, int b, int ls, double (&acc)[kMaxRhs]) {
            double alpha[kMaxRhs];
            int act[kMaxRhs];
#pragma unroll
            for (int r = 0; r < kMaxRhs; r++) {
                act[r] = r < R ? sc.act[ls * kMaxRhs + r] : 0;
                alpha[r] = act[r] ? sc.rz[ls * kMaxRhs + r] / sc.t[ls * kMaxRhs + r] : 0.0;
            }
#pragma unroll
            for (int r = 0; r < kMaxRhs; r++)
                if (r < R) {
                    const size_t o = (size_t)r * n;
                    acc[r] = batch_update_rows<T>(A.X + (size_t)r * A.ldb, A.r + o, A.p + o, A.Ap + o, zg + o, a, b,
                                                  act[r] != 0, alpha[r], acc[r]);
                }
        });
        BAAS_BARRIER();
        batch_totals(A, red++ & 1, sc);
        // residual test per instance; the first CTA of a system retires its newly converged
        // instances from the global count
        for (int q = threadIdx.x; q < nls * kMaxRhs; q += blockDim.x) {
            const int ls = q / kMaxRhs, r = q - ls * kMaxRhs;
            if (r >= R || !sc.act[q]) continue;
            const double rel = sqrt(sc.t[q]) / sc.norm0[q];
            sc.its[q] = k;
            if (rel < A.tol) {
                sc.act[q] = 0;
                if (c == __ldg(A.bp.cta_lo + s0 + ls)) atomicSub(A.active, 1u);
            }
            if (c == __ldg(A.bp.cta_lo + s0 + ls)) {
                A.out_iters[(s0 + ls) * R + r] = k;
                A.out_relres[(s0 + ls) * R + r] = rel;
            }
        }
        __syncthreads();

        if (!batch_precond<T, MR, IEEE, RW>(A, ws, smem, w)) {
            ws.drain(A.spin_limit);
            return;
        }
        BAAS_BARRIER();
        batch_partials(A, red & 1, [&](int a, int b, int, double (&acc)[kMaxRhs]) {
#pragma unroll
            for (int r = 0; r < kMaxRhs; r++)
                if (r < R) acc[r] = batch_rz_rows<T>(A.r + (size_t)r * n, zg + (size_t)r * n, a, b, acc[r]);
        });
        BAAS_BARRIER();
        // every CTA reads the same count after this barrier
        if (ld_relaxed_u32(A.active) == 0u) break;
        batch_totals(A, red++ & 1, sc);
        // p = z + beta p (active instances)
        for (int ls = 0; ls < nls; ls++) {
            const int s = s0 + ls;
            const int a = max(__ldg(A.bp.vlo + c), __ldg(A.bp.sys_off + s));
            const int b = min(__ldg(A.bp.vlo + c + 1), __ldg(A.bp.sys_off + s + 1));
            double beta[kMaxRhs];
            int act[kMaxRhs];
#pragma unroll
            for (int r = 0; r < kMaxRhs; r++) {
                act[r] = r < R ? sc.act[ls * kMaxRhs + r] : 0;
                beta[r] = act[r] ? sc.t[ls * kMaxRhs + r] / sc.rz[ls * kMaxRhs + r] : 0.0;
            }
#pragma unroll
            for (int r = 0; r < kMaxRhs; r++)
                if (r < R && act[r]) batch_p_rows<T>(A.p + (size_t)r * n, zg + (size_t)r * n, a, b, beta[r]);
        }
        __syncthreads();
        for (int q = threadIdx.x; q < nls * kMaxRhs; q += blockDim.x)
            if (sc.act[q]) sc.rz[q] = sc.t[q];
        __syncthreads();
        BAAS_BARRIER();
    }
    ws.drain(A.spin_limit);
#undef BAAS_BARRIER
}

}  // namespace baas
