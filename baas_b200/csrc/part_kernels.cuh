// Partitioned, level-synchronous factorisation kernels (IC0, ILU0): the factor step of the BAAS
// hot path. (The triangular sweeps run from the chunked plan of staged.cuh.)
//
// Rows are owned by P CTAs (contiguous row ranges by default; one CTA per SM). The schedule's
// coarsened groups are the work items, and each CTA walks the group DAG's dependency levels in
// order: at level l it runs its own groups of level l (one group per thread, the group's rows in
// ascending order, exactly as one reference thread runs a group, merge/SpTRSV.cpp:458-471),
// then a CTA barrier. So
//   - a dependency on a row of the same CTA needs no wait at all: the barrier (or program
//     order, inside a group) already made it visible;
//   - a dependency on a row of another CTA is a point-to-point wait on that row's epoch-stamped
//     release/acquire flag, the analogue of the reference's taskFinsished waits
//     (merge/include/SpTRSV.hpp:16-35).
// A group of level l depends only on groups of levels < l and every CTA walks the levels in
// the same increasing order, so by induction on l every CTA finishes every level: no deadlock
// while all CTAs are resident (cooperative launch). With contiguous row ranges every cross-CTA
// dependency points to an earlier CTA.
//
// Dependency encoding per factor entry: dep >= 0 is a global row index (remote), dep < 0 is
// -(slot + 1) with slot the CTA-local index of a row computed earlier by this CTA.
#pragma once

#include "device_common.cuh"

namespace baas {

constexpr int kPartBlock = 512;

struct PartView {
    int P;
    const int *cta_seg;   // P + 1: level segments of each CTA
    const int *seg_item;  // nseg + 1: items (groups) of each segment
    const int *item_pos;  // nitem + 1: positions (rows) of each item
    const int *cta_pos;   // P + 1: first position of each CTA (local slot = pos - cta_pos[c])
    const int *row;       // position -> row
    const int *eptr;      // position -> off-diagonal entries [eptr[pos], eptr[pos+1])
    const int *dep;       // entry -> encoded dependency
    // factorisations: entry -> A position of its pivot (the other row's diagonal), and its
    // column-match pairs [mptr[e], mptr[e+1]) of mpair = {offset in the own row, A position}
    const int *epiv;
    const int *mptr;
    const int2 *mpair;
};

// Walks this CTA's level segments; `row_fn(pos, slot)` computes one row (false = give up).
// Every thread passes every barrier, also after a failed wait, so the CTA never splits.
template <typename RowFn>
__device__ __forceinline__ bool walk_levels(const PartView &pv, RowFn row_fn) {
    const int c = blockIdx.x;
    const int pos0 = __ldg(pv.cta_pos + c);
    const int sb = __ldg(pv.cta_seg + c), se = __ldg(pv.cta_seg + c + 1);
    bool alive = true;
    for (int sg = sb; sg < se; sg++) {
        const int ib = __ldg(pv.seg_item + sg), ie = __ldg(pv.seg_item + sg + 1);
        for (int it = ib + (int)threadIdx.x; it < ie && alive; it += blockDim.x) {
            const int pb = __ldg(pv.item_pos + it), pe = __ldg(pv.item_pos + it + 1);
            for (int pos = pb; pos < pe; pos++)
                if (!row_fn(pos, pos - pos0)) {
                    alive = false;
                    break;
                }
        }
        __syncthreads();
    }
    return alive;
}

// ---------------------------------------------------------------------------------------
// Level-synchronous IC0 / ILU0. A row of this CTA from an earlier level is final after the
// barrier and is read through L1; a row of another CTA is waited for on its epoch-stamped
// global flag (acquire) and read from L2. Every row publishes its flag with a release store.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double ld_l2(const double *p) { return Sent<double>::load(p); }

template <bool LOCAL>
__device__ __forceinline__ double ldv(const double *p) {
    if constexpr (LOCAL)
        return *p;
    else
        return ld_l2(p);
}

// IC0 row i (merge/IC.cpp:296-393; sparse_dot_product :6-29), correctly rounded FP64.
// Rows wider than the register path: the same operations, with each entry's dot product taken
// from the host-built column-match pairs (the merge's matches, in its order) instead of a merge
// over column indices, and eight pairs' loads in flight at once.
__device__ __forceinline__ bool ic0_row_part(const PartView &pv, int pos, int i, const int *__restrict__ rowptr,
                                             const int *__restrict__ colidx, const int *__restrict__ diagptr, double *lu,
                                             const int *gflag, int epoch, Waiter &w, DevStatus *st) {
    constexpr int B = 8;
    const int rb = __ldg(rowptr + i), di = __ldg(diagptr + i), e0 = __ldg(pv.eptr + pos);
    for (int k = rb; k < di; k++) {
        const int t = k - rb;
        const int d = __ldg(pv.dep + e0 + t);
        const bool loc = d < 0;
        if (!loc && !wait_flag(gflag + __ldg(colidx + k), epoch, w, i)) return false;
        const int pj = __ldg(pv.epiv + e0 + t);
        const double ljj = loc ? ldv<true>(lu + pj) : ldv<false>(lu + pj);
        double dp = 0.0;
        for (int m0 = __ldg(pv.mptr + e0 + t), m1 = __ldg(pv.mptr + e0 + t + 1); m0 < m1; m0 += B) {
            int2 pr[B];
            double av[B], bv[B];
#pragma unroll
            for (int u = 0; u < B; u++) pr[u] = m0 + u < m1 ? __ldg(pv.mpair + m0 + u) : make_int2(0, -1);
#pragma unroll
            for (int u = 0; u < B; u++) {
                av[u] = pr[u].y < 0 ? 0.0 : lu[rb + pr[u].x];
                bv[u] = pr[u].y < 0 ? 0.0 : (loc ? ldv<true>(lu + pr[u].y) : ldv<false>(lu + pr[u].y));
            }
#pragma unroll
            for (int u = 0; u < B; u++)
                if (m0 + u < m1) dp = __dadd_rn(dp, __dmul_rn(av[u], bv[u]));
        }
        lu[k] = __ddiv_rn(__dsub_rn(lu[k], dp), ljj);
    }
    double dv = 0.0;
    for (int k = rb; k < di; k++) dv = __dadd_rn(dv, __dmul_rn(lu[k], lu[k]));
    const double t = __dsub_rn(lu[di], dv);
    if (t > 0.0)
        lu[di] = __dsqrt_rn(t);
    else
        atomicAdd(&st->zero_pivots, 1);
    return true;
}

// ILU0 row i (merge/ILU.cpp:638-720).
template <bool LOCAL>
__device__ __forceinline__ void ilu0_update(int j, int re, int dc, int ec, double tmp, const int *__restrict__ colidx,
                                            double *lu) {
    int k1 = j + 1, k2 = dc + 1;
    while (k1 < re && k2 < ec) {
        const int c1 = __ldg(colidx + k1), c2 = __ldg(colidx + k2);
        if (c1 < c2) {
            k1++;
        } else if (c1 > c2) {
            k2++;
        } else {
            lu[k1] = __dsub_rn(lu[k1], __dmul_rn(tmp, ldv<LOCAL>(lu + k2)));
            k1++;
            k2++;
        }
    }
}

__device__ __forceinline__ bool ilu0_row_part(const PartView &pv, int pos, int i, const int *__restrict__ rowptr,
                                              const int *__restrict__ colidx, const int *__restrict__ diagptr, double *lu,
                                              const int *gflag, int epoch, Waiter &w, DevStatus *st) {
    const int rb = __ldg(rowptr + i), di = __ldg(diagptr + i), re = __ldg(rowptr + i + 1), e0 = __ldg(pv.eptr + pos);
    for (int j = rb; j < di; j++) {
        const int c = __ldg(colidx + j);
        const int d = __ldg(pv.dep + e0 + (j - rb));
        const int dc = __ldg(diagptr + c), ec = __ldg(rowptr + c + 1);
        if (d >= 0 && !wait_flag(gflag + c, epoch, w, i)) return false;
        const double pivot = d < 0 ? ldv<true>(lu + dc) : ldv<false>(lu + dc);
        if (pivot == 0.0) atomicAdd(&st->zero_pivots, 1);
        const double tmp = __ddiv_rn(lu[j], pivot);
        lu[j] = tmp;
        if (d < 0)
            ilu0_update<true>(j, re, dc, ec, tmp, colidx, lu);
        else
            ilu0_update<false>(j, re, dc, ec, tmp, colidx, lu);
    }
    return true;
}

// Rows of at most kFacRegs entries (the lower part for IC0, the whole row for ILU0) run from
// registers: the row's values and all its pivots are loaded at once (after the waits for remote
// rows), the column matches come from the host-built pair lists instead of a merge loop over
// column indices, and the row is written back once. Same operations in the same order as
// ic0_row_part / ilu0_row_part, so the factor is bit-identical.
constexpr int kFacRegs = 8;

__device__ __forceinline__ double pick(const double (&v)[kFacRegs], int k) {
    double r = 0.0;
#pragma unroll
    for (int u = 0; u < kFacRegs; u++) r = u == k ? v[u] : r;
    return r;
}

// Waits for the rows of the entries [rb, rb + ne) that another CTA computes (their flags, by
// column index, as ic0_row_part / ilu0_row_part wait).
__device__ __forceinline__ bool wait_remote(const PartView &pv, int e0, int rb, int ne, const int *__restrict__ colidx,
                                            const int *gflag, int epoch, Waiter &w, int i) {
#pragma unroll
    for (int t = 0; t < kFacRegs; t++)
        if (t < ne && __ldg(pv.dep + e0 + t) >= 0 && !wait_flag(gflag + __ldg(colidx + rb + t), epoch, w, i)) return false;
    return true;
}

__device__ __forceinline__ bool ic0_row_reg(const PartView &pv, int pos, int i, int rb, int di,
                                            const int *__restrict__ colidx, double *lu, const int *gflag, int epoch,
                                            Waiter &w, DevStatus *st) {
    const int ne = di - rb, e0 = __ldg(pv.eptr + pos);
    if (!wait_remote(pv, e0, rb, ne, colidx, gflag, epoch, w, i)) return false;
    double v[kFacRegs], piv[kFacRegs];
#pragma unroll
    for (int t = 0; t < kFacRegs; t++) {
        v[t] = piv[t] = 0.0;
        if (t < ne) {
            v[t] = lu[rb + t];
            const int pj = __ldg(pv.epiv + e0 + t);
            piv[t] = __ldg(pv.dep + e0 + t) < 0 ? ldv<true>(lu + pj) : ldv<false>(lu + pj);
        }
    }
    const double dval = lu[di];
#pragma unroll
    for (int t = 0; t < kFacRegs; t++)
        if (t < ne) {
            const bool loc = __ldg(pv.dep + e0 + t) < 0;
            double dp = 0.0;
            for (int m = __ldg(pv.mptr + e0 + t), m1 = __ldg(pv.mptr + e0 + t + 1); m < m1; m++) {
                const int2 pr = __ldg(pv.mpair + m);
                const double bv = loc ? ldv<true>(lu + pr.y) : ldv<false>(lu + pr.y);
                dp = __dadd_rn(dp, __dmul_rn(pick(v, pr.x), bv));
            }
            v[t] = __ddiv_rn(__dsub_rn(v[t], dp), piv[t]);
        }
    double dv = 0.0;
#pragma unroll
    for (int t = 0; t < kFacRegs; t++)
        if (t < ne) {
            dv = __dadd_rn(dv, __dmul_rn(v[t], v[t]));
            lu[rb + t] = v[t];
        }
    const double tt = __dsub_rn(dval, dv);
    if (tt > 0.0)
        lu[di] = __dsqrt_rn(tt);
    else
        atomicAdd(&st->zero_pivots, 1);
    return true;
}

__device__ __forceinline__ bool ilu0_row_reg(const PartView &pv, int pos, int i, int rb, int di, int re,
                                             const int *__restrict__ colidx, double *lu, const int *gflag, int epoch,
                                             Waiter &w, DevStatus *st) {
    const int nlow = di - rb, nrow = re - rb, e0 = __ldg(pv.eptr + pos);
    if (!wait_remote(pv, e0, rb, nlow, colidx, gflag, epoch, w, i)) return false;
    double v[kFacRegs], piv[kFacRegs];
#pragma unroll
    for (int t = 0; t < kFacRegs; t++) {
        v[t] = piv[t] = 0.0;
        if (t < nrow) v[t] = lu[rb + t];
        if (t < nlow) {
            const int pj = __ldg(pv.epiv + e0 + t);
            piv[t] = __ldg(pv.dep + e0 + t) < 0 ? ldv<true>(lu + pj) : ldv<false>(lu + pj);
        }
    }
#pragma unroll
    for (int t = 0; t < kFacRegs; t++)
        if (t < nlow) {
            const bool loc = __ldg(pv.dep + e0 + t) < 0;
            if (piv[t] == 0.0) atomicAdd(&st->zero_pivots, 1);
            const double tmp = __ddiv_rn(v[t], piv[t]);
            v[t] = tmp;
            for (int m = __ldg(pv.mptr + e0 + t), m1 = __ldg(pv.mptr + e0 + t + 1); m < m1; m++) {
                const int2 pr = __ldg(pv.mpair + m);
                const double bv = loc ? ldv<true>(lu + pr.y) : ldv<false>(lu + pr.y);
                const double u = __dsub_rn(pick(v, pr.x), __dmul_rn(tmp, bv));
#pragma unroll
                for (int q = 0; q < kFacRegs; q++)
                    if (q == pr.x) v[q] = u;
            }
        }
#pragma unroll
    for (int t = 0; t < kFacRegs; t++)
        if (t < nrow) lu[rb + t] = v[t];
    return true;
}

template <bool ILU>
__device__ __forceinline__ bool factor_part(const PartView &pv, const int *rowptr, const int *colidx, const int *diagptr,
                                            double *lu, int *gflag, int epoch, Waiter &w, DevStatus *st) {
    return walk_levels(pv, [&](int pos, int) {
        const int row = __ldg(pv.row + pos);
        const int rb = __ldg(rowptr + row), di = __ldg(diagptr + row), re = __ldg(rowptr + row + 1);
        bool ok;
        if constexpr (ILU)
            ok = re - rb <= kFacRegs ? ilu0_row_reg(pv, pos, row, rb, di, re, colidx, lu, gflag, epoch, w, st)
                                     : ilu0_row_part(pv, pos, row, rowptr, colidx, diagptr, lu, gflag, epoch, w, st);
        else
            ok = di - rb <= kFacRegs ? ic0_row_reg(pv, pos, row, rb, di, colidx, lu, gflag, epoch, w, st)
                                     : ic0_row_part(pv, pos, row, rowptr, colidx, diagptr, lu, gflag, epoch, w, st);
        if (!ok) return false;
        // the release store orders this thread's writes of the row before the flag
        st_release_s32(gflag + row, epoch);
        return true;
    });
}

template <bool ILU>
__global__ void __launch_bounds__(kPartBlock, 1) k_factor_part(PartView pv, const int *__restrict__ rowptr,
                                                              const int *__restrict__ colidx,
                                                              const int *__restrict__ diagptr, double *lu, int *gflag,
                                                              int epoch, DevStatus *st, unsigned int spin_limit) {
    Waiter w(spin_limit, st);
    factor_part<ILU>(pv, rowptr, colidx, diagptr, lu, gflag, epoch, w, st);
}

template <int BLOCK>
__device__ __forceinline__ void put_partial(double *part, double v) {
    const double s = block_sum<BLOCK>(v);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

}  // namespace baas
