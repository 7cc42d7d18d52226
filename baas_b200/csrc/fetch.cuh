// Fetch walk: the triangular sweep for rows of at most three off-diagonal entries and one
// right-hand side (the stencil systems), with a fetcher warp that brings other CTAs' results into
// shared memory.
//
// Why: a level step of the chunked walk (staged.cuh) costs ~0.4 us, and a CTA whose rows depend
// on another CTA's rows pays an L2 round trip on almost every step, because its remote values
// are loaded one step ahead and the producer has written them only just before. Measured on the
// 64^3 lower sweep, the branches around remote loads and waits cost more than the arithmetic.
// So here:
//   - every dependency of a row is a SLOT in shared memory: a row of this CTA (its position in
//     the CTA's row list), the zero slot (an absent entry: it holds -0, and -0 times the
//     coefficient +0 is -0, which added to any sum -- +0 and -0 included -- returns that sum
//     bit for bit, in the FP64 add as in the FP32 fused multiply-add), or a STAGING slot that
//     the fetcher warp fills with another CTA's result;
//   - the compute warps run the step without branches: lanes beyond the step's row count repeat
//     its last row (within a warp they read before any of them stores, so they store the same
//     value to the same places; a warp wholly past the row count stores nothing), all loads are
//     unconditional, and a staged value that has not arrived yet is awaited behind one
//     warp-wide vote;
//   - the fetcher warp (the CTA's last warp) walks the CTA's fetch list -- the remote rows in
//     order of first use, kept in shared memory -- with four polls in flight per lane, and stores each value into its
//     staging slot as soon as it is no longer the sentinel. It never joins the compute warps'
//     step barrier (a named barrier), so its polls never delay a step.
// Row operations are the reference's (merge/SpTRSV.cpp:421-478 forward, :601-660 backward):
// entries in the plan's order (ascending columns for L, descending for U = L^T), then the
// division by the diagonal; so results are bit-identical to the chunked walk's.
//
// Plan, per direction and CTA (built on the host, capi.cu build_fetch):
//   int block  [step table int4 x (ns + 2) | records int4 x nrows]
//              step k: {first record, row count nl, 0, 0}; two terminal copies of the last step
//              let the walk read one step ahead without a test.
//              record: {own, slot0, slot1, slot2}: own is the row's position in the CTA's row
//              list (its slot, where its right-hand side is staged and its result goes; the
//              row itself is srow[own], kept in shared memory beside the slots).
//   values     one record's worth per row, in record order: FP64 {diag, 1/diag, a0, a1, a2, 0}
//              (48 bytes; 1/diag = div_recip(diag)), FP32 {1/diag, a0, a1, a2} (16 bytes).
//   fetch list rows of other CTAs, in order of first use; entry f fills staging slot
//              nrows + 1 + f.
// Dependency deadlock-freedom: a fetch entry's first use is at a step no later than any later
// entry's, and its producer row sits at a lower level than that use, so by induction on levels
// every entry is eventually written (all CTAs are co-resident: cooperative launch).
#pragma once

#include "device_common.cuh"

namespace baas {

constexpr int kFetchBlock = 256;                  // threads of a CTA that runs a fetch walk
constexpr int kFetchWarp = kFetchBlock / 32 - 1;  // the last warp fetches
constexpr int kFetchMaxRows = kFetchBlock - 32;   // widest step the compute warps take
constexpr int kFetchVal64 = 6;                    // doubles per record
constexpr int kFetchVal32 = 4;                    // floats per record

struct FetchDir {
    const int4 *ints;    // int blocks, CTA by CTA
    const int4 *cblk;    // per CTA: {first int4 of its block, int4 count, ns, first record}
    const int *code;     // 4 per record: A positions of {diag, a0, a1, a2} (-1: absent)
    const int *codeT;    // the same for the caller's triangular CSR (standalone sweeps)
    const int *cfetch;   // P + 1: fetch list of each CTA
    const int *frow;     // fetch list rows
};

struct FetchPlan {
    int P;
    FetchDir dir[2];
    const int *soff, *srow;  // rows of each CTA (its row list: position -> row)
    int nslot;               // slots per CTA: rows + 1 + staging of both directions (the most of any CTA)
    int srow_bytes;          // shared bytes reserved for the CTA's row list and both fetch lists
    int ints_bytes[2];       // shared bytes reserved for each direction's int block
    int vals_bytes;          // shared bytes of the value buffer
    int ncomp;               // compute threads (a multiple of 32, at most kFetchMaxRows)
};

// Shared-memory layout of a fetch walk: [slots | row list | fetch lists (lower, upper) | int block
// lower | int block upper | values | control]; all but the slots and values stay resident for the
// launch.
struct FetchCtl {
    unsigned long long mbar_ints, mbar_vals, mbar_fac;  // int blocks; record values; IC0's A values
    int err;
    int pad;
};
__host__ __device__ constexpr int fetch_smem_bytes(int slot_bytes, int srow_bytes, int ib0, int ib1, int vb) {
    return slot_bytes + srow_bytes + ib0 + ib1 + vb + 64;
}

// Bounded wait of one fetcher lane or compute lane: gives up after `limit` polls, or when the
// CTA's error word or the launch's status word is set.
struct FetchWait {
    unsigned int polls, limit;
    __device__ __forceinline__ bool tick(DevStatus *st, volatile int *cta_err, int where) {
        ++polls;
        if ((polls & 127u) == 0u) {
            if (*cta_err || ld_relaxed_u32(&st->code) != 0u) return false;
            if (polls >= limit) {
                if (atomicCAS(&st->code, kOk, kTimeout) == kOk) st->where = where;
                return false;
            }
        }
        return true;
    }
};

// Fetcher: lane l stages entries l, l + 32, l + 64, l + 96, then l + 128, ...: four polls in
// flight per lane. The CTA's fetch list sits in shared memory (FL: its shared address); entry f
// goes to staging slot `stage + f`.
template <typename T>
__device__ __forceinline__ void fetch_run(unsigned int FL, int nf, const T *xg, unsigned int stage, unsigned int limit,
                                          DevStatus *st, FetchCtl *ctl) {
    constexpr unsigned int S = sizeof(T);
    constexpr int U = 4;
    const int l = (int)(threadIdx.x & 31);
    volatile int *cerr = &ctl->err;
    for (int k0 = l; k0 < nf; k0 += 32 * U) {
        int r[U];
        T v[U];
        bool done[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int k = k0 + 32 * u;
            done[u] = k >= nf;
            r[u] = Sh<int>::ldu(FL + 4u * (unsigned int)(done[u] ? k0 : k));
        }
#pragma unroll
        for (int u = 0; u < U; u++) v[u] = Sent<T>::load(xg + r[u]);
        FetchWait w{0u, limit};
        for (;;) {
            bool all = true;
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (!done[u] && !Sent<T>::is(v[u])) {
                    Sh<T>::stu(stage + S * (unsigned int)(k0 + 32 * u), v[u]);
                    done[u] = true;
                }
                all &= done[u];
            }
            if (all) break;
            if (!w.tick(st, cerr, r[0])) {
                *cerr = 1;
                return;
            }
#pragma unroll
            for (int u = 0; u < U; u++)
                if (!done[u]) v[u] = Sent<T>::load(xg + r[u]);
        }
    }
}

__device__ __forceinline__ void bar_compute(int nthreads) {
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}
__device__ __forceinline__ int4 ldsh4(unsigned int a) {
    int4 v;
    asm volatile("ld.shared.v4.s32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
    return v;
}
__device__ __forceinline__ double2 ldsh_d2(unsigned int a) {
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
    return v;
}
__device__ __forceinline__ float4 ldsh_f4(unsigned int a) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}

// One direction's walk by the compute threads [0, ncomp). I: shared address of the direction's
// int block; V: shared address of its first record's values; SL: shared address of slot 0; RW:
// shared address of the CTA's row list. Each row's result goes to its own slot (where its
// right-hand side was staged) and, as its own ready flag, to xg[row]. DIV: 1 = FP64 with
// div_fast (a quotient outside its proven range sets `slow`, and the launch is repeated with
// DIV = 2), 2 = FP64 with __ddiv_rn, 0 = FP32 (the value block holds 1/diag). A wait that gives
// up sets the CTA's error word; the walk then finishes without waiting, and the caller reads the
// word after a CTA barrier.
template <typename T, int DIV>
__device__ __forceinline__ void walk_fetch(unsigned int I, unsigned int V, unsigned int SL, unsigned int RW, int ns,
                                           int ncomp, T *xg, unsigned int limit, DevStatus *st, FetchCtl *ctl,
                                           bool &slow) {
    constexpr unsigned int S = sizeof(T);
    constexpr unsigned int RB = sizeof(T) == 8 ? 8u * kFetchVal64 : 4u * kFetchVal32;
    const int tid = (int)threadIdx.x;
    if (ns == 0) return;  // a CTA without rows
    const unsigned int R0 = I + 16u * (unsigned int)(ns + 2);
    volatile int *cerr = &ctl->err;
    int4 stp = ldsh4(I);
    int4 rec = ldsh4(R0 + 16u * (unsigned int)(stp.x + min(tid, stp.y - 1)));
    int row = Sh<int>::ldu(RW + 4u * (unsigned int)rec.x);
    for (int s = 0; s < ns; s++) {
        const int4 stn = ldsh4(I + 16u * (unsigned int)(s + 1));
        const int nl = stp.y;
        const int q = min(tid, nl - 1);
        const unsigned int va = V + RB * (unsigned int)(stp.x + q);
        const unsigned int ko = SL + S * (unsigned int)rec.x;
        T x0 = Sh<T>::ldu(SL + S * (unsigned int)rec.y);
        T x1 = Sh<T>::ldu(SL + S * (unsigned int)rec.z);
        T x2 = Sh<T>::ldu(SL + S * (unsigned int)rec.w);
        const T rhs = Sh<T>::ldu(ko);
        const int4 recn = ldsh4(R0 + 16u * (unsigned int)(stn.x + min(tid, stn.y - 1)));
        {
            T o;
            if constexpr (sizeof(T) == 8) {
                const double2 dr = ldsh_d2(va), a01 = ldsh_d2(va + 16u), a2 = ldsh_d2(va + 32u);
                const bool miss = Sent<T>::is(x0) | Sent<T>::is(x1) | Sent<T>::is(x2);
                if (__any_sync(0xffffffffu, miss)) {
                    FetchWait w{0u, limit};
                    while ((Sent<T>::is(x0) | Sent<T>::is(x1) | Sent<T>::is(x2)) && !*cerr) {
                        if (!w.tick(st, cerr, row)) *cerr = 1;
                        x0 = Sh<T>::ldu(SL + S * (unsigned int)rec.y);
                        x1 = Sh<T>::ldu(SL + S * (unsigned int)rec.z);
                        x2 = Sh<T>::ldu(SL + S * (unsigned int)rec.w);
                    }
                }
                double sum = 0.0;
                sum = __dadd_rn(sum, __dmul_rn(x0, a01.x));
                sum = __dadd_rn(sum, __dmul_rn(x1, a01.y));
                sum = __dadd_rn(sum, __dmul_rn(x2, a2.x));
                if constexpr (DIV == 2)
                    o = __ddiv_rn(__dsub_rn(rhs, sum), dr.x);
                else
                    o = div_fast(__dsub_rn(rhs, sum), dr.x, dr.y, slow);
            } else {
                const float4 v = ldsh_f4(va);
                const bool miss = Sent<T>::is(x0) | Sent<T>::is(x1) | Sent<T>::is(x2);
                if (__any_sync(0xffffffffu, miss)) {
                    FetchWait w{0u, limit};
                    while ((Sent<T>::is(x0) | Sent<T>::is(x1) | Sent<T>::is(x2)) && !*cerr) {
                        if (!w.tick(st, cerr, row)) *cerr = 1;
                        x0 = Sh<T>::ldu(SL + S * (unsigned int)rec.y);
                        x1 = Sh<T>::ldu(SL + S * (unsigned int)rec.z);
                        x2 = Sh<T>::ldu(SL + S * (unsigned int)rec.w);
                    }
                }
                float sum = 0.0f;
                sum = fmaf(x0, v.y, sum);
                sum = fmaf(x1, v.z, sum);
                sum = fmaf(x2, v.w, sum);
                o = (rhs - sum) * v.x;
            }
            // a warp past the step's rows computed a copy of the last row and stores nothing:
            // another warp may already have replaced that row's right-hand side by its result
            if ((tid & ~31) < nl) {
                Sh<T>::stu(ko, o);
                Sent<T>::store(xg + row, o);
            }
        }
        row = Sh<int>::ldu(RW + 4u * (unsigned int)recn.x);
        rec = recn;
        stp = stn;
        bar_compute(ncomp);
    }
}

// Slot reset before a pass: the zero slot to -0, both directions' staging slots to the sentinel.
// nrows: this CTA's rows; nst: its staging slots (both directions). All threads take part.
template <typename T>
__device__ __forceinline__ void fetch_reset_slots(unsigned int SL, int nrows, int nst) {
    constexpr unsigned int S = sizeof(T);
    for (int k = (int)threadIdx.x; k <= nst; k += blockDim.x)
        Sh<T>::stu(SL + S * (unsigned int)(nrows + k), k == 0 ? T(-0.0) : Sent<T>::value());
}

// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from global memory
// into shared memory, completing on `bar`, whose phase the issuing thread has armed with
// mbar_expect_tx for all of the phase's bytes. The issuing thread calls fence_async_shared()
// first, after its own and (through a barrier) every other thread's last reads of dst.
__device__ __forceinline__ void fetch_copy(unsigned int dst, const void *src, unsigned int bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Values of a direction's records from the factor lu (positions in A; FP64: {diag, div_recip(diag),
// a0, a1, a2, 0}; FP32: {1/diag, a0, a1, a2} rounded from FP64) or from the caller's triangular
// values (codeT). This CTA's records only.
template <typename T>
__device__ __forceinline__ void fetch_pack(const FetchDir &D, const int *code, const double *src, T *gv) {
    const int4 cb = __ldg(D.cblk + blockIdx.x);
    const int rb = cb.w, nr = __ldg(D.cblk + blockIdx.x + 1).w - rb;
    for (int k = (int)threadIdx.x; k < nr; k += blockDim.x) {
        const int4 c4 = __ldg(reinterpret_cast<const int4 *>(code) + rb + k);
        const double dg = Sent<double>::load(src + c4.x);
        const double a0 = c4.y >= 0 ? Sent<double>::load(src + c4.y) : 0.0;
        const double a1 = c4.z >= 0 ? Sent<double>::load(src + c4.z) : 0.0;
        const double a2 = c4.w >= 0 ? Sent<double>::load(src + c4.w) : 0.0;
        if constexpr (sizeof(T) == 8) {
            double *g = reinterpret_cast<double *>(gv) + (size_t)(rb + k) * kFetchVal64;
            g[0] = dg;
            g[1] = div_recip(dg);
            g[2] = a0;
            g[3] = a1;
            g[4] = a2;
            g[5] = 0.0;
        } else {
            float *g = reinterpret_cast<float *>(gv) + (size_t)(rb + k) * kFetchVal32;
            g[0] = __frcp_rn(__double2float_rn(dg));
            g[1] = __double2float_rn(a0);
            g[2] = __double2float_rn(a1);
            g[3] = __double2float_rn(a2);
        }
    }
}

// IC0 on the lower fetch plan, for patterns in which no entry's dot product has a column match
// (the 5- and 7-point stencils): row i's entry (i, j) is then l_ij = a_ij / l_jj and its diagonal
// l_ii = sqrt(a_ii - sum_j l_ij^2) (merge/IC.cpp:296-393 with an empty sparse_dot_product;
// a_ij - 0.0 is a_ij bit for bit, so that subtraction is left out), the same correctly rounded
// operations in the same order as k_factor_part. A row needs only its dependencies' final
// diagonals, so the walk passes l_jj where the sweeps pass x_j: the row's own slot and dg[row]
// (its ready flag for other CTAs) receive l_ii. A non-positive pivot leaves a_ii in place (and is
// counted once per row), as the reference does. Absent entries read the zero slot, which holds
// +1 here: 0 / 1 = +0 adds +0 to the sum of squares, which starts at +0 and never becomes -0.
// V holds the records' A values in the FP64 record layout {a_ii, -, a0, a1, a2, -}; code are the
// records' A positions (global; the lu writes), rec0 the CTA's first record.
__device__ __forceinline__ void walk_ic0_fetch(unsigned int I, unsigned int V, unsigned int SL, unsigned int RW, int ns,
                                               int ncomp, double *dg, double *lu, const int4 *__restrict__ code,
                                               int rec0, unsigned int limit, DevStatus *st, FetchCtl *ctl) {
    constexpr unsigned int S = 8u, RB = 8u * kFetchVal64;
    if (ns == 0) return;
    const int tid = (int)threadIdx.x;
    const unsigned int R0 = I + 16u * (unsigned int)(ns + 2);
    volatile int *cerr = &ctl->err;
    int4 stp = ldsh4(I);
    int4 rec = ldsh4(R0 + 16u * (unsigned int)(stp.x + min(tid, stp.y - 1)));
    int row = Sh<int>::ldu(RW + 4u * (unsigned int)rec.x);
    int4 cd = __ldg(code + rec0 + stp.x + min(tid, stp.y - 1));
    for (int s = 0; s < ns; s++) {
        const int4 stn = ldsh4(I + 16u * (unsigned int)(s + 1));
        const int nl = stp.y;
        const int q = min(tid, nl - 1);
        const unsigned int va = V + RB * (unsigned int)(stp.x + q);
        const unsigned int ko = SL + S * (unsigned int)rec.x;
        double x0 = Sh<double>::ldu(SL + S * (unsigned int)rec.y);
        double x1 = Sh<double>::ldu(SL + S * (unsigned int)rec.z);
        double x2 = Sh<double>::ldu(SL + S * (unsigned int)rec.w);
        const int4 recn = ldsh4(R0 + 16u * (unsigned int)(stn.x + min(tid, stn.y - 1)));
        const int4 cdn = __ldg(code + rec0 + stn.x + min(tid, stn.y - 1));
        const double2 d0 = ldsh_d2(va), a01 = ldsh_d2(va + 16u), a2 = ldsh_d2(va + 32u);
        const bool miss = Sent<double>::is(x0) | Sent<double>::is(x1) | Sent<double>::is(x2);
        if (__any_sync(0xffffffffu, miss)) {
            FetchWait w{0u, limit};
            while ((Sent<double>::is(x0) | Sent<double>::is(x1) | Sent<double>::is(x2)) && !*cerr) {
                if (!w.tick(st, cerr, row)) *cerr = 1;
                x0 = Sh<double>::ldu(SL + S * (unsigned int)rec.y);
                x1 = Sh<double>::ldu(SL + S * (unsigned int)rec.z);
                x2 = Sh<double>::ldu(SL + S * (unsigned int)rec.w);
            }
        }
        const double v0 = __ddiv_rn(a01.x, x0), v1 = __ddiv_rn(a01.y, x1), v2 = __ddiv_rn(a2.x, x2);
        double dv = 0.0;
        dv = __dadd_rn(dv, __dmul_rn(v0, v0));
        dv = __dadd_rn(dv, __dmul_rn(v1, v1));
        dv = __dadd_rn(dv, __dmul_rn(v2, v2));
        const double t = __dsub_rn(d0.x, dv);
        const bool pos = t > 0.0;
        const double lii = pos ? __dsqrt_rn(t) : d0.x;
        if ((tid & ~31) < nl) {  // a warp wholly past the step's rows stores nothing
            Sh<double>::stu(ko, lii);
            if (cd.y >= 0) lu[cd.y] = v0;
            if (cd.z >= 0) lu[cd.z] = v1;
            if (cd.w >= 0) lu[cd.w] = v2;
            lu[cd.x] = lii;
            Sent<double>::store(dg + row, lii);
            if (!pos && tid < nl) atomicAdd(&st->zero_pivots, 1);
        }
        row = Sh<int>::ldu(RW + 4u * (unsigned int)recn.x);
        rec = recn;
        stp = stn;
        cd = cdn;
        bar_compute(ncomp);
    }
}

}  // namespace baas
