// Chunked, shared-memory-staged, step-synchronous sweeps: the production triangular sweeps.
//
// Each CTA owns a set of rows (part_kernels.cuh explains the partition and why it is
// deadlock-free). The CTA walks the schedule's group levels in the global order. A level whose
// groups hold up to m rows is split into m steps; step j holds the j-th row of every group of
// the level, so the rows of a group (a tree coarsened by the reference, merge/Coarsen.cpp:
// 73-403) still run in their order, separated by a CTA barrier. Inside a step, row k belongs to
// thread k (k, k + blockDim, ... when a step is wider than the CTA).
//
// The plan of a step is a self-contained CHUNK (a wide step is cut into several):
//   int block   [nl, E, 0, 0 | rowid (nl) | slot (nl) | ne (nl) | dep (nl*E)], padded to 8 ints
//   value block [diag (nl) | val (nl*E)], padded to 4 values
// with E the widest row of the CTA (one stride for all of a CTA's chunks, so the walk is
// specialised on it once per window), and row `pos` finds its entries at pos*E + j.
// dep >= 0 is a CTA-local slot (final after the barrier that ended the producing step); dep < 0
// is -(row+1) of a row owned by another CTA (a value-as-flag wait on its global slot). The
// slot of a row is its position in the CTA's lower-sweep order; the lower and the upper sweep
// use the same slots, so the upper sweep finds its right-hand side (the lower result) in place.
//
// A CTA's chunks are contiguous in global memory. Consecutive chunks are grouped into WINDOWS
// that fit one of two shared-memory buffers; a window arrives through two bulk copies (ints,
// values) issued by one thread and completes on an mbarrier, so the copy of window k+1 (or of the
// next sweep's first windows) overlaps the walk of window k. When all of a CTA's windows fit the
// two buffers they are copied once and stay resident. Solution slots (one value per row and
// right-hand side) sit in front of the buffers.
#pragma once

#include "device_common.cuh"
#include "part_kernels.cuh"

namespace baas {

constexpr int kStageBlock = 512;
constexpr int kChunkHdr = 4;
constexpr int kIssuer = kStageBlock - 32;  // lane 0 of the last warp issues the bulk copies
constexpr int kMaxRhs = 8;                 // right-hand sides walked together

__host__ __device__ constexpr int pad4(int x) { return (x + 3) & ~3; }
__host__ __device__ constexpr int pad8(int x) { return (x + 7) & ~7; }
__host__ __device__ constexpr int chunk_nint(int nl, int E) { return pad8(kChunkHdr + 3 * nl + nl * E); }
__host__ __device__ constexpr int chunk_nval(int nl, int E) { return pad4(nl + nl * E); }
// value-source code of a diagonal entry at position p (off-diagonals: p >= 0; padding: -1)
__host__ __device__ constexpr int diag_code(int p) { return -2 - p; }

struct ChunkDir {
    const int *ints;           // chunk int blocks, CTA by CTA
    const int *vsrcT, *vsrcA;  // per value slot: source position in the caller's CSR / in A
    const int *cval;           // P + 1: value slots of each CTA
    const int4 *swrec;         // windows: {int offset, ints, value offset, values}
    const int *swptr;          // P + 1: windows of each CTA
};

struct ChunkPlan {
    int P;
    ChunkDir dir[2];
    const int *soff;  // P + 1: slots of each CTA
    const int *srow;  // row of each slot, CTA by CTA
    int xs_bytes;     // shared-memory bytes of the solution slots
    int cap;          // bytes of each window buffer
    int nrec;         // most windows of one CTA, both directions together
};

// shared memory: [slots | buffer 0 | buffer 1 | stream control block with the CTA's window
// records]; nrec = the most windows one CTA has (both directions)
struct WinCtl {
    unsigned long long mbar[2];
    int nint[2];              // int count of the window in each buffer
    const int *ints0, *ints1; // chunk int blocks of the first / second direction
    const void *vals0, *vals1;
    int n0, n1;               // windows of this CTA in each direction
    unsigned int limit;       // no copy is issued for sequence numbers >= limit
    int resident;             // all windows fit the two buffers: copied once
    int4 rec[1];              // n0 + n1 window records {int offset, ints, value offset, values}
};
__host__ __device__ constexpr int win_ctl_bytes(int nrec) { return 128 + 16 * nrec; }
__host__ __device__ constexpr int chunk_smem_bytes(int xs_bytes, int cap, int nrec) {
    return xs_bytes + 2 * cap + win_ctl_bytes(nrec);
}

// Value of source code s in array v (the packing of a window's value slots).
template <typename V>
__device__ __forceinline__ double src_value(const V *v, int s) {
    return s >= 0 ? (double)v[s] : (s <= -2 ? (double)v[-2 - s] : 0.0);
}

// The stream of windows one CTA walks: the windows of direction `first`, then (two_dirs)
// those of direction 1, pass after pass. Its configuration sits in shared memory; every thread
// holds the same two counters; one thread issues the copies.
template <typename T>
struct WinStream {
    WinCtl *ctl;
    unsigned char *buf;
    int cap;
    unsigned int issued, consumed;  // sequence numbers
    bool loaded;

    __device__ void init(const ChunkPlan &pl, int first, bool two_dirs, const T *v0, const T *v1, unsigned char *smem,
                         unsigned int lim) {
        const int c = blockIdx.x;
        cap = pl.cap;
        buf = smem + pl.xs_bytes;
        ctl = reinterpret_cast<WinCtl *>(smem + pl.xs_bytes + 2 * pl.cap);
        issued = consumed = 0;
        loaded = false;
        const ChunkDir &A = first ? pl.dir[1] : pl.dir[0];
        const int q0 = __ldg(A.swptr + c), n0 = __ldg(A.swptr + c + 1) - q0;
        const int q1 = two_dirs ? __ldg(pl.dir[1].swptr + c) : 0;
        const int n1 = two_dirs ? __ldg(pl.dir[1].swptr + c + 1) - q1 : 0;
        if (threadIdx.x == 0) {
            ctl->ints0 = A.ints;
            ctl->ints1 = pl.dir[1].ints;
            ctl->vals0 = v0;
            ctl->vals1 = v1;
            ctl->n0 = n0;
            ctl->n1 = n1;
            ctl->limit = lim;
            ctl->resident = n0 + n1 <= 2;
            mbar_init(&ctl->mbar[0], 1);
            mbar_init(&ctl->mbar[1], 1);
            fence_mbar_init();
        }
        for (int i = threadIdx.x; i < n0 + n1; i += blockDim.x)
            ctl->rec[i] = i < n0 ? __ldg(A.swrec + q0 + i) : __ldg(pl.dir[1].swrec + q1 + (i - n0));
        __syncthreads();
    }
    __device__ int total() const { return ctl->n0 + ctl->n1; }

    // Issues the copy of sequence number `issued` into buffer issued % 2. All threads call it.
    __device__ void issue_next() {
        if (threadIdx.x == kIssuer) {
            const int i = (int)(issued % (unsigned int)total());
            const int4 r = ctl->rec[i];
            const bool second = i >= ctl->n0;
            const unsigned int b = issued & 1u;
            unsigned char *dst = buf + b * cap;
            const unsigned int ib = (unsigned int)r.y * 4u, vb = (unsigned int)r.w * (unsigned int)sizeof(T);
            ctl->nint[b] = r.y;
            fence_async_shared();
            mbar_expect_tx(&ctl->mbar[b], ib + vb);
            bulk_g2s(dst, (second ? ctl->ints1 : ctl->ints0) + r.x, ib, &ctl->mbar[b]);
            bulk_g2s(dst + ib, static_cast<const T *>(second ? ctl->vals1 : ctl->vals0) + r.z, vb, &ctl->mbar[b]);
        }
        issued++;
    }
    // Item i of the current pass: waits for its window and returns the buffer holding it.
    // False (uniformly for the CTA) if the wait gave up.
    __device__ bool acquire(int i, unsigned int spin, DevStatus *st, const unsigned char *&b, int &nint) {
        unsigned int s;
        bool ok = true;
        if (ctl->resident) {
            s = (unsigned int)i;
            if (!loaded) {
                if (i == 0)
                    while (issued < (unsigned int)total() && issued < ctl->limit) issue_next();
                ok = mbar_wait(&ctl->mbar[s & 1u], (s >> 1) & 1u, spin);
            }
        } else {
            s = consumed;
            while (issued < s + 2u && issued < ctl->limit) issue_next();
            ok = mbar_wait(&ctl->mbar[s & 1u], (s >> 1) & 1u, spin);
        }
        if (!ok && atomicCAS(&st->code, kOk, kTimeout) == kOk) st->where = -1000000 - (int)s;
        if (__syncthreads_or(!ok)) return false;
        b = buf + (s & 1u) * cap;
        nint = ctl->nint[s & 1u];
        return true;
    }
    // After the walk of item i (which ended with a CTA barrier): refill its buffer.
    __device__ void release(int i) {
        if (ctl->resident) {
            if (i == total() - 1) loaded = true;
            return;
        }
        consumed++;
        while (issued < consumed + 2u && issued < ctl->limit) issue_next();
    }
    // Wait (bounded) for copies still in flight, before the CTA exits.
    __device__ void drain(unsigned int spin) {
        const unsigned int from = ctl->resident ? (loaded ? issued : 0u) : consumed;
        for (unsigned int s = from; s < issued; s++) mbar_wait(&ctl->mbar[s & 1u], (s >> 1) & 1u, spin);
        __syncthreads();
    }
};

// The plan of one row of a chunk, loaded into registers before the barrier that precedes its
// step (the plan is read-only; only the solution slots change from step to step).
template <typename T, int EK>
struct RowPlan {
    int row, sl, ne;
    int d[EK];
    T a[EK];
    T diag;
};

template <typename T, int EK>
__device__ __forceinline__ void load_row(const int *I, const T *V, int nl, int pos, RowPlan<T, EK> &p) {
    const int *rowid = I + kChunkHdr;
    p.row = rowid[pos];
    p.sl = rowid[nl + pos];
    p.ne = rowid[2 * nl + pos];
    const int *dp = rowid + 3 * nl + pos * EK;
    const T *vp = V + nl + pos * EK;
#pragma unroll
    for (int j = 0; j < EK; j++) {
        p.d[j] = dp[j];
        p.a[j] = vp[j];
    }
    p.diag = V[pos];
}

// Loads of the row's remote dependencies (their values, or the sentinel if not yet written);
// issued before the barrier, they complete while the CTA waits at it.
template <typename T, int EK>
__device__ __forceinline__ void load_remote(const RowPlan<T, EK> &p, const T *xg, T (&pf)[EK]) {
#pragma unroll
    for (int j = 0; j < EK; j++) pf[j] = (j < p.ne && p.d[j] < 0) ? Sent<T>::load(xg + (-p.d[j] - 1)) : T(0);
}

// One row: dependency values gathered without branches (local slot, or the prefetched remote
// value), one sentinel test for the whole row, and a wait only for a remote value that was not
// yet written when it was prefetched. EXACT: the reference's FP64 operation order with correctly
// rounded operations; else FP32 with 1/diag.
template <typename T, bool EXACT, int EK>
__device__ __forceinline__ bool row_compute(const RowPlan<T, EK> &p, const T (&pf)[EK], const T *xs, const T *xg,
                                            Waiter &w, T &out) {
    T xv[EK];
    bool miss = false;
#pragma unroll
    for (int j = 0; j < EK; j++) {
        const int dj = p.d[j];
        const T loc = xs[dj >= 0 ? dj : 0];
        xv[j] = dj >= 0 ? loc : pf[j];
        miss |= j < p.ne && Sent<T>::is(xv[j]);
    }
    if (miss) {
#pragma unroll
        for (int j = 0; j < EK; j++)
            if (j < p.ne && p.d[j] < 0 && Sent<T>::is(xv[j]) && !wait_value<T>(xg + (-p.d[j] - 1), xv[j], w, -p.d[j] - 1))
                return false;
    }
    T sum = T(0);
#pragma unroll
    for (int j = 0; j < EK; j++)
        if (j < p.ne) {
            if constexpr (EXACT)
                sum = __dadd_rn(sum, __dmul_rn(xv[j], p.a[j]));
            else
                sum = fmaf(xv[j], p.a[j], sum);
        }
    const T rhs = xs[p.sl];
    if constexpr (EXACT)
        out = __ddiv_rn(__dsub_rn(rhs, sum), p.diag);
    else
        out = (rhs - sum) * p.diag;  // FP32 value blocks hold 1/diag
    return true;
}

// Walk one window whose chunks all have entry stride EK (1..4). Thread t owns row t of every
// chunk (rows beyond the block width loop, without prefetch); its next row's plan and remote
// values are loaded before each barrier.
template <typename T, bool EXACT, int EK>
__device__ __forceinline__ bool walk_window_e(const int *I, const int *Iend, const T *V, T *xs, T *xg, Waiter &w,
                                              bool alive) {
    const int tid = threadIdx.x;
    int nl = I[0];
    RowPlan<T, EK> rp;
    T pf[EK];
    bool mine = tid < nl;
    if (mine) {
        load_row<T, EK>(I, V, nl, tid, rp);
        load_remote<T, EK>(rp, xg, pf);
    }
    for (;;) {
        if (alive && mine) {
            T out;
            if (row_compute<T, EXACT, EK>(rp, pf, xs, xg, w, out)) {
                xs[rp.sl] = out;
                Sent<T>::store(xg + rp.row, out);
            } else {
                alive = false;
            }
        }
        for (int pos = tid + (int)blockDim.x; alive && pos < nl; pos += blockDim.x) {
            RowPlan<T, EK> q;
            T qf[EK];
            load_row<T, EK>(I, V, nl, pos, q);
#pragma unroll
            for (int j = 0; j < EK; j++) qf[j] = Sent<T>::value();
            T out;
            if (!row_compute<T, EXACT, EK>(q, qf, xs, xg, w, out)) {
                alive = false;
                break;
            }
            xs[q.sl] = out;
            Sent<T>::store(xg + q.row, out);
        }
        const int *In = I + chunk_nint(nl, EK);
        const T *Vn = V + chunk_nval(nl, EK);
        const int nln = In < Iend ? In[0] : 0;
        mine = tid < nln;
        if (mine) {
            load_row<T, EK>(In, Vn, nln, tid, rp);
            if (alive) load_remote<T, EK>(rp, xg, pf);
        }
        __syncthreads();
        if (In >= Iend) break;
        I = In;
        V = Vn;
        nl = nln;
    }
    return alive;
}

// Any entry stride (the CTA's widest row has more than 4 entries): plain loop, waits in place.
template <typename T, bool EXACT>
__device__ __forceinline__ bool walk_window_any(const int *I, const int *Iend, const T *V, T *xs, T *xg, Waiter &w,
                                                bool alive) {
    while (I < Iend) {
        const int nl = I[0], E = I[1];
        const int *rowid = I + kChunkHdr, *slot = rowid + nl, *ne = slot + nl, *dep = ne + nl;
        const T *diag = V, *val = V + nl;
        for (int pos = threadIdx.x; alive && pos < nl; pos += blockDim.x) {
            T sum = T(0);
            for (int j = 0; j < ne[pos]; j++) {
                const int d = dep[pos * E + j];
                T xv;
                if (d >= 0) {
                    xv = xs[d];
                } else if (!wait_value<T>(xg + (-d - 1), xv, w, -d - 1)) {
                    alive = false;
                    break;
                }
                if constexpr (EXACT)
                    sum = __dadd_rn(sum, __dmul_rn(xv, val[pos * E + j]));
                else
                    sum = fmaf(xv, val[pos * E + j], sum);
            }
            if (!alive) break;
            const int sl = slot[pos];
            T out;
            if constexpr (EXACT)
                out = __ddiv_rn(__dsub_rn(xs[sl], sum), diag[pos]);
            else
                out = (xs[sl] - sum) * diag[pos];
            xs[sl] = out;
            Sent<T>::store(xg + rowid[pos], out);
        }
        I += chunk_nint(nl, E);
        V += chunk_nval(nl, E);
        __syncthreads();
    }
    return alive;
}

// Walk one window (nint ints of chunk blocks, then their values) held in shared memory. All
// chunks of a CTA share one entry stride. Every thread passes every barrier, also after a
// failed wait, so the CTA never splits.
template <typename T, bool EXACT>
__device__ __forceinline__ bool walk_window(const unsigned char *b, int nint, T *xs, T *xg, Waiter &w, bool alive) {
    const int *I = reinterpret_cast<const int *>(b);
    const int *Iend = I + nint;
    const T *V = reinterpret_cast<const T *>(b + (size_t)nint * 4);
    switch (I[1]) {
        case 1: return walk_window_e<T, EXACT, 1>(I, Iend, V, xs, xg, w, alive);
        case 2: return walk_window_e<T, EXACT, 2>(I, Iend, V, xs, xg, w, alive);
        case 3: return walk_window_e<T, EXACT, 3>(I, Iend, V, xs, xg, w, alive);
        case 4: return walk_window_e<T, EXACT, 4>(I, Iend, V, xs, xg, w, alive);
        default: return walk_window_any<T, EXACT>(I, Iend, V, xs, xg, w, alive);
    }
}

// Multi-right-hand-side walk (R <= kMaxRhs, runtime): slots hold R values per row
// (xs[slot*R + r]); right-hand side r of row `row` lives at xg[r*ldx + row]. FP64, exact.
__device__ __forceinline__ bool walk_window_multi(const unsigned char *b, int nint, double *xs, double *xg, int ldx, int R,
                                                  Waiter &w, bool alive) {
    const int *I = reinterpret_cast<const int *>(b);
    const int *Iend = I + nint;
    const double *V = reinterpret_cast<const double *>(b + (size_t)nint * 4);
    while (I < Iend) {
        const int nl = I[0], E = I[1];
        const int *rowid = I + kChunkHdr, *slot = rowid + nl, *ne = slot + nl, *dep = ne + nl;
        const double *diag = V, *val = V + nl;
        for (int pos = threadIdx.x; pos < nl && alive; pos += blockDim.x) {
            double sum[kMaxRhs];
#pragma unroll
            for (int r = 0; r < kMaxRhs; r++) sum[r] = 0.0;
            const int n_ = ne[pos];
            for (int j = 0; j < n_ && alive; j++) {
                const int d = dep[pos * E + j];
                const double a = val[pos * E + j];
#pragma unroll
                for (int r = 0; r < kMaxRhs; r++)
                    if (r < R) {
                        double xv = 0.0;
                        if (d >= 0)
                            xv = xs[d * R + r];
                        else if (alive && !wait_value<double>(xg + (size_t)r * ldx + (-d - 1), xv, w, -d - 1))
                            alive = false;
                        sum[r] = __dadd_rn(sum[r], __dmul_rn(xv, a));
                    }
            }
            if (!alive) break;
            const int sl = slot[pos], row = rowid[pos];
#pragma unroll
            for (int r = 0; r < kMaxRhs; r++)
                if (r < R) {
                    const double out = __ddiv_rn(__dsub_rn(xs[sl * R + r], sum[r]), diag[pos]);
                    xs[sl * R + r] = out;
                    Sent<double>::store(xg + (size_t)r * ldx + row, out);
                }
        }
        I += chunk_nint(nl, E);
        V += chunk_nval(nl, E);
        __syncthreads();
    }
    return alive;
}

// Standalone FP64 sweep of the caller's triangular CSR (values gathered through vsrcT into the
// packed scratch gv), right-hand sides R at a time. d = 0: lower (L), 1: upper (U = L^T).
template <bool MULTI>
__global__ void __launch_bounds__(kStageBlock, 1) k_sweep_chunked(ChunkPlan pl, int d, const double *__restrict__ tval,
                                                                 double *gv, const double *__restrict__ b, int ldb,
                                                                 double *x, int ldx, int nrhs, int R, DevStatus *st,
                                                                 unsigned int spin, unsigned long long *trace) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int c = blockIdx.x;
    Waiter w(spin, st);
    trace_mark(trace, 0);
    {
        const ChunkDir &D = d ? pl.dir[1] : pl.dir[0];
        const int vb = __ldg(D.cval + c), ve = __ldg(D.cval + c + 1);
        for (int i = vb + (int)threadIdx.x; i < ve; i += blockDim.x) gv[i] = src_value(tval, __ldg(D.vsrcT + i));
        fence_async_global();
    }
    const int npass = (nrhs + R - 1) / R;
    WinStream<double> ws;
    {
        const ChunkDir &D = d ? pl.dir[1] : pl.dir[0];
        ws.init(pl, d, false, gv, gv, smem, (unsigned int)(npass * (__ldg(D.swptr + c + 1) - __ldg(D.swptr + c))));
    }
    trace_mark(trace, 1);
    double *xs = reinterpret_cast<double *>(smem);
    const int s0 = __ldg(pl.soff + c), nl = __ldg(pl.soff + c + 1) - s0;
    const int *srow = pl.srow + s0;
    for (int r0 = 0; r0 < nrhs; r0 += R) {
        const int Rb = min(R, nrhs - r0);
        for (int k = threadIdx.x; k < nl * Rb; k += blockDim.x) {
            const int sl = k / Rb, r = k - sl * Rb;
            xs[k] = __ldg(b + (size_t)(r0 + r) * ldb + __ldg(srow + sl));
        }
        __syncthreads();
        trace_mark(trace, 2 + 2 * (r0 / R));
        bool alive = true;
        for (int i = 0; i < ws.total(); i++) {
            const unsigned char *buf;
            int nint;
            if (!ws.acquire(i, spin, st, buf, nint)) {
                ws.drain(spin);
                return;
            }
            if (MULTI)
                alive = walk_window_multi(buf, nint, xs, x + (size_t)r0 * ldx, ldx, Rb, w, alive);
            else
                alive = walk_window<double, true>(buf, nint, xs, x + (size_t)r0 * ldx, w, alive);
            ws.release(i);
            if (__syncthreads_or(!alive)) {
                ws.drain(spin);
                return;
            }
        }
        trace_mark(trace, 3 + 2 * (r0 / R));
    }
    ws.drain(spin);
}

// ---------------------------------------------------------------------------------------
// Persistent ICCG: IC0 (level-synchronous, part_kernels.cuh), packing of L and U = L^T into
// the chunk value slots, and the pcg_opt loop (test/iccg_level_merge.cpp:380-533, break at
// tol) in one cooperative launch of P CTAs.
// ---------------------------------------------------------------------------------------
struct IccgArgs {
    int n;
    const int *a_rowptr, *a_colidx, *a_diag;
    const double *a_val;
    const double *b;
    double *x;
    PartView fac;     // level plan of the factorisation
    ChunkPlan pl;     // chunked sweep plan (dir 0: L, dir 1: U = L^T)
    double *gv64[2];  // packed FP64 value slots, per direction
    float *gv32[2];   // packed FP32 value slots (1/diag on the diagonal), per direction
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
    int reuse;         // 1: the value slots already hold the factors (adjoint solves)
    const double *xf;  // with grad_a: the forward solution x
    double *grad_a;    // if set: grad_a[e] = -x_i * xf_j for each entry e = (i, j) of A
};

// z = U^-1 L^-1 r on this CTA's rows; p = z if set_p; adds this thread's share of r.z to rz
// (a pass over the CTA's slots after the upper walk, which leaves z in them).
template <typename T>
__device__ bool chunk_precond(const IccgArgs &A, WinStream<T> &ws, T *xs, bool set_p, double &rz, Waiter &w) {
    const int c = blockIdx.x;
    T *yg = sizeof(T) == 8 ? (T *)A.y : (T *)A.y32;
    T *zg = sizeof(T) == 8 ? (T *)A.z : (T *)A.z32;
    const int s0 = __ldg(A.pl.soff + c), nl = __ldg(A.pl.soff + c + 1) - s0;
    for (int k = threadIdx.x; k < nl; k += blockDim.x) xs[k] = (T)A.r[__ldg(A.pl.srow + s0 + k)];
    __syncthreads();
    bool alive = true;
    trace_mark(A.trace, 56);
    for (int i = 0; i < ws.total(); i++) {
        const unsigned char *buf;
        int nint;
        if (!ws.acquire(i, A.spin_limit, A.st, buf, nint)) return false;
        const bool lower = i < ws.ctl->n0;
        alive = walk_window<T, sizeof(T) == 8>(buf, nint, xs, lower ? yg : zg, w, alive);
        if (lower && i == ws.ctl->n0 - 1) trace_mark(A.trace, 57);
        ws.release(i);
        if (__syncthreads_or(!alive)) return false;
    }
    for (int k = threadIdx.x; k < nl; k += blockDim.x) {
        const int row = __ldg(A.pl.srow + s0 + k);
        const double zd = (double)xs[k];
        rz = __dadd_rn(rz, __dmul_rn(A.r[row], zd));
        if (set_p) A.p[row] = zd;
    }
    trace_mark(A.trace, 59);
    return true;
}

// T = double: FP64 factors; T = float: FP32 factors (one instantiation each keeps the register
// budget of each variant to one precision).
template <typename T>
__global__ void __launch_bounds__(kStageBlock, 1) k_iccg_chunked(IccgArgs A) {
    constexpr bool kMixed = sizeof(T) == 4;
    extern __shared__ __align__(128) unsigned char smem[];
    const int n = A.n;
    const int W = gridDim.x * blockDim.x;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned int nb = 0;
    Waiter w(A.spin_limit, A.st);
    WinStream<T> ws;
    ws.init(A.pl, 0, true, kMixed ? (const T *)A.gv32[0] : (const T *)A.gv64[0],
            kMixed ? (const T *)A.gv32[1] : (const T *)A.gv64[1], smem, 0xFFFFFFFFu);
    T *xs = reinterpret_cast<T *>(smem);
#define BAAS_BARRIER()                                            \
    do {                                                          \
        if (!grid_barrier(A.bar, nb, A.st, A.spin_limit)) {       \
            ws.drain(A.spin_limit);                               \
            return;                                               \
        }                                                         \
    } while (0)

    trace_mark(A.trace, 0);
    if (!A.reuse) {
        const int nnz = __ldg(A.a_rowptr + n);
        for (int e = gt; e < nnz; e += W) A.lu[e] = A.a_val[e];
        BAAS_BARRIER();
        trace_mark(A.trace, 1);

        factor_part<false>(A.fac, A.a_rowptr, A.a_colidx, A.a_diag, A.lu, A.gflag, A.epoch, w, A.st);
        BAAS_BARRIER();
        trace_mark(A.trace, 2);

        // pack this CTA's value slots of L and U = L^T (IC0_preconditioner split,
        // test/iccg_level_merge.cpp:874-891)
        for (int d = 0; d < 2; d++) {
            const ChunkDir &D = A.pl.dir[d];
            const int vb = __ldg(D.cval + blockIdx.x), ve = __ldg(D.cval + blockIdx.x + 1);
            for (int i = vb + (int)threadIdx.x; i < ve; i += blockDim.x) {
                const int s = __ldg(D.vsrcA + i);
                const double v = s >= 0 ? ld_l2(A.lu + s) : (s <= -2 ? ld_l2(A.lu + (-2 - s)) : 0.0);
                if constexpr (kMixed)
                    A.gv32[d][i] = s <= -2 ? __frcp_rn(__double2float_rn(v)) : __double2float_rn(v);
                else
                    A.gv64[d][i] = v;
            }
        }
        fence_async_global();
    }
    // r = b - A x; sentinels
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
    const double norm0 = sqrt(grid_total<kStageBlock>(A.part_b, gridDim.x));
    trace_mark(A.trace, 3);

    double rzl = 0.0;
    if (!chunk_precond<T>(A, ws, xs, true, rzl, w)) {
        ws.drain(A.spin_limit);
        return;
    }
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
        if (!chunk_precond<T>(A, ws, xs, false, rzl, w)) {
            ws.drain(A.spin_limit);
            return;
        }
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
    if (A.grad_a) {
        // gradient on the sparsity pattern: dL/dA_ij = -lambda_i x_j (this launch solved for
        // lambda = A^-T dL/dx)
        BAAS_BARRIER();
        for (int i = gt; i < n; i += W) {
            const double li = -A.x[i];
            for (int e = __ldg(A.a_rowptr + i); e < __ldg(A.a_rowptr + i + 1); e++)
                A.grad_a[e] = __dmul_rn(li, __ldg(A.xf + __ldg(A.a_colidx + e)));
        }
    }
    ws.drain(A.spin_limit);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *A.out_iters = iters;
        *A.out_relres = rel;
    }
#undef BAAS_BARRIER
}

}  // namespace baas
