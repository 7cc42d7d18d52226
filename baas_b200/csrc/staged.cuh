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
//   int block   [nl, E, nl_next, 0 | rowid (nl) | slot (nl) | ne (nl) | kpos (nl) | dep (nl*E)],
//               padded to 8 ints
//   value block [diag (nl) | 1/diag (nl) | val (nl*E)], padded to 4 values
// with E the widest row of the CTA (one stride for all of a CTA's chunks, so the walk is
// specialised on it once per direction), and row `pos` finds its entries at pos*E + j.
// nl_next is the next chunk's row count (what the pipelined walk needs to address it early).
// dep >= 0 is a CTA-local solution slot (final after the barrier that ended the producing
// step); dep < 0 is -(row+1) of a row owned by another CTA (a value-as-flag wait on its global
// result). A row has a slot (slot >= 0) only while a later row of the same CTA still has to read
// it. kpos is the row's position in the CTA's row list: where its right-hand side sits when
// the CTA's right-hand sides are staged in shared memory (when they fit; else they come from
// global memory).
//
// A CTA's chunks are contiguous in global memory. Consecutive chunks are grouped into WINDOWS
// that fit one of two shared-memory buffers; a window arrives through two bulk copies (ints,
// values) issued by one thread and completes on an mbarrier, so the copy of window k+1 (or of the
// next sweep's first windows) overlaps the walk of window k. When all of a CTA's windows fit the
// two buffers they are copied once and stay resident. Solution slots (one value per row and
// right-hand side) sit in front of the buffers.
#pragma once

#include "device_common.cuh"
#include "fetch.cuh"
#include "part_kernels.cuh"

namespace baas {

// 256 threads: steps hold tens of rows per CTA, so more threads would only add idle warps to
// every step barrier; and the pipelined walk gets up to 255 registers.
constexpr int kStageBlock = 256;
static_assert(kStageBlock == kFetchBlock, "the fetch walk runs in the chunked kernels' CTAs");
// walks of the persistent ICCG kernel
constexpr int kWalkChunked = 0, kWalkFetch = 1, kWalkLevels = 2;
constexpr int kChunkHdr = 4;
constexpr int kIssuer = kStageBlock - 32;  // lane 0 of the last warp issues the bulk copies
constexpr int kMaxRhs = 8;                 // right-hand sides walked together

__host__ __device__ constexpr int pad4(int x) { return (x + 3) & ~3; }
__host__ __device__ constexpr int pad8(int x) { return (x + 7) & ~7; }
__host__ __device__ constexpr int chunk_nint(int nl, int E) { return pad8(kChunkHdr + 4 * nl + nl * E); }
__host__ __device__ constexpr int chunk_nval(int nl, int E) { return pad4(2 * nl + nl * E); }
// value-source codes: off-diagonal entry at position p: p; padding: -1; diagonal entry at p:
// -2 - p; the diagonal's correctly rounded reciprocal: kRcpBase + p (positions < 2^30)
constexpr int kRcpBase = -2147483647 - 1;
__host__ __device__ constexpr int diag_code(int p) { return -2 - p; }
__host__ __device__ constexpr int rcp_code(int p) { return kRcpBase + p; }

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
    int rhs_bytes;    // shared-memory bytes of the staged right-hand sides (0: read from global)
    int cap;          // bytes of each window buffer
    int nrec;         // most windows of one CTA, both directions together
};

// shared memory: [slots | staged right-hand sides | buffer 0 | buffer 1 | stream control block
// with the CTA's window records]; nrec = the most windows one CTA has (both directions)
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
__host__ __device__ constexpr int chunk_smem_bytes(int xs_bytes, int rhs_bytes, int cap, int nrec) {
    return xs_bytes + rhs_bytes + 2 * cap + win_ctl_bytes(nrec);
}

// Value of source code s in array v (the packing of a window's value slots); reciprocal slots
// hold div_recip of the diagonal.
template <typename V>
__device__ __forceinline__ double src_value(const V *v, int s) {
    if (s >= 0) return (double)v[s];
    if (s == -1) return 0.0;
    if (s < -(1 << 30)) {
        return div_recip((double)v[s - kRcpBase]);
    }
    return (double)v[-2 - s];
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
        buf = smem + pl.xs_bytes + pl.rhs_bytes;
        ctl = reinterpret_cast<WinCtl *>(buf + 2 * pl.cap);
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
    // The window after item i of the current pass, from one thread's view: waits (bounded) for its
    // copy without a CTA barrier; the caller makes the outcome uniform at its next barrier. The
    // buffer and size are returned also when the wait gave up (the caller then reads nothing).
    __device__ bool peek(int i, unsigned int spin, const unsigned char *&b, int &nint) {
        unsigned int s;
        bool ok = true;
        if (ctl->resident) {
            s = (unsigned int)(i + 1);
            if (!loaded) ok = mbar_wait(&ctl->mbar[s & 1u], (s >> 1) & 1u, spin);
        } else {
            s = consumed + 1u;
            ok = mbar_wait(&ctl->mbar[s & 1u], (s >> 1) & 1u, spin);
        }
        b = buf + (s & 1u) * cap;
        nint = ctl->rec[s % (unsigned int)total()].y;
        return ok;
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

// Where a walk finds its right-hand sides and puts its results, and which (row, right-hand
// side) pairs a thread computes. MR = false: one right-hand side, thread t takes rows t,
// t + blockDim, ... of every chunk. MR = true: thread t takes right-hand side t % R of rows
// t / R, t / R + stride, ... (stride = blockDim / R rows per pass). STG: the CTA's right-hand
// sides are staged in shared memory at rs[kpos * R + r], and each result is written back there.
template <typename T, typename RT, bool MR, bool STG>
struct WalkIO {
    T *xs;          // solution slots: xs[slot * R + r]
    T *xg;          // results, value-as-flag: xg[r * ldx + row]
    const RT *rhs;  // right-hand sides in global memory: rhs[r * ldr + row] (unless STG)
    T *rs;          // staged right-hand sides (STG)
    int ldx, ldr, R_;
    __device__ int R() const { return MR ? R_ : 1; }
    __device__ int stride() const { return MR ? (int)blockDim.x / R_ : (int)blockDim.x; }
    __device__ int rr() const { return MR ? (int)threadIdx.x % R_ : 0; }
    // this thread's first row of a chunk (a huge value: the thread is idle)
    __device__ int lane_row() const {
        if (!MR) return (int)threadIdx.x;
        return (int)threadIdx.x < stride() * R_ ? (int)threadIdx.x / R_ : 0x3fffffff;
    }
    __device__ T *out() const { return MR ? xg + (size_t)rr() * ldx : xg; }
    __device__ const RT *in() const { return MR ? rhs + (size_t)rr() * ldr : rhs; }
    __device__ int slot(int sl) const { return MR ? sl * R_ + rr() : sl; }
    // shared-window addresses of slot / staged entry k (as io.slot indexes them)
    __device__ unsigned int xs_at(int k) const { return smem_u32(xs) + (unsigned int)k * (unsigned int)sizeof(T); }
    __device__ unsigned int rs_at(int k) const { return smem_u32(rs) + (unsigned int)k * (unsigned int)sizeof(T); }
};

// Dependency indices, entry count, row and staging position of one row: loaded one step
// ahead, because the loads issued before the barrier need them.
template <int EK>
struct RowDeps {
    int row, ne, kpos;
    int d[EK];
};
// The rest of a row's plan and its right-hand side.
template <typename T, int EK>
struct RowVals {
    int sl;
    T a[EK];
    T diag, rcp, rhs;
};

// I, V: shared-window addresses of the chunk's int block and value block.
template <int EK>
__device__ __forceinline__ void load_deps(unsigned int I, int nl, int pos, RowDeps<EK> &p) {
    const unsigned int r = I + 4u * (unsigned int)(kChunkHdr + pos), n4 = 4u * (unsigned int)nl;
    p.row = Sh<int>::ldu(r);
    p.ne = Sh<int>::ldu(r + 2u * n4);
    p.kpos = Sh<int>::ldu(r + 3u * n4);
    const unsigned int dp = I + 4u * (unsigned int)(kChunkHdr + 4 * nl + pos * EK);
#pragma unroll
    for (int j = 0; j < EK; j++) p.d[j] = Sh<int>::ldu(dp + 4u * j);
}

// The rest of a row's plan, and its staged right-hand side (STG).
template <typename T, typename RT, bool RL2, bool MR, bool STG, int EK>
__device__ __forceinline__ void load_vals(unsigned int I, unsigned int V, int nl, int pos, const RowDeps<EK> &p,
                                          const WalkIO<T, RT, MR, STG> &io, RowVals<T, EK> &v) {
    constexpr unsigned int S = sizeof(T);
    v.sl = Sh<int>::ldu(I + 4u * (unsigned int)(kChunkHdr + nl + pos));
    const unsigned int vp = V + S * (unsigned int)(2 * nl + pos * EK);
#pragma unroll
    for (int j = 0; j < EK; j++) v.a[j] = Sh<T>::ldu(vp + S * j);
    v.diag = Sh<T>::ldu(V + S * (unsigned int)pos);
    if constexpr (sizeof(T) == 8) v.rcp = Sh<T>::ldu(V + S * (unsigned int)(nl + pos));
    if constexpr (STG) v.rhs = Sh<T>::ldu(io.rs_at(io.slot(p.kpos)));
}

// A row's right-hand side: staged in shared memory, or from global memory (RL2: written
// earlier in the same launch by this CTA, so read from L2, where those writes went).
template <typename T, typename RT, bool RL2, bool MR, bool STG>
__device__ __forceinline__ T load_rhs(int row, int kpos, const WalkIO<T, RT, MR, STG> &io) {
    if constexpr (STG) {
        return Sh<T>::ldu(io.rs_at(io.slot(kpos)));
    } else {
        const RT *src = io.in() + row;
        if constexpr (RL2)
            return (T)Sent<RT>::load(src);
        else
            return (T)*src;
    }
}

// Loads of the row's remote dependencies (their values, or the sentinel if not yet written);
// issued before a barrier, they complete while the CTA waits at it.
// One branch per row: a row with no remote dependency (most rows) issues nothing; a row with one
// loads every entry, pointing its local ones at its own (unused) result slot, so no entry needs
// a branch of its own.
template <typename T, typename RT, bool MR, bool STG, int EK>
__device__ __forceinline__ void load_remote(const RowDeps<EK> &p, const WalkIO<T, RT, MR, STG> &io, T (&pf)[EK]) {
    const T *xg = io.out();
    bool rem = false;
#pragma unroll
    for (int j = 0; j < EK; j++) rem |= j < p.ne && p.d[j] < 0;
    if (rem) {
#pragma unroll
        for (int j = 0; j < EK; j++) pf[j] = Sent<T>::load(xg + ((j < p.ne && p.d[j] < 0) ? -p.d[j] - 1 : p.row));
    }
}

// One row: dependency values gathered without branches (local slot, or the prefetched remote
// value), one sentinel test for the whole row, and a wait only for a remote value that was not
// yet written when it was prefetched. DIV != 0: the reference's FP64 operation order with
// correctly rounded operations, the division by div_fast (DIV == 1; a division outside its
// range marks the thread's Waiter and the launch is repeated with DIV == 2) or by __ddiv_rn
// (DIV == 2); DIV == 0: FP32 with 1/diag. Writes the slot (if a later row of the CTA reads it),
// the staged copy (STG) and the global result.
template <typename T, typename RT, bool MR, bool STG, int DIV, int EK>
__device__ __forceinline__ bool row_compute(const RowDeps<EK> &p, const RowVals<T, EK> &v, const T (&pf)[EK],
                                            const WalkIO<T, RT, MR, STG> &io, Waiter &w) {
    T *xg = io.out();
    T xv[EK];
    bool miss = false;
#pragma unroll
    for (int j = 0; j < EK; j++) {
        const int dj = p.d[j];
        const T loc = Sh<T>::ldu(io.xs_at(io.slot(dj >= 0 ? dj : 0)));
        xv[j] = dj >= 0 ? loc : pf[j];
        miss |= j < p.ne && dj < 0 && Sent<T>::is(pf[j]);
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
            if constexpr (DIV != 0)
                sum = __dadd_rn(sum, __dmul_rn(xv[j], v.a[j]));
            else
                sum = fmaf(xv[j], v.a[j], sum);
        }
    T o;
    if constexpr (DIV == 2)
        o = __ddiv_rn(__dsub_rn(v.rhs, sum), v.diag);
    else if constexpr (DIV == 1)
        o = div_fast(__dsub_rn(v.rhs, sum), v.diag, v.rcp, w.slow);
    else
        o = (v.rhs - sum) * v.diag;  // FP32 value blocks hold 1/diag
    if (v.sl >= 0) Sh<T>::stu(io.xs_at(io.slot(v.sl)), o);
    if constexpr (STG) Sh<T>::stu(io.rs_at(io.slot(p.kpos)), o);
    Sent<T>::store(xg + p.row, o);
    return true;
}

// Walk a direction's chunks with entry stride EK (1..3) from window item `i` (held in buf)
// through its last window, crossing windows without a break in the step pipeline. At the start
// of step s a thread issues the loads of its step-s+1 row's dependency indices; they complete
// while step s computes, so the loads of that row's remote values (and, without staging, of its
// right-hand side) go out before the barrier that ends step s without waiting. The rest of a
// row's plan is loaded after the barrier, together with its dependencies' slots. Rows beyond one
// pass of the block loop go without prefetch. When step s+1 opens the next window, its copy is
// awaited at the start of step s (it was issued a window earlier), the barrier ending step s also
// decides, for the whole CTA, whether every wait so far succeeded, and the window of step s is
// then released for refilling. Returns with `i` on the last window walked (not released).
template <typename T, typename RT, bool RL2, bool MR, bool STG, int DIV, int EK>
__device__ __forceinline__ bool walk_run_e(WinStream<T> &ws, int &i, const unsigned char *buf, int nint,
                                           const WalkIO<T, RT, MR, STG> &io, Waiter &w, unsigned int spin,
                                           DevStatus *st) {
    constexpr unsigned int S = sizeof(T);
    const int lr = io.lane_row(), stp = io.stride();
    unsigned int I0 = smem_u32(buf);
    unsigned int Iend = I0 + 4u * (unsigned int)nint;
    unsigned int V0 = Iend;  // the value blocks follow the int blocks
    bool alive = true;
    int nl0 = Sh<int>::ldu(I0);
    RowDeps<EK> q0, q1;
    T pf0[EK];
    T rhs0 = T(0), rhs1 = T(0);
    bool m0 = lr < nl0;
    if (m0) {
        load_deps<EK>(I0, nl0, lr, q0);
        load_remote<T, RT, MR, STG, EK>(q0, io, pf0);
        if constexpr (!STG) rhs0 = load_rhs<T, RT, RL2, MR, STG>(q0.row, q0.kpos, io);
    }
    for (;;) {
        const int nl1 = Sh<int>::ldu(I0 + 8u);  // 0 after the direction's last chunk
        unsigned int I1 = I0 + 4u * (unsigned int)chunk_nint(nl0, EK);
        unsigned int V1 = V0 + S * (unsigned int)chunk_nval(nl0, EK);
        unsigned int Iend1 = Iend;
        const bool cross = nl1 != 0 && I1 == Iend;  // uniform: step s+1 opens the next window
        bool okw = true;
        if (cross) {
            const unsigned char *nb;
            int nn;
            okw = ws.peek(i, spin, nb, nn);
            I1 = smem_u32(nb);
            Iend1 = I1 + 4u * (unsigned int)nn;
            V1 = Iend1;
        }
        const bool m1 = okw && lr < nl1;
        if (m1) load_deps<EK>(I1, nl1, lr, q1);
        if (alive && m0) {
            RowVals<T, EK> v;
            load_vals<T, RT, RL2, MR, STG, EK>(I0, V0, nl0, lr, q0, io, v);
            if constexpr (!STG) v.rhs = rhs0;
            if (!row_compute<T, RT, MR, STG, DIV, EK>(q0, v, pf0, io, w)) alive = false;
        }
        for (int pos = lr + stp; alive && pos < nl0; pos += stp) {
            RowDeps<EK> q;
            RowVals<T, EK> v;
            T qf[EK];
            load_deps<EK>(I0, nl0, pos, q);
            load_vals<T, RT, RL2, MR, STG, EK>(I0, V0, nl0, pos, q, io, v);
            if constexpr (!STG) v.rhs = load_rhs<T, RT, RL2, MR, STG>(q.row, q.kpos, io);
#pragma unroll
            for (int j = 0; j < EK; j++) qf[j] = Sent<T>::value();
            if (!row_compute<T, RT, MR, STG, DIV, EK>(q, v, qf, io, w)) alive = false;
        }
        if (m1 && alive) {
            load_remote<T, RT, MR, STG, EK>(q1, io, pf0);
            if constexpr (!STG) rhs1 = load_rhs<T, RT, RL2, MR, STG>(q1.row, q1.kpos, io);
        }
        if (cross) {
            if (!okw && atomicCAS(&st->code, kOk, kTimeout) == kOk) st->where = -1000000 - i - 1;
            if (__syncthreads_or(!okw || !alive)) return false;
            ws.release(i);
            i++;
            Iend = Iend1;
        } else {
            __syncthreads();
        }
        if (nl1 == 0) break;
        I0 = I1;
        V0 = V1;
        nl0 = nl1;
        m0 = m1;
        q0 = q1;
        rhs0 = rhs1;
    }
    return alive;
}

// ---------------------------------------------------------------------------------------
// Row-wide multi-right-hand-side walk (FP32 factors, RW = 2 or 4 right-hand sides, not staged):
// thread t takes rows t, t + blockDim, ... of every chunk with all RW right-hand sides. A row's
// plan is then read once instead of once per right-hand side, its RW solves are independent
// chains, and a chunk of up to blockDim rows is one pass instead of RW. The slot layout
// (xs[slot * RW + r]), the operations and so every result are those of the MR walk, which gives
// each (row, right-hand side) pair a thread of its own.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void sh_ldv(unsigned int a, float (&v)[4]) {
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]) : "r"(a));
}
__device__ __forceinline__ void sh_stv(unsigned int a, const float (&v)[4]) {
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(a), "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]));
}
__device__ __forceinline__ void sh_ldv(unsigned int a, float (&v)[2]) {
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v[0]), "=f"(v[1]) : "r"(a));
}
__device__ __forceinline__ void sh_stv(unsigned int a, const float (&v)[2]) {
    asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v[0]), "f"(v[1]));
}

template <typename RT, bool RL2, int RW>
__device__ __forceinline__ void load_rhs_rw(int row, const WalkIO<float, RT, true, false> &io, float (&rh)[RW]) {
#pragma unroll
    for (int r = 0; r < RW; r++) {
        const RT *src = io.rhs + (size_t)r * io.ldr + row;
        if constexpr (RL2)
            rh[r] = (float)Sent<RT>::load(src);
        else
            rh[r] = (float)*src;
    }
}

template <typename RT, int RW, int EK>
__device__ __forceinline__ void load_remote_rw(const RowDeps<EK> &p, const WalkIO<float, RT, true, false> &io,
                                               float (&pf)[RW][EK]) {
    bool rem = false;
#pragma unroll
    for (int j = 0; j < EK; j++) rem |= j < p.ne && p.d[j] < 0;
    if (rem) {
#pragma unroll
        for (int r = 0; r < RW; r++)
#pragma unroll
            for (int j = 0; j < EK; j++)
                pf[r][j] = Sent<float>::load(io.xg + (size_t)r * io.ldx + ((j < p.ne && p.d[j] < 0) ? -p.d[j] - 1 : p.row));
    }
}

// row_compute for all RW right-hand sides of one row (DIV == 0: multiply by the stored 1/diag).
template <typename RT, int RW, int EK>
__device__ __forceinline__ bool row_compute_rw(const RowDeps<EK> &p, const RowVals<float, EK> &v, const float (&rh)[RW],
                                               const float (&pf)[RW][EK], const WalkIO<float, RT, true, false> &io,
                                               Waiter &w) {
    static_assert(RW == 2 || RW == 4, "the row-wide walk moves slots as 2- or 4-float vectors");
    float xv[EK][RW];
    bool miss = false;
#pragma unroll
    for (int j = 0; j < EK; j++) {
        const int dj = p.d[j];
        float loc[RW];
        sh_ldv(io.xs_at((dj >= 0 ? dj : 0) * RW), loc);
#pragma unroll
        for (int r = 0; r < RW; r++) {
            xv[j][r] = dj >= 0 ? loc[r] : pf[r][j];
            miss |= j < p.ne && dj < 0 && Sent<float>::is(pf[r][j]);
        }
    }
    if (miss) {
#pragma unroll
        for (int r = 0; r < RW; r++)
#pragma unroll
            for (int j = 0; j < EK; j++)
                if (j < p.ne && p.d[j] < 0 && Sent<float>::is(xv[j][r]) &&
                    !wait_value<float>(io.xg + (size_t)r * io.ldx + (-p.d[j] - 1), xv[j][r], w, -p.d[j] - 1))
                    return false;
    }
    float o[RW];
#pragma unroll
    for (int r = 0; r < RW; r++) {
        float sum = 0.0f;
#pragma unroll
        for (int j = 0; j < EK; j++)
            if (j < p.ne) sum = fmaf(xv[j][r], v.a[j], sum);
        o[r] = (rh[r] - sum) * v.diag;  // FP32 value blocks hold 1/diag
    }
    if (v.sl >= 0) sh_stv(io.xs_at(v.sl * RW), o);
#pragma unroll
    for (int r = 0; r < RW; r++) Sent<float>::store(io.xg + (size_t)r * io.ldx + p.row, o[r]);
    return true;
}

// walk_run_e with the row-wide mapping: the same window crossing and step pipeline, the
// step-s+1 row's remote values and right-hand sides loaded before the barrier ending step s.
template <typename RT, bool RL2, int RW, int EK>
__device__ __forceinline__ bool walk_run_rw(WinStream<float> &ws, int &i, const unsigned char *buf, int nint,
                                            const WalkIO<float, RT, true, false> &io, Waiter &w, unsigned int spin,
                                            DevStatus *st) {
    constexpr unsigned int S = sizeof(float);
    const int lr = (int)threadIdx.x, stp = (int)blockDim.x;
    unsigned int I0 = smem_u32(buf);
    unsigned int Iend = I0 + 4u * (unsigned int)nint;
    unsigned int V0 = Iend;
    bool alive = true;
    int nl0 = Sh<int>::ldu(I0);
    RowDeps<EK> q0, q1;
    float pf0[RW][EK];
    float rh0[RW], rh1[RW];
    bool m0 = lr < nl0;
    if (m0) {
        load_deps<EK>(I0, nl0, lr, q0);
        load_remote_rw<RT, RW, EK>(q0, io, pf0);
        load_rhs_rw<RT, RL2, RW>(q0.row, io, rh0);
    }
    for (;;) {
        const int nl1 = Sh<int>::ldu(I0 + 8u);
        unsigned int I1 = I0 + 4u * (unsigned int)chunk_nint(nl0, EK);
        unsigned int V1 = V0 + S * (unsigned int)chunk_nval(nl0, EK);
        unsigned int Iend1 = Iend;
        const bool cross = nl1 != 0 && I1 == Iend;
        bool okw = true;
        if (cross) {
            const unsigned char *nb;
            int nn;
            okw = ws.peek(i, spin, nb, nn);
            I1 = smem_u32(nb);
            Iend1 = I1 + 4u * (unsigned int)nn;
            V1 = Iend1;
        }
        const bool m1 = okw && lr < nl1;
        if (m1) load_deps<EK>(I1, nl1, lr, q1);
        if (alive && m0) {
            RowVals<float, EK> v;
            load_vals<float, RT, RL2, true, false, EK>(I0, V0, nl0, lr, q0, io, v);
            if (!row_compute_rw<RT, RW, EK>(q0, v, rh0, pf0, io, w)) alive = false;
        }
        for (int pos = lr + stp; alive && pos < nl0; pos += stp) {
            RowDeps<EK> q;
            RowVals<float, EK> v;
            float qf[RW][EK], rh[RW];
            load_deps<EK>(I0, nl0, pos, q);
            load_vals<float, RT, RL2, true, false, EK>(I0, V0, nl0, pos, q, io, v);
            load_rhs_rw<RT, RL2, RW>(q.row, io, rh);
#pragma unroll
            for (int r = 0; r < RW; r++)
#pragma unroll
                for (int j = 0; j < EK; j++) qf[r][j] = Sent<float>::value();
            if (!row_compute_rw<RT, RW, EK>(q, v, rh, qf, io, w)) alive = false;
        }
        if (m1 && alive) {
            load_remote_rw<RT, RW, EK>(q1, io, pf0);
            load_rhs_rw<RT, RL2, RW>(q1.row, io, rh1);
        }
        if (cross) {
            if (!okw && atomicCAS(&st->code, kOk, kTimeout) == kOk) st->where = -1000000 - i - 1;
            if (__syncthreads_or(!okw || !alive)) return false;
            ws.release(i);
            i++;
            Iend = Iend1;
        } else {
            __syncthreads();
        }
        if (nl1 == 0) break;
        I0 = I1;
        V0 = V1;
        nl0 = nl1;
        m0 = m1;
        q0 = q1;
#pragma unroll
        for (int r = 0; r < RW; r++) rh0[r] = rh1[r];
    }
    return alive;
}

// Any entry stride (the CTA's widest row has more than 3 entries): plain loop, waits in place.
template <typename T, typename RT, bool RL2, bool MR, bool STG, int DIV>
__device__ __forceinline__ bool walk_window_any(const int *I, const int *Iend, const T *V,
                                                const WalkIO<T, RT, MR, STG> &io, Waiter &w, bool alive) {
    T *xg = io.out();
    while (I < Iend) {
        const int nl = I[0], E = I[1];
        const int *rowid = I + kChunkHdr, *slot = rowid + nl, *ne = slot + nl, *kpos = ne + nl, *dep = kpos + nl;
        const T *diag = V, *rcp = V + nl, *val = V + 2 * nl;
        for (int pos = io.lane_row(); alive && pos < nl; pos += io.stride()) {
            const int row = rowid[pos];
            T rhs;
            if constexpr (STG) {
                rhs = io.rs[io.slot(kpos[pos])];
            } else {
                const RT *src = io.in() + row;
                if constexpr (RL2)
                    rhs = (T)Sent<RT>::load(src);
                else
                    rhs = (T)*src;
            }
            T sum = T(0);
            for (int j = 0; j < ne[pos]; j++) {
                const int d = dep[pos * E + j];
                T xv;
                if (d >= 0) {
                    xv = io.xs[io.slot(d)];
                } else if (!wait_value<T>(xg + (-d - 1), xv, w, -d - 1)) {
                    alive = false;
                    break;
                }
                if constexpr (DIV != 0)
                    sum = __dadd_rn(sum, __dmul_rn(xv, val[pos * E + j]));
                else
                    sum = fmaf(xv, val[pos * E + j], sum);
            }
            if (!alive) break;
            T o;
            if constexpr (DIV == 2)
                o = __ddiv_rn(__dsub_rn(rhs, sum), diag[pos]);
            else if constexpr (DIV == 1)
                o = div_fast(__dsub_rn(rhs, sum), diag[pos], rcp[pos], w.slow);
            else
                o = (rhs - sum) * diag[pos];
            if (slot[pos] >= 0) io.xs[io.slot(slot[pos])] = o;
            if constexpr (STG) io.rs[io.slot(kpos[pos])] = o;
            Sent<T>::store(xg + row, o);
        }
        I += chunk_nint(nl, E);
        V += chunk_nval(nl, E);
        __syncthreads();
    }
    return alive;
}

// Walk the windows [i, iend) of one direction (all of a CTA's chunks in a direction share one
// entry stride). Every thread passes every barrier, also after a failed wait, so the CTA never
// splits; the result is uniform. Each window is released after its walk.
// RW > 1: the row-wide walk (FP32 factors, MR, not staged, io.R_ == RW) for entry strides up to
// 2; wider strides keep the MR walk (a stride-3 row-wide walk pushed the batched kernel to 255
// registers with spills, and its 64-system batch ran 13% slower than with strides up to 2).
template <typename T, typename RT, bool RL2, bool MR, bool STG, int DIV, int RW = 1>
__device__ __forceinline__ bool walk_dir(WinStream<T> &ws, int i, int iend, const WalkIO<T, RT, MR, STG> &io,
                                         Waiter &w, unsigned int spin, DevStatus *st) {
    static_assert(RW == 1 || (sizeof(T) == 4 && MR && !STG && DIV == 0), "row-wide walk: FP32, MR, not staged");
    const unsigned char *b;
    int nint;
    if (i >= iend) return true;
    if (!ws.acquire(i, spin, st, b, nint)) return false;
    bool alive = true;
    switch (Sh<int>::ld(reinterpret_cast<const int *>(b) + 1)) {
        case 1:
            if constexpr (RW > 1)
                alive = walk_run_rw<RT, RL2, RW, 1>(ws, i, b, nint, io, w, spin, st);
            else
                alive = walk_run_e<T, RT, RL2, MR, STG, DIV, 1>(ws, i, b, nint, io, w, spin, st);
            break;
        case 2:
            if constexpr (RW > 1)
                alive = walk_run_rw<RT, RL2, RW, 2>(ws, i, b, nint, io, w, spin, st);
            else
                alive = walk_run_e<T, RT, RL2, MR, STG, DIV, 2>(ws, i, b, nint, io, w, spin, st);
            break;
        case 3: alive = walk_run_e<T, RT, RL2, MR, STG, DIV, 3>(ws, i, b, nint, io, w, spin, st); break;
        default:
            for (;;) {
                const int *I = reinterpret_cast<const int *>(b);
                alive = walk_window_any<T, RT, RL2, MR, STG, DIV>(I, I + nint,
                                                                    reinterpret_cast<const T *>(b + (size_t)nint * 4),
                                                                    io, w, alive);
                if (i + 1 == iend) break;
                ws.release(i);
                if (__syncthreads_or(!alive)) return false;
                if (!ws.acquire(++i, spin, st, b, nint)) return false;
            }
    }
    if (!alive && i + 1 < iend) {
        // walk_run_e returned early (uniformly) at a window crossing
        return false;
    }
    ws.release(i);
    if (DIV == 1 && w.slow) st->slow_div = 1;
    return !__syncthreads_or(!alive);
}

// Standalone FP64 sweep of the caller's triangular CSR (values gathered through vsrcT into the
// packed scratch gv), right-hand sides R at a time (MR: R > 1; STG: staged in shared memory).
// d = 0: lower (L), 1: upper (U = L^T). IEEE: divide with __ddiv_rn (the repeat of a launch
// whose div_fast divisions left their range); else div_fast.
template <bool MR, bool STG, bool IEEE>
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
    const int s0 = __ldg(pl.soff + c), nl = __ldg(pl.soff + c + 1) - s0;
    for (int r0 = 0; r0 < nrhs; r0 += R) {
        WalkIO<double, double, MR, STG> io;
        io.xs = reinterpret_cast<double *>(smem);
        io.rs = reinterpret_cast<double *>(smem + pl.xs_bytes);
        io.xg = x + (size_t)r0 * ldx;
        io.rhs = b + (size_t)r0 * ldb;
        io.ldx = ldx;
        io.ldr = ldb;
        io.R_ = min(R, nrhs - r0);
        if constexpr (STG) {
            const int Rb = io.R();
            for (int k = threadIdx.x; k < nl * Rb; k += blockDim.x) {
                const int kk = k / Rb, r = k - kk * Rb;
                io.rs[k] = __ldg(b + (size_t)(r0 + r) * ldb + __ldg(pl.srow + s0 + kk));
            }
            __syncthreads();
        }
        trace_mark(trace, 2 + 2 * (r0 / R));
        if (!walk_dir<double, double, false, MR, STG, IEEE ? 2 : 1>(ws, 0, ws.total(), io, w, spin, st)) {
            ws.drain(spin);
            return;
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
// ---------------------------------------------------------------------------------------
// Level walk: for shallow group DAGs (a few dozen levels, each thousands of groups wide: an
// unstructured or randomly permuted pattern), where per-row waits between CTAs would cost more
// than one grid barrier per level. Every thread of the launch takes groups of the current level
// in turn (grid stride) and solves their rows in order, reading the rows of earlier levels from
// L2; a grid barrier ends the level (its fences publish the level's results). Entries are summed
// in the plan's order with the same correctly rounded operations as the other walks (the FP64
// quotient by __ddiv_rn, which the chunked walk's div_fast reproduces), so results are
// bit-identical to theirs.
// ---------------------------------------------------------------------------------------
struct LevelDir {
    const int *lev;    // nlev + 1: items (groups) of each level, in execution order
    const int *item;   // nitem + 1: positions (rows) of each item
    const int *row;    // position -> row
    const int *eptr;   // position -> its entries
    const int *dep;    // entry -> the row it reads
    const int *src;    // entry -> A position (factor values)
    const int *dsrc;   // position -> the diagonal's A position
    const int *srcT;   // entry -> position in the caller's triangular CSR
    const int *dsrcT;  // position -> the diagonal's position there
    int nlev, nent, npos;
};

// Packs a direction's values (grid stride): v[e] per entry, d[pos] per row (FP64: the diagonal;
// FP32: 1/diag, as the other FP32 walks store it).
template <typename T>
__device__ __forceinline__ void level_pack(const LevelDir &D, const int *src, const int *dsrc, const double *vals,
                                           T *v, T *d, int gt, int W) {
    for (int e = gt; e < D.nent; e += W) v[e] = (T)Sent<double>::load(vals + __ldg(src + e));
    for (int p = gt; p < D.npos; p += W) {
        const double dv = Sent<double>::load(vals + __ldg(dsrc + p));
        if constexpr (sizeof(T) == 4)
            d[p] = __frcp_rn(__double2float_rn(dv));
        else
            d[p] = dv;
    }
}

// One direction: out[row] = (rhs[row] - sum_e v[e] out[dep[e]]) / d[pos], level by level. False
// (uniformly) if a grid barrier gave up.
template <typename T, typename RT>
__device__ __forceinline__ bool level_walk(const LevelDir &D, const T *v, const T *d, const RT *rhs, T *out,
                                           unsigned int *bar, unsigned int &nb, DevStatus *st, unsigned int limit) {
    const int W = gridDim.x * blockDim.x;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    for (int l = 0; l < D.nlev; l++) {
        const int ib = __ldg(D.lev + l), ie = __ldg(D.lev + l + 1);
        for (int it = ib + gt; it < ie; it += W) {
            // the group's last kWin results stay in registers: a row that reads one of them (the
            // rows of a coarsened group form chains) takes it from there, not from L2
            constexpr int kWin = 4;
            int wr[kWin];
            T wv[kWin];
#pragma unroll
            for (int k = 0; k < kWin; k++) {
                wr[k] = -1;
                wv[k] = T(0);
            }
            for (int p = __ldg(D.item + it), pe = __ldg(D.item + it + 1); p < pe; p++) {
                const int row = bounded(__ldg(D.row + bounded(p, D.npos, st, 130)), D.npos, st, 131);
                T sum = T(0);
                // eight entries' loads in flight at once (dependency rows, then their values),
                // then their products summed in entry order
                for (int e0 = __ldg(D.eptr + p), ee = __ldg(D.eptr + p + 1); e0 < ee; e0 += 8) {
                    int dr[8];
                    T vv[8], xv[8];
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        const bool in = e0 + u < ee;
                        dr[u] = in ? bounded(__ldg(D.dep + bounded(e0 + u, D.nent, st, 132)), D.npos, st, 133) : row;
                        vv[u] = in ? __ldg(v + bounded(e0 + u, D.nent, st, 134)) : T(0);
                    }
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        bool hit = false;
                        T hv = T(0);
#pragma unroll
                        for (int k = 0; k < kWin; k++)
                            if (dr[u] == wr[k]) {
                                hit = true;
                                hv = wv[k];
                            }
                        xv[u] = hv;
                        if (!hit) xv[u] = __ldcg(out + dr[u]);
                    }
#pragma unroll
                    for (int u = 0; u < 8; u++)
                        if (e0 + u < ee) {
                            if constexpr (sizeof(T) == 8)
                                sum = __dadd_rn(sum, __dmul_rn(xv[u], vv[u]));
                            else
                                sum = fmaf(xv[u], vv[u], sum);
                        }
                }
                const T r = (T)__ldcg(rhs + row);
                T o;
                if constexpr (sizeof(T) == 8)
                    o = __ddiv_rn(__dsub_rn(r, sum), __ldg(d + p));
                else
                    o = (r - sum) * __ldg(d + p);
                __stcg(out + row, o);
#pragma unroll
                for (int k = kWin - 1; k > 0; k--) {
                    wr[k] = wr[k - 1];
                    wv[k] = wv[k - 1];
                }
                wr[0] = row;
                wv[0] = o;
            }
        }
        if (!grid_barrier(bar, nb, st, limit)) return false;
    }
    return true;
}

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
    LevelDir lv[2];     // level-walk plan per direction (kernels instantiated with the level walk)
    double *lv64[2], *ld64[2];  // its packed values and diagonals, FP64 factors
    float *lv32[2], *ld32[2];   // the same, FP32 factors (1/diag)
    FetchPlan fp;      // fetch-walk plan (kernels instantiated with FW)
    double *gf64[2];   // fetch-walk record values per direction, FP64 factors
    float *gf32[2];    // the same, FP32 factors
    int fac_fetch;     // FW: IC0 by the fetch walk (no entry's dot product has a column match)
    double *dg;        // with fac_fetch: each row's final diagonal, its ready flag for other CTAs
};

// Vector phases take L rows (or elements) per thread per pass: rows i, i + W, ..., i + (L-1) W
// in lockstep, so their loads are in flight together (one CTA of 8 warps per SM leaves little
// other parallelism to hide them). Each row still sums in CSR order, and the caller consumes
// the rows in the grid-stride order i, i + W, ..., so every result and every partial dot product
// is bit-identical to the row-at-a-time loop. The FP64-factor solve uses 4; the FP32-factor
// solve keeps 1, because the extra registers slowed its FP32 sweeps (26.5 -> 30.1 ms on 64^3).
template <int kLanes, typename F>
__device__ __forceinline__ void csr_rows(const int *__restrict__ rowptr, const int *__restrict__ colidx,
                                         const double *val, const double *v, int i0, int W, int n, F consume) {
    int e[kLanes], ee[kLanes], len = 0;
    double s[kLanes];
#pragma unroll
    for (int u = 0; u < kLanes; u++) {
        const int i = i0 + u * W;
        e[u] = i < n ? __ldg(rowptr + i) : 0;
        ee[u] = i < n ? __ldg(rowptr + i + 1) : 0;
        s[u] = 0.0;
        len = max(len, ee[u] - e[u]);
    }
    for (int k = 0; k < len; k++) {
#pragma unroll
        for (int u = 0; u < kLanes; u++)
            if (e[u] + k < ee[u]) {
                const int q = e[u] + k;
                s[u] = __dadd_rn(s[u], __dmul_rn(val[q], v[__ldg(colidx + q)]));
            }
    }
#pragma unroll
    for (int u = 0; u < kLanes; u++)
        if (i0 + u * W < n) consume(i0 + u * W, s[u]);
}

// Division mode of a walk over factors of type T (FP32 factors multiply by 1/diag).
template <typename T, bool IEEE>
constexpr int kDiv = sizeof(T) == 8 ? (IEEE ? 2 : 1) : 0;

// z = U^-1 L^-1 r on this CTA's rows; p = z if set_p; adds this thread's share of r.z to rz in
// a pass over the CTA's rows afterwards. STG: r is staged in shared memory, the lower walk
// leaves y there for the upper walk, which leaves z there for the r.z pass; else the right-hand
// sides come from r and from y (in L2) and z is read back from L2.
template <typename T, bool STG, bool IEEE>
__device__ __forceinline__ bool chunk_precond(const IccgArgs &A, WinStream<T> &ws, unsigned char *smem, bool set_p, double &rz,
                              Waiter &w) {
    const int c = blockIdx.x;
    T *yg = sizeof(T) == 8 ? (T *)A.y : (T *)A.y32;
    T *zg = sizeof(T) == 8 ? (T *)A.z : (T *)A.z32;
    T *xs = reinterpret_cast<T *>(smem);
    T *rs = reinterpret_cast<T *>(smem + A.pl.xs_bytes);
    const int s0 = __ldg(A.pl.soff + c), nl = __ldg(A.pl.soff + c + 1) - s0;
    if constexpr (STG) {
        for (int k = threadIdx.x; k < nl; k += blockDim.x) rs[k] = (T)A.r[__ldg(A.pl.srow + s0 + k)];
        __syncthreads();
    }
    trace_mark(A.trace, 56);
    const int n0 = ws.ctl->n0;
    {
        const WalkIO<T, double, false, STG> lo{xs, yg, A.r, rs, 0, 0, 1};
        if (!walk_dir<T, double, false, false, STG, kDiv<T, IEEE>>(ws, 0, n0, lo, w, A.spin_limit, A.st)) return false;
    }
    trace_mark(A.trace, 57);
    {
        const WalkIO<T, T, false, STG> up{xs, zg, yg, rs, 0, 0, 1};
        if (!walk_dir<T, T, true, false, STG, kDiv<T, IEEE>>(ws, n0, ws.total(), up, w, A.spin_limit, A.st)) return false;
    }
    for (int k = threadIdx.x; k < nl; k += blockDim.x) {
        const int row = __ldg(A.pl.srow + s0 + k);
        const double zd = STG ? (double)rs[k] : (double)Sent<T>::load(zg + row);
        rz = __dadd_rn(rz, __dmul_rn(A.r[row], zd));
        if (set_p) A.p[row] = zd;
    }
    trace_mark(A.trace, 59);
    return true;
}

// Level-walk preconditioner: z = U^-1 L^-1 r by the level walk (lower into y, upper into z, both
// in global memory), p = z if set_p, and this thread's share of r.z (grid stride). nb: the
// caller's grid-barrier count. False (uniformly) if a barrier gave up.
template <typename T>
__device__ __forceinline__ bool level_precond(const IccgArgs &A, bool set_p, double &rz, unsigned int &nb) {
    constexpr bool kMixed = sizeof(T) == 4;
    T *yg = kMixed ? (T *)A.y32 : (T *)A.y;
    T *zg = kMixed ? (T *)A.z32 : (T *)A.z;
    const T *v0 = kMixed ? (const T *)A.lv32[0] : (const T *)A.lv64[0];
    const T *d0 = kMixed ? (const T *)A.ld32[0] : (const T *)A.ld64[0];
    const T *v1 = kMixed ? (const T *)A.lv32[1] : (const T *)A.lv64[1];
    const T *d1 = kMixed ? (const T *)A.ld32[1] : (const T *)A.ld64[1];
    trace_mark(A.trace, 56);
    if (!level_walk<T, double>(A.lv[0], v0, d0, A.r, yg, A.bar, nb, A.st, A.spin_limit)) return false;
    if (!level_walk<T, T>(A.lv[1], v1, d1, yg, zg, A.bar, nb, A.st, A.spin_limit)) return false;
    trace_mark(A.trace, 57);
    const int W = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += W) {
        const double zd = (double)__ldcg(zg + i);
        rz = __dadd_rn(rz, __dmul_rn(A.r[i], zd));
        if (set_p) A.p[i] = zd;
    }
    trace_mark(A.trace, 59);
    return true;
}

// Shared-memory addresses of a fetch walk (fetch.cuh): slots, the int blocks (both directions
// resident), the value buffer (FP64: one direction at a time; FP32: both), the control block.
struct FetchSh {
    unsigned int SL, RW, FL[2], I[2], V[2];
    FetchCtl *ctl;
    int nrows, s0, nf0, nf1, ns[2];
};
template <typename T>
__device__ __forceinline__ FetchSh fetch_layout(const FetchPlan &fp, unsigned char *smem, bool two_dirs) {
    const int c = blockIdx.x;
    FetchSh F;
    // an ICCG (two_dirs) reserves 8-byte slots in both precisions: its IC0 walk passes FP64 diagonals
    const unsigned int slot_elem = two_dirs ? 8u : (unsigned int)sizeof(T);
    const unsigned int slot_bytes = ((unsigned int)fp.nslot * slot_elem + 15u) & ~15u;
    F.s0 = __ldg(fp.soff + c);
    F.nrows = __ldg(fp.soff + c + 1) - F.s0;
    F.SL = smem_u32(smem);
    F.RW = F.SL + slot_bytes;
    F.I[0] = F.RW + (unsigned int)fp.srow_bytes;
    F.I[1] = F.I[0] + (unsigned int)fp.ints_bytes[0];
    const unsigned int vb = F.I[1] + (two_dirs ? (unsigned int)fp.ints_bytes[1] : 0u);
    F.V[0] = vb;
    F.V[1] = sizeof(T) == 4 && two_dirs ? vb + 16u * (unsigned int)F.nrows : vb;
    F.ctl = reinterpret_cast<FetchCtl *>(smem + (vb - F.SL) + (unsigned int)fp.vals_bytes);
    F.nf0 = __ldg(fp.dir[0].cfetch + c + 1) - __ldg(fp.dir[0].cfetch + c);
    F.nf1 = __ldg(fp.dir[1].cfetch + c + 1) - __ldg(fp.dir[1].cfetch + c);
    F.ns[0] = __ldg(fp.dir[0].cblk + c).z;
    F.ns[1] = __ldg(fp.dir[1].cblk + c).z;
    F.FL[0] = F.RW + 4u * (unsigned int)F.nrows;
    F.FL[1] = F.FL[0] + 4u * (unsigned int)F.nf0;
    return F;
}
// The CTA's row list and both directions' fetch lists into shared memory (all threads; the
// caller's next barrier publishes them).
__device__ __forceinline__ void fetch_stage_lists(const FetchPlan &fp, const FetchSh &F) {
    const int c = blockIdx.x;
    const int *f0 = fp.dir[0].frow + __ldg(fp.dir[0].cfetch + c), *f1 = fp.dir[1].frow + __ldg(fp.dir[1].cfetch + c);
    for (int k = threadIdx.x; k < F.nrows; k += blockDim.x) Sh<int>::stu(F.RW + 4u * (unsigned int)k, __ldg(fp.srow + F.s0 + k));
    for (int k = threadIdx.x; k < F.nf0; k += blockDim.x) Sh<int>::stu(F.FL[0] + 4u * (unsigned int)k, __ldg(f0 + k));
    for (int k = threadIdx.x; k < F.nf1; k += blockDim.x) Sh<int>::stu(F.FL[1] + 4u * (unsigned int)k, __ldg(f1 + k));
}
// Issues the copies of the int blocks (both directions when two_dirs, else direction d at I[0])
// on mbar_ints. One thread.
__device__ __forceinline__ void fetch_issue_ints(const FetchPlan &fp, const FetchSh &F, bool two_dirs, int d) {
    const int4 c0 = __ldg(fp.dir[two_dirs ? 0 : d].cblk + blockIdx.x);
    const int4 c1 = __ldg(fp.dir[1].cblk + blockIdx.x);
    fence_async_shared();
    mbar_expect_tx(&F.ctl->mbar_ints, 16u * (unsigned int)(c0.y + (two_dirs ? c1.y : 0)));
    fetch_copy(F.I[0], fp.dir[two_dirs ? 0 : d].ints + c0.x, 16u * (unsigned int)c0.y, &F.ctl->mbar_ints);
    if (two_dirs) fetch_copy(F.I[1], fp.dir[1].ints + c1.x, 16u * (unsigned int)c1.y, &F.ctl->mbar_ints);
}
// Issues the copy of this CTA's record values of direction d (both directions, FP32 only, when
// both) into V[d] (V[0], V[1]) on mbar_vals. One thread.
template <typename T>
__device__ __forceinline__ void fetch_issue_vals(const FetchPlan &fp, const FetchSh &F, T *const gv[2], int d, bool both) {
    constexpr unsigned int RB = sizeof(T) == 8 ? 8u * kFetchVal64 : 4u * kFetchVal32;
    const unsigned int bytes = RB * (unsigned int)F.nrows;
    fence_async_shared();
    mbar_expect_tx(&F.ctl->mbar_vals, both ? 2u * bytes : bytes);  // 0 bytes (no rows): the phase completes here
    for (int k = both ? 0 : d; bytes > 0 && k <= (both ? 1 : d); k++) {
        const int rb = __ldg(fp.dir[k].cblk + blockIdx.x).w;
        fetch_copy(F.V[k], reinterpret_cast<const unsigned char *>(gv[k]) + (size_t)RB * (size_t)rb, bytes, &F.ctl->mbar_vals);
    }
}

// Fetch-walk preconditioner (fetch.cuh): z = U^-1 L^-1 r on this CTA's rows, p = z if set_p, and
// this thread's share of r.z. r is staged in the row slots; the lower walk leaves y there, the
// upper walk z. The compute warps walk both directions while the last warp fetches both
// directions' remote values. FP64 values: the lower block was copied in before this call (by
// the caller, or by the previous call's tail); the upper block is copied once the lower walk
// is over, and this call's tail starts the copy of the next lower block. Thread 0 issues every
// copy and keeps in vpend the mbarrier parity of the one in flight (-1: none), which it awaits
// before the kernel exits. false (uniform) if a wait gave up.
template <typename T, bool IEEE>
__device__ __forceinline__ bool fetch_precond(const IccgArgs &A, const FetchSh &F, bool set_p, double &rz, int &vpend) {
    constexpr unsigned int S = sizeof(T);
    const FetchPlan &fp = A.fp;
    const int tid = (int)threadIdx.x;
    T *yg = sizeof(T) == 8 ? (T *)A.y : (T *)A.y32;
    T *zg = sizeof(T) == 8 ? (T *)A.z : (T *)A.z32;
    for (int k = tid; k < F.nrows; k += blockDim.x) Sh<T>::stu(F.SL + S * (unsigned int)k, (T)A.r[__ldg(fp.srow + F.s0 + k)]);
    fetch_reset_slots<T>(F.SL, F.nrows, F.nf0 + F.nf1);
    if constexpr (sizeof(T) == 8) {
        if (!mbar_wait(&F.ctl->mbar_vals, 0u, A.spin_limit) && atomicCAS(&A.st->code, kOk, kTimeout) == kOk)
            A.st->where = -3000000;
        if (tid == 0) vpend = -1;
    }
    __syncthreads();
    trace_mark(A.trace, 56);
    bool slow = false;
    if (tid >= kFetchWarp * 32) {
        fetch_run<T>(F.FL[0], F.nf0, yg, F.SL + S * (unsigned int)(F.nrows + 1), A.spin_limit, A.st, F.ctl);
        fetch_run<T>(F.FL[1], F.nf1, zg, F.SL + S * (unsigned int)(F.nrows + 1 + F.nf0), A.spin_limit, A.st, F.ctl);
    } else if (tid < fp.ncomp) {
        walk_fetch<T, kDiv<T, IEEE>>(F.I[0], F.V[0], F.SL, F.RW, F.ns[0], fp.ncomp, yg, A.spin_limit, A.st, F.ctl, slow);
        trace_mark(A.trace, 60);
        if constexpr (sizeof(T) == 8) {
            // the lower walk's last step barrier has passed: every compute thread is done with
            // the lower values
            if (tid == 0) {
                fetch_issue_vals<T>(fp, F, reinterpret_cast<T *const *>(A.gf64), 1, false);
                vpend = 1;
            }
            if (!mbar_wait(&F.ctl->mbar_vals, 1u, A.spin_limit)) {
                F.ctl->err = 1;
            } else if (tid == 0) {
                vpend = -1;
            }
        }
        trace_mark(A.trace, 61);
        walk_fetch<T, kDiv<T, IEEE>>(F.I[1], F.V[1], F.SL, F.RW, F.ns[1], fp.ncomp, zg, A.spin_limit, A.st, F.ctl, slow);
    }
    if (kDiv<T, IEEE> == 1 && slow) A.st->slow_div = 1;
    trace_mark(A.trace, 57);
    if (__syncthreads_or(F.ctl->err)) return false;
    if constexpr (sizeof(T) == 8) {
        if (tid == 0) {
            fetch_issue_vals<T>(fp, F, reinterpret_cast<T *const *>(A.gf64), 0, false);
            vpend = 0;
        }
    }
    for (int k = tid; k < F.nrows; k += blockDim.x) {
        const int row = __ldg(fp.srow + F.s0 + k);
        const double zd = (double)Sh<T>::ldu(F.SL + S * (unsigned int)k);
        rz = __dadd_rn(rz, __dmul_rn(A.r[row], zd));
        if (set_p) A.p[row] = zd;
    }
    trace_mark(A.trace, 59);
    return true;
}

// This CTA's value slots of one direction from the IC0 factor lu (FP32: the diagonal as its
// reciprocal).
template <typename T>
__device__ __forceinline__ void pack_factor(const ChunkDir &D, const double *lu, double *g64, float *g32) {
    const int vb = __ldg(D.cval + blockIdx.x), ve = __ldg(D.cval + blockIdx.x + 1);
    for (int i = vb + (int)threadIdx.x; i < ve; i += blockDim.x) {
        const int s = __ldg(D.vsrcA + i);
        const bool rcp = s < -(1 << 30), dg = s <= -2 && !rcp;
        const int src = s >= 0 ? s : (rcp ? s - kRcpBase : (dg ? -2 - s : -1));
        const double v = src >= 0 ? ld_l2(lu + src) : 0.0;
        if constexpr (sizeof(T) == 4)
            g32[i] = (dg || rcp) ? __frcp_rn(__double2float_rn(v)) : __double2float_rn(v);
        else
            g64[i] = rcp ? div_recip(v) : v;
    }
}

// T = double: FP64 factors; T = float: FP32 factors. STG: the right-hand sides of the sweeps are
// staged in shared memory (when they fit). One instantiation per combination keeps each one's
// register budget to what it uses. IEEE (FP64 factors only): sweep divisions by __ddiv_rn, for the
// repeat of a launch whose div_fast divisions left their range.
template <typename T, bool STG, bool IEEE, int WK>
__global__ void __launch_bounds__(kStageBlock, 1) k_iccg_chunked(IccgArgs A) {
    constexpr bool FW = WK == kWalkFetch, LW = WK == kWalkLevels;
    constexpr bool kMixed = sizeof(T) == 4;
    constexpr int kLanes = 4;  // rows whose SpMV loads a thread keeps in flight together (8: slower)
    extern __shared__ __align__(128) unsigned char smem[];
    const int n = A.n;
    const int W = gridDim.x * blockDim.x;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned int nb = 0;
    Waiter w(A.spin_limit, A.st);
    WinStream<T> ws;
    FetchSh F;
    int vpend = -1;           // thread 0: parity of the value copy in flight (fetch walk)
    bool ints_pending = FW;   // the int blocks' copy has not been awaited yet
    if constexpr (FW) {
        F = fetch_layout<T>(A.fp, smem, true);
        if (threadIdx.x == 0) {
            F.ctl->err = 0;
            mbar_init(&F.ctl->mbar_ints, 1);
            mbar_init(&F.ctl->mbar_vals, 1);
            mbar_init(&F.ctl->mbar_fac, 1);
            fence_mbar_init();
        }
        __syncthreads();
        if (threadIdx.x == 0) fetch_issue_ints(A.fp, F, true, 0);
        fetch_stage_lists(A.fp, F);
    } else if constexpr (!LW) {
        ws.init(A.pl, 0, true, kMixed ? (const T *)A.gv32[0] : (const T *)A.gv64[0],
                kMixed ? (const T *)A.gv32[1] : (const T *)A.gv64[1], smem, 0xFFFFFFFFu);
    }
    // waits (bounded) for this CTA's bulk copies still in flight before it exits
    auto drain = [&]() {
        if constexpr (FW) {
            if (threadIdx.x == 0) {
                if (ints_pending) mbar_wait(&F.ctl->mbar_ints, 0u, A.spin_limit);
                if (vpend >= 0) mbar_wait(&F.ctl->mbar_vals, (unsigned int)vpend, A.spin_limit);
            }
            __syncthreads();
        } else if constexpr (!LW) {
            ws.drain(A.spin_limit);
        }
    };
#define BAAS_BARRIER()                                            \
    do {                                                          \
        if (!grid_barrier(A.bar, nb, A.st, A.spin_limit)) {       \
            drain();                                              \
            return;                                               \
        }                                                         \
    } while (0)

    trace_mark(A.trace, 0);
    if (!A.reuse) {
        const int nnz = __ldg(A.a_rowptr + n);
        for (int e = gt; e < nnz; e += W) A.lu[e] = A.a_val[e];
        if (FW && A.fac_fetch)
            for (int i = gt; i < n; i += W) A.dg[i] = Sent<double>::value();
        BAAS_BARRIER();
        trace_mark(A.trace, 1);

        if constexpr (FW) {
            if (A.fac_fetch) {
                // IC0 by the fetch walk: the lower records' A values into shared memory (FP64
                // layout), the zero slot to +1, then the lower walk with l_jj as the value passed
                fetch_pack<double>(A.fp.dir[0], A.fp.dir[0].code, A.a_val, A.gf64[0]);
                fence_async_global();
                fetch_reset_slots<double>(F.SL, F.nrows, F.nf0 + F.nf1);
                if (threadIdx.x == 0) Sh<double>::stu(F.SL + 8u * (unsigned int)F.nrows, 1.0);
                __syncthreads();
                if (threadIdx.x == 0) {
                    fence_async_shared();
                    const unsigned int bytes = 8u * kFetchVal64 * (unsigned int)F.nrows;
                    mbar_expect_tx(&F.ctl->mbar_fac, bytes);
                    if (bytes > 0)
                        fetch_copy(F.V[0], A.gf64[0] + (size_t)kFetchVal64 * (size_t)__ldg(A.fp.dir[0].cblk + blockIdx.x).w,
                                   bytes, &F.ctl->mbar_fac);
                }
                bool ok = mbar_wait(&F.ctl->mbar_ints, 0u, A.spin_limit);
                ok = mbar_wait(&F.ctl->mbar_fac, 0u, A.spin_limit) && ok;
                if (!ok && atomicCAS(&A.st->code, kOk, kTimeout) == kOk) A.st->where = -3000003;
                if (__syncthreads_or(!ok)) {
                    if (threadIdx.x == 0) mbar_wait(&F.ctl->mbar_fac, 0u, A.spin_limit);
                    drain();
                    return;
                }
                ints_pending = false;
                const int tid = (int)threadIdx.x;
                if (tid >= kFetchWarp * 32) {
                    fetch_run<double>(F.FL[0], F.nf0, A.dg, F.SL + 8u * (unsigned int)(F.nrows + 1), A.spin_limit, A.st, F.ctl);
                } else if (tid < A.fp.ncomp) {
                    walk_ic0_fetch(F.I[0], F.V[0], F.SL, F.RW, F.ns[0], A.fp.ncomp, A.dg, A.lu,
                                   reinterpret_cast<const int4 *>(A.fp.dir[0].code), __ldg(A.fp.dir[0].cblk + blockIdx.x).w,
                                   A.spin_limit, A.st, F.ctl);
                }
                if (__syncthreads_or(F.ctl->err)) {
                    drain();
                    return;
                }
            } else {
                factor_part<false>(A.fac, A.a_rowptr, A.a_colidx, A.a_diag, A.lu, A.gflag, A.epoch, w, A.st);
            }
        } else {
            factor_part<false>(A.fac, A.a_rowptr, A.a_colidx, A.a_diag, A.lu, A.gflag, A.epoch, w, A.st);
        }
        BAAS_BARRIER();
        trace_mark(A.trace, 2);

        // pack this CTA's value slots of L and U = L^T (IC0_preconditioner split,
        // test/iccg_level_merge.cpp:874-891)
        if constexpr (FW) {
            for (int d = 0; d < 2; d++)
                fetch_pack<T>(A.fp.dir[d], A.fp.dir[d].code, A.lu, kMixed ? (T *)A.gf32[d] : (T *)A.gf64[d]);
        } else if constexpr (LW) {
            for (int d = 0; d < 2; d++)
                level_pack<T>(A.lv[d], A.lv[d].src, A.lv[d].dsrc, A.lu, kMixed ? (T *)A.lv32[d] : (T *)A.lv64[d],
                              kMixed ? (T *)A.ld32[d] : (T *)A.ld64[d], gt, W);
        } else {
            pack_factor<T>(A.pl.dir[0], A.lu, A.gv64[0], A.gv32[0]);
            pack_factor<T>(A.pl.dir[1], A.lu, A.gv64[1], A.gv32[1]);
        }
        fence_async_global();
    }
    if constexpr (FW) {
        // the record values this CTA walks first: FP32 both directions (they stay), FP64 the
        // lower block (the upper one follows each lower walk)
        __syncthreads();
        if (threadIdx.x == 0) {
            if constexpr (kMixed) {
                fetch_issue_vals<T>(A.fp, F, reinterpret_cast<T *const *>(A.gf32), 0, true);
            } else {
                fetch_issue_vals<T>(A.fp, F, reinterpret_cast<T *const *>(A.gf64), 0, false);
            }
            vpend = 0;
        }
    }
    // r = b - A x; sentinels
    double acc = 0.0;
    for (int i0 = gt; i0 < n; i0 += kLanes * W)
        csr_rows<kLanes>(A.a_rowptr, A.a_colidx, A.a_val, A.x, i0, W, n, [&](int i, double s) {
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
        });
    put_partial<kStageBlock>(A.part_b, acc);
    BAAS_BARRIER();
    const double norm0 = sqrt(grid_total<kStageBlock>(A.part_b, gridDim.x));
    trace_mark(A.trace, 3);

    double rzl = 0.0;
    if constexpr (FW) {
        bool ok = mbar_wait(&F.ctl->mbar_ints, 0u, A.spin_limit);
        if (kMixed) ok = mbar_wait(&F.ctl->mbar_vals, 0u, A.spin_limit) && ok;
        if (!ok && atomicCAS(&A.st->code, kOk, kTimeout) == kOk) A.st->where = -3000001;
        if (__syncthreads_or(!ok)) {
            drain();
            return;
        }
        ints_pending = false;
        if (kMixed && threadIdx.x == 0) vpend = -1;
    }
    auto precond = [&](bool set_p, double &rzp) -> bool {
        if constexpr (FW)
            return fetch_precond<T, IEEE>(A, F, set_p, rzp, vpend);
        else if constexpr (LW)
            return level_precond<T>(A, set_p, rzp, nb);
        else
            return chunk_precond<T, STG, IEEE>(A, ws, smem, set_p, rzp, w);
    };
    if (!precond(true, rzl)) {
        drain();
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
        for (int i0 = gt; i0 < n; i0 += kLanes * W)
            csr_rows<kLanes>(A.a_rowptr, A.a_colidx, A.a_val, A.p, i0, W, n, [&](int i, double s) {
                A.Ap[i] = s;
                acc = __dadd_rn(acc, __dmul_rn(A.p[i], s));
                if constexpr (kMixed)
                    A.y32[i] = Sent<float>::value();
                else
                    A.y[i] = Sent<double>::value();
            });
        put_partial<kStageBlock>(A.part_a, acc);
        BAAS_BARRIER();
        const double alpha = old_rz / grid_total<kStageBlock>(A.part_a, gridDim.x);
        if (k <= 8) trace_mark(A.trace, 6 + 5 * (k - 1));

        acc = 0.0;
        for (int i0 = gt; i0 < n; i0 += kLanes * W) {
            double xv[kLanes], pv[kLanes], rv[kLanes], av[kLanes];
#pragma unroll
            for (int u = 0; u < kLanes; u++) {
                const int i = i0 + u * W;
                if (i < n) {
                    xv[u] = A.x[i];
                    pv[u] = A.p[i];
                    rv[u] = A.r[i];
                    av[u] = A.Ap[i];
                }
            }
#pragma unroll
            for (int u = 0; u < kLanes; u++) {
                const int i = i0 + u * W;
                if (i < n) {
                    A.x[i] = __dadd_rn(xv[u], __dmul_rn(alpha, pv[u]));
                    const double ri = __dadd_rn(rv[u], __dmul_rn(-alpha, av[u]));
                    A.r[i] = ri;
                    acc = __dadd_rn(acc, __dmul_rn(ri, ri));
                    if constexpr (kMixed)
                        A.z32[i] = Sent<float>::value();
                    else
                        A.z[i] = Sent<double>::value();
                }
            }
        }
        put_partial<kStageBlock>(A.part_b, acc);
        BAAS_BARRIER();
        rel = sqrt(grid_total<kStageBlock>(A.part_b, gridDim.x)) / norm0;
        if (k <= 8) trace_mark(A.trace, 7 + 5 * (k - 1));
        iters = k;
        if (rel < A.tol) break;

        rzl = 0.0;
        if (!precond(false, rzl)) {
            drain();
            return;
        }
        if (k <= 8) trace_mark(A.trace, 8 + 5 * (k - 1));
        put_partial<kStageBlock>(A.part_c, rzl);
        BAAS_BARRIER();
        rz = grid_total<kStageBlock>(A.part_c, gridDim.x);
        const double beta = rz / old_rz;
        if (k <= 8) trace_mark(A.trace, 9 + 5 * (k - 1));

        for (int i0 = gt; i0 < n; i0 += kLanes * W) {
            double zv[kLanes], pv[kLanes];
#pragma unroll
            for (int u = 0; u < kLanes; u++) {
                const int i = i0 + u * W;
                if (i < n) {
                    zv[u] = kMixed ? (double)A.z32[i] : A.z[i];
                    pv[u] = A.p[i];
                }
            }
#pragma unroll
            for (int u = 0; u < kLanes; u++) {
                const int i = i0 + u * W;
                if (i < n) A.p[i] = __dadd_rn(zv[u], __dmul_rn(beta, pv[u]));
            }
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
    drain();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *A.out_iters = iters;
        *A.out_relres = rel;
    }
#undef BAAS_BARRIER
}

// Standalone sweep of the caller's triangular CSR by the fetch walk (fetch.cuh): one right-hand
// side, direction d (0: L, 1: U = L^T). gv: this direction's record values, gathered from tval
// here. xg: the schedule's publication buffer for this call (every entry holds the sentinel on
// entry; the rows' results are published there for the other CTAs' fetchers, the values being
// their own ready flags); xnext: the other buffer, which each CTA resets to the sentinel for its
// rows once its walk is done, so that the next call finds it ready without a separate fill
// launch; x: the caller's solution, written from the CTA's slots. IEEE: divide with __ddiv_rn
// (the repeat of a launch whose div_fast divisions left their range).
template <bool IEEE>
__global__ void __launch_bounds__(kStageBlock, 1) k_sweep_fetch(FetchPlan fp, int d, const double *__restrict__ tval,
                                                               double *gv, const double *__restrict__ b, double *x,
                                                               double *xg, double *xnext, DevStatus *st,
                                                               unsigned int spin, unsigned long long *trace) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr unsigned int S = sizeof(double);
    const int tid = (int)threadIdx.x;
    trace_mark(trace, 0);
    const FetchSh F = fetch_layout<double>(fp, smem, false);
    if (tid == 0) {
        F.ctl->err = 0;
        mbar_init(&F.ctl->mbar_ints, 1);
        mbar_init(&F.ctl->mbar_vals, 1);
        fence_mbar_init();
    }
    fetch_pack<double>(fp.dir[d], fp.dir[d].codeT, tval, gv);
    fence_async_global();
    __syncthreads();
    if (tid == 0) {
        fetch_issue_ints(fp, F, false, d);
        double *const gvs[2] = {gv, gv};
        fetch_issue_vals<double>(fp, F, gvs, d, false);
    }
    fetch_stage_lists(fp, F);
    for (int k = tid; k < F.nrows; k += blockDim.x) Sh<double>::stu(F.SL + S * (unsigned int)k, b[__ldg(fp.srow + F.s0 + k)]);
    fetch_reset_slots<double>(F.SL, F.nrows, F.nf0 + F.nf1);
    bool ok = mbar_wait(&F.ctl->mbar_ints, 0u, spin);
    ok = mbar_wait(&F.ctl->mbar_vals, 0u, spin) && ok;
    if (!ok && atomicCAS(&st->code, kOk, kTimeout) == kOk) st->where = -3000002;
    if (__syncthreads_or(!ok)) {
        if (tid == 0) {  // both copies were issued: let them land before the CTA exits
            mbar_wait(&F.ctl->mbar_ints, 0u, spin);
            mbar_wait(&F.ctl->mbar_vals, 0u, spin);
        }
        return;
    }
    trace_mark(trace, 1);
    bool slow = false;
    if (tid >= kFetchWarp * 32) {
        fetch_run<double>(F.FL[d], d ? F.nf1 : F.nf0, xg, F.SL + S * (unsigned int)(F.nrows + 1 + (d ? F.nf0 : 0)), spin,
                          st, F.ctl);
    } else if (tid < fp.ncomp) {
        walk_fetch<double, IEEE ? 2 : 1>(F.I[0], F.V[d], F.SL, F.RW, F.ns[d], fp.ncomp, xg, spin, st, F.ctl, slow);
    }
    if (!IEEE && slow) st->slow_div = 1;
    // every slot holds its row's result (or, after a failed wait, whatever it held): the caller's
    // solution, and the next call's publication buffer reset for this CTA's rows
    if (__syncthreads_or(F.ctl->err)) return;
    for (int k = tid; k < F.nrows; k += blockDim.x) {
        const int row = __ldg(fp.srow + F.s0 + k);
        x[row] = Sh<double>::ldu(F.SL + S * (unsigned int)k);
        xnext[row] = Sent<double>::value();
    }
    trace_mark(trace, 2);
}

// Standalone sweep of the caller's triangular CSR by the level walk: one right-hand side,
// values packed from tval into v/d here; bar must be 0 on entry.
__global__ void __launch_bounds__(kStageBlock, 1) k_sweep_levels(LevelDir D, const double *__restrict__ tval, double *v,
                                                                double *d, const double *b, double *x, unsigned int *bar,
                                                                DevStatus *st, unsigned int spin) {
    unsigned int nb = 0;
    const int W = gridDim.x * blockDim.x, gt = blockIdx.x * blockDim.x + threadIdx.x;
    level_pack<double>(D, D.srcT, D.dsrcT, tval, v, d, gt, W);
    if (!grid_barrier(bar, nb, st, spin)) return;
    level_walk<double, double>(D, v, d, b, x, bar, nb, st, spin);
}

}  // namespace baas

namespace baas {

// ILU0 by the level walk's plan: every thread of the launch takes groups of the current level
// (grid stride), factors their rows in order, and a grid barrier ends the level, so no row waits
// on a flag. Row i (merge/ILU.cpp:638-720): for each lower entry j in ascending column order,
// lu_ij /= lu_jj, then every later entry of row i whose column row j's upper part also holds loses
// lu_ij * lu_j,col -- the same operations on the same values as k_factor_part<true>, so the factor
// is bit-identical. Rows of at most kFacRegs entries whose lower entries (at most kIluLow) each
// name a row with at most kIluUp upper entries run from registers: the row, its pivots and its
// partners' upper entries are loaded first, all at once; each entry of row i matches at most one
// upper entry of a given row j, so applying row j's matches in any order gives the merge's result.
// Other rows take ilu0_row_merge, the reference's merge loop.
constexpr int kIluLow = 4, kIluUp = 4;

__device__ __forceinline__ void ilu0_row_merge(int i, const int *__restrict__ rowptr, const int *__restrict__ colidx,
                                               const int *__restrict__ diagptr, double *lu, DevStatus *st) {
    const int rb = __ldg(rowptr + i), di = __ldg(diagptr + i), re = __ldg(rowptr + i + 1);
    for (int j = rb; j < di; j++) {
        const int c = __ldg(colidx + j);
        const int dc = __ldg(diagptr + c), ec = __ldg(rowptr + c + 1);
        const double pivot = ld_l2(lu + dc);
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
                lu[k1] = __dsub_rn(lu[k1], __dmul_rn(tmp, ld_l2(lu + k2)));
                k1++;
                k2++;
            }
        }
    }
}

// A row of the level ILU0 in registers: its record (host-built per plan position: row, first
// entry, entries, lower entries -- entries < 0 sends the row down the merge path), its columns and
// values, and per lower entry the partner row's diagonal position and upper-entry count. All of it
// is static or not yet written when a level starts, so the next level's first row is loaded before
// the barrier; only the pivots and the partners' upper values wait for it.
struct IluRow {
    int i, rb, n, nlow;
    int c[kFacRegs];
    double v[kFacRegs];
    int dc[kIluLow], nu[kIluLow];
};

__device__ __forceinline__ void ilu_load(int p, const int4 *__restrict__ irec, const int2 *__restrict__ idep,
                                         const int *__restrict__ colidx, const double *lu, IluRow &R) {
    const int4 r = __ldg(irec + p);
    R.i = r.x;
    R.rb = r.y;
    R.n = r.z;
    R.nlow = r.w;
#pragma unroll
    for (int t = 0; t < kFacRegs; t++)
        if (t < R.n) {
            R.c[t] = __ldg(colidx + R.rb + t);
            R.v[t] = lu[R.rb + t];
        }
#pragma unroll
    for (int t = 0; t < kIluLow; t++)
        if (t < R.nlow) {
            const int2 d = __ldg(idep + (size_t)p * kIluLow + t);
            R.dc[t] = d.x;
            R.nu[t] = d.y;
        }
}

__device__ __forceinline__ void ilu_finish(IluRow &R, const int *__restrict__ rowptr, const int *__restrict__ colidx,
                                           const int *__restrict__ diagptr, double *lu, DevStatus *st) {
    if (R.n < 0) {
        ilu0_row_merge(R.i, rowptr, colidx, diagptr, lu, st);
        return;
    }
    double piv[kIluLow], uv[kIluLow][kIluUp];
    int uc[kIluLow][kIluUp];
#pragma unroll
    for (int t = 0; t < kIluLow; t++)
        if (t < R.nlow) {
            piv[t] = ld_l2(lu + R.dc[t]);
#pragma unroll
            for (int q = 0; q < kIluUp; q++)
                if (q < R.nu[t]) {
                    uc[t][q] = __ldg(colidx + R.dc[t] + 1 + q);
                    uv[t][q] = ld_l2(lu + R.dc[t] + 1 + q);
                }
        }
#pragma unroll
    for (int t = 0; t < kIluLow; t++)
        if (t < R.nlow) {
            if (piv[t] == 0.0) atomicAdd(&st->zero_pivots, 1);
            const double tmp = __ddiv_rn(R.v[t], piv[t]);
            R.v[t] = tmp;
#pragma unroll
            for (int q = 0; q < kIluUp; q++)
                if (q < R.nu[t]) {
#pragma unroll
                    for (int u = 0; u < kFacRegs; u++)
                        if (u > t && u < R.n && R.c[u] == uc[t][q]) R.v[u] = __dsub_rn(R.v[u], __dmul_rn(tmp, uv[t][q]));
                }
        }
#pragma unroll
    for (int t = 0; t < kFacRegs; t++)
        if (t < R.n) lu[R.rb + t] = R.v[t];
}

__global__ void __launch_bounds__(kStageBlock, 1) k_ilu0_levels(LevelDir D, const int4 *__restrict__ irec,
                                                                const int2 *__restrict__ idep,
                                                                const int *__restrict__ rowptr,
                                                                const int *__restrict__ colidx,
                                                                const int *__restrict__ diagptr, double *lu,
                                                                unsigned int *bar, DevStatus *st, unsigned int limit) {
    const int W = gridDim.x * blockDim.x;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned int nb = 0;
    IluRow cur, nxt;
    cur.i = -1;
    // this thread's first item of level l: its first position is prefetched one level ahead
    auto first = [&](int l) -> int {
        const int it = __ldg(D.lev + l) + gt;
        return it < __ldg(D.lev + l + 1) ? bounded(__ldg(D.item + it), D.npos, st, 141) : -1;
    };
    if (D.nlev > 0) {
        const int p0 = first(0);
        if (p0 >= 0) ilu_load(p0, irec, idep, colidx, lu, cur);
    }
    for (int l = 0; l < D.nlev; l++) {
        const int ib = __ldg(D.lev + l), ie = __ldg(D.lev + l + 1);
        nxt.i = -1;
        if (l + 1 < D.nlev) {
            const int pn = first(l + 1);
            if (pn >= 0) ilu_load(pn, irec, idep, colidx, lu, nxt);
        }
        for (int it = ib + gt; it < ie; it += W) {
            int p = __ldg(D.item + it);
            const int pe = __ldg(D.item + it + 1);
            if (it == ib + gt && cur.i >= 0) {
                ilu_finish(cur, rowptr, colidx, diagptr, lu, st);
                p++;
            }
            for (; p < pe; p++) {  // the group's later rows, and the thread's further groups
                IluRow r;
                ilu_load(bounded(p, D.npos, st, 142), irec, idep, colidx, lu, r);
                ilu_finish(r, rowptr, colidx, diagptr, lu, st);
            }
        }
        if (!grid_barrier(bar, nb, st, limit)) return;
        cur = nxt;
    }
}

}  // namespace baas
