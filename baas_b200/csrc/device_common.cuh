// Device helpers shared by the sparse kernels: memory-model-explicit loads and stores, the
// "not yet written" sentinel used by the sweeps, bounded waits, a bounded grid barrier and a
// deterministic block reduction.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace baas {

// Status words written by kernels (mirrors baas_status).
enum : int { kOk = 0, kTimeout = 3, kZeroPivot = 4, kBounds = 5 };

struct DevStatus {
    int code;        // first error (kOk if none)
    int zero_pivots; // count of non-positive IC0 / zero ILU0 pivots
    int where;       // row or barrier index where a wait gave up
    int slow_div;    // set when an FP64 sweep division left div_fast's proven range (rerun with IEEE)
};

// --- relaxed / acquire / release accesses at GPU scope (PTX memory model) ---
// The relaxed forms carry values that are their own ready flags, so they order nothing else:
// they are `asm volatile` (never removed, merged or hoisted out of a polling loop) but have no
// "memory" clobber, which would make every one of them a compiler barrier and serialise the
// surrounding shared-memory loads (measured: ~5x slower sweep steps). The acquire / release /
// fence forms below do order other accesses and keep the clobber.
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const void *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ unsigned int ld_relaxed_u32(const void *p) {
    unsigned int v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(void *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v));
}
__device__ __forceinline__ void st_relaxed_u32(void *p, unsigned int v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v));
}
__device__ __forceinline__ int ld_acquire_s32(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_s32(int *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned int atom_add_release_u32(unsigned int *p, unsigned int v) {
    unsigned int old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// --- sentinels: signalling-NaN bit patterns. Arithmetic never produces a signalling NaN
// (results of NaN inputs are quiet), so a solution slot holding the sentinel has not been
// written yet. The value itself is the ready flag: one load both waits and fetches. ---
constexpr unsigned long long kSent64 = 0xFFF0DEADBEEF0001ull;
constexpr unsigned int kSent32 = 0xFF80DEADu;

template <typename T> struct Sent;
template <> struct Sent<double> {
    static __device__ __forceinline__ bool is(double v) { return (unsigned long long)__double_as_longlong(v) == kSent64; }
    static __device__ __forceinline__ double value() { return __longlong_as_double((long long)kSent64); }
    static __device__ __forceinline__ double load(const double *p) { return __longlong_as_double((long long)ld_relaxed_u64(p)); }
    static __device__ __forceinline__ void store(double *p, double v) { st_relaxed_u64(p, (unsigned long long)__double_as_longlong(v)); }
};
template <> struct Sent<float> {
    static __device__ __forceinline__ bool is(float v) { return __float_as_uint(v) == kSent32; }
    static __device__ __forceinline__ float value() { return __uint_as_float(kSent32); }
    static __device__ __forceinline__ float load(const float *p) { return __uint_as_float(ld_relaxed_u32(p)); }
    static __device__ __forceinline__ void store(float *p, float v) { st_relaxed_u32(p, __float_as_uint(v)); }
};

// Bounded wait bookkeeping: the limit applies to each wait on its own (every wait starts with
// begin()). Every 128 polls the wait also looks at the shared status word so that one failure
// ends every waiting thread promptly. tick() returns false when the caller must stop.
struct Waiter {
    unsigned int polls;
    unsigned int limit;
    DevStatus *st;
    bool slow;  // this thread met a division outside div_fast's range
    __device__ __forceinline__ Waiter(unsigned int lim, DevStatus *s) : polls(0), limit(lim), st(s), slow(false) {}
    __device__ __forceinline__ void begin() { polls = 0; }
    __device__ __forceinline__ bool tick(int where) {
        ++polls;
        if ((polls & 127u) == 0u) {
            if (ld_relaxed_u32(&st->code) != 0u) return false;
            if (polls >= limit) {
                if (atomicCAS(&st->code, kOk, kTimeout) == kOk) st->where = where;
                return false;
            }
        }
        return true;
    }
};

// Bounds-checked builds (-DBAAS_DEBUG_BOUNDS: python -m baas_b200.build --debug-bounds): an index
// outside [0, n) is recorded (status kBounds, `where` = the check's site) and replaced by 0, so the
// kernel goes on without touching memory outside the array and the host reports the first site.
// In the ordinary build the check compiles to nothing.
__device__ __forceinline__ int bounded(int i, int n, DevStatus *st, int site) {
#ifdef BAAS_DEBUG_BOUNDS
    if ((unsigned int)i >= (unsigned int)n) {
        if (atomicCAS(&st->code, kOk, kBounds) == kOk) st->where = site;
        return 0;
    }
#else
    (void)n;
    (void)st;
    (void)site;
#endif
    return i;
}

// Shared-memory value-as-flag (producer and consumer in the same CTA).
template <typename T> struct SSent;
template <> struct SSent<double> {
    static __device__ __forceinline__ double load(const double *p) { return *(const volatile double *)p; }
    static __device__ __forceinline__ void store(double *p, double v) { *(volatile double *)p = v; }
};
template <> struct SSent<float> {
    static __device__ __forceinline__ float load(const float *p) { return *(const volatile float *)p; }
    static __device__ __forceinline__ void store(float *p, float v) { *(volatile float *)p = v; }
};

template <typename T>
__device__ __forceinline__ bool wait_smem(const T *p, T &out, Waiter &w, int where) {
    w.begin();
    T v = SSent<T>::load(p);
    while (Sent<T>::is(v)) {
        if (!w.tick(where)) return false;
        v = SSent<T>::load(p);
    }
    out = v;
    return true;
}

// Wait until *p no longer holds the sentinel; returns false if the wait was abandoned.
template <typename T>
__device__ __forceinline__ bool wait_value(const T *p, T &out, Waiter &w, int where) {
    w.begin();
    T v = Sent<T>::load(p);
    while (Sent<T>::is(v)) {
        if (!w.tick(where)) return false;
        v = Sent<T>::load(p);
    }
    out = v;
    return true;
}

// Wait until an epoch-stamped ready flag reaches `epoch` (acquire).
__device__ __forceinline__ bool wait_flag(const int *flag, int epoch, Waiter &w, int where) {
    w.begin();
    while (ld_acquire_s32(flag) != epoch) {
        if (!w.tick(where)) return false;
    }
    return true;
}

// Grid barrier over all CTAs of a co-resident (cooperative) launch. `counter` starts at 0 for
// the launch and only grows; barrier number k (0-based) completes when it reaches
// (k+1)*gridDim.x. The wait is bounded. Returns false -- uniformly for the whole CTA -- when
// the wait gave up or the status word carries an error, so every CTA leaves at the same
// barrier or, at the latest, at the next one.
__device__ __forceinline__ bool grid_barrier(unsigned int *counter, unsigned int &k, DevStatus *st, unsigned int limit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int target = (k + 1) * gridDim.x;
        __threadfence();
        atom_add_release_u32(counter, 1u);
        Waiter w(limit, st);
        int ok = 1;
        while (ld_acquire_u32(counter) < target) {
            if (!w.tick(-1 - (int)k)) {
                ok = 0;
                break;
            }
        }
        __threadfence();
        if (ld_relaxed_u32(&st->code) != 0u) ok = 0;
        s_ok = ok;
    }
    ++k;
    __syncthreads();
    return s_ok != 0;
}

// --- shared-memory mbarriers and untiled bulk copies (the TMA engine's cp.async.bulk form):
// global -> shared copies of contiguous, 16-byte aligned blocks whose size is a multiple of
// 16 bytes, completion counted in bytes on an mbarrier. ---
__device__ __forceinline__ unsigned int smem_u32(const void *p) { return (unsigned int)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes mbarrier initialisation visible to the async proxy (the bulk-copy engine)
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// orders this thread's earlier shared-memory accesses before its later async-proxy ones
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// orders this thread's generic-proxy global writes before later async-proxy reads of them
__device__ __forceinline__ void fence_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned int bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned int bytes, unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned int parity) {
    unsigned int ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}
// Bounded wait for the completion of phase `parity` of `bar` (each try_wait may suspend the
// thread for a while, so `limit` tries last far longer than `limit` polls).
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned int parity, unsigned int limit) {
    for (unsigned int i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Reciprocal stored beside a diagonal entry d for div_fast: RN(1/d) (__drcp_rn) when
// 2^-500 <= |d| < 2^500, else 0, which sends every division by d to __ddiv_rn.
__device__ __forceinline__ double div_recip(double d) {
    const unsigned int e = ((unsigned int)__double2hiint(d) >> 20) & 0x7ffu;  // biased exponent
    return e - (1023u - 500u) <= 999u ? __drcp_rn(d) : 0.0;
}

// Correctly rounded FP64 quotient a / b from y = div_recip(b), by Markstein's method
// (P. Markstein, "Computation of elementary functions on the IBM RISC System/6000 processor",
// IBM J. Res. Dev. 34(1), 1990; Muller et al., Handbook of Floating-Point Arithmetic, division
// with an FMA): q0 = RN(a*y) lies within two ulps of a/b; one correction
// q1 = RN(q0 + RN(a - b*q0)*y) makes it a faithful rounding; then, y being RN(1/b) and the
// remainder a - b*q1 exact in an FMA, q2 = RN(q1 + (a - b*q1)*y) = RN(a/b). The remainders are
// exact and nothing under- or overflows while 2^-500 <= |b| < 2^500 (y != 0) and
// 2^-460 <= |a| < 2^461: then 2^-961 <= |a/b| <= 2^961 and the remainders' lowest bits stay
// above 2^-570. a = +0 also comes out right (+0 / b: every step keeps the zero and its sign
// follows y); a = -0 does not (the first remainder turns it into +0). Every other a (-0,
// subnormals, the far ranges, infinities, NaNs) and every b outside the range set `slow`, and
// the caller must then compute the quotient with __ddiv_rn instead. The range test reads a's
// bits and runs beside the FMA chain.
__device__ __forceinline__ double div_fast(double a, double b, double y, bool &slow) {
    const unsigned int hi = (unsigned int)__double2hiint(a), lo = (unsigned int)__double2loint(a);
    const unsigned int ea = (hi >> 20) & 0x7ffu;
    const bool fast = (ea - (1023u - 460u) <= 920u || (hi | lo) == 0u) && y != 0.0;
    const double q0 = __dmul_rn(a, y);
    const double r0 = __fma_rn(-q0, b, a);
    const double q1 = __fma_rn(r0, y, q0);
    const double r1 = __fma_rn(-q1, b, a);
    const double q2 = __fma_rn(r1, y, q1);
    slow |= !fast;
    return q2;
}

// div_fast with its fall-back: always RN(a/b). The sweeps do not use it (they repeat a flagged
// launch instead); baas_test_divide does, to check div_fast quotient by quotient.
__device__ __forceinline__ double div_rcp(double a, double b, double y) {
    bool slow = false;
    const double q = div_fast(a, b, y, slow);
    return slow ? __ddiv_rn(a, b) : q;
}

// Explicit shared-memory accesses for data reached through pointers the compiler cannot prove
// to be shared (window buffers, staged arrays handed through structures): a generic access to
// shared memory is resolved in the L1TEX unit and costs far more than ld/st.shared. Volatile,
// so they keep their order relative to one another and to barriers; no "memory" clobber, so
// they do not serialise the surrounding code.
template <typename T> struct Sh;
// ldu / stu take 32-bit shared-window addresses, so address arithmetic stays in 32 bits: one
// integer add per access instead of a 64-bit generic address and its conversion.
template <> struct Sh<int> {
    static __device__ __forceinline__ int ldu(unsigned int a) {
        int v;
        asm volatile("ld.shared.s32 %0, [%1];" : "=r"(v) : "r"(a));
        return v;
    }
    static __device__ __forceinline__ void stu(unsigned int a, int v) { asm volatile("st.shared.s32 [%0], %1;" ::"r"(a), "r"(v)); }
    static __device__ __forceinline__ int ld(const int *p) { return ldu(smem_u32(p)); }
    static __device__ __forceinline__ void st(int *p, int v) { stu(smem_u32(p), v); }
};
template <> struct Sh<float> {
    static __device__ __forceinline__ float ldu(unsigned int a) {
        float v;
        asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
        return v;
    }
    static __device__ __forceinline__ void stu(unsigned int a, float v) { asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v)); }
    static __device__ __forceinline__ float ld(const float *p) { return ldu(smem_u32(p)); }
    static __device__ __forceinline__ void st(float *p, float v) { stu(smem_u32(p), v); }
};
template <> struct Sh<double> {
    static __device__ __forceinline__ double ldu(unsigned int a) {
        double v;
        asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
        return v;
    }
    static __device__ __forceinline__ void stu(unsigned int a, double v) { asm volatile("st.shared.f64 [%0], %1;" ::"r"(a), "d"(v)); }
    static __device__ __forceinline__ double ld(const double *p) { return ldu(smem_u32(p)); }
    static __device__ __forceinline__ void st(double *p, double v) { stu(smem_u32(p), v); }
};

// Phase tracing (BAAS_TRACE=1): thread 0 of the first and last CTA record %globaltimer (ns)
// at phase boundaries into trace[cta_sel * kTraceSlots + k]; a NULL trace disables it.
constexpr int kTraceSlots = 64;
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void trace_mark(unsigned long long *trace, int k) {
    if (trace && threadIdx.x == 0 && k < kTraceSlots && (blockIdx.x == 0 || blockIdx.x == gridDim.x - 1))
        trace[(blockIdx.x == 0 ? 0 : kTraceSlots) + k] = gtimer();
}

// Deterministic sum over the block (fixed shuffle tree, fixed warp order). All threads
// receive the result.
template <int BLOCK>
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double s_part[BLOCK / 32];
    __shared__ double s_total;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) s_part[wid] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < BLOCK / 32; i++) t += s_part[i];
        s_total = t;
    }
    __syncthreads();
    double r = s_total;
    __syncthreads();
    return r;
}

// Every CTA sums the per-CTA partials in CTA order and gets the bitwise-same value.
template <int BLOCK>
__device__ __forceinline__ double grid_total(const double *partials, int nparts) {
    double v = 0.0;
    // each thread sums a strided subset in a fixed order, then a fixed block tree
    for (int i = threadIdx.x; i < nparts; i += BLOCK) v += Sent<double>::load(partials + i);
    return block_sum<BLOCK>(v);
}

}  // namespace baas
