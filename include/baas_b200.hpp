// C++ facade over the C ABI (baas_b200.h) with the reference's runtime surface, so that code
// written against the reference's Schedule::Scheduler and its runtime classes switches to the
// GPU by changing the include and the namespace:
//
//   reference (test/Schedule.hpp:39-177)          this header
//   Schedule::Scheduler(csrA, isSymmetric,         baas_b200::Scheduler<CSR>(same arguments)
//       isTRSVPerm, ALG_SCHEDULE, num_thread)
//   preprocessing()                                preprocessing()          -> baas_analyze
//   runIC0(mat, lu)                                runIC0(mat, lu)          -> baas_ic0
//   runForwardTRSVNoPerm(L, x, b)                  runForwardTRSVNoPerm     -> baas_sptrsv(upper=0)
//   runBackwardTRSVNoPerm(U, x, b)                 runBackwardTRSVNoPerm    -> baas_sptrsv(upper=1)
//   SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRule  SpTRSVRuntime<CSR>  (test/SpTRSVRuntime.hpp:617-852)
//   IC_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRule      ICRuntime<CSR>      (test/ICRuntime.hpp:353-583)
//   ILU_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRule     ILURuntime<CSR>     (test/ILURuntime.hpp:207-436)
//
// CSR is any type with the members of the reference's SPM::CSR that these calls read
// (spm/include/CSR.hpp:16-30): int m, n; int *rowptr, *colidx; double *values -- the reference's
// own SPM::CSR works unchanged. As in the reference, matrices and vectors are HOST arrays owned by
// the caller; the facade keeps device mirrors and copies in and out around each call (the C ABI
// itself takes device arrays, for callers that keep their data on the GPU). Errors throw
// std::runtime_error, as the reference does for unsupported configurations
// (test/Schedule.hpp:252, 278). Like the reference, an object is not re-entrant.
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "baas_b200.h"

namespace baas_b200 {

// test/Schedule.hpp:31-37. All four are built: P2P_RULE (the BAAS four-rule mapping), P2P
// (level merge and a cost-balanced split per level), P2P_MAPPING (parent-thread affinity with
// load rebalancing) and P2P_TIME (earliest-finishing threads first).
enum ALG_SCHEDULE { P2P, P2P_MAPPING, P2P_TIME, P2P_RULE };

namespace detail {

inline void check(baas_status st, const char *where) {
    if (st != BAAS_OK) throw std::runtime_error(std::string(where) + ": " + baas_last_error_string());
}
inline void check_cuda(cudaError_t e, const char *where) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e));
}

// A device array that grows on demand.
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t cap = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    T *get(size_t n) {
        if (n > cap) {
            if (p) cudaFree(p);
            p = nullptr;
            check_cuda(cudaMalloc((void **)&p, (n ? n : 1) * sizeof(T)), "cudaMalloc");
            cap = n;
        }
        return p;
    }
    T *put(const T *h, size_t n) {
        T *d = get(n);
        check_cuda(cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
        return d;
    }
    void take(T *h, size_t n) const { check_cuda(cudaMemcpy(h, p, n * sizeof(T), cudaMemcpyDeviceToHost), "cudaMemcpy D2H"); }
};

// Device mirror of a host CSR (pattern uploaded once per distinct pattern pointer).
struct DevCsr {
    DevBuf<int> rowptr, colidx;
    DevBuf<double> values;
    const int *host_rowptr = nullptr;
    int n = 0, nnz = 0;
    template <typename CSR>
    baas_csr upload(const CSR *A, bool with_values = true) {
        n = A->m;
        nnz = A->rowptr[A->m];
        if (host_rowptr != A->rowptr) {
            rowptr.put(A->rowptr, (size_t)n + 1);
            colidx.put(A->colidx, (size_t)nnz);
            host_rowptr = A->rowptr;
        }
        if (with_values) values.put(A->values, (size_t)nnz);
        return baas_csr{n, nnz, rowptr.p, colidx.p, with_values ? values.p : values.get((size_t)nnz)};
    }
};

template <typename CSR>
baas_csr host_pattern(const CSR *A) {
    return baas_csr{A->m, A->rowptr[A->m], A->rowptr, A->colidx, nullptr};
}

}  // namespace detail

// Schedule::Scheduler (test/Schedule.hpp:39-353): owns the BAAS schedule of A's lower triangle
// and runs IC0 and the two sweeps. isSymmetric = false builds the same schedule without the
// backward one, as the reference's preprocessing does (test/Schedule.hpp:289-292): IC0 and the
// forward sweep run, and a backward sweep throws (the reference has no schedule for it then).
// isTRSVPerm = false only (the thread-contiguous permuted variant is not built).
template <typename CSR>
class Scheduler {
   public:
    Scheduler(const CSR *csrA, bool isSymmetric, bool isTRSVPerm, ALG_SCHEDULE alg, int num_thread)
        : csrA_(csrA), num_thread_(num_thread), symmetric_(isSymmetric) {
        if (isTRSVPerm) throw std::runtime_error("Scheduler: the permuted (isTRSVPerm) variant is not built");
        mapping_ = alg == P2P           ? BAAS_MAPPING_COST_SPLIT
                   : alg == P2P_TIME    ? BAAS_MAPPING_FINISH_TIME
                   : alg == P2P_MAPPING ? BAAS_MAPPING_AFFINITY
                                        : BAAS_MAPPING_FOUR_RULE;
    }
    ~Scheduler() { baas_destroy(s_); }
    Scheduler(const Scheduler &) = delete;
    Scheduler &operator=(const Scheduler &) = delete;

    // Schedule construction (Scheduler::preprocessing, test/Schedule.hpp:181-296).
    void preprocessing() {
        baas_options o;
        baas_options_default(&o);
        o.nthread = num_thread_;
        o.mapping = mapping_;
        const baas_csr a = detail::host_pattern(csrA_);
        baas_destroy(s_);
        s_ = nullptr;
        detail::check(baas_analyze(&a, BAAS_KERNEL_ICCG, &o, &s_), "Scheduler::preprocessing");
    }
    // IC0 in place on lu (host, pre-filled with mat->values, merge/IC.hpp:54).
    void runIC0(const CSR *mat, double *lu) {
        baas_csr a = dA_.upload(mat, false);
        double *d = dlu_.put(lu, (size_t)a.nnz);
        detail::check(baas_ic0(sched(), &a, d, nullptr), "Scheduler::runIC0");
        dlu_.take(lu, (size_t)a.nnz);
    }
    // x = L^-1 b, L lower with the diagonal last in each row.
    void runForwardTRSVNoPerm(const CSR *L, double *x, const double *b) { sweep(L, x, b, 0); }
    // x = U^-1 b, U = L^T upper with the diagonal first in each row.
    void runBackwardTRSVNoPerm(const CSR *U, double *x, const double *b) {
        if (!symmetric_) throw std::runtime_error("Scheduler: built with isSymmetric = false, so it has no backward schedule");
        sweep(U, x, b, 1);
    }
    void runForwardTRSV(const CSR *L, double *x, const double *b, bool isPerm) {
        if (isPerm) throw std::runtime_error("Scheduler: the permuted variant is not built");
        runForwardTRSVNoPerm(L, x, b);
    }
    void runBackwardTRSV(const CSR *U, double *x, const double *b, bool isPerm) {
        if (isPerm) throw std::runtime_error("Scheduler: the permuted variant is not built");
        runBackwardTRSVNoPerm(U, x, b);
    }
    baas_schedule *handle() const { return s_; }

   private:
    baas_schedule *sched() {
        if (!s_) preprocessing();
        return s_;
    }
    void sweep(const CSR *T, double *x, const double *b, int upper) {
        baas_csr t = (upper ? dU_ : dL_).upload(T);
        const int n = T->m;
        double *db = db_.put(b, (size_t)n);
        double *dx = dx_.get((size_t)n);
        detail::check(baas_sptrsv(sched(), &t, upper, db, dx, 1, n, nullptr), "Scheduler::sweep");
        dx_.take(x, (size_t)n);
    }
    const CSR *csrA_;
    int num_thread_;
    bool symmetric_;
    int mapping_ = BAAS_MAPPING_FOUR_RULE;
    baas_schedule *s_ = nullptr;
    detail::DevCsr dA_, dL_, dU_;
    detail::DevBuf<double> dlu_, db_, dx_;
};

// Shared part of the runtime classes (FusionDemo / ICDemo / ILUDemo): analysis in buildset(),
// the timed kernel in fused_code(), checked against the caller's correct result in testing();
// evaluate() runs them like FusionDemo::evaluate (test/FusionDemo.cpp:118-178).
class RuntimeBase {
   public:
    virtual ~RuntimeBase() { baas_destroy(s_); }
    double evaluate() {
        setup();
        const auto t0 = std::chrono::steady_clock::now();
        buildset();
        analysis_time_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        double total = 0.0;
        for (int k = 0; k < num_test_; k++) total += fused_code();
        elapsed_time_ = total / num_test_;
        testing();
        return elapsed_time_;
    }
    void set_num_test(int v) { num_test_ = v; }
    void set_num_thread(int v) { num_thread_ = v; }
    double getAnalysisTime() const { return analysis_time_; }
    double getElaspedTime() const { return elapsed_time_; }
    std::string getAlgName() const { return alg_name_; }
    double getMaxError() const { return max_error_; }

   protected:
    virtual void setup() {}
    virtual void buildset() = 0;
    virtual double fused_code() = 0;  // milliseconds of one GPU run (CUDA events)
    virtual void testing() = 0;
    void analyze(const baas_csr &pattern, baas_kernel kind) {
        baas_options o;
        baas_options_default(&o);
        o.nthread = num_thread_;
        o.ablation = ablation_;
        baas_destroy(s_);
        s_ = nullptr;
        detail::check(baas_analyze(&pattern, kind, &o, &s_), alg_name_.c_str());
    }
    template <typename F>
    static double timed(F f) {
        cudaEvent_t a, b;
        detail::check_cuda(cudaEventCreate(&a), "cudaEventCreate");
        detail::check_cuda(cudaEventCreate(&b), "cudaEventCreate");
        cudaEventRecord(a);
        f();
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return ms;
    }
    baas_schedule *s_ = nullptr;
    int num_test_ = 10, num_thread_ = 8;
    int ablation_ = BAAS_ABLATION_NONE;
    double analysis_time_ = 0.0, elapsed_time_ = 0.0, max_error_ = 0.0;
    std::string alg_name_;
};

// SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRule (test/SpTRSVRuntime.hpp:617-852): forward sweep
// of the lower triangle csrL (diagonal last); the result is checked against correct_x.
template <typename CSR>
class SpTRSVRuntime : public RuntimeBase {
   public:
    // ablation: BAAS_ABLATION_NONE for SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRule, or one of the
    // ablation classes' schedules (the aliases below)
    SpTRSVRuntime(const CSR *csrL, const double *correct_x, int n, int nnz, double alpha, std::string algName,
                  int num_thread, int ablation = BAAS_ABLATION_NONE)
        : L_(csrL), correct_x_(correct_x), n_(n), alpha_(alpha), x_(n, 0.0), b_(n, 0.0) {
        (void)nnz;
        alg_name_ = std::move(algName);
        num_thread_ = num_thread;
        ablation_ = ablation;
    }
    const double *getSolution() const { return x_.data(); }

   protected:
    void setup() override {
        // b = L * correct_x * alpha (FusionDemo::setup builds b from the known solution)
        for (int i = 0; i < n_; i++) {
            double s = 0.0;
            for (int e = L_->rowptr[i]; e < L_->rowptr[i + 1]; e++) s += L_->values[e] * correct_x_[L_->colidx[e]];
            b_[i] = s * alpha_;
        }
    }
    void buildset() override {
        analyze(detail::host_pattern(L_), BAAS_KERNEL_SPTRSV);
        t_ = dL_.upload(L_);
        db_.put(b_.data(), (size_t)n_);
    }
    double fused_code() override {
        double *dx = dx_.get((size_t)n_);
        const double ms = timed([&] { detail::check(baas_sptrsv(s_, &t_, 0, db_.p, dx, 1, n_, nullptr), "SpTRSVRuntime"); });
        dx_.take(x_.data(), (size_t)n_);
        return ms;
    }
    void testing() override {
        max_error_ = 0.0;
        for (int i = 0; i < n_; i++) max_error_ = std::max(max_error_, std::fabs(x_[i] - correct_x_[i] * alpha_));
    }

   private:
    const CSR *L_;
    const double *correct_x_;
    int n_;
    double alpha_;
    std::vector<double> x_, b_;
    baas_csr t_{};
    detail::DevCsr dL_;
    detail::DevBuf<double> db_, dx_;
};

// The SpTRSV runtime's ablation classes (test/SpTRSV_level_merge.cpp:156-299), same constructor
// as the reference's: BAASWOS (test/SpTRSVRuntime.hpp:389-615), BAASWOAS (:855-1054), BAASWOA
// (:1056-1262). Their schedules are the reference classes' array for array; the sweep is the GPU's.
template <typename CSR>
class SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P : public SpTRSVRuntime<CSR> {
   public:
    SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P(const CSR *csrL, const double *correct_x, int n, int nnz, double alpha,
                                      std::string algName, int num_thread)
        : SpTRSVRuntime<CSR>(csrL, correct_x, n, nnz, alpha, std::move(algName), num_thread, BAAS_ABLATION_WOS) {}
};
template <typename CSR>
class SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRuleAblationBase : public SpTRSVRuntime<CSR> {
   public:
    SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRuleAblationBase(const CSR *csrL, const double *correct_x, int n, int nnz,
                                                              double alpha, std::string algName, int num_thread)
        : SpTRSVRuntime<CSR>(csrL, correct_x, n, nnz, alpha, std::move(algName), num_thread, BAAS_ABLATION_WOAS) {}
};
template <typename CSR>
class SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRuleAblationWOAggregation : public SpTRSVRuntime<CSR> {
   public:
    SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRuleAblationWOAggregation(const CSR *csrL, const double *correct_x, int n,
                                                                       int nnz, double alpha, std::string algName,
                                                                       int num_thread)
        : SpTRSVRuntime<CSR>(csrL, correct_x, n, nnz, alpha, std::move(algName), num_thread, BAAS_ABLATION_WOA) {}
};

// IC_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRule (test/ICRuntime.hpp:353-583) and
// ILU_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRule (test/ILURuntime.hpp:207-436): in-place
// factorisation of A's values; checked against correct_lu.
template <typename CSR, bool ILU>
class FactorRuntime : public RuntimeBase {
   public:
    FactorRuntime(const CSR *csrA, const double *correct_lu, int n, int nnz, std::string algName, int num_thread)
        : A_(csrA), correct_lu_(correct_lu), nnz_(nnz), lu_((size_t)nnz, 0.0) {
        (void)n;
        alg_name_ = std::move(algName);
        num_thread_ = num_thread;
    }
    const double *getSolution() const { return lu_.data(); }

   protected:
    void buildset() override {
        analyze(detail::host_pattern(A_), ILU ? BAAS_KERNEL_ILU0 : BAAS_KERNEL_IC0);
        a_ = dA_.upload(A_);
    }
    double fused_code() override {
        double *dlu = dlu_.get((size_t)nnz_);
        detail::check_cuda(cudaMemcpy(dlu, a_.values, sizeof(double) * (size_t)nnz_, cudaMemcpyDeviceToDevice), "cudaMemcpy");
        const double ms = timed([&] {
            detail::check(ILU ? baas_ilu0(s_, &a_, dlu, nullptr) : baas_ic0(s_, &a_, dlu, nullptr), alg_name_.c_str());
        });
        dlu_.take(lu_.data(), (size_t)nnz_);
        return ms;
    }
    void testing() override {
        max_error_ = 0.0;
        if (!correct_lu_) return;
        for (int e = 0; e < nnz_; e++) max_error_ = std::max(max_error_, std::fabs(lu_[e] - correct_lu_[e]));
    }

   private:
    const CSR *A_;
    const double *correct_lu_;
    int nnz_;
    std::vector<double> lu_;
    baas_csr a_{};
    detail::DevCsr dA_;
    detail::DevBuf<double> dlu_;
};

template <typename CSR>
using ICRuntime = FactorRuntime<CSR, false>;
template <typename CSR>
using ILURuntime = FactorRuntime<CSR, true>;

}  // namespace baas_b200
