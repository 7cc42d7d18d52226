// C ABI of the B200 BAAS hot path (declarations and contracts: include/baas_b200.h).
//
// baas_analyze builds the reference-identical schedule on the host (schedule.cpp) and the
// device execution plan from it: the schedule's groups listed level by level become the work
// items of the persistent kernels (kernels.cuh), in forward order for the lower sweep and the
// factorisations and in exactly reversed order for the upper sweep. The plan is uploaded on
// the first GPU call; the device is the current device of that call.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/baas_b200.h"
#include "kernels.cuh"
#include "schedule.hpp"

using baas::DevStatus;

namespace {

thread_local std::string g_err;

baas_status fail(baas_status st, const std::string &msg) {
    g_err = msg;
    return st;
}

#define BAAS_CUDA(call)                                                                         \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return fail(BAAS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
    } while (0)

constexpr unsigned int kDefaultSpin = 1u << 22;

template <typename T>
baas_status upload(T *&d, const std::vector<T> &h) {
    d = nullptr;
    if (h.empty()) return BAAS_OK;
    BAAS_CUDA(cudaMalloc((void **)&d, h.size() * sizeof(T)));
    BAAS_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return BAAS_OK;
}

template <typename T>
baas_status dalloc(T *&d, size_t count) {
    d = nullptr;
    if (count == 0) count = 1;
    BAAS_CUDA(cudaMalloc((void **)&d, count * sizeof(T)));
    BAAS_CUDA(cudaMemset(d, 0, count * sizeof(T)));
    return BAAS_OK;
}

}  // namespace

struct baas_schedule {
    baas::HostSchedule hs;
    baas_options opt{};
    int nnz_a = 0, nnz_l = 0;

    // host plan
    std::vector<int> f_item_ptr, f_ord, b_item_ptr, b_ord;
    std::vector<int> fp_ptr, fp_col, fp_src, fp_dsrc;  // packed L (A positions)
    std::vector<int> bp_ptr, bp_col, bp_src, bp_dsrc;  // packed U = L^T (A positions)

    // device plan
    int device = -1;
    bool uploaded = false;
    int num_sms = 0;
    int *d_f_item_ptr = nullptr, *d_f_ord = nullptr, *d_b_item_ptr = nullptr, *d_b_ord = nullptr;
    int *d_a_diag = nullptr;
    int *d_fp_ptr = nullptr, *d_fp_col = nullptr, *d_fp_src = nullptr, *d_fp_dsrc = nullptr;
    int *d_bp_ptr = nullptr, *d_bp_col = nullptr, *d_bp_src = nullptr, *d_bp_dsrc = nullptr;
    DevStatus *d_status = nullptr;
    DevStatus *h_status = nullptr;  // pinned
    int *d_flags = nullptr;
    int epoch = 0;
    unsigned int *d_bar = nullptr;

    // ICCG workspace
    bool ws_ready = false;
    double *d_lu = nullptr, *d_r = nullptr, *d_y = nullptr, *d_z = nullptr, *d_p = nullptr, *d_Ap = nullptr;
    float *d_y32 = nullptr, *d_z32 = nullptr;
    double *d_fp_val = nullptr, *d_fp_diag = nullptr, *d_bp_val = nullptr, *d_bp_diag = nullptr;
    float *d_fp_val32 = nullptr, *d_fp_diag32 = nullptr, *d_bp_val32 = nullptr, *d_bp_diag32 = nullptr;
    double *d_part = nullptr;
    int *d_iters = nullptr;
    double *d_relres = nullptr;
    int part_cap = 0;

    unsigned int spin() const { return opt.spin_limit > 0 ? (unsigned int)opt.spin_limit : kDefaultSpin; }
    int block() const { return baas::kBlock; }
};

namespace {

void build_plan(baas_schedule *s) {
    const baas::HostSchedule &h = s->hs;
    const int n = h.n;
    const int ng = h.ngroups;
    // forward items: groups level by level (LevelSet permToOrig), rows ascending
    s->f_item_ptr.assign(ng + 1, 0);
    s->f_ord.clear();
    s->f_ord.reserve(n);
    for (int q = 0; q < ng; q++) {
        const int g = h.perm_to_orig[q];
        for (int e = h.group_ptr[g]; e < h.group_ptr[g + 1]; e++) s->f_ord.push_back(h.group_set[e]);
        s->f_item_ptr[q + 1] = (int)s->f_ord.size();
    }
    // backward items: the exact reverse (items reversed, rows descending)
    s->b_item_ptr.assign(ng + 1, 0);
    s->b_ord.assign(s->f_ord.rbegin(), s->f_ord.rend());
    for (int q = 0; q < ng; q++) {
        const int fq = ng - 1 - q;
        s->b_item_ptr[q + 1] = s->b_item_ptr[q] + (s->f_item_ptr[fq + 1] - s->f_item_ptr[fq]);
    }
    // packed L: off-diagonals ascending, in forward order
    s->fp_ptr.assign(n + 1, 0);
    s->fp_col.clear();
    s->fp_src.clear();
    s->fp_dsrc.assign(n, 0);
    for (int p = 0; p < n; p++) {
        const int row = s->f_ord[p];
        const int lb = h.l_rowptr[row], le = h.l_rowptr[row + 1];
        for (int e = lb; e < le - 1; e++) {
            s->fp_col.push_back(h.l_colidx[e]);
            s->fp_src.push_back(h.l_src[e]);
        }
        s->fp_dsrc[p] = h.l_src[le - 1];
        s->fp_ptr[p + 1] = (int)s->fp_col.size();
    }
    // packed U = L^T: row j of U = column j of L; off-diagonals DESCENDING, in backward order
    std::vector<int> cptr(n + 1, 0), crow, cpos;
    for (int e = 0; e < (int)h.l_colidx.size(); e++) cptr[h.l_colidx[e] + 1]++;
    for (int i = 0; i < n; i++) cptr[i + 1] += cptr[i];
    crow.resize(h.l_colidx.size());
    cpos.resize(h.l_colidx.size());
    {
        std::vector<int> cur(cptr.begin(), cptr.end() - 1);
        for (int i = 0; i < n; i++)
            for (int e = h.l_rowptr[i]; e < h.l_rowptr[i + 1]; e++) {
                const int c = h.l_colidx[e];
                crow[cur[c]] = i;
                cpos[cur[c]] = e;
                cur[c]++;
            }
    }
    s->bp_ptr.assign(n + 1, 0);
    s->bp_col.clear();
    s->bp_src.clear();
    s->bp_dsrc.assign(n, 0);
    for (int p = 0; p < n; p++) {
        const int j = s->b_ord[p];
        // column j of L: rows ascending, first is the diagonal
        for (int e = cptr[j + 1] - 1; e > cptr[j]; e--) {
            s->bp_col.push_back(crow[e]);
            s->bp_src.push_back(h.l_src[cpos[e]]);
        }
        s->bp_dsrc[p] = h.l_src[cpos[cptr[j]]];
        s->bp_ptr[p + 1] = (int)s->bp_col.size();
    }
}

baas_status ensure_device(baas_schedule *s) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(BAAS_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (s->uploaded) {
        if (dev != s->device) return fail(BAAS_ERR_STATE, "schedule was uploaded to another device");
        return BAAS_OK;
    }
    cudaDeviceProp prop;
    BAAS_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (!prop.cooperativeLaunch) return fail(BAAS_ERR_NO_DEVICE, "device lacks cooperative launch");
    s->num_sms = prop.multiProcessorCount;
    s->device = dev;
    baas_status st;
#define UP(d, h)                               \
    if ((st = upload(d, h)) != BAAS_OK) return st;
    UP(s->d_f_item_ptr, s->f_item_ptr);
    UP(s->d_f_ord, s->f_ord);
    UP(s->d_b_item_ptr, s->b_item_ptr);
    UP(s->d_b_ord, s->b_ord);
    UP(s->d_a_diag, s->hs.a_diagptr);
    UP(s->d_fp_ptr, s->fp_ptr);
    UP(s->d_fp_col, s->fp_col);
    UP(s->d_fp_src, s->fp_src);
    UP(s->d_fp_dsrc, s->fp_dsrc);
    UP(s->d_bp_ptr, s->bp_ptr);
    UP(s->d_bp_col, s->bp_col);
    UP(s->d_bp_src, s->bp_src);
    UP(s->d_bp_dsrc, s->bp_dsrc);
#undef UP
    if ((st = dalloc(s->d_status, 1)) != BAAS_OK) return st;
    if ((st = dalloc(s->d_flags, (size_t)s->hs.n)) != BAAS_OK) return st;
    if ((st = dalloc(s->d_bar, 1)) != BAAS_OK) return st;
    BAAS_CUDA(cudaMallocHost((void **)&s->h_status, sizeof(DevStatus)));
    s->uploaded = true;
    return BAAS_OK;
}

// Persistent grid: co-resident CTAs (capped by the options and by the work available).
template <typename K>
baas_status grid_for(baas_schedule *s, K kernel, int work_items, int &grid) {
    int per_sm = 0;
    BAAS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, s->block(), 0));
    if (per_sm <= 0) return fail(BAAS_ERR_CUDA, "kernel cannot be resident");
    if (s->opt.ctas_per_sm > 0) per_sm = std::min(per_sm, s->opt.ctas_per_sm);
    grid = per_sm * s->num_sms;
    if (work_items > 0) grid = std::min(grid, std::max(1, (work_items + s->block() - 1) / s->block()));
    return BAAS_OK;
}

baas_status next_epoch(baas_schedule *s, cudaStream_t stream) {
    if (s->epoch == INT_MAX) {
        BAAS_CUDA(cudaMemsetAsync(s->d_flags, 0, sizeof(int) * (size_t)s->hs.n, stream));
        s->epoch = 0;
    }
    s->epoch++;
    return BAAS_OK;
}

baas_status read_status(baas_schedule *s, cudaStream_t stream) {
    BAAS_CUDA(cudaMemcpyAsync(s->h_status, s->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
    BAAS_CUDA(cudaStreamSynchronize(stream));
    const DevStatus &ds = *s->h_status;
    if (ds.code == baas::kTimeout)
        return fail(BAAS_ERR_TIMEOUT, "a device wait ran out (at " + std::to_string(ds.where) + ")");
    if (ds.code != 0) return fail(BAAS_ERR_CUDA, "device status " + std::to_string(ds.code));
    if (ds.zero_pivots > 0)
        return fail(BAAS_ERR_ZERO_PIVOT, std::to_string(ds.zero_pivots) + " non-positive / zero pivot(s)");
    return BAAS_OK;
}

bool csr_ok(const baas_csr *m, int n, int nnz) {
    return m && m->n == n && m->nnz == nnz && m->rowptr && m->colidx && m->values;
}

}  // namespace

extern "C" {

void baas_options_default(baas_options *opt) {
    if (!opt) return;
    opt->nthread = 8;
    opt->spin_limit = 0;
    opt->block_size = 0;
    opt->ctas_per_sm = 0;
}

const char *baas_last_error_string(void) { return g_err.c_str(); }

const char *baas_version(void) { return "baas_b200 0.1.0 (sm_100a)"; }

baas_status baas_analyze(const baas_csr *A, baas_kernel kind, const baas_options *opt, baas_schedule **out) {
    if (!A || !out) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    *out = nullptr;
    if (kind < BAAS_KERNEL_SPTRSV || kind > BAAS_KERNEL_ILU0) return fail(BAAS_ERR_BAD_ARG, "unknown kernel kind");
    baas_options o;
    baas_options_default(&o);
    if (opt) o = *opt;
    if (o.nthread < 1) return fail(BAAS_ERR_BAD_ARG, "nthread must be >= 1");
    if (!A->rowptr || !A->colidx || A->n <= 0) return fail(BAAS_ERR_BAD_ARG, "empty or NULL pattern");
    if (A->rowptr[A->n] != A->nnz) return fail(BAAS_ERR_BAD_ARG, "nnz != rowptr[n]");
    const baas::SchedKind sk = (baas::SchedKind)kind;
    const char *why = baas::validate_pattern(A->n, A->rowptr, A->colidx, sk);
    if (why[0]) return fail(BAAS_ERR_BAD_ARG, why);
    baas_schedule *s = new baas_schedule();
    s->opt = o;
    s->nnz_a = A->nnz;
    baas::build_schedule(s->hs, A->n, A->rowptr, A->colidx, sk, o.nthread);
    s->nnz_l = (int)s->hs.l_colidx.size();
    if (sk != baas::SchedKind::SpTRSV && s->nnz_a != 2 * s->nnz_l - A->n) {
        delete s;
        return fail(BAAS_ERR_BAD_ARG, "the pattern must be structurally symmetric");
    }
    build_plan(s);
    *out = s;
    return BAAS_OK;
}

int baas_schedule_export(const baas_schedule *s, int field, int *out) {
    if (!s) return -1;
    const baas::HostSchedule &h = s->hs;
    auto put = [out](const std::vector<int> &v) -> int {
        if (out && !v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(int));
        return (int)v.size();
    };
    auto scalar = [out](int v) -> int {
        if (out) *out = v;
        return 1;
    };
    switch (field) {
        case BAAS_FIELD_NGROUPS: return scalar(h.ngroups);
        case BAAS_FIELD_NLEVELS: return scalar(h.nlevels);
        case BAAS_FIELD_NTASKS: return scalar(h.ntasks);
        case BAAS_FIELD_GROUP_PTR: return put(h.group_ptr);
        case BAAS_FIELD_GROUP_SET: return put(h.group_set);
        case BAAS_FIELD_LEVEL_PTR: return put(h.level_ptr);
        case BAAS_FIELD_PERM_TO_ORIG: return put(h.perm_to_orig);
        case BAAS_FIELD_NODE_TO_LEVEL: return put(h.node_to_level);
        case BAAS_FIELD_NTHREAD_PER_LEVEL: return put(h.nthread_per_level);
        case BAAS_FIELD_THREAD_BOUNDARIES: return put(h.thread_boundaries);
        case BAAS_FIELD_TASK_BOUNDARIES: return put(h.task_boundaries);
        case BAAS_FIELD_THREAD_CONT_TO_ORIG: return put(h.thread_cont_to_orig);
        case BAAS_FIELD_ORIG_TO_THREAD_CONT: return put(h.orig_to_thread_cont);
        case BAAS_FIELD_TASK_PTR: return put(h.task_ptr);
        case BAAS_FIELD_TASK_SET: return put(h.task_set);
        case BAAS_FIELD_BTASK_PTR: return put(h.btask_ptr);
        case BAAS_FIELD_BTASK_SET: return put(h.btask_set);
        case BAAS_FIELD_COST: {
            std::vector<int> c(h.cost.size());
            for (size_t i = 0; i < c.size(); i++) c[i] = (int)h.cost[i];
            return put(c);
        }
        default: return -1;
    }
}

double baas_schedule_analysis_ms(const baas_schedule *s) { return s ? s->hs.analysis_ms : 0.0; }

void baas_destroy(baas_schedule *s) {
    if (!s) return;
    if (s->uploaded) {
        int cur = -1;
        cudaGetDevice(&cur);
        if (cur != s->device) cudaSetDevice(s->device);
        void *ptrs[] = {s->d_f_item_ptr, s->d_f_ord, s->d_b_item_ptr, s->d_b_ord, s->d_a_diag, s->d_fp_ptr, s->d_fp_col,
                        s->d_fp_src, s->d_fp_dsrc, s->d_bp_ptr, s->d_bp_col, s->d_bp_src, s->d_bp_dsrc, s->d_status,
                        s->d_flags, s->d_bar, s->d_lu, s->d_r, s->d_y, s->d_z, s->d_p, s->d_Ap, s->d_y32, s->d_z32,
                        s->d_fp_val, s->d_fp_diag, s->d_bp_val, s->d_bp_diag, s->d_fp_val32, s->d_fp_diag32,
                        s->d_bp_val32, s->d_bp_diag32, s->d_part, s->d_iters, s->d_relres};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        if (s->h_status) cudaFreeHost(s->h_status);
        if (cur >= 0 && cur != s->device) cudaSetDevice(cur);
    }
    delete s;
}

baas_status baas_sptrsv(baas_schedule *s, const baas_csr *T, int upper, const double *b, double *x, int nrhs, int ldb,
                        void *stream_) {
    if (!s || !b || !x) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    const int n = s->hs.n;
    if (!csr_ok(T, n, s->nnz_l)) return fail(BAAS_ERR_BAD_ARG, "triangular factor does not match the analysed pattern");
    if (nrhs < 1 || ldb < n) return fail(BAAS_ERR_BAD_ARG, "nrhs must be >= 1 and ldb >= n");
    if (x == b) return fail(BAAS_ERR_BAD_ARG, "x must not alias b");
    baas_status st = ensure_device(s);
    if (st != BAAS_OK) return st;
    cudaStream_t stream = (cudaStream_t)stream_;
    BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
    {
        const int fill_blocks = std::min(4 * s->num_sms, (int)(((long long)n * nrhs + 255) / 256));
        baas::k_fill_sentinel<double><<<std::max(fill_blocks, 1), 256, 0, stream>>>(x, n, nrhs, ldb);
        BAAS_CUDA(cudaGetLastError());
    }
    const int nitems = s->hs.ngroups;
    const int *item_ptr = upper ? s->d_b_item_ptr : s->d_f_item_ptr;
    const int *ord = upper ? s->d_b_ord : s->d_f_ord;
    unsigned int spin = s->spin();
    int grid = 0;
    void *args[] = {(void *)&nitems, (void *)&item_ptr, (void *)&ord, (void *)&T->rowptr, (void *)&T->colidx,
                    (void *)&T->values, (void *)&b, (void *)&ldb, (void *)&x, (void *)&ldb, (void *)&nrhs,
                    (void *)&s->d_status, (void *)&spin};
    if (upper) {
        if ((st = grid_for(s, baas::k_sweep_csr<true>, nitems, grid)) != BAAS_OK) return st;
        BAAS_CUDA(cudaLaunchCooperativeKernel((void *)baas::k_sweep_csr<true>, grid, s->block(), args, 0, stream));
    } else {
        if ((st = grid_for(s, baas::k_sweep_csr<false>, nitems, grid)) != BAAS_OK) return st;
        BAAS_CUDA(cudaLaunchCooperativeKernel((void *)baas::k_sweep_csr<false>, grid, s->block(), args, 0, stream));
    }
    return read_status(s, stream);
}

static baas_status factor(baas_schedule *s, const baas_csr *A, double *lu, void *stream_, bool ilu) {
    if (!s || !lu) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    if (s->hs.kind == baas::SchedKind::SpTRSV) return fail(BAAS_ERR_STATE, "a SpTRSV schedule cannot drive a factorisation");
    if (!A || A->n != s->hs.n || A->nnz != s->nnz_a || !A->rowptr || !A->colidx)
        return fail(BAAS_ERR_BAD_ARG, "matrix does not match the analysed pattern");
    baas_status st = ensure_device(s);
    if (st != BAAS_OK) return st;
    cudaStream_t stream = (cudaStream_t)stream_;
    if ((st = next_epoch(s, stream)) != BAAS_OK) return st;
    BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
    const int nitems = s->hs.ngroups;
    unsigned int spin = s->spin();
    int grid = 0;
    void *args[] = {(void *)&nitems, (void *)&s->d_f_item_ptr, (void *)&s->d_f_ord, (void *)&A->rowptr,
                    (void *)&A->colidx, (void *)&s->d_a_diag, (void *)&lu, (void *)&s->d_flags, (void *)&s->epoch,
                    (void *)&s->d_status, (void *)&spin};
    if (ilu) {
        if ((st = grid_for(s, baas::k_factor<true>, nitems, grid)) != BAAS_OK) return st;
        BAAS_CUDA(cudaLaunchCooperativeKernel((void *)baas::k_factor<true>, grid, s->block(), args, 0, stream));
    } else {
        if ((st = grid_for(s, baas::k_factor<false>, nitems, grid)) != BAAS_OK) return st;
        BAAS_CUDA(cudaLaunchCooperativeKernel((void *)baas::k_factor<false>, grid, s->block(), args, 0, stream));
    }
    return read_status(s, stream);
}

baas_status baas_ic0(baas_schedule *s, const baas_csr *A, double *lu, void *stream) { return factor(s, A, lu, stream, false); }

baas_status baas_ilu0(baas_schedule *s, const baas_csr *A, double *lu, void *stream) { return factor(s, A, lu, stream, true); }

baas_status baas_iccg(baas_schedule *s, const baas_csr *A, const double *b, double *x, double tol, int maxiter,
                      int precision, int *iters, double *relres, void *stream_) {
    if (!s || !b || !x) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    if (s->hs.kind != baas::SchedKind::ICCG) return fail(BAAS_ERR_STATE, "ICCG needs a schedule of kind BAAS_KERNEL_ICCG");
    if (!csr_ok(A, s->hs.n, s->nnz_a)) return fail(BAAS_ERR_BAD_ARG, "matrix does not match the analysed pattern");
    if (maxiter < 0 || !(tol >= 0.0)) return fail(BAAS_ERR_BAD_ARG, "maxiter must be >= 0 and tol >= 0");
    if (precision != BAAS_PREC_FP64 && precision != BAAS_PREC_FP32_FACTORS) return fail(BAAS_ERR_BAD_ARG, "unknown precision");
    baas_status st = ensure_device(s);
    if (st != BAAS_OK) return st;
    cudaStream_t stream = (cudaStream_t)stream_;
    const int n = s->hs.n;
    int grid = 0;
    if ((st = grid_for(s, baas::k_iccg, 0, grid)) != BAAS_OK) return st;
    if (!s->ws_ready) {
        const size_t nf = std::max<size_t>(s->fp_col.size(), 1), nbk = std::max<size_t>(s->bp_col.size(), 1);
        if ((st = dalloc(s->d_lu, (size_t)s->nnz_a)) != BAAS_OK) return st;
        if ((st = dalloc(s->d_r, n)) || (st = dalloc(s->d_y, n)) || (st = dalloc(s->d_z, n)) || (st = dalloc(s->d_p, n)) ||
            (st = dalloc(s->d_Ap, n)) || (st = dalloc(s->d_y32, n)) || (st = dalloc(s->d_z32, n)))
            return st;
        if ((st = dalloc(s->d_fp_val, nf)) || (st = dalloc(s->d_bp_val, nbk)) || (st = dalloc(s->d_fp_val32, nf)) ||
            (st = dalloc(s->d_bp_val32, nbk)) || (st = dalloc(s->d_fp_diag, n)) || (st = dalloc(s->d_bp_diag, n)) ||
            (st = dalloc(s->d_fp_diag32, n)) || (st = dalloc(s->d_bp_diag32, n)))
            return st;
        s->part_cap = grid;
        if ((st = dalloc(s->d_part, (size_t)3 * grid)) || (st = dalloc(s->d_iters, 1)) || (st = dalloc(s->d_relres, 1)))
            return st;
        s->ws_ready = true;
    }
    if (grid > s->part_cap) return fail(BAAS_ERR_STATE, "grid grew after the workspace was sized");
    if ((st = next_epoch(s, stream)) != BAAS_OK) return st;
    BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
    BAAS_CUDA(cudaMemsetAsync(s->d_bar, 0, sizeof(unsigned int), stream));

    baas::IccgArgs a{};
    a.n = n;
    a.a_rowptr = A->rowptr;
    a.a_colidx = A->colidx;
    a.a_diag = s->d_a_diag;
    a.a_val = A->values;
    a.b = b;
    a.x = x;
    a.nitems = s->hs.ngroups;
    a.f_item_ptr = s->d_f_item_ptr;
    a.f_ord = s->d_f_ord;
    a.b_item_ptr = s->d_b_item_ptr;
    a.b_ord = s->d_b_ord;
    a.fp_ptr = s->d_fp_ptr;
    a.fp_col = s->d_fp_col;
    a.fp_src = s->d_fp_src;
    a.fp_dsrc = s->d_fp_dsrc;
    a.bp_ptr = s->d_bp_ptr;
    a.bp_col = s->d_bp_col;
    a.bp_src = s->d_bp_src;
    a.bp_dsrc = s->d_bp_dsrc;
    a.fp_val = s->d_fp_val;
    a.fp_diag = s->d_fp_diag;
    a.bp_val = s->d_bp_val;
    a.bp_diag = s->d_bp_diag;
    a.fp_val32 = s->d_fp_val32;
    a.fp_diag32 = s->d_fp_diag32;
    a.bp_val32 = s->d_bp_val32;
    a.bp_diag32 = s->d_bp_diag32;
    a.nnzf = (int)s->fp_col.size();
    a.nnzb = (int)s->bp_col.size();
    a.lu = s->d_lu;
    a.flags = s->d_flags;
    a.epoch = s->epoch;
    a.r = s->d_r;
    a.y = s->d_y;
    a.z = s->d_z;
    a.p = s->d_p;
    a.Ap = s->d_Ap;
    a.y32 = s->d_y32;
    a.z32 = s->d_z32;
    a.part_a = s->d_part;
    a.part_b = s->d_part + grid;
    a.part_c = s->d_part + 2 * grid;
    a.bar = s->d_bar;
    a.st = s->d_status;
    a.maxiter = maxiter;
    a.tol = tol;
    a.mixed = precision == BAAS_PREC_FP32_FACTORS;
    a.out_iters = s->d_iters;
    a.out_relres = s->d_relres;
    a.spin_limit = s->spin();
    void *args[] = {(void *)&a};
    BAAS_CUDA(cudaLaunchCooperativeKernel((void *)baas::k_iccg, grid, s->block(), args, 0, stream));
    int it = 0;
    double rr = 0.0;
    BAAS_CUDA(cudaMemcpyAsync(&it, s->d_iters, sizeof(int), cudaMemcpyDeviceToHost, stream));
    BAAS_CUDA(cudaMemcpyAsync(&rr, s->d_relres, sizeof(double), cudaMemcpyDeviceToHost, stream));
    st = read_status(s, stream);
    if (iters) *iters = it;
    if (relres) *relres = rr;
    if (st != BAAS_OK) return st;
    if (!(rr < tol)) return fail(BAAS_ERR_NOT_CONVERGED, "maxiter reached before tol");
    return BAAS_OK;
}

}  // extern "C"
