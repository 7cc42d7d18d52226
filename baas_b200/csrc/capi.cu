// C ABI of the B200 BAAS hot path (declarations and contracts: include/baas_b200.h).
//
// baas_analyze builds the reference-identical schedule on the host (schedule.cpp). From it the
// device plan is derived: the schedule's groups listed level by level (the BAAS LevelSet
// order, rows ascending inside a group) give one global topological order of the rows; rows
// are given to P CTAs (contiguous row ranges by default, or the four-rule thread mapping);
// each CTA walks its rows in the global order (part_kernels.cuh). The backward sweep uses the
// exact reverse order. The plan is uploaded on the first GPU call, to the current device.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <mutex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/baas_b200.h"
#include "kernels.cuh"
#include "part_kernels.cuh"
#include "staged.cuh"
#include "schedule.hpp"

using baas::DevStatus;

namespace {

thread_local std::string g_err;

baas_status fail(baas_status st, const std::string &msg) {
    g_err = msg;
    return st;
}

#define BAAS_CUDA(call)                                                                      \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(BAAS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define BAAS_TRY(expr)                       \
    do {                                     \
        baas_status s_ = (expr);             \
        if (s_ != BAAS_OK) return s_;        \
    } while (0)

constexpr unsigned int kDefaultSpin = 1u << 22;
// shared memory one CTA may use for its rows' solution values (B200: 227 KB per CTA)
constexpr size_t kSmemBudget = 220 * 1024;

template <typename T>
baas_status upload(T *&d, const std::vector<T> &h) {
    d = nullptr;
    const size_t cnt = std::max<size_t>(h.size(), 1);
    BAAS_CUDA(cudaMalloc((void **)&d, cnt * sizeof(T)));
    if (!h.empty()) BAAS_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
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

// One sweep direction of the partitioned plan (host side). Positions are CTA-major; inside a
// CTA they run level segment by level segment, group (item) by group, row by row.
struct PartHost {
    std::vector<int> cta_seg, seg_item, item_pos, cta_pos, row, eptr, dep;
    std::vector<int> srcT, dsrcT;  // positions in the caller's triangular CSR (L or U)
    std::vector<int> srcA, dsrcA;  // positions in A's value array (IC0 factor on A's pattern)
    int max_local = 0;
};

struct PartDev {
    int *cta_seg = nullptr, *seg_item = nullptr, *item_pos = nullptr, *cta_pos = nullptr;
    int *row = nullptr, *eptr = nullptr, *dep = nullptr;
    int *srcT = nullptr, *dsrcT = nullptr, *srcA = nullptr, *dsrcA = nullptr;
    baas::PartView view(int P) const { return baas::PartView{P, cta_seg, seg_item, item_pos, cta_pos, row, eptr, dep}; }
    void release() {
        int *ptrs[] = {cta_seg, seg_item, item_pos, cta_pos, row, eptr, dep, srcT, dsrcT, srcA, dsrcA};
        for (int *p : ptrs)
            if (p) cudaFree(p);
        *this = PartDev();
    }
};

baas_status upload_part(PartDev &d, const PartHost &h) {
    BAAS_TRY(upload(d.cta_seg, h.cta_seg));
    BAAS_TRY(upload(d.seg_item, h.seg_item));
    BAAS_TRY(upload(d.item_pos, h.item_pos));
    BAAS_TRY(upload(d.cta_pos, h.cta_pos));
    BAAS_TRY(upload(d.row, h.row));
    BAAS_TRY(upload(d.eptr, h.eptr));
    BAAS_TRY(upload(d.dep, h.dep));
    BAAS_TRY(upload(d.srcT, h.srcT));
    BAAS_TRY(upload(d.dsrcT, h.dsrcT));
    BAAS_TRY(upload(d.srcA, h.srcA));
    BAAS_TRY(upload(d.dsrcA, h.dsrcA));
    return BAAS_OK;
}

// Staged plan (staged.cuh), host side: per direction the packed per-CTA int and value-source
// blocks.
struct StagedHostDir {
    std::vector<int> ioff, voff, ns, nl, ne, ints, vsrcT, vsrcA;
};
struct StagedHost {
    StagedHostDir dir[2];
    size_t smem64 = 0, smem32 = 0;  // dynamic shared memory per CTA (FP64 / FP32 values)
};
struct StagedDevDir {
    int *ioff = nullptr, *voff = nullptr, *ns = nullptr, *nl = nullptr, *ne = nullptr, *ints = nullptr,
        *vsrcT = nullptr, *vsrcA = nullptr;
};
struct StagedDev {
    StagedDevDir dir[2];
    baas::StagedPlan plan(int P) const {
        baas::StagedPlan p;
        p.P = P;
        for (int d = 0; d < 2; d++)
            p.dir[d] = baas::StagedDir{dir[d].ioff, dir[d].voff, dir[d].ns, dir[d].nl, dir[d].ne,
                                      dir[d].ints, dir[d].vsrcT, dir[d].vsrcA};
        return p;
    }
    void release() {
        for (auto &D : dir) {
            int *ptrs[] = {D.ioff, D.voff, D.ns, D.nl, D.ne, D.ints, D.vsrcT, D.vsrcA};
            for (int *p : ptrs)
                if (p) cudaFree(p);
        }
        *this = StagedDev();
    }
};

baas_status upload_staged(StagedDev &d, const StagedHost &h) {
    for (int k = 0; k < 2; k++) {
        const StagedHostDir &H = h.dir[k];
        StagedDevDir &D = d.dir[k];
        BAAS_TRY(upload(D.ioff, H.ioff));
        BAAS_TRY(upload(D.voff, H.voff));
        BAAS_TRY(upload(D.ns, H.ns));
        BAAS_TRY(upload(D.nl, H.nl));
        BAAS_TRY(upload(D.ne, H.ne));
        BAAS_TRY(upload(D.ints, H.ints));
        BAAS_TRY(upload(D.vsrcT, H.vsrcT));
        BAAS_TRY(upload(D.vsrcA, H.vsrcA));
    }
    return BAAS_OK;
}

}  // namespace

struct baas_schedule {
    baas::HostSchedule hs;
    baas_options opt{};
    int nnz_a = 0, nnz_l = 0;

    // global topological order of rows (forward) and the transpose of L (for U = L^T)
    std::vector<int> f_ord;
    std::vector<int> cptr, crow, cpos;  // CSC of L: rows ascending per column (diagonal first)

    // partition (built at first GPU use, when the SM count is known)
    int P = 0;
    std::vector<int> group_cta, row_cta;
    PartHost fwd, bwd;
    StagedHost stg;
    int fault_row = -1;  // test hook: forward row made to wait on its own output

    // device
    int device = -1;
    bool uploaded = false;
    int num_sms = 0;
    PartDev d_fwd, d_bwd;
    StagedDev d_stg;
    int *d_a_diag = nullptr;
    DevStatus *d_status = nullptr;
    DevStatus *h_status = nullptr;  // pinned
    int *d_flags = nullptr;
    int epoch = 0;
    unsigned int *d_bar = nullptr;

    // ICCG workspace
    bool ws_ready = false;
    double *d_lu = nullptr, *d_r = nullptr, *d_y = nullptr, *d_z = nullptr, *d_p = nullptr, *d_Ap = nullptr;
    float *d_y32 = nullptr, *d_z32 = nullptr;
    double *d_gv64[2] = {nullptr, nullptr};
    float *d_gv32[2] = {nullptr, nullptr};
    double *d_part = nullptr;
    int *d_iters = nullptr;
    double *d_relres = nullptr;

    unsigned long long *d_trace = nullptr;  // BAAS_TRACE=1: phase timestamps of the last launch

    unsigned int spin() const { return opt.spin_limit > 0 ? (unsigned int)opt.spin_limit : kDefaultSpin; }
};

namespace {

void build_order(baas_schedule *s) {
    const baas::HostSchedule &h = s->hs;
    const int n = h.n;
    s->f_ord.clear();
    s->f_ord.reserve(n);
    for (int q = 0; q < h.ngroups; q++) {
        const int g = h.perm_to_orig[q];
        for (int e = h.group_ptr[g]; e < h.group_ptr[g + 1]; e++) s->f_ord.push_back(h.group_set[e]);
    }
    s->cptr.assign(n + 1, 0);
    for (int c : h.l_colidx) s->cptr[c + 1]++;
    for (int i = 0; i < n; i++) s->cptr[i + 1] += s->cptr[i];
    s->crow.resize(h.l_colidx.size());
    s->cpos.resize(h.l_colidx.size());
    std::vector<int> cur(s->cptr.begin(), s->cptr.end() - 1);
    for (int i = 0; i < n; i++)
        for (int e = h.l_rowptr[i]; e < h.l_rowptr[i + 1]; e++) {
            const int c = h.l_colidx[e];
            s->crow[cur[c]] = i;
            s->cpos[cur[c]] = e;
            cur[c]++;
        }
}

// Groups -> CTAs. RANGES: the CTA whose row range holds the group's first row (P contiguous,
// row-balanced ranges). BAAS_THREADS: the four-rule mapping's thread of the group.
void build_partition(baas_schedule *s, int P) {
    const baas::HostSchedule &h = s->hs;
    const int n = h.n;
    s->P = P;
    s->group_cta.assign(h.ngroups, 0);
    if (s->opt.partition == BAAS_PARTITION_BAAS_THREADS) {
        for (int t = 0; t < h.nthread; t++)
            for (int task = h.thread_boundaries[t]; task < h.thread_boundaries[t + 1]; task++)
                for (int q = h.task_boundaries[task]; q < h.task_boundaries[task + 1]; q++) s->group_cta[h.thread_cont_to_orig[q]] = t;
    } else {
        for (int g = 0; g < h.ngroups; g++) {
            const int r0 = h.group_set[h.group_ptr[g]];
            s->group_cta[g] = (int)(((long long)r0 * P) / n);
        }
    }
    s->row_cta.assign(n, 0);
    for (int g = 0; g < h.ngroups; g++)
        for (int e = h.group_ptr[g]; e < h.group_ptr[g + 1]; e++) s->row_cta[h.group_set[e]] = s->group_cta[g];
}

// One direction of the plan. Forward: levels ascending, groups in LevelSet order, rows
// ascending. Backward (U = L^T): the exact reverse.
void build_dir(baas_schedule *s, bool upper, PartHost &out) {
    const baas::HostSchedule &h = s->hs;
    const int n = h.n, P = s->P, nl = h.nlevels;
    out = PartHost();
    // per CTA: list of (level, group) in processing order
    std::vector<std::vector<std::pair<int, int>>> items(P);
    for (int li = 0; li < nl; li++) {
        const int l = upper ? nl - 1 - li : li;
        const int qb = h.level_ptr[l], qe = h.level_ptr[l + 1];
        for (int qi = 0; qi < qe - qb; qi++) {
            const int q = upper ? qe - 1 - qi : qb + qi;
            const int g = h.perm_to_orig[q];
            items[s->group_cta[g]].push_back({l, g});
        }
    }
    out.cta_seg.assign(1, 0);
    out.seg_item.assign(1, 0);
    out.item_pos.assign(1, 0);
    out.cta_pos.assign(1, 0);
    out.row.clear();
    out.row.reserve(n);
    for (int c = 0; c < P; c++) {
        int last_level = -1;
        for (auto &lg : items[c]) {
            if (lg.first != last_level) {
                if (last_level != -1) out.seg_item.push_back((int)out.item_pos.size() - 1);
                last_level = lg.first;
            }
            const int g = lg.second;
            const int rb = h.group_ptr[g], re = h.group_ptr[g + 1];
            for (int k = 0; k < re - rb; k++) out.row.push_back(h.group_set[upper ? re - 1 - k : rb + k]);
            out.item_pos.push_back((int)out.row.size());
        }
        if (last_level != -1) out.seg_item.push_back((int)out.item_pos.size() - 1);
        out.cta_seg.push_back((int)out.seg_item.size() - 1);
        out.cta_pos.push_back((int)out.row.size());
        out.max_local = std::max(out.max_local, out.cta_pos[c + 1] - out.cta_pos[c]);
    }
    std::vector<int> slot(n, 0);
    for (int c = 0; c < P; c++)
        for (int pos = out.cta_pos[c]; pos < out.cta_pos[c + 1]; pos++) slot[out.row[pos]] = pos - out.cta_pos[c];
    out.eptr.assign(n + 1, 0);
    out.dsrcT.assign(n, 0);
    out.dsrcA.assign(n, 0);
    auto add = [&](int row, int col, int posT, int posA) {
        out.dep.push_back(s->row_cta[col] == s->row_cta[row] ? -(slot[col] + 1) : col);
        out.srcT.push_back(posT);
        out.srcA.push_back(posA);
    };
    for (int pos = 0; pos < n; pos++) {
        const int r = out.row[pos];
        if (!upper) {
            // L row r: off-diagonals ascending, diagonal last
            const int lb = h.l_rowptr[r], le = h.l_rowptr[r + 1];
            for (int e = lb; e < le - 1; e++) add(r, h.l_colidx[e], e, h.l_src[e]);
            out.dsrcT[pos] = le - 1;
            out.dsrcA[pos] = h.l_src[le - 1];
        } else {
            // U = L^T row r = column r of L: diagonal first, off-diagonals DESCENDING
            const int cb = s->cptr[r], ce = s->cptr[r + 1];
            for (int e = ce - 1; e > cb; e--) add(r, s->crow[e], e, h.l_src[s->cpos[e]]);
            out.dsrcT[pos] = cb;
            out.dsrcA[pos] = h.l_src[s->cpos[cb]];
        }
        out.eptr[pos + 1] = (int)out.dep.size();
    }
    if (!upper && s->fault_row >= 0) {
        for (int pos = 0; pos < n; pos++)
            if (out.row[pos] == s->fault_row && out.eptr[pos + 1] > out.eptr[pos]) out.dep[out.eptr[pos]] = s->fault_row;
    }
}

// Staged plan from the two position plans: per CTA, each level segment becomes as many steps
// as its largest group has rows; step j holds the j-th row of every group of the level. Slots
// are the rows' local positions in the lower sweep's step order. Entries are laid out with the
// CTA's uniform stride E (its widest row), padding unused entries.
void build_staged(baas_schedule *s) {
    const int n = s->hs.n, P = s->P;
    StagedHost &S = s->stg;
    S = StagedHost();
    std::vector<int> slot_of(n, 0);  // lower-sweep local position of each row
    size_t smem64 = 0, smem32 = 0;
    for (int d = 0; d < 2; d++) {
        const PartHost &H = d == 0 ? s->fwd : s->bwd;
        StagedHostDir &D = S.dir[d];
        D.ioff.assign(P + 1, 0);
        D.voff.assign(P + 1, 0);
        for (int c = 0; c < P; c++) {
            std::vector<int> step_row(1, 0), order;
            int E = 0;
            for (int sg = H.cta_seg[c]; sg < H.cta_seg[c + 1]; sg++) {
                int m = 0;
                for (int it = H.seg_item[sg]; it < H.seg_item[sg + 1]; it++) m = std::max(m, H.item_pos[it + 1] - H.item_pos[it]);
                for (int j = 0; j < m; j++) {
                    for (int it = H.seg_item[sg]; it < H.seg_item[sg + 1]; it++)
                        if (H.item_pos[it] + j < H.item_pos[it + 1]) {
                            const int pos = H.item_pos[it] + j;
                            order.push_back(pos);
                            E = std::max(E, H.eptr[pos + 1] - H.eptr[pos]);
                        }
                    step_row.push_back((int)order.size());
                }
            }
            const int nl = (int)order.size(), S_ = (int)step_row.size() - 1;
            if (d == 0)
                for (int k = 0; k < nl; k++) slot_of[H.row[order[k]]] = k;
            std::vector<int> ne(nl), rowid(nl), slot(nl), dep((size_t)nl * E, 0);
            std::vector<int> dT(nl), dA(nl), vT((size_t)nl * E, -1), vA((size_t)nl * E, -1);
            for (int k = 0; k < nl; k++) {
                const int pos = order[k];
                const int r = H.row[pos];
                ne[k] = H.eptr[pos + 1] - H.eptr[pos];
                rowid[k] = r;
                slot[k] = slot_of[r];
                dT[k] = H.dsrcT[pos];
                dA[k] = H.dsrcA[pos];
                for (int j = 0; j < ne[k]; j++) {
                    const int e = H.eptr[pos] + j;
                    const int dd = H.dep[e];
                    // local: the dependency's slot; remote: -(row + 1)
                    dep[(size_t)k * E + j] = dd < 0 ? slot_of[H.row[H.cta_pos[c] + (-dd - 1)]] : -(dd + 1);
                    vT[(size_t)k * E + j] = H.srcT[e];
                    vA[(size_t)k * E + j] = H.srcA[e];
                }
            }
            const int ent = nl * E;
            D.ns.push_back(S_);
            D.nl.push_back(nl);
            D.ne.push_back(ent);
            D.ints.push_back(E);
            D.ints.insert(D.ints.end(), step_row.begin(), step_row.end());
            D.ints.insert(D.ints.end(), ne.begin(), ne.end());
            D.ints.insert(D.ints.end(), rowid.begin(), rowid.end());
            D.ints.insert(D.ints.end(), slot.begin(), slot.end());
            D.ints.insert(D.ints.end(), dep.begin(), dep.end());
            D.ints.resize(baas::pad4((int)D.ints.size()), 0);
            D.ioff[c + 1] = (int)D.ints.size();
            D.vsrcT.insert(D.vsrcT.end(), dT.begin(), dT.end());
            D.vsrcT.insert(D.vsrcT.end(), vT.begin(), vT.end());
            D.vsrcA.insert(D.vsrcA.end(), dA.begin(), dA.end());
            D.vsrcA.insert(D.vsrcA.end(), vA.begin(), vA.end());
            const int padded = baas::pad4((int)D.vsrcA.size());
            D.vsrcT.resize(padded, -1);
            D.vsrcA.resize(padded, -1);
            D.voff[c + 1] = padded;
            baas::StageLayout L64, L32;
            L64.make<double>(S_, nl, ent);
            L32.make<float>(S_, nl, ent);
            smem64 = std::max(smem64, (size_t)L64.total);
            smem32 = std::max(smem32, (size_t)L32.total);
        }
        // slack so the last block's 16-byte copies stay inside the arrays
        D.ints.resize(D.ints.size() + 4, 0);
        D.vsrcT.resize(D.vsrcT.size() + 4, -1);
        D.vsrcA.resize(D.vsrcA.size() + 4, -1);
    }
    S.smem64 = smem64;
    S.smem32 = smem32;
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

    // partition size: the fewest CTAs whose staged plan slice fits in shared memory
    const int n = s->hs.n;
    int P;
    if (s->opt.partition == BAAS_PARTITION_BAAS_THREADS) {
        P = s->hs.nthread;
        if (s->opt.parts > 0 && s->opt.parts != P) return fail(BAAS_ERR_BAD_ARG, "BAAS_THREADS partition needs parts == nthread");
    } else if (s->opt.parts > 0) {
        P = std::min(s->opt.parts, n);
    } else {
        P = (int)std::max<long long>(1, ((long long)n * 48 + kSmemBudget - 1) / (long long)kSmemBudget);
    }
    for (;;) {
        if (P > s->num_sms) return fail(BAAS_ERR_BAD_ARG, "the partition needs more CTAs than the device has SMs");
        build_partition(s, P);
        build_dir(s, false, s->fwd);
        build_dir(s, true, s->bwd);
        build_staged(s);
        if (s->stg.smem64 <= kSmemBudget) break;
        if (s->opt.parts > 0 || s->opt.partition == BAAS_PARTITION_BAAS_THREADS)
            return fail(BAAS_ERR_BAD_ARG, "a CTA's plan slice does not fit in shared memory: raise `parts`");
        P = std::min(s->num_sms, std::max(P + 1, (int)(P * 1.25)));
    }

    BAAS_TRY(upload_part(s->d_fwd, s->fwd));
    BAAS_TRY(upload_part(s->d_bwd, s->bwd));
    BAAS_TRY(upload_staged(s->d_stg, s->stg));
    BAAS_TRY(upload(s->d_a_diag, s->hs.a_diagptr));
    BAAS_TRY(dalloc(s->d_status, 1));
    BAAS_TRY(dalloc(s->d_flags, (size_t)n));
    BAAS_TRY(dalloc(s->d_bar, 1));
    BAAS_CUDA(cudaMallocHost((void **)&s->h_status, sizeof(DevStatus)));
    if (getenv("BAAS_TRACE") && atoi(getenv("BAAS_TRACE")) > 0) BAAS_TRY(dalloc(s->d_trace, 2 * baas::kTraceSlots));
    // the partitioned kernels take up to kSmemBudget bytes of dynamic shared memory
    BAAS_CUDA(cudaFuncSetAttribute(baas::k_factor_part<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBudget));
    BAAS_CUDA(cudaFuncSetAttribute(baas::k_factor_part<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBudget));
    BAAS_CUDA(cudaFuncSetAttribute(baas::k_sweep_staged<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBudget));
    BAAS_CUDA(cudaFuncSetAttribute(baas::k_sweep_staged<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBudget));
    BAAS_CUDA(cudaFuncSetAttribute(baas::k_iccg_staged<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBudget));
    BAAS_CUDA(cudaFuncSetAttribute(baas::k_iccg_staged<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBudget));
    s->uploaded = true;
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

// BAAS_TRACE=1: print the phase timestamps of the last launch (microseconds from its start).
void dump_trace(baas_schedule *s, const char *what, cudaStream_t stream) {
    if (!s->d_trace) return;
    unsigned long long h[2 * baas::kTraceSlots];
    if (cudaMemcpyAsync(h, s->d_trace, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess) return;
    cudaStreamSynchronize(stream);
    for (int c = 0; c < 2; c++) {
        const unsigned long long *t = h + c * baas::kTraceSlots;
        fprintf(stderr, "[baas trace] %s cta=%s:", what, c == 0 ? "first" : "last");
        for (int k = 0; k < baas::kTraceSlots; k++)
            if (t[k]) fprintf(stderr, " %d:%.1f", k, (double)(t[k] - t[0]) / 1000.0);
        fprintf(stderr, "\n");
    }
    cudaMemsetAsync(s->d_trace, 0, sizeof(h), stream);
}

bool csr_ok(const baas_csr *m, int n, int nnz) {
    return m && m->n == n && m->nnz == nnz && m->rowptr && m->colidx && m->values;
}


// ---------------------------------------------------------------------------------------
// Allocation-free IC0 (baas_ic0_noalloc). The factorisation's scratch -- one ready flag per
// row plus the status word -- lives in this file-scope device array instead of memory the
// schedule allocates. Every GPU that loads this library holds the array (8 MB) until the
// process exits. Host code must not use the symbol as an address: the device address is looked
// up once per device with cudaGetSymbolAddress while that device is current.
// ---------------------------------------------------------------------------------------
constexpr int kNoAllocMaxRows = 1 << 21;  // 2,097,152 rows
constexpr int kNoAllocStatusInts = 4;     // a DevStatus at the front
static __device__ __align__(256) int g_noalloc_scratch[kNoAllocStatusInts + kNoAllocMaxRows];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
int *g_noalloc_ptr[kMaxDevices] = {};

baas_status noalloc_scratch(int dev, int **out) {
    if (dev < 0 || dev >= kMaxDevices) return fail(BAAS_ERR_NO_DEVICE, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(BAAS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_noalloc_ptr[dev] = static_cast<int *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return BAAS_OK;
}

}  // namespace

extern "C" {

void baas_options_default(baas_options *opt) {
    if (!opt) return;
    opt->nthread = 8;
    opt->spin_limit = 0;
    opt->parts = 0;
    opt->partition = BAAS_PARTITION_RANGES;
}

const char *baas_last_error_string(void) { return g_err.c_str(); }

const char *baas_version(void) { return "baas_b200 0.2.0 (sm_100a)"; }

baas_status baas_analyze(const baas_csr *A, baas_kernel kind, const baas_options *opt, baas_schedule **out) {
    if (!A || !out) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    *out = nullptr;
    if (kind < BAAS_KERNEL_SPTRSV || kind > BAAS_KERNEL_ILU0) return fail(BAAS_ERR_BAD_ARG, "unknown kernel kind");
    baas_options o;
    baas_options_default(&o);
    if (opt) o = *opt;
    if (o.nthread < 1) return fail(BAAS_ERR_BAD_ARG, "nthread must be >= 1");
    if (o.partition != BAAS_PARTITION_RANGES && o.partition != BAAS_PARTITION_BAAS_THREADS)
        return fail(BAAS_ERR_BAD_ARG, "unknown partition");
    if (o.parts < 0) return fail(BAAS_ERR_BAD_ARG, "parts must be >= 0");
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
    build_order(s);
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

baas_status baas_test_inject_unsatisfiable_wait(baas_schedule *s, int row) {
    if (!s || row < 0 || row >= s->hs.n) return fail(BAAS_ERR_BAD_ARG, "bad row");
    const int lb = s->hs.l_rowptr[row], le = s->hs.l_rowptr[row + 1];
    if (le - lb < 2) return fail(BAAS_ERR_BAD_ARG, "the row has no off-diagonal entry");
    if (s->uploaded) return fail(BAAS_ERR_STATE, "inject before the first GPU call on the schedule");
    s->fault_row = row;
    return BAAS_OK;
}

void baas_destroy(baas_schedule *s) {
    if (!s) return;
    if (s->uploaded) {
        int cur = -1;
        cudaGetDevice(&cur);
        if (cur != s->device) cudaSetDevice(s->device);
        s->d_fwd.release();
        s->d_bwd.release();
        s->d_stg.release();
        for (int d = 0; d < 2; d++) {
            if (s->d_gv64[d]) cudaFree(s->d_gv64[d]);
            if (s->d_gv32[d]) cudaFree(s->d_gv32[d]);
        }
        void *ptrs[] = {s->d_a_diag, s->d_status, s->d_flags, s->d_bar, s->d_lu, s->d_r, s->d_y, s->d_z, s->d_p,
                        s->d_Ap, s->d_y32, s->d_z32, s->d_part, s->d_iters, s->d_relres};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        if (s->h_status) cudaFreeHost(s->h_status);
        if (s->d_trace) cudaFree(s->d_trace);
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
    BAAS_TRY(ensure_device(s));
    cudaStream_t stream = (cudaStream_t)stream_;
    BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
    {
        const int fill_blocks = (int)std::min<long long>(4LL * s->num_sms, ((long long)n * nrhs + 255) / 256);
        baas::k_fill_sentinel<double><<<std::max(fill_blocks, 1), 256, 0, stream>>>(x, n, nrhs, ldb);
        BAAS_CUDA(cudaGetLastError());
    }
    baas::StagedPlan pl = s->d_stg.plan(s->P);
    unsigned int spin = s->spin();
    void *args[] = {(void *)&pl, (void *)&T->values, (void *)&b, (void *)&ldb, (void *)&x, (void *)&ldb,
                    (void *)&nrhs, (void *)&s->d_status, (void *)&spin, (void *)&s->d_trace};
    void *kern = upper ? (void *)baas::k_sweep_staged<true> : (void *)baas::k_sweep_staged<false>;

    BAAS_CUDA(cudaLaunchCooperativeKernel(kern, s->P, baas::kStageBlock, args, s->stg.smem64, stream));
    dump_trace(s, upper ? "sptrsv-upper" : "sptrsv-lower", stream);
    return read_status(s, stream);
}

static baas_status factor(baas_schedule *s, const baas_csr *A, double *lu, void *stream_, bool ilu) {
    if (!s || !lu) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    if (s->hs.kind == baas::SchedKind::SpTRSV) return fail(BAAS_ERR_STATE, "a SpTRSV schedule cannot drive a factorisation");
    if (!A || A->n != s->hs.n || A->nnz != s->nnz_a || !A->rowptr || !A->colidx)
        return fail(BAAS_ERR_BAD_ARG, "matrix does not match the analysed pattern");
    BAAS_TRY(ensure_device(s));
    cudaStream_t stream = (cudaStream_t)stream_;
    BAAS_TRY(next_epoch(s, stream));
    BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
    baas::PartView pv = s->d_fwd.view(s->P);
    unsigned int spin = s->spin();
    void *args[] = {(void *)&pv, (void *)&A->rowptr, (void *)&A->colidx, (void *)&s->d_a_diag, (void *)&lu,
                    (void *)&s->d_flags, (void *)&s->epoch, (void *)&s->d_status, (void *)&spin};
    void *kern = ilu ? (void *)baas::k_factor_part<true> : (void *)baas::k_factor_part<false>;
    BAAS_CUDA(cudaLaunchCooperativeKernel(kern, s->P, baas::kPartBlock, args, (size_t)s->fwd.max_local * 4, stream));
    return read_status(s, stream);
}

baas_status baas_ic0(baas_schedule *s, const baas_csr *A, double *lu, void *stream) { return factor(s, A, lu, stream, false); }

baas_status baas_ilu0(baas_schedule *s, const baas_csr *A, double *lu, void *stream) { return factor(s, A, lu, stream, true); }

// IC0 that allocates nothing: the same level-synchronous kernel as baas_ic0, given the static
// scratch array above for its row flags and status word. The schedule's device plan must already
// be resident (it is uploaded by the first ordinary GPU call on this schedule); this call does
// not upload it, because uploading allocates. It clears the flags and the status it uses, then
// launches on `stream` and reads the status back from device memory into a local variable.
baas_status baas_ic0_noalloc(baas_schedule *s, const baas_csr *A, double *lu, void *stream_) {
    if (!s || !lu) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    if (s->hs.kind == baas::SchedKind::SpTRSV) return fail(BAAS_ERR_STATE, "a SpTRSV schedule cannot drive a factorisation");
    if (!A || A->n != s->hs.n || A->nnz != s->nnz_a || !A->rowptr || !A->colidx)
        return fail(BAAS_ERR_BAD_ARG, "matrix does not match the analysed pattern");
    if (s->hs.n > kNoAllocMaxRows)
        return fail(BAAS_ERR_BAD_ARG, "baas_ic0_noalloc takes at most " + std::to_string(kNoAllocMaxRows) +
                                          " rows (its static scratch size); use baas_ic0");
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(BAAS_ERR_NO_DEVICE, "no CUDA device");
    if (!s->uploaded || dev != s->device)
        return fail(BAAS_ERR_STATE, "the schedule's device plan is not resident on this device: run one ordinary GPU "
                                    "call (e.g. baas_ic0) on it first");
    int *scratch = nullptr;
    BAAS_TRY(noalloc_scratch(dev, &scratch));
    DevStatus *status = reinterpret_cast<DevStatus *>(scratch);
    int *flags = scratch + kNoAllocStatusInts;
    cudaStream_t stream = (cudaStream_t)stream_;
    // the array keeps the previous call's contents: flags and status must start at zero
    BAAS_CUDA(cudaMemsetAsync(scratch, 0, sizeof(int) * ((size_t)kNoAllocStatusInts + (size_t)s->hs.n), stream));
    int epoch = 1;
    baas::PartView pv = s->d_fwd.view(s->P);
    unsigned int spin = s->spin();
    void *args[] = {(void *)&pv, (void *)&A->rowptr, (void *)&A->colidx, (void *)&s->d_a_diag, (void *)&lu,
                    (void *)&flags, (void *)&epoch, (void *)&status, (void *)&spin};
    BAAS_CUDA(cudaLaunchCooperativeKernel((void *)baas::k_factor_part<false>, s->P, baas::kPartBlock, args, 0, stream));
    DevStatus hs{};
    BAAS_CUDA(cudaMemcpyAsync(&hs, status, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
    BAAS_CUDA(cudaStreamSynchronize(stream));
    if (hs.code == baas::kTimeout) return fail(BAAS_ERR_TIMEOUT, "a device wait ran out (at " + std::to_string(hs.where) + ")");
    if (hs.code != 0) return fail(BAAS_ERR_CUDA, "device status " + std::to_string(hs.code));
    if (hs.zero_pivots > 0) return fail(BAAS_ERR_ZERO_PIVOT, std::to_string(hs.zero_pivots) + " non-positive pivot(s)");
    return BAAS_OK;
}

baas_status baas_iccg(baas_schedule *s, const baas_csr *A, const double *b, double *x, double tol, int maxiter,
                      int precision, int *iters, double *relres, void *stream_) {
    if (!s || !b || !x) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    if (s->hs.kind != baas::SchedKind::ICCG) return fail(BAAS_ERR_STATE, "ICCG needs a schedule of kind BAAS_KERNEL_ICCG");
    if (!csr_ok(A, s->hs.n, s->nnz_a)) return fail(BAAS_ERR_BAD_ARG, "matrix does not match the analysed pattern");
    if (maxiter < 0 || !(tol >= 0.0)) return fail(BAAS_ERR_BAD_ARG, "maxiter must be >= 0 and tol >= 0");
    if (precision != BAAS_PREC_FP64 && precision != BAAS_PREC_FP32_FACTORS) return fail(BAAS_ERR_BAD_ARG, "unknown precision");
    BAAS_TRY(ensure_device(s));
    cudaStream_t stream = (cudaStream_t)stream_;
    const int n = s->hs.n;
    const int P = s->P;
    if (!s->ws_ready) {
        BAAS_TRY(dalloc(s->d_lu, (size_t)s->nnz_a));
        BAAS_TRY(dalloc(s->d_r, n));
        BAAS_TRY(dalloc(s->d_y, n));
        BAAS_TRY(dalloc(s->d_z, n));
        BAAS_TRY(dalloc(s->d_p, n));
        BAAS_TRY(dalloc(s->d_Ap, n));
        BAAS_TRY(dalloc(s->d_y32, n));
        BAAS_TRY(dalloc(s->d_z32, n));
        for (int d = 0; d < 2; d++) {
            BAAS_TRY(dalloc(s->d_gv64[d], s->stg.dir[d].vsrcA.size()));
            BAAS_TRY(dalloc(s->d_gv32[d], s->stg.dir[d].vsrcA.size()));
        }
        BAAS_TRY(dalloc(s->d_part, (size_t)3 * P));
        BAAS_TRY(dalloc(s->d_iters, 1));
        BAAS_TRY(dalloc(s->d_relres, 1));
        s->ws_ready = true;
    }
    BAAS_TRY(next_epoch(s, stream));
    BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
    BAAS_CUDA(cudaMemsetAsync(s->d_bar, 0, sizeof(unsigned int), stream));

    baas::StagedIccgArgs a{};
    a.n = n;
    a.a_rowptr = A->rowptr;
    a.a_colidx = A->colidx;
    a.a_diag = s->d_a_diag;
    a.a_val = A->values;
    a.b = b;
    a.x = x;
    a.fac = s->d_fwd.view(P);
    a.pl = s->d_stg.plan(P);
    a.nv[0] = (int)s->stg.dir[0].vsrcA.size();
    a.nv[1] = (int)s->stg.dir[1].vsrcA.size();
    for (int d = 0; d < 2; d++) {
        a.gv64[d] = s->d_gv64[d];
        a.gv32[d] = s->d_gv32[d];
    }
    a.lu = s->d_lu;
    a.gflag = s->d_flags;
    a.epoch = s->epoch;
    a.r = s->d_r;
    a.y = s->d_y;
    a.z = s->d_z;
    a.p = s->d_p;
    a.Ap = s->d_Ap;
    a.y32 = s->d_y32;
    a.z32 = s->d_z32;
    a.part_a = s->d_part;
    a.part_b = s->d_part + P;
    a.part_c = s->d_part + 2 * P;
    a.bar = s->d_bar;
    a.st = s->d_status;
    a.maxiter = maxiter;
    a.tol = tol;
    a.out_iters = s->d_iters;
    a.out_relres = s->d_relres;
    a.spin_limit = s->spin();
    a.trace = s->d_trace;
    void *args[] = {(void *)&a};
    const bool mixed = precision == BAAS_PREC_FP32_FACTORS;
    void *kern = mixed ? (void *)baas::k_iccg_staged<float> : (void *)baas::k_iccg_staged<double>;
    BAAS_CUDA(cudaLaunchCooperativeKernel(kern, P, baas::kStageBlock, args, mixed ? s->stg.smem32 : s->stg.smem64, stream));
    int it = 0;
    double rr = 0.0;
    BAAS_CUDA(cudaMemcpyAsync(&it, s->d_iters, sizeof(int), cudaMemcpyDeviceToHost, stream));
    BAAS_CUDA(cudaMemcpyAsync(&rr, s->d_relres, sizeof(double), cudaMemcpyDeviceToHost, stream));
    dump_trace(s, "iccg", stream);
    baas_status st = read_status(s, stream);
    if (iters) *iters = it;
    if (relres) *relres = rr;
    if (st != BAAS_OK) return st;
    if (!(rr < tol)) return fail(BAAS_ERR_NOT_CONVERGED, "maxiter reached before tol");
    return BAAS_OK;
}

}  // extern "C"
