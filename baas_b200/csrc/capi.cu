// C ABI of the B200 BAAS hot path (declarations and contracts: include/baas_b200.h).
//
// baas_analyze builds the reference-identical schedule on the host (schedule.cpp). From it the
// device plan is derived: the schedule's groups listed level by level (the BAAS LevelSet
// order, rows ascending inside a group) give one global topological order of the rows; rows
// are given to P CTAs (contiguous row ranges by default, or the four-rule thread mapping);
// each CTA walks its rows in the global order (part_kernels.cuh). The backward sweep uses the
// exact reverse order. The plan is uploaded on the first GPU call, to the current device.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <map>
#include <mutex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/baas_b200.h"
#include "kernels.cuh"
#include "part_kernels.cuh"
#include "batched.cuh"
#include "staged.cuh"
#include "small.cuh"
#include "schedule.hpp"

using baas::DevStatus;

namespace baas {
baas_status set_error(baas_status code, const std::string &msg);
}

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
    // factorisations (forward direction): per entry, the A position of its pivot (the diagonal
    // of the row it depends on) and its column-match pairs in merge order (mptr ranges of
    // mpair = {offset in the own row, A position in the other row})
    std::vector<int> epiv, mptr, mpair;
    int max_local = 0;
};

struct PartDev {
    int *cta_seg = nullptr, *seg_item = nullptr, *item_pos = nullptr, *cta_pos = nullptr;
    int *row = nullptr, *eptr = nullptr, *dep = nullptr;
    int *srcT = nullptr, *dsrcT = nullptr, *srcA = nullptr, *dsrcA = nullptr;
    int *epiv = nullptr, *mptr = nullptr, *mpair = nullptr;
    baas::PartView view(int P) const {
        return baas::PartView{P, cta_seg, seg_item, item_pos, cta_pos, row, eptr, dep, epiv, mptr,
                              reinterpret_cast<const int2 *>(mpair)};
    }
    void release() {
        int *ptrs[] = {cta_seg, seg_item, item_pos, cta_pos, row, eptr, dep, srcT, dsrcT, srcA, dsrcA, epiv, mptr, mpair};
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
    if (!h.mptr.empty()) {
        BAAS_TRY(upload(d.epiv, h.epiv));
        BAAS_TRY(upload(d.mptr, h.mptr));
        BAAS_TRY(upload(d.mpair, h.mpair));
    }
    BAAS_TRY(upload(d.srcT, h.srcT));
    BAAS_TRY(upload(d.dsrcT, h.dsrcT));
    BAAS_TRY(upload(d.srcA, h.srcA));
    BAAS_TRY(upload(d.dsrcA, h.dsrcA));
    return BAAS_OK;
}

// Chunk plan (staged.cuh), host side: per direction the chunk int blocks and value-slot
// sources, CTA by CTA; the slot order rows of every CTA.
struct ChunkHostDir {
    std::vector<int> ints, vsrcT, vsrcA;
    std::vector<int> cval;                    // P + 1: value slots of each CTA
    std::vector<int> cchunk;                  // P + 1: chunks of each CTA
    std::vector<int> chunk_ioff, chunk_voff;  // nchunk + 1
};
struct ChunkHost {
    ChunkHostDir dir[2];
    std::vector<int> soff, srow;  // the rows of each CTA
    int slot_max = 0;             // most solution slots one CTA needs in one direction
};
struct ChunkDevDir {
    int *ints = nullptr, *vsrcT = nullptr, *vsrcA = nullptr, *cval = nullptr;
};
struct ChunkDev {
    ChunkDevDir dir[2];
    int *soff = nullptr, *srow = nullptr;
    void release() {
        for (auto &D : dir) {
            int *ptrs[] = {D.ints, D.vsrcT, D.vsrcA, D.cval};
            for (int *p : ptrs)
                if (p) cudaFree(p);
        }
        if (soff) cudaFree(soff);
        if (srow) cudaFree(srow);
        *this = ChunkDev();
    }
};
// Windows of one launch configuration (value width, right-hand sides walked together).
struct WinCfg {
    int4 *rec[2] = {nullptr, nullptr};
    int *swptr[2] = {nullptr, nullptr};
    int xs_bytes = 0, rhs_bytes = 0, cap = 0;
    size_t smem = 0;
    int nrec = 0;  // most windows of one CTA, both directions
    void release() {
        for (int d = 0; d < 2; d++) {
            if (rec[d]) cudaFree(rec[d]);
            if (swptr[d]) cudaFree(swptr[d]);
        }
    }
};

// Fetch-walk plan (fetch.cuh): per direction and CTA an int block [step table | records], the
// value-source codes of its records and the CTA's fetch list.
struct FetchHostDir {
    std::vector<int4> ints;        // int blocks, CTA by CTA
    std::vector<int4> cblk;        // P + 1: {first int4, int4 count, steps, first record}
    std::vector<int> code, codeT;  // 4 per record: {diag, a0, a1, a2} positions in A / in the caller's T
    std::vector<int> cfetch, frow; // P + 1 and the fetch lists
    int ints_max = 0;              // most int4 of one CTA's block
};
struct FetchHost {
    bool ok = false;  // every row has at most 3 off-diagonal entries and every step fits the compute warps
    FetchHostDir dir[2];
    int ncomp = 32;     // compute threads: the widest step, rounded up to a warp
    int rows_max = 0;   // most rows of one CTA
    int nslot_max = 0;  // most slots of one CTA: rows + 1 + staging of both directions
};
struct FetchDevDir {
    int4 *ints = nullptr, *cblk = nullptr;
    int *code = nullptr, *codeT = nullptr, *cfetch = nullptr, *frow = nullptr;
};
struct FetchDev {
    FetchDevDir dir[2];
    void release() {
        for (auto &D : dir) {
            void *ptrs[] = {D.ints, D.cblk, D.code, D.codeT, D.cfetch, D.frow};
            for (void *p : ptrs)
                if (p) cudaFree(p);
        }
        *this = FetchDev();
    }
};

// Single-CTA walk plan (small.cuh): row levels of both directions and each row's record in the
// caller's triangular layouts (rec_t: L diagonal last, U = L^T diagonal first) and in the full
// matrix's layouts ICCG and IC0 read (rec_a: A's lower part; U's off-diagonal entries gathered
// from the IC0 factor), plus the IC0 column-match pairs.
struct SmallHost {
    bool built = false;
    int nlev[2] = {0, 0};
    std::vector<int> lev[2];
    std::vector<int4> rec_t[2], rec_a[2];
    std::vector<int> ic_ptr, ub_col, ub_pos;
    std::vector<int2> ic_pair;
};

// Level-walk plan (staged.cuh level_walk): the whole schedule as one partition, per direction.
struct LevelHostDir {
    std::vector<int> lev, item, row, eptr, dep, src, dsrc, srcT, dsrcT;
};
struct LevelDevDir {
    int *lev = nullptr, *item = nullptr, *row = nullptr, *eptr = nullptr, *dep = nullptr, *src = nullptr,
        *dsrc = nullptr, *srcT = nullptr, *dsrcT = nullptr;
    int nlev = 0, nent = 0, npos = 0;
    baas::LevelDir view() const { return baas::LevelDir{lev, item, row, eptr, dep, src, dsrc, srcT, dsrcT, nlev, nent, npos}; }
    void release() {
        int *ptrs[] = {lev, item, row, eptr, dep, src, dsrc, srcT, dsrcT};
        for (int *p : ptrs)
            if (p) cudaFree(p);
        *this = LevelDevDir();
    }
};

baas_status upload_fetch(FetchDev &d, const FetchHost &h) {
    for (int k = 0; k < 2; k++) {
        const FetchHostDir &H = h.dir[k];
        FetchDevDir &D = d.dir[k];
        BAAS_TRY(upload(D.ints, H.ints));
        BAAS_TRY(upload(D.cblk, H.cblk));
        BAAS_TRY(upload(D.code, H.code));
        BAAS_TRY(upload(D.codeT, H.codeT));
        BAAS_TRY(upload(D.cfetch, H.cfetch));
        BAAS_TRY(upload(D.frow, H.frow));
    }
    return BAAS_OK;
}

baas_status upload_chunks(ChunkDev &d, const ChunkHost &h) {
    for (int k = 0; k < 2; k++) {
        const ChunkHostDir &H = h.dir[k];
        ChunkDevDir &D = d.dir[k];
        BAAS_TRY(upload(D.ints, H.ints));
        BAAS_TRY(upload(D.vsrcT, H.vsrcT));
        BAAS_TRY(upload(D.vsrcA, H.vsrcA));
        BAAS_TRY(upload(D.cval, H.cval));
    }
    BAAS_TRY(upload(d.soff, h.soff));
    BAAS_TRY(upload(d.srow, h.srow));
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
    std::vector<int> custom_part;  // BAAS_PARTITION_CUSTOM: the caller's row -> CTA map
    bool use_boxes = false;        // grid-box partition (choose_partition)
    int grid[3] = {1, 1, 1}, box[3] = {1, 1, 1}, nbox[3] = {1, 1, 1};
    PartHost fwd, bwd;
    ChunkHost chk;
    FetchHost fch;
    int fault_row = -1;  // test hook: forward row made to wait on its own output

    // device
    int device = -1;
    bool uploaded = false;
    int num_sms = 0;
    PartDev d_fwd, d_bwd;
    ChunkDev d_chk;
    FetchDev d_fch;
    double *d_gf64[2] = {nullptr, nullptr};  // fetch-walk record values: ICCG factors, FP64
    float *d_gf32[2] = {nullptr, nullptr};   // the same, FP32
    double *d_gfT[2] = {nullptr, nullptr};   // record values of the caller's factor (sweeps)
    int last_walk = 0;                       // walk of the last sweep / ICCG launch (BAAS_WALK_*)
    double *d_dg = nullptr;                  // fetch-walk IC0: each row's diagonal (its ready flag)
    LevelDevDir d_lv[2];                     // level-walk plan, per direction
    double *d_lv64[2] = {nullptr, nullptr}, *d_ld64[2] = {nullptr, nullptr};  // its values (ICCG, FP64)
    float *d_lv32[2] = {nullptr, nullptr}, *d_ld32[2] = {nullptr, nullptr};   // (ICCG, FP32 factors)
    double *d_lvT[2] = {nullptr, nullptr}, *d_ldT[2] = {nullptr, nullptr};    // (caller's factor, sweeps)
    double *d_fbuf[2] = {nullptr, nullptr};  // standalone fetch sweeps: publication buffers, used in turn
    int fbuf_cur = 0;                        // the buffer the next sweep publishes into
    bool fbuf_ready = false;                 // both hold the sentinel wherever the next sweep will look
    int4 *d_ilu_rec = nullptr;               // level ILU0: per plan position {row, first entry, entries, lower}
    int2 *d_ilu_dep = nullptr;               // ... and per lower entry {partner diagonal, partner upper entries}
    SmallHost sm;                            // single-CTA walk plan (host), built on first use
    int *d_sm_lev[2] = {nullptr, nullptr};
    int4 *d_sm_rec_t[2] = {nullptr, nullptr}, *d_sm_rec_a[2] = {nullptr, nullptr};
    int *d_sm_ic_ptr = nullptr, *d_sm_ub_col = nullptr, *d_sm_ub_pos = nullptr;
    int2 *d_sm_ic_pair = nullptr;
    double *d_sm_ut = nullptr;
    float *d_sm_lf32 = nullptr, *d_sm_ut32 = nullptr, *d_sm_rcp32 = nullptr;
    std::map<int, WinCfg> wins;  // key: value bytes * 16 + right-hand sides
    int smem_budget = 0;
    int rmax64 = 1;  // most FP64 right-hand sides one sweep walks together
    int factor_prec = -1;  // precision of the IC0 factors the last baas_iccg left in the value slots
    double *d_gvT[2] = {nullptr, nullptr};  // packed values of the caller's factor (sweeps)
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
    // the initial guess of an FP64 ICCG launch, kept for its repeat with IEEE divisions
    double *d_x0 = nullptr;
    size_t x0_cap = 0;

    // batched systems (baas_analyze_batch): row offsets of the systems, and the vector-phase
    // decomposition (built at the first batched solve)
    std::vector<int> sys_off;
    int nsys = 0, maxls = 0;
    int *d_sys_off = nullptr, *d_vlo = nullptr, *d_sys_lo = nullptr, *d_nls = nullptr, *d_cta_lo = nullptr,
        *d_cta_hi = nullptr;
    int batch_R = 0;  // right-hand sides the batched workspace is sized for
    double *d_br = nullptr, *d_bp = nullptr, *d_bAp = nullptr, *d_by = nullptr, *d_bz = nullptr, *d_bpart = nullptr,
           *d_brelres = nullptr, *d_blu = nullptr;
    float *d_by32 = nullptr, *d_bz32 = nullptr;
    double *d_bgv64[2] = {nullptr, nullptr};
    float *d_bgv32[2] = {nullptr, nullptr};
    int *d_biters = nullptr;
    unsigned int *d_active = nullptr;

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

// Structured-grid detection: the off-diagonal offsets r - c of L's rows are {1}, {1, n1} or
// {1, n1, n1 n2} (a 1-, 2- or 3-D stencil in natural ordering, x fastest), with n a multiple of
// the grid's plane size. Only a hint for the partition: any partition gives the same results.
bool detect_grid(const baas::HostSchedule &h, int dims[3]) {
    const int n = h.n;
    int off[4], no = 0;
    for (int r = 0; r < n; r++)
        for (int e = h.l_rowptr[r]; e < h.l_rowptr[r + 1] - 1; e++) {
            const int o = r - h.l_colidx[e];
            int t = 0;
            while (t < no && off[t] != o) t++;
            if (t == no) {
                if (no == 3) return false;
                off[no++] = o;
            }
        }
    std::sort(off, off + no);
    if (no == 0 || off[0] != 1) return false;
    dims[0] = n, dims[1] = 1, dims[2] = 1;
    if (no >= 2) {
        if (n % off[1]) return false;
        dims[0] = off[1];
        dims[1] = n / off[1];
    }
    if (no == 3) {
        if (off[2] % off[1] || n % off[2]) return false;
        dims[1] = off[2] / off[1];
        dims[2] = n / off[2];
    }
    return dims[0] >= 2 || n == 1;
}

// Box shape for the BLOCKS partition of an n1 x n2 x n3 grid: boxes of at most vmax rows, at
// most max_boxes of them, whose widest level (anti-diagonal) fits the fetch walk's compute warps.
// The shape minimises a model of the fetch walk's sweep time: one step per level of the grid
// (~0.15 us, 10% more per extra compute warp) plus ~1.8 us for every box boundary the
// critical path crosses -- the constants measured on B200 for 64^3 with 2,048-row boxes.
bool choose_boxes(const int dims[3], int max_boxes, int vmax, int box[3], int nbox[3]) {
    auto cand = [](int m) {
        std::vector<int> v;
        for (int b = 1; b < m; b *= 2) v.push_back(b);
        v.push_back(m);
        return v;
    };
    double best = 1e30;
    bool found = false;
    for (int b1 : cand(dims[0]))
        for (int b2 : cand(dims[1]))
            for (int b3 : cand(dims[2])) {
                if ((long long)b1 * b2 * b3 > vmax) continue;
                const int c1 = (dims[0] + b1 - 1) / b1, c2 = (dims[1] + b2 - 1) / b2, c3 = (dims[2] + b3 - 1) / b3;
                if ((long long)c1 * c2 * c3 > max_boxes) continue;
                std::vector<int> lev(b1 + b2 + b3, 0);
                for (int i = 0; i < b1; i++)
                    for (int j = 0; j < b2; j++)
                        for (int k = 0; k < b3; k++) lev[i + j + k]++;
                const int width = *std::max_element(lev.begin(), lev.end());
                if (width > baas::kFetchMaxRows) continue;
                const int warps = (width + 31) / 32;
                const double est = (dims[0] + dims[1] + dims[2] - 2) * 0.15 * (1.0 + 0.1 * (warps - 1)) +
                                   1.8 * (c1 - 1 + c2 - 1 + c3 - 1);
                if (est < best - 1e-9 || (est < best + 1e-9 && found && b1 > box[0])) {
                    best = est;
                    box[0] = b1, box[1] = b2, box[2] = b3;
                    nbox[0] = c1, nbox[1] = c2, nbox[2] = c3;
                    found = true;
                }
            }
    return found;
}

// The partition a plan uses and its CTA count. AUTO: grid boxes when the pattern is a
// natural-order stencil whose rows (of L and of U = L^T) hold at most 3 off-diagonal entries and
// the fetch walk is allowed (those are the plans the fetch walk runs fastest on), else RANGES.
// BLOCKS: grid boxes whenever the pattern is a grid, else RANGES. RANGES: `parts`, or about one
// CTA per 2,048 rows (at most one per SM).
int choose_partition(baas_schedule *s, int num_sms) {
    const baas::HostSchedule &h = s->hs;
    const int n = h.n;
    s->use_boxes = false;
    if (s->opt.partition == BAAS_PARTITION_BAAS_THREADS) return h.nthread;
    if (s->opt.partition == BAAS_PARTITION_CUSTOM) return s->opt.parts;
    const bool may_box = s->opt.parts == 0 && (s->opt.partition == BAAS_PARTITION_BLOCKS ||
                                               (s->opt.partition == BAAS_PARTITION_AUTO && s->opt.walk != BAAS_WALK_CHUNKED));
    if (may_box) {
        bool narrow = true;
        for (int r = 0; r < n && narrow; r++) narrow = h.l_rowptr[r + 1] - h.l_rowptr[r] - 1 <= 3 && s->cptr[r + 1] - s->cptr[r] - 1 <= 3;
        int dims[3];
        if ((narrow || s->opt.partition == BAAS_PARTITION_BLOCKS) && detect_grid(h, dims) &&
            choose_boxes(dims, num_sms, 2048, s->box, s->nbox)) {
            s->use_boxes = true;
            s->grid[0] = dims[0], s->grid[1] = dims[1], s->grid[2] = dims[2];
            return s->nbox[0] * s->nbox[1] * s->nbox[2];
        }
    }
    if (s->opt.parts > 0) return std::min(s->opt.parts, n);
    return std::max(1, std::min((n + 2047) / 2048, num_sms));
}

// Groups -> CTAs. RANGES: the CTA whose row range holds the group's first row (P contiguous,
// row-balanced ranges). BAAS_THREADS: the four-rule mapping's thread of the group. Boxes
// (use_boxes): the grid box that holds the group's first row.
void build_partition(baas_schedule *s, int P) {
    const baas::HostSchedule &h = s->hs;
    const int n = h.n;
    s->P = P;
    s->group_cta.assign(h.ngroups, 0);
    if (s->opt.partition == BAAS_PARTITION_CUSTOM) {
        for (int g = 0; g < h.ngroups; g++) s->group_cta[g] = s->custom_part[h.group_set[h.group_ptr[g]]];
    } else if (s->opt.partition == BAAS_PARTITION_BAAS_THREADS) {
        for (int t = 0; t < h.nthread; t++)
            for (int task = h.thread_boundaries[t]; task < h.thread_boundaries[t + 1]; task++)
                for (int q = h.task_boundaries[task]; q < h.task_boundaries[task + 1]; q++) s->group_cta[h.thread_cont_to_orig[q]] = t;
    } else if (s->use_boxes) {
        for (int g = 0; g < h.ngroups; g++) {
            const int r0 = h.group_set[h.group_ptr[g]];
            const int i = r0 % s->grid[0], j = (r0 / s->grid[0]) % s->grid[1], k = r0 / (s->grid[0] * s->grid[1]);
            s->group_cta[g] = i / s->box[0] + s->nbox[0] * (j / s->box[1] + s->nbox[1] * (k / s->box[2]));
        }
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
    const int n = h.n, P = s->P, nl = (int)h.exec_level_ptr.size() - 1;
    out = PartHost();
    // per CTA: list of (level, group) in processing order
    std::vector<std::vector<std::pair<int, int>>> items(P);
    for (int li = 0; li < nl; li++) {
        const int l = upper ? nl - 1 - li : li;
        const int qb = h.exec_level_ptr[l], qe = h.exec_level_ptr[l + 1];
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
    if (!upper && h.kind != baas::SchedKind::SpTRSV) {
        // factorisation entries: entry t of a row is A position rb + t (the row's lower part,
        // ascending). IC0 (merge/IC.cpp sparse_dot_product): row i's entry at column j pairs with
        // row j's entries of equal column, both lower parts; ILU0 (merge/ILU.cpp): entry t with
        // column c updates row i's later entries whose column row c holds in its upper part.
        const bool ilu = h.kind == baas::SchedKind::ILU0;
        const std::vector<int> &rp = h.a_rowptr, &ci = h.a_colidx, &dg = h.a_diagptr;
        out.epiv.assign(out.dep.size(), 0);
        out.mptr.assign(out.dep.size() + 1, 0);
        out.mpair.clear();
        for (int pos = 0; pos < n; pos++) {
            const int r = out.row[pos], rb = rp[r], di = dg[r], re = rp[r + 1];
            for (int t = 0; t < di - rb; t++) {
                const int e = out.eptr[pos] + t, j = ci[rb + t];
                out.epiv[e] = dg[j];
                int a = ilu ? rb + t + 1 : rb, ae = ilu ? re : di;
                int b = ilu ? dg[j] + 1 : rp[j], be = ilu ? rp[j + 1] : dg[j];
                while (a < ae && b < be) {
                    if (ci[a] == ci[b]) {
                        out.mpair.push_back(a - rb);
                        out.mpair.push_back(b);
                        a++;
                        b++;
                    } else if (ci[a] < ci[b]) {
                        a++;
                    } else {
                        b++;
                    }
                }
                out.mptr[e + 1] = (int)(out.mpair.size() / 2);
            }
        }
    }
    if (!upper && s->fault_row >= 0) {
        for (int pos = 0; pos < n; pos++)
            if (out.row[pos] == s->fault_row && out.eptr[pos + 1] > out.eptr[pos]) out.dep[out.eptr[pos]] = s->fault_row;
    }
}

// Chunk plan from the two position plans: per CTA, each level segment becomes as many steps as
// its largest group has rows; step j holds the j-th row of every group of the level. A step is
// one chunk, cut into several when its block would exceed kChunkBytes (FP64 values). All chunks
// of a CTA and direction share one entry stride, the CTA's widest row. A row gets a solution slot
// only if a later row of the same CTA reads it, and only until that last read: slots are
// allocated by liveness, so a CTA needs about two levels' worth of them, not one per row.
constexpr int kChunkBytes = 16 * 1024;

int chunk_bytes64(int nl, int E) { return baas::chunk_nint(nl, E) * 4 + baas::chunk_nval(nl, E) * 8; }

void build_chunks(baas_schedule *s) {
    const int n = s->hs.n, P = s->P;
    ChunkHost &C = s->chk;
    C = ChunkHost();
    C.soff.assign(P + 1, 0);
    C.srow.reserve(n);
    std::vector<int> ordidx(n, -1);  // part position -> index in the CTA's step order
    std::vector<int> kpos_of(n, 0);  // row -> its position in its CTA's row list
    for (int d = 0; d < 2; d++) {
        const PartHost &H = d == 0 ? s->fwd : s->bwd;
        ChunkHostDir &D = C.dir[d];
        D.cval.assign(P + 1, 0);
        D.cchunk.assign(P + 1, 0);
        D.chunk_ioff.assign(1, 0);
        D.chunk_voff.assign(1, 0);
        for (int c = 0; c < P; c++) {
            // steps of this CTA: positions in order
            std::vector<int> order, step_end;
            for (int sg = H.cta_seg[c]; sg < H.cta_seg[c + 1]; sg++) {
                int m = 0;
                for (int it = H.seg_item[sg]; it < H.seg_item[sg + 1]; it++) m = std::max(m, H.item_pos[it + 1] - H.item_pos[it]);
                for (int j = 0; j < m; j++) {
                    for (int it = H.seg_item[sg]; it < H.seg_item[sg + 1]; it++)
                        if (H.item_pos[it] + j < H.item_pos[it + 1]) order.push_back(H.item_pos[it] + j);
                    step_end.push_back((int)order.size());
                }
            }
            if (d == 0) {
                for (int pos : order) {
                    kpos_of[H.row[pos]] = (int)C.srow.size() - C.soff[c];
                    C.srow.push_back(H.row[pos]);
                }
                C.soff[c + 1] = (int)C.srow.size();
            }
            const int no = (int)order.size();
            for (int k = 0; k < no; k++) ordidx[order[k]] = k;
            // one entry stride for all of the CTA's chunks: its widest row (at least 1)
            int E = 1;
            for (int pos : order) E = std::max(E, H.eptr[pos + 1] - H.eptr[pos]);
            // chunks: each step, cut into pieces of at most kChunkBytes
            std::vector<std::pair<int, int>> chunks;
            int kb = 0;
            for (int se : step_end) {
                int cb = kb;
                for (int k = kb; k < se; k++)
                    if (k > cb && chunk_bytes64(k + 1 - cb, E) > kChunkBytes) {
                        chunks.push_back({cb, k});
                        cb = k;
                    }
                if (se > cb) chunks.push_back({cb, se});
                kb = se;
            }
            // liveness: the last chunk in which a row of this CTA reads each row's value
            std::vector<int> chunk_of(no), last_use(no, -1);
            for (size_t t = 0; t < chunks.size(); t++)
                for (int k = chunks[t].first; k < chunks[t].second; k++) chunk_of[k] = (int)t;
            for (int k = 0; k < no; k++) {
                const int pos = order[k];
                for (int e = H.eptr[pos]; e < H.eptr[pos + 1]; e++)
                    if (H.dep[e] < 0) {
                        const int kp = ordidx[H.cta_pos[c] + (-H.dep[e] - 1)];
                        last_use[kp] = std::max(last_use[kp], chunk_of[k]);
                    }
            }
            // slots: a row holds one from its own chunk to its last local reader's chunk; a
            // slot freed after chunk t serves rows of chunk t+1 onwards
            std::vector<int> slot(no, -1), free_slots;
            std::vector<std::vector<int>> release((size_t)chunks.size() + 1);
            int nslots = 0;
            for (size_t t = 0; t < chunks.size(); t++) {
                if (t > 0)
                    for (int sl : release[t - 1]) free_slots.push_back(sl);
                for (int k = chunks[t].first; k < chunks[t].second; k++) {
                    if (last_use[k] < 0) continue;
                    int sl;
                    if (!free_slots.empty()) {
                        sl = free_slots.back();
                        free_slots.pop_back();
                    } else {
                        sl = nslots++;
                    }
                    slot[k] = sl;
                    release[last_use[k]].push_back(sl);
                }
            }
            C.slot_max = std::max(C.slot_max, nslots);
            for (size_t t = 0; t < chunks.size(); t++) {
                const int cb = chunks[t].first, ce = chunks[t].second, nl = ce - cb;
                const size_t i0 = D.ints.size();
                D.ints.resize(i0 + baas::chunk_nint(nl, E), 0);
                int *I = D.ints.data() + i0;
                I[0] = nl;
                I[1] = E;
                I[2] = t + 1 < chunks.size() ? chunks[t + 1].second - chunks[t + 1].first : 0;
                int *rowid = I + baas::kChunkHdr, *sl = rowid + nl, *ne = sl + nl, *kp = ne + nl, *dep = kp + nl;
                const size_t v0 = D.vsrcT.size();
                D.vsrcT.resize(v0 + baas::chunk_nval(nl, E), -1);
                D.vsrcA.resize(v0 + baas::chunk_nval(nl, E), -1);
                int *vT = D.vsrcT.data() + v0, *vA = D.vsrcA.data() + v0;
                for (int k = cb; k < ce; k++) {
                    const int q = k - cb, pos = order[k];
                    rowid[q] = H.row[pos];
                    sl[q] = slot[k];
                    kp[q] = kpos_of[H.row[pos]];
                    ne[q] = H.eptr[pos + 1] - H.eptr[pos];
                    vT[q] = baas::diag_code(H.dsrcT[pos]);
                    vA[q] = baas::diag_code(H.dsrcA[pos]);
                    vT[nl + q] = baas::rcp_code(H.dsrcT[pos]);
                    vA[nl + q] = baas::rcp_code(H.dsrcA[pos]);
                    for (int j = 0; j < ne[q]; j++) {
                        const int e = H.eptr[pos] + j;
                        const int dd = H.dep[e];
                        // local: the producer's slot; remote: -(row + 1)
                        dep[q * E + j] = dd < 0 ? slot[ordidx[H.cta_pos[c] + (-dd - 1)]] : -(dd + 1);
                        vT[2 * nl + q * E + j] = H.srcT[e];
                        vA[2 * nl + q * E + j] = H.srcA[e];
                    }
                }
                D.chunk_ioff.push_back((int)D.ints.size());
                D.chunk_voff.push_back((int)D.vsrcT.size());
            }
            D.cchunk[c + 1] = (int)D.chunk_ioff.size() - 1;
            D.cval[c + 1] = (int)D.vsrcT.size();
        }
    }
}

// Fetch-walk plan (fetch.cuh) from the same per-CTA steps as the chunk plan: a level segment
// whose groups hold up to m rows is m steps, step j holding the j-th row of every group.
// Records carry the row's own slot (its position in the CTA's row list, C.srow) and one slot
// per off-diagonal entry, in the entry order of the position plan (ascending columns for L,
// descending for U): the producer's own slot when it belongs to this CTA, the zero slot (rows)
// for an absent entry, or the staging slot of the producer's fetch-list entry (rows + 1 + f in
// the lower direction, rows + 1 + nf_lower + f in the upper). The plan is marked unusable (and
// the chunked walk runs) when a row has more than 3 off-diagonal entries or a step more rows
// than the compute warps hold.
void build_fetch(baas_schedule *s) {
    const int n = s->hs.n, P = s->P;
    const ChunkHost &C = s->chk;
    FetchHost &F = s->fch;
    F = FetchHost();
    std::vector<int> kpos_of(n, 0);
    for (int c = 0; c < P; c++) {
        for (int k = C.soff[c]; k < C.soff[c + 1]; k++) kpos_of[C.srow[k]] = k - C.soff[c];
        F.rows_max = std::max(F.rows_max, C.soff[c + 1] - C.soff[c]);
    }
    std::vector<int> fidx(n, -1), nf0(P, 0), nslot(P, 0);
    bool ok = true;
    int widest = 1;
    for (int d = 0; d < 2 && ok; d++) {
        const PartHost &H = d == 0 ? s->fwd : s->bwd;
        FetchHostDir &D = F.dir[d];
        D.cfetch.assign(1, 0);
        D.code.reserve(4 * (size_t)n);
        D.codeT.reserve(4 * (size_t)n);
        for (int c = 0; c < P && ok; c++) {
            const int nrows = C.soff[c + 1] - C.soff[c];
            const int sbase = nrows + 1 + (d ? nf0[c] : 0);
            std::vector<int> order, step_end;
            for (int sg = H.cta_seg[c]; sg < H.cta_seg[c + 1]; sg++) {
                int m = 0;
                for (int it = H.seg_item[sg]; it < H.seg_item[sg + 1]; it++) m = std::max(m, H.item_pos[it + 1] - H.item_pos[it]);
                for (int j = 0; j < m; j++) {
                    for (int it = H.seg_item[sg]; it < H.seg_item[sg + 1]; it++)
                        if (H.item_pos[it] + j < H.item_pos[it + 1]) order.push_back(H.item_pos[it] + j);
                    step_end.push_back((int)order.size());
                }
            }
            const int ns = (int)step_end.size();
            const int i0 = (int)D.ints.size();
            // step table: {first record, rows, 0, 0}, then two copies of the last step
            int kb = 0;
            for (int t = 0; t < ns; t++) {
                const int nl = step_end[t] - kb;
                if (nl > baas::kFetchMaxRows) ok = false;
                widest = std::max(widest, nl);
                D.ints.push_back(make_int4(kb, nl, 0, 0));
                kb = step_end[t];
            }
            const int4 last = ns > 0 ? D.ints.back() : make_int4(0, 1, 0, 0);
            D.ints.push_back(last);
            D.ints.push_back(last);
            const int fb = (int)D.frow.size();
            for (int pos : order) {
                const int row = H.row[pos], ne = H.eptr[pos + 1] - H.eptr[pos];
                if (ne > 3) {
                    ok = false;
                    break;
                }
                int sl[3] = {nrows, nrows, nrows}, ca[4] = {H.dsrcA[pos], -1, -1, -1}, ct[4] = {H.dsrcT[pos], -1, -1, -1};
                for (int j = 0; j < ne; j++) {
                    const int e = H.eptr[pos] + j, dd = H.dep[e];
                    if (dd < 0) {
                        sl[j] = kpos_of[H.row[H.cta_pos[c] + (-dd - 1)]];
                    } else {
                        if (fidx[dd] < 0) {
                            fidx[dd] = (int)D.frow.size() - fb;
                            D.frow.push_back(dd);
                        }
                        sl[j] = sbase + fidx[dd];
                    }
                    ca[j + 1] = H.srcA[e];
                    ct[j + 1] = H.srcT[e];
                }
                D.ints.push_back(make_int4(kpos_of[row], sl[0], sl[1], sl[2]));
                for (int j = 0; j < 4; j++) {
                    D.code.push_back(ca[j]);
                    D.codeT.push_back(ct[j]);
                }
            }
            for (size_t f = fb; f < D.frow.size(); f++) fidx[D.frow[f]] = -1;
            const int nf = (int)D.frow.size() - fb;
            if (d == 0) nf0[c] = nf;
            nslot[c] = std::max(nslot[c], nrows + 1 + nf0[c] + (d ? nf : 0));
            D.cblk.push_back(make_int4(i0, (int)D.ints.size() - i0, ns, C.soff[c]));
            D.cfetch.push_back((int)D.frow.size());
            D.ints_max = std::max(D.ints_max, (int)D.ints.size() - i0);
        }
        D.cblk.push_back(make_int4((int)D.ints.size(), 0, 0, n));
    }
    for (int c = 0; c < P; c++) F.nslot_max = std::max(F.nslot_max, nslot[c]);
    F.ncomp = (widest + 31) / 32 * 32;
    F.ok = ok && F.ncomp <= baas::kFetchMaxRows;
    if (!F.ok) F = FetchHost();
}

// Level-walk plan of one direction: levels in execution order (descending for U = L^T), the
// groups of a level in LevelSet order (reversed for U), a group's rows ascending (descending for
// U); each row's entries in the reference's order -- L: off-diagonals ascending, diagonal last;
// U = L^T: diagonal first, off-diagonals descending -- with the row each reads and the value's
// position in A (through the lower triangle's source map) and in the caller's triangular CSR.
void build_level_dir(const baas_schedule *s, bool upper, LevelHostDir &D) {
    const baas::HostSchedule &h = s->hs;
    const int nl = (int)h.exec_level_ptr.size() - 1;
    D = LevelHostDir();
    D.lev.assign(1, 0);
    D.item.assign(1, 0);
    D.eptr.assign(1, 0);
    for (int li = 0; li < nl; li++) {
        const int l = upper ? nl - 1 - li : li;
        const int qb = h.exec_level_ptr[l], qe = h.exec_level_ptr[l + 1];
        for (int qi = 0; qi < qe - qb; qi++) {
            const int g = h.perm_to_orig[upper ? qe - 1 - qi : qb + qi];
            const int rb = h.group_ptr[g], re = h.group_ptr[g + 1];
            for (int k = 0; k < re - rb; k++) {
                const int r = h.group_set[upper ? re - 1 - k : rb + k];
                D.row.push_back(r);
                if (!upper) {
                    const int lb = h.l_rowptr[r], le = h.l_rowptr[r + 1];
                    for (int e = lb; e < le - 1; e++) {
                        D.dep.push_back(h.l_colidx[e]);
                        D.src.push_back(h.l_src[e]);
                        D.srcT.push_back(e);
                    }
                    D.dsrc.push_back(h.l_src[le - 1]);
                    D.dsrcT.push_back(le - 1);
                } else {
                    const int cb = s->cptr[r], ce = s->cptr[r + 1];
                    for (int e = ce - 1; e > cb; e--) {
                        D.dep.push_back(s->crow[e]);
                        D.src.push_back(h.l_src[s->cpos[e]]);
                        D.srcT.push_back(e);
                    }
                    D.dsrc.push_back(h.l_src[s->cpos[cb]]);
                    D.dsrcT.push_back(cb);
                }
                D.eptr.push_back((int)D.dep.size());
            }
            D.item.push_back((int)D.row.size());
        }
        D.lev.push_back((int)D.item.size() - 1);
    }
}

baas_status upload_level(baas_schedule *s) {
    for (int d = 0; d < 2; d++) {
        LevelHostDir H;
        build_level_dir(s, d == 1, H);
        LevelDevDir &D = s->d_lv[d];
        BAAS_TRY(upload(D.lev, H.lev));
        BAAS_TRY(upload(D.item, H.item));
        BAAS_TRY(upload(D.row, H.row));
        BAAS_TRY(upload(D.eptr, H.eptr));
        BAAS_TRY(upload(D.dep, H.dep));
        BAAS_TRY(upload(D.src, H.src));
        BAAS_TRY(upload(D.dsrc, H.dsrc));
        BAAS_TRY(upload(D.srcT, H.srcT));
        BAAS_TRY(upload(D.dsrcT, H.dsrcT));
        D.nlev = (int)H.lev.size() - 1;
        D.nent = (int)H.dep.size();
        D.npos = (int)H.row.size();
    }
    return BAAS_OK;
}

// Shared bytes of a fetch-walk launch: ICCG (both directions' int blocks resident; values: FP64
// one direction at a time, FP32 both) or a standalone sweep (one direction).
size_t fetch_smem(const FetchHost &F, int vbytes, bool iccg) {
    // an ICCG launch reserves 8-byte slots in both precisions (its IC0 walk passes FP64 diagonals)
    const int slot_bytes = (F.nslot_max * (iccg ? 8 : vbytes) + 15) / 16 * 16;
    const int srow_bytes = (F.nslot_max * 4 + 15) / 16 * 16;
    const int ib0 = 16 * (iccg ? F.dir[0].ints_max : std::max(F.dir[0].ints_max, F.dir[1].ints_max));
    const int ib1 = iccg ? 16 * F.dir[1].ints_max : 0;
    const int rb = vbytes == 8 ? 8 * baas::kFetchVal64 : 4 * baas::kFetchVal32;
    const int vb = iccg ? std::max(rb * F.rows_max * (vbytes == 4 ? 2 : 1), 8 * baas::kFetchVal64 * F.rows_max)
                        : rb * F.rows_max;
    return (size_t)baas::fetch_smem_bytes(slot_bytes, srow_bytes, ib0, ib1, vb);
}

// Windows for values of `vbytes` bytes and R right-hand sides: each CTA's chunks grouped
// greedily into blocks that fit one of the two buffers. False if a chunk does not fit.
// Window buffers: at most kWindowTarget bytes each unless the budget was set explicitly (then
// as large as it allows), and never larger than the largest window formed, so that shared
// memory the plan does not need stays L1 cache for the SpMV and vector phases.
constexpr int kWindowTarget = 32 * 1024;
constexpr int kStagedMinCap = 16 * 1024;

bool plan_windows(const ChunkHost &C, int P, int budget, bool explicit_budget, int vbytes, int R,
                  std::vector<int4> rec[2], std::vector<int> swptr[2], int &xs_bytes, int &rhs_bytes, int &cap,
                  int &nrec) {
    xs_bytes = (int)(((long long)C.slot_max * R * vbytes + 127) / 128 * 128);
    // right-hand sides staged in shared memory when the CTA's rows' values fit beside the slots
    // and two buffers of at least kStagedMinCap
    int rows_max = 0;
    for (int c = 0; c < P; c++) rows_max = std::max(rows_max, C.soff[c + 1] - C.soff[c]);
    rhs_bytes = (int)(((long long)rows_max * R * vbytes + 127) / 128 * 128);
    long long big = 0;  // every chunk must fit a buffer
    for (int d = 0; d < 2; d++) {
        const ChunkHostDir &D = C.dir[d];
        for (size_t k = 0; k + 1 < D.chunk_ioff.size(); k++)
            big = std::max(big, (long long)(D.chunk_ioff[k + 1] - D.chunk_ioff[k]) * 4 +
                                    (long long)(D.chunk_voff[k + 1] - D.chunk_voff[k]) * vbytes);
    }
    // the control block holds one record per window of a CTA: reserve room for it, and grow
    // the reserve if the windows outnumber it
    for (int reserve = 1024;;) {
        if (rhs_bytes > 0 && ((budget - xs_bytes - rhs_bytes - reserve) / 2 < std::max<long long>(big, kStagedMinCap)))
            rhs_bytes = 0;
        const int cap_max = ((budget - xs_bytes - rhs_bytes - reserve) / 2) & ~127;
        if (cap_max < 1024 || big > cap_max) return false;
        cap = explicit_budget ? cap_max : std::min(cap_max, kWindowTarget);
        cap = std::max(cap, (int)((big + 127) / 128 * 128));
        std::vector<int> count(P, 0);
        for (int d = 0; d < 2; d++) {
            const ChunkHostDir &D = C.dir[d];
            rec[d].clear();
            swptr[d].assign(P + 1, 0);
            for (int c = 0; c < P; c++) {
                const int kb = D.cchunk[c], ke = D.cchunk[c + 1];
                int a = kb;
                auto bytes = [&](int x, int y) {
                    return (long long)(D.chunk_ioff[y] - D.chunk_ioff[x]) * 4 +
                           (long long)(D.chunk_voff[y] - D.chunk_voff[x]) * vbytes;
                };
                auto close = [&](int x, int y) {
                    rec[d].push_back(make_int4(D.chunk_ioff[x], D.chunk_ioff[y] - D.chunk_ioff[x], D.chunk_voff[x],
                                               D.chunk_voff[y] - D.chunk_voff[x]));
                };
                for (int k = kb; k < ke; k++)
                    if (k > a && bytes(a, k + 1) > cap) {
                        close(a, k);
                        a = k;
                    }
                if (ke > a) close(a, ke);
                swptr[d][c + 1] = (int)rec[d].size();
                count[c] += swptr[d][c + 1] - swptr[d][c];
            }
        }
        nrec = 1;
        for (int c = 0; c < P; c++) nrec = std::max(nrec, count[c]);
        if (baas::win_ctl_bytes(nrec) <= reserve) break;
        reserve = baas::win_ctl_bytes(nrec) + 512;
        if (reserve > budget / 4) return false;
    }
    long long widest = 0;
    for (int d = 0; d < 2; d++)
        for (const int4 &r : rec[d]) widest = std::max(widest, (long long)r.y * 4 + (long long)r.w * vbytes);
    cap = std::min(cap, (int)((widest + 127) / 128 * 128));
    return true;
}

baas_status get_windows(baas_schedule *s, int vbytes, int R, WinCfg **out) {
    const int key = vbytes * 16 + R;
    auto it = s->wins.find(key);
    if (it != s->wins.end()) {
        *out = &it->second;
        return BAAS_OK;
    }
    std::vector<int4> rec[2];
    std::vector<int> swptr[2];
    int xs_bytes = 0, rhs_bytes = 0, cap = 0, mw = 0;
    if (!plan_windows(s->chk, s->P, s->smem_budget, s->opt.smem_budget > 0, vbytes, R, rec, swptr, xs_bytes, rhs_bytes,
                      cap, mw))
        return fail(BAAS_ERR_BAD_ARG, "a CTA's rows do not fit its shared memory: raise `parts` or smem_budget");
    WinCfg w;
    for (int d = 0; d < 2; d++) {
        BAAS_TRY(upload(w.rec[d], rec[d]));
        BAAS_TRY(upload(w.swptr[d], swptr[d]));
    }
    w.xs_bytes = xs_bytes;
    w.rhs_bytes = rhs_bytes;
    w.cap = cap;
    w.smem = (size_t)baas::chunk_smem_bytes(xs_bytes, rhs_bytes, cap, mw);
    w.nrec = mw;
    *out = &(s->wins[key] = w);
    return BAAS_OK;
}

baas::ChunkPlan chunk_plan(const baas_schedule *s, const WinCfg &w) {
    baas::ChunkPlan p;
    p.P = s->P;
    for (int d = 0; d < 2; d++) {
        const ChunkDevDir &D = s->d_chk.dir[d];
        p.dir[d] = baas::ChunkDir{D.ints, D.vsrcT, D.vsrcA, D.cval, w.rec[d], w.swptr[d]};
    }
    p.soff = s->d_chk.soff;
    p.srow = s->d_chk.srow;
    p.xs_bytes = w.xs_bytes;
    p.rhs_bytes = w.rhs_bytes;
    p.cap = w.cap;
    p.nrec = w.nrec;
    return p;
}

// Device view of the fetch-walk plan for values of `vbytes` bytes, for an ICCG launch (both
// directions resident) or a standalone sweep.
baas::FetchPlan fetch_plan(const baas_schedule *s, int vbytes, bool iccg) {
    const FetchHost &F = s->fch;
    baas::FetchPlan p{};
    p.P = s->P;
    for (int d = 0; d < 2; d++) {
        const FetchDevDir &D = s->d_fch.dir[d];
        p.dir[d] = baas::FetchDir{D.ints, D.cblk, D.code, D.codeT, D.cfetch, D.frow};
    }
    p.soff = s->d_chk.soff;
    p.srow = s->d_chk.srow;
    p.nslot = F.nslot_max;
    p.srow_bytes = (F.nslot_max * 4 + 15) / 16 * 16;  // the row list and both fetch lists
    p.ints_bytes[0] = 16 * (iccg ? F.dir[0].ints_max : std::max(F.dir[0].ints_max, F.dir[1].ints_max));
    p.ints_bytes[1] = iccg ? 16 * F.dir[1].ints_max : 0;
    const int rb = vbytes == 8 ? 8 * baas::kFetchVal64 : 4 * baas::kFetchVal32;
    // ICCG: FP64 one direction, FP32 both; at least the FP64 layout of one direction, which the
    // fetch-walk IC0 reads its A values in
    p.vals_bytes = iccg ? std::max(rb * F.rows_max * (vbytes == 4 ? 2 : 1), 8 * baas::kFetchVal64 * F.rows_max)
                        : rb * F.rows_max;
    p.ncomp = F.ncomp;
    return p;
}

constexpr int kMaxSmemBudget = 224 * 1024;
// dynamic shared memory a kernel may request: B200's 227 KB per block less room for the
// kernels' static shared memory
constexpr int kMaxDynSmem = 227 * 1024 - 2048;

// Builds every plan of the partition choose_partition picked. When AUTO picked grid boxes but
// the fetch walk cannot run them (a step too wide, or the ICCG plan too large for shared memory),
// the plans are rebuilt on RANGES, where the chunked walk is faster than on boxes.
void build_plans(baas_schedule *s, int P, int num_sms) {
    for (int pass = 0; pass < 2; pass++) {
        build_partition(s, P);
        build_dir(s, false, s->fwd);
        build_dir(s, true, s->bwd);
        build_chunks(s);
        build_fetch(s);
        const bool fits = s->fch.ok && fetch_smem(s->fch, 8, s->hs.kind != baas::SchedKind::SpTRSV) <= (size_t)kMaxDynSmem;
        if (!s->use_boxes || s->opt.partition != BAAS_PARTITION_AUTO || fits) return;
        s->use_boxes = false;
        P = s->opt.parts > 0 ? std::min(s->opt.parts, s->hs.n) : std::max(1, std::min((s->hs.n + 2047) / 2048, num_sms));
    }
}

// Most group levels for which AUTO takes the level walk: one grid barrier (~2 us) per level and
// direction then costs less than the chunked walk's per-row waits between CTAs on such wide,
// unstructured levels.
constexpr int kLevelWalkMaxLevels = 64;

// The walk of a launch (values of vbytes bytes; ICCG, or a standalone sweep of one right-hand
// side): FETCH where the fetch plan qualifies and fits shared memory, else LEVELS for shallow
// group DAGs, else CHUNKED. An explicitly requested walk that cannot run is an error.
// Dynamic shared memory the single-CTA walk may use: 227 KB less its static level offsets.
constexpr size_t kSmallMaxDyn = 227 * 1024 - 2 * baas::kSmallLevShared * sizeof(int) - 2048;
// Automatic choice of the single-CTA walk: row DAGs of at most this many levels per direction.
constexpr int kSmallAutoLevels = 64;

// The single-CTA walk's host plan (small.cuh): row levels from the analysed lower pattern, U's
// pattern by a transpose that keeps each entry's L position, and the IC0 column-match pairs.
void build_small(baas_schedule *s) {
    SmallHost &m = s->sm;
    if (m.built) return;
    const baas::HostSchedule &h = s->hs;
    const int n = h.n;
    const std::vector<int> &lp = h.l_rowptr, &lc = h.l_colidx;
    const bool full = h.kind != baas::SchedKind::SpTRSV;
    // U = L^T: row c holds its diagonal first, then the rows k > c whose L row has column c
    std::vector<int> urp(n + 1, 0), ucol(lc.size()), upos(lc.size());
    for (int c : lc) urp[c + 1]++;
    for (int i = 0; i < n; i++) urp[i + 1] += urp[i];
    std::vector<int> cur(urp.begin(), urp.end() - 1);
    for (int k = 0; k < n; k++)
        for (int e = lp[k]; e < lp[k + 1]; e++) {
            const int c = lc[e];
            ucol[cur[c]] = k;
            upos[cur[c]++] = e;
        }
    // row levels: forward over L's off-diagonal columns, backward over U's
    std::vector<int> lv[2] = {std::vector<int>(n), std::vector<int>(n)};
    for (int i = 0; i < n; i++) {
        int v = 0;
        for (int e = lp[i]; e < lp[i + 1] - 1; e++) v = std::max(v, lv[0][lc[e]]);
        lv[0][i] = v + 1;
    }
    for (int i = n - 1; i >= 0; i--) {
        int v = 0;
        for (int e = urp[i] + 1; e < urp[i + 1]; e++) v = std::max(v, lv[1][ucol[e]]);
        lv[1][i] = v + 1;
    }
    for (int d = 0; d < 2; d++) {
        int nl = 0;
        for (int i = 0; i < n; i++) nl = std::max(nl, lv[d][i]);
        m.nlev[d] = nl;
        m.lev[d].assign(nl + 1, 0);
        for (int i = 0; i < n; i++) m.lev[d][lv[d][i]]++;
        for (int l = 0; l < nl; l++) m.lev[d][l + 1] += m.lev[d][l];
        std::vector<int> at(m.lev[d].begin(), m.lev[d].end() - 1);
        m.rec_t[d].assign(n, int4{0, 0, 0, 0});
        if (full) m.rec_a[d].assign(n, int4{0, 0, 0, 0});
        for (int i = 0; i < n; i++) {  // rows ascending inside each level
            const int q = at[lv[d][i] - 1]++;
            if (d == 0) {
                m.rec_t[0][q] = int4{i, lp[i], lp[i + 1] - 1 - lp[i], lp[i + 1] - 1};
                if (full) m.rec_a[0][q] = int4{i, h.a_rowptr[i], h.a_diagptr[i] - h.a_rowptr[i], h.a_diagptr[i]};
            } else {
                m.rec_t[1][q] = int4{i, urp[i] + 1, urp[i + 1] - urp[i] - 1, urp[i]};
                if (full) m.rec_a[1][q] = int4{i, urp[i] - i, urp[i + 1] - urp[i] - 1, h.a_diagptr[i]};
            }
        }
    }
    if (full) {
        for (int i = 0; i < n; i++)
            for (int e = urp[i] + 1; e < urp[i + 1]; e++) {
                m.ub_col.push_back(ucol[e]);
                m.ub_pos.push_back(h.l_src[upos[e]]);
            }
        // IC0: for lower entry k of row i (column j), the positions in rows i and j of the columns
        // both hold below j, ascending (sparse_dot's merge, merge/IC.cpp:6-29)
        const std::vector<int> &rp = h.a_rowptr, &ci = h.a_colidx, &dg = h.a_diagptr;
        m.ic_ptr.assign(rp[n] + 1, 0);
        for (int i = 0; i < n; i++)
            for (int k = rp[i]; k < dg[i]; k++) {
                const int j = ci[k];
                int a = rp[i], b = rp[j];
                while (a < dg[i] && b < dg[j]) {
                    if (ci[a] == ci[b]) {
                        m.ic_pair.push_back(int2{a, b});
                        a++;
                        b++;
                    } else if (ci[a] < ci[b]) {
                        a++;
                    } else {
                        b++;
                    }
                }
                m.ic_ptr[k + 1] = (int)m.ic_pair.size();
            }
        for (int k = 0; k < rp[n]; k++) m.ic_ptr[k + 1] = std::max(m.ic_ptr[k + 1], m.ic_ptr[k]);
    }
    m.built = true;
}

baas_status upload_small(baas_schedule *s, bool full) {
    build_small(s);
    const SmallHost &m = s->sm;
    for (int d = 0; d < 2; d++) {
        if (!s->d_sm_lev[d]) BAAS_TRY(upload(s->d_sm_lev[d], m.lev[d]));
        if (!s->d_sm_rec_t[d]) BAAS_TRY(upload(s->d_sm_rec_t[d], m.rec_t[d]));
        if (full && !s->d_sm_rec_a[d]) BAAS_TRY(upload(s->d_sm_rec_a[d], m.rec_a[d]));
    }
    if (full && !s->d_sm_ic_ptr) {
        BAAS_TRY(upload(s->d_sm_ic_ptr, m.ic_ptr));
        BAAS_TRY(upload(s->d_sm_ic_pair, m.ic_pair));
        BAAS_TRY(upload(s->d_sm_ub_col, m.ub_col));
        BAAS_TRY(upload(s->d_sm_ub_pos, m.ub_pos));
        BAAS_TRY(dalloc(s->d_sm_ut, std::max<size_t>(m.ub_col.size(), 1)));
        BAAS_TRY(dalloc(s->d_sm_ut32, std::max<size_t>(m.ub_col.size(), 1)));
        BAAS_TRY(dalloc(s->d_sm_lf32, (size_t)s->nnz_a));
        BAAS_TRY(dalloc(s->d_sm_rcp32, (size_t)s->hs.n));
    }
    return BAAS_OK;
}

baas::SmallArgs small_args(const baas_schedule *s, bool full) {
    baas::SmallArgs a{};
    a.n = s->hs.n;
    a.nnz_a = s->nnz_a;
    a.nnz_t = s->nnz_l;
    a.npair = (int)s->sm.ic_pair.size();
    for (int d = 0; d < 2; d++)
        a.dir[d] = baas::SmallDir{s->sm.nlev[d], s->d_sm_lev[d], full ? s->d_sm_rec_a[d] : s->d_sm_rec_t[d]};
    a.st = s->d_status;
    if (full) {
        a.a_diag = s->d_a_diag;
        a.ic_ptr = s->d_sm_ic_ptr;
        a.ic_pair = s->d_sm_ic_pair;
        a.ub_col = s->d_sm_ub_col;
        a.ub_pos = s->d_sm_ub_pos;
        a.nub = (int)s->sm.ub_col.size();
        a.ut = s->d_sm_ut;
        a.lf32 = s->d_sm_lf32;
        a.ut32 = s->d_sm_ut32;
        a.rcp32 = s->d_sm_rcp32;
    }
    return a;
}

// The single-CTA walk runs as a cluster of kSmallCluster CTAs (each holding a full copy of the
// solution) from kSmallClusterMinRows rows up, of 16 CTAs from kSmallCluster16MinRows rows up (k-NN
// n = 12,000 ICCG: 8 CTAs 2.58 ms, 16 CTAs 2.23 ms); below it, as one CTA.
constexpr int kSmallCluster = 8;
constexpr int kSmallClusterMinRows = 2048;

// 16-CTA clusters (non-portable) from this many rows up, where the device can hold one
constexpr int kSmallCluster16MinRows = 8192;

int small_cs(const baas_schedule *s) {
    if (s->opt.small_cluster > 0) return s->opt.small_cluster;
    if (s->hs.n >= kSmallCluster16MinRows) return 16;
    return s->hs.n >= kSmallClusterMinRows ? kSmallCluster : 1;
}
static_assert(baas::kIcScratch <= kSmallMaxDyn, "the IC0 scratch must fit the walk's dynamic shared memory");

// The single-CTA walk's kernels for a cluster size (1, 2, 4 or 8).
template <int CS>
const void *small_kernel_cs(int which, bool flag) {
    switch (which) {
        case 0: return flag ? (const void *)baas::k_sweep_small<true, CS> : (const void *)baas::k_sweep_small<false, CS>;
        case 1: return flag ? (const void *)baas::k_iccg_small<float, CS> : (const void *)baas::k_iccg_small<double, CS>;
        default: return (const void *)baas::k_ic0_small<CS>;
    }
}
// which: 0 sweep (flag = upper), 1 ICCG (flag = FP32 factors), 2 IC0
const void *small_kernel(int cs, int which, bool flag) {
    switch (cs) {
        case 1: return small_kernel_cs<1>(which, flag);
        case 2: return small_kernel_cs<2>(which, flag);
        case 4: return small_kernel_cs<4>(which, flag);
        case 16: return small_kernel_cs<16>(which, flag);
        default: return small_kernel_cs<8>(which, flag);
    }
}

// One launch of a single-CTA walk kernel (small_kernel's `which` / `flag`) with `dyn` bytes of
// dynamic shared memory: one CTA (cs = 1), or one cluster of cs CTAs. A cluster size the device
// cannot hold is refused when the caller asked for it, and halved when it was the automatic choice.
baas_status launch_small(const baas_schedule *s, int which, bool flag, size_t dyn, void **args, cudaStream_t stream) {
    int cs = small_cs(s);
    const bool forced = s->opt.small_cluster > 0;
    for (;;) {
        const void *kern = small_kernel(cs, which, flag);
        if (dyn > 0) BAAS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
        if (cs > 8) BAAS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(cs);
        cfg.blockDim = dim3(baas::kSmallBlock);
        cfg.dynamicSmemBytes = dyn;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cs;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = cs > 1 ? 1 : 0;
        if (cs > 1) {
            int nclusters = 0;
            const cudaError_t e = cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg);
            if (e != cudaSuccess || nclusters < 1) {
                cudaGetLastError();
                if (forced) return fail(BAAS_ERR_CUDA, "this device cannot hold a cluster of " + std::to_string(cs) + " CTAs");
                cs /= 2;
                continue;
            }
        }
        BAAS_CUDA(cudaLaunchKernelExC(&cfg, kern, args));
        return BAAS_OK;
    }
}


baas_status pick_walk(baas_schedule *s, int vbytes, bool iccg, int &walk) {
    const bool fits = s->fch.ok && fetch_smem(s->fch, vbytes, iccg) <= (size_t)kMaxDynSmem;
    const int nlev = (int)s->hs.exec_level_ptr.size() - 1;
    // the single-CTA walk keeps the sweep's solution (and ICCG's p, FP64) in shared memory
    const size_t small_row = iccg ? 8 + (size_t)vbytes : 8;
    const bool small_fits = (size_t)s->hs.n * small_row <= kSmallMaxDyn;
    switch (s->opt.walk) {
        case BAAS_WALK_SMALL:
            if (!small_fits)
                return fail(BAAS_ERR_BAD_ARG, "the single-CTA walk holds at most " + std::to_string(kSmallMaxDyn / small_row) +
                                                  " rows here");
            walk = BAAS_WALK_SMALL;
            return BAAS_OK;
        case BAAS_WALK_FETCH:
            if (!fits)
                return fail(BAAS_ERR_BAD_ARG, "the fetch walk needs rows of at most 3 off-diagonal entries, steps of at most " +
                                                  std::to_string(baas::kFetchMaxRows) + " rows and a plan that fits shared memory");
            walk = BAAS_WALK_FETCH;
            break;
        case BAAS_WALK_CHUNKED: walk = BAAS_WALK_CHUNKED; break;
        case BAAS_WALK_LEVELS: walk = BAAS_WALK_LEVELS; break;
        default:
            if (fits) {
                walk = BAAS_WALK_FETCH;
            } else if (small_fits && (build_small(s), std::max(s->sm.nlev[0], s->sm.nlev[1]) <= kSmallAutoLevels)) {
                walk = BAAS_WALK_SMALL;
            } else {
                walk = nlev <= kLevelWalkMaxLevels ? BAAS_WALK_LEVELS : BAAS_WALK_CHUNKED;
            }
    }
    return BAAS_OK;
}

// The launched variants. ieee: sweep divisions by __ddiv_rn, for the repeat of a launch whose
// div_fast divisions left their range (DevStatus::slow_div); FP32 factors never divide.
void *sweep_kernel(bool mr, bool stg, bool ieee) {
    if (ieee)
        return mr ? (stg ? (void *)baas::k_sweep_chunked<true, true, true> : (void *)baas::k_sweep_chunked<true, false, true>)
                  : (stg ? (void *)baas::k_sweep_chunked<false, true, true> : (void *)baas::k_sweep_chunked<false, false, true>);
    return mr ? (stg ? (void *)baas::k_sweep_chunked<true, true, false> : (void *)baas::k_sweep_chunked<true, false, false>)
              : (stg ? (void *)baas::k_sweep_chunked<false, true, false> : (void *)baas::k_sweep_chunked<false, false, false>);
}
// walk: BAAS_WALK_CHUNKED, BAAS_WALK_FETCH or BAAS_WALK_LEVELS (the level walk divides with
// __ddiv_rn and never needs the IEEE repeat).
void *iccg_kernel(bool mixed, bool stg, bool ieee, int walk = BAAS_WALK_CHUNKED) {
    using baas::k_iccg_chunked;
    constexpr int C = baas::kWalkChunked, F = baas::kWalkFetch, L = baas::kWalkLevels;
    if (walk == BAAS_WALK_LEVELS)
        return mixed ? (void *)k_iccg_chunked<float, false, false, L> : (void *)k_iccg_chunked<double, false, false, L>;
    if (walk == BAAS_WALK_FETCH) {
        if (mixed) return (void *)k_iccg_chunked<float, false, false, F>;
        return ieee ? (void *)k_iccg_chunked<double, false, true, F> : (void *)k_iccg_chunked<double, false, false, F>;
    }
    if (mixed) return stg ? (void *)k_iccg_chunked<float, true, false, C> : (void *)k_iccg_chunked<float, false, false, C>;
    if (ieee) return stg ? (void *)k_iccg_chunked<double, true, true, C> : (void *)k_iccg_chunked<double, false, true, C>;
    return stg ? (void *)k_iccg_chunked<double, true, false, C> : (void *)k_iccg_chunked<double, false, false, C>;
}
void *sweep_fetch_kernel(bool ieee) {
    return ieee ? (void *)baas::k_sweep_fetch<true> : (void *)baas::k_sweep_fetch<false>;
}
// rw: FP32 factors with exactly 2 or 4 right-hand sides take the row-wide sweeps (one thread per
// row for all of them; rw = that count, else 1); BAAS_BATCH_PAIRS=1 keeps the
// one-pair-per-thread sweeps (same results).
void *batched_kernel(bool mixed, bool mr, bool ieee, int rw = 1) {
    if (mixed && mr && rw == 4) return (void *)baas::k_iccg_batched<float, true, false, 4>;
    if (mixed && mr && rw == 2) return (void *)baas::k_iccg_batched<float, true, false, 2>;
    if (mixed) return mr ? (void *)baas::k_iccg_batched<float, true, false, 1> : (void *)baas::k_iccg_batched<float, false, false, 1>;
    if (ieee) return mr ? (void *)baas::k_iccg_batched<double, true, true, 1> : (void *)baas::k_iccg_batched<double, false, true, 1>;
    return mr ? (void *)baas::k_iccg_batched<double, true, false, 1> : (void *)baas::k_iccg_batched<double, false, false, 1>;
}

// Keeps `count` doubles from src (device) for a repeat of the launch.
baas_status save_x0(baas_schedule *s, const double *src, size_t count, cudaStream_t stream) {
    if (count > s->x0_cap) {
        if (s->d_x0) cudaFree(s->d_x0);
        s->d_x0 = nullptr;
        s->x0_cap = 0;
        BAAS_CUDA(cudaMalloc((void **)&s->d_x0, count * sizeof(double)));
        s->x0_cap = count;
    }
    BAAS_CUDA(cudaMemcpyAsync(s->d_x0, src, count * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    return BAAS_OK;
}

// After read_status: the launch ran without a device error but some div_fast division left its
// range, so it must be repeated with the IEEE variant.
bool needs_ieee_repeat(const baas_schedule *s) { return s->h_status->code == 0 && s->h_status->slow_div != 0; }

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
    s->smem_budget = s->opt.smem_budget > 0 ? std::min(s->opt.smem_budget, kMaxSmemBudget) : (int)kSmemBudget;

    // partition size: BAAS_THREADS: the schedule's threads; else `parts`, or about one CTA per
    // 2,048 rows (at most one per SM)
    const int n = s->hs.n;
    if (s->opt.partition == BAAS_PARTITION_BAAS_THREADS && s->opt.parts > 0 && s->opt.parts != s->hs.nthread)
        return fail(BAAS_ERR_BAD_ARG, "BAAS_THREADS partition needs parts == nthread");
    const int P = choose_partition(s, s->num_sms);
    if (P > s->num_sms) return fail(BAAS_ERR_BAD_ARG, "the partition needs more CTAs than the device has SMs");
    build_plans(s, P, s->num_sms);

    BAAS_TRY(upload_part(s->d_fwd, s->fwd));
    BAAS_TRY(upload_part(s->d_bwd, s->bwd));
    BAAS_TRY(upload_chunks(s->d_chk, s->chk));
    if (s->fch.ok) BAAS_TRY(upload_fetch(s->d_fch, s->fch));
    BAAS_TRY(upload(s->d_a_diag, s->hs.a_diagptr));
    BAAS_TRY(dalloc(s->d_status, 1));
    BAAS_TRY(dalloc(s->d_flags, (size_t)n));
    BAAS_TRY(dalloc(s->d_bar, 1));
    BAAS_CUDA(cudaMallocHost((void **)&s->h_status, sizeof(DevStatus)));
    if (getenv("BAAS_TRACE") && atoi(getenv("BAAS_TRACE")) > 0) BAAS_TRY(dalloc(s->d_trace, 2 * baas::kTraceSlots));
    {
        for (int v = 0; v < 8; v++) {
            const bool a = v & 1, b = v & 2, c = v & 4;
            const void *kerns[] = {sweep_kernel(a, b, c), iccg_kernel(a, b, c), batched_kernel(a, b, c),
                                   batched_kernel(true, true, false, 4), batched_kernel(true, true, false, 2)};
            for (const void *k : kerns)
                BAAS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem));
            const void *fk[] = {iccg_kernel(a, false, b, BAAS_WALK_FETCH), sweep_fetch_kernel(a),
                                iccg_kernel(a, false, b, BAAS_WALK_LEVELS)};
            for (const void *k : fk)
                BAAS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem));
        }
    }
    s->uploaded = true;
    // the single-right-hand-side FP64 windows must exist for every kind of call
    WinCfg *w = nullptr;
    BAAS_TRY(get_windows(s, 8, 1, &w));
    // multi-right-hand-side sweeps: the widest batch that leaves both window buffers >= 8 KiB
    s->rmax64 = 1;
    for (int R = baas::kMaxRhs; R > 1; R--) {
        const long long xs = ((long long)s->chk.slot_max * R * 8 + 127) / 128 * 128;
        if ((s->smem_budget - xs - 32) / 2 < 8 * 1024) continue;
        std::vector<int4> rec[2];
        std::vector<int> swptr[2];
        int xb = 0, rb = 0, cap = 0, mw = 0;
        if (plan_windows(s->chk, s->P, s->smem_budget, s->opt.smem_budget > 0, 8, R, rec, swptr, xb, rb, cap, mw)) {
            s->rmax64 = R;
            break;
        }
    }
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
    if (ds.code == baas::kBounds)
        return fail(BAAS_ERR_CUDA, "a device bounds check failed (site " + std::to_string(ds.where) + ")");
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
static_assert(sizeof(DevStatus) <= kNoAllocStatusInts * sizeof(int), "the status word must fit in front of the row flags");
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
    opt->partition = BAAS_PARTITION_AUTO;
    opt->smem_budget = 0;
    opt->mapping = BAAS_MAPPING_FOUR_RULE;
    opt->walk = BAAS_WALK_AUTO;
    opt->analysis = BAAS_ANALYSIS_HOST;
    opt->ablation = BAAS_ABLATION_NONE;
    opt->small_cluster = 0;
    const baas::ScoreParams sp;
    opt->level_window = sp.level_window;
    opt->amplify = sp.amplify;
    opt->over_gamma = sp.over_gamma;
    opt->award_alpha = sp.award_alpha;
    opt->load_beta = sp.load_beta;
}

const char *baas_last_error_string(void) { return g_err.c_str(); }

}  // extern "C"

// error reporting for the library's other host sources (mtx.cpp)
baas_status baas::set_error(baas_status code, const std::string &msg) { return fail(code, msg); }

// NVTX ranges named after the reference's phase timers (pcg_opt, test/iccg_level_merge.cpp:384-521:
// pre, ic, trsv, ... ) around each entry point, for a profiler's timeline; free without one.
struct PhaseRange {
    explicit PhaseRange(const char *name) { nvtxRangePushA(name); }
    ~PhaseRange() { nvtxRangePop(); }
    PhaseRange(const PhaseRange &) = delete;
    PhaseRange &operator=(const PhaseRange &) = delete;
};

extern "C" {

const char *baas_version(void) { return "baas_b200 0.2.0 (sm_100a)"; }

static baas_status analyze_common(const baas_csr *A, baas_kernel kind, const baas_options *opt, baas_schedule **out,
                                  const std::vector<int> *sys_off);

baas_status baas_analyze(const baas_csr *A, baas_kernel kind, const baas_options *opt, baas_schedule **out) {
    return analyze_common(A, kind, opt, out, nullptr);
}

}  // extern "C"

// sys_off: row offsets of a block-diagonal batch (baas_analyze_batch), or nullptr
static baas_status analyze_common(const baas_csr *A, baas_kernel kind, const baas_options *opt, baas_schedule **out,
                                  const std::vector<int> *sys_off) {
    PhaseRange range("pre");
    if (!A || !out) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    *out = nullptr;
    if (kind < BAAS_KERNEL_SPTRSV || kind > BAAS_KERNEL_ILU0) return fail(BAAS_ERR_BAD_ARG, "unknown kernel kind");
    baas_options o;
    baas_options_default(&o);
    if (opt) o = *opt;
    if (o.nthread < 1) return fail(BAAS_ERR_BAD_ARG, "nthread must be >= 1");
    if (o.partition != BAAS_PARTITION_RANGES && o.partition != BAAS_PARTITION_BAAS_THREADS &&
        o.partition != BAAS_PARTITION_BLOCKS && o.partition != BAAS_PARTITION_AUTO)
        return fail(BAAS_ERR_BAD_ARG, "unknown partition");
    if (o.parts < 0) return fail(BAAS_ERR_BAD_ARG, "parts must be >= 0");
    if (o.smem_budget < 0) return fail(BAAS_ERR_BAD_ARG, "smem_budget must be >= 0");
    if (o.walk < BAAS_WALK_AUTO || o.walk > BAAS_WALK_SMALL) return fail(BAAS_ERR_BAD_ARG, "unknown walk");
    if (o.mapping < BAAS_MAPPING_FOUR_RULE || o.mapping > BAAS_MAPPING_AFFINITY)
        return fail(BAAS_ERR_BAD_ARG, "unknown mapping");
    if (o.analysis != BAAS_ANALYSIS_HOST && o.analysis != BAAS_ANALYSIS_DEVICE)
        return fail(BAAS_ERR_BAD_ARG, "unknown analysis placement");
    if (o.small_cluster != 0 && o.small_cluster != 1 && o.small_cluster != 2 && o.small_cluster != 4 &&
        o.small_cluster != 8 && o.small_cluster != 16)
        return fail(BAAS_ERR_BAD_ARG, "small_cluster must be 0, 1, 2, 4, 8 or 16");
    if (o.level_window < 0 || o.level_window > 1024 || !std::isfinite(o.amplify) || !std::isfinite(o.over_gamma) ||
        !std::isfinite(o.award_alpha) || !std::isfinite(o.load_beta))
        return fail(BAAS_ERR_BAD_ARG, "scoring constants: level_window in [0, 1024] and finite weights");
    if (o.ablation < BAAS_ABLATION_NONE || o.ablation > BAAS_ABLATION_WOAS)
        return fail(BAAS_ERR_BAD_ARG, "unknown ablation");
    if (o.ablation != BAAS_ABLATION_NONE && (kind != BAAS_KERNEL_SPTRSV || o.mapping != BAAS_MAPPING_FOUR_RULE))
        return fail(BAAS_ERR_BAD_ARG, "the ablations are the SpTRSV runtime's (kind BAAS_KERNEL_SPTRSV, mapping FOUR_RULE)");
    if (o.mapping != BAAS_MAPPING_FOUR_RULE && kind != BAAS_KERNEL_ICCG)
        return fail(BAAS_ERR_BAD_ARG, "the P2P, barrier, P2P_TIME and P2P_MAPPING mappings are the Scheduler's (kind BAAS_KERNEL_ICCG)");
    if (!A->rowptr || !A->colidx || A->n <= 0) return fail(BAAS_ERR_BAD_ARG, "empty or NULL pattern");
    if (A->rowptr[A->n] != A->nnz) return fail(BAAS_ERR_BAD_ARG, "nnz != rowptr[n]");
    // value-source codes of the sweep plan address positions below 2^30
    if (A->nnz >= (1 << 30) - 2) return fail(BAAS_ERR_BAD_ARG, "nnz must be below 2^30 - 2");
    const baas::SchedKind sk = (baas::SchedKind)kind;
    const char *why = baas::validate_pattern(A->n, A->rowptr, A->colidx, sk);
    if (why[0]) return fail(BAAS_ERR_BAD_ARG, why);
    baas_schedule *s = new baas_schedule();
    s->opt = o;
    s->nnz_a = A->nnz;
    const bool dev = o.analysis == BAAS_ANALYSIS_DEVICE;
    if (dev) {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
            cudaGetLastError();
            delete s;
            return fail(BAAS_ERR_NO_DEVICE, "BAAS_ANALYSIS_DEVICE needs a CUDA device");
        }
    }
    std::string reason;
    baas::ScoreParams score;
    score.level_window = o.level_window;
    score.amplify = o.amplify;
    score.over_gamma = o.over_gamma;
    score.award_alpha = o.award_alpha;
    score.load_beta = o.load_beta;
    if (!baas::build_schedule(s->hs, A->n, A->rowptr, A->colidx, sk, o.nthread, (baas::Mapping)o.mapping,
                              (baas::Ablation)o.ablation, dev, reason, sys_off, score)) {
        delete s;
        return fail(dev && reason.rfind("device analysis", 0) == 0 ? BAAS_ERR_CUDA : BAAS_ERR_BAD_ARG, reason);
    }
    s->nnz_l = (int)s->hs.l_colidx.size();
    if (sk != baas::SchedKind::SpTRSV && s->nnz_a != 2 * s->nnz_l - A->n) {
        delete s;
        return fail(BAAS_ERR_BAD_ARG, "the pattern must be structurally symmetric");
    }
    build_order(s);
    *out = s;
    return BAAS_OK;
}

extern "C" {

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
        case BAAS_FIELD_GROUP_DAG_PTR: return put(h.fdag_ptr);
        case BAAS_FIELD_GROUP_DAG_SET: return put(h.fdag_set);
        case BAAS_FIELD_COST: {
            std::vector<int> c(h.cost.size());
            for (size_t i = 0; i < c.size(); i++) c[i] = (int)h.cost[i];
            return put(c);
        }
        default: return -1;
    }
}

double baas_schedule_analysis_ms(const baas_schedule *s) { return s ? s->hs.analysis_ms : 0.0; }

int baas_schedule_last_walk(const baas_schedule *s) { return s ? s->last_walk : 0; }

int baas_plan_parts(const baas_schedule *s, int *box) {
    if (!s) return 0;
    if (box)
        for (int t = 0; t < 3; t++) {
            box[t] = s->use_boxes ? s->box[t] : 0;
            box[3 + t] = s->use_boxes ? s->nbox[t] : 0;
        }
    return s->P;
}

baas_status baas_test_inject_unsatisfiable_wait(baas_schedule *s, int row) {
    if (!s || row < 0 || row >= s->hs.n) return fail(BAAS_ERR_BAD_ARG, "bad row");
    const int lb = s->hs.l_rowptr[row], le = s->hs.l_rowptr[row + 1];
    if (le - lb < 2) return fail(BAAS_ERR_BAD_ARG, "the row has no off-diagonal entry");
    if (s->uploaded) return fail(BAAS_ERR_STATE, "inject before the first GPU call on the schedule");
    s->fault_row = row;
    return BAAS_OK;
}

namespace {
__global__ void k_test_divide(const double *a, const double *b, double *q, long long n, int mode) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double x = a[i], d = b[i];
        if (mode == 2) {
            bool slow = false;
            baas::div_fast(x, d, baas::div_recip(d), slow);
            q[i] = slow ? 1.0 : 0.0;
        } else {
            q[i] = mode == 0 ? baas::div_rcp(x, d, baas::div_recip(d)) : __ddiv_rn(x, d);
        }
    }
}
}  // namespace

baas_status baas_test_divide(const double *a, const double *b, double *q, long long n, int mode, void *stream) {
    if (n < 0 || (n > 0 && (!a || !b || !q))) return fail(BAAS_ERR_BAD_ARG, "NULL argument or negative n");
    if (mode < 0 || mode > 2) return fail(BAAS_ERR_BAD_ARG, "mode must be 0, 1 or 2");
    if (n == 0) return BAAS_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const long long blocks = std::min<long long>((n + 255) / 256, 148LL * 16);
    k_test_divide<<<(int)blocks, 256, 0, st>>>(a, b, q, n, mode);
    BAAS_CUDA(cudaGetLastError());
    BAAS_CUDA(cudaStreamSynchronize(st));
    return BAAS_OK;
}

baas_status baas_test_emulate_sweep(baas_schedule *s, int parts, int smem_budget, int upper, const double *tval,
                                    const double *b, double *x) {
    if (!s || !tval || !b || !x) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    if (s->uploaded) return fail(BAAS_ERR_STATE, "the schedule's plan is resident on a GPU");
    const int n = s->hs.n;
    const int saved_parts = s->opt.parts;
    if (parts > 0 && s->opt.partition != BAAS_PARTITION_CUSTOM && s->opt.partition != BAAS_PARTITION_BAAS_THREADS)
        s->opt.parts = parts;
    build_plans(s, choose_partition(s, 148), 148);  // plans as for a 148-SM B200
    s->opt.parts = saved_parts;
    const int P = s->P;
    const int budget = smem_budget > 0 ? std::min(smem_budget, kMaxSmemBudget) : (int)kSmemBudget;
    std::vector<int4> rec[2];
    std::vector<int> swptr[2];
    int xs_bytes = 0, rhs_bytes = 0, cap = 0, mw = 0;
    if (!plan_windows(s->chk, P, budget, smem_budget > 0, 8, 1, rec, swptr, xs_bytes, rhs_bytes, cap, mw))
        return fail(BAAS_ERR_BAD_ARG, "emulate: a chunk does not fit the window buffer");
    if (baas::chunk_smem_bytes(xs_bytes, rhs_bytes, cap, mw) > budget)
        return fail(BAAS_ERR_BAD_ARG, "emulate: shared memory over budget");
    const int d = upper ? 1 : 0;
    const ChunkHostDir &D = s->chk.dir[d];
    const ChunkHost &C = s->chk;
    auto bad = [](const std::string &m) { return fail(BAAS_ERR_BAD_ARG, "emulate: " + m); };
    if (s->fault_row >= 0) return fail(BAAS_ERR_STATE, "emulate: the schedule carries an injected fault");
    // packing of the value slots, as the sweep kernel does
    std::vector<double> gv(D.vsrcT.size());
    for (size_t i = 0; i < gv.size(); i++) {
        const int code = D.vsrcT[i];
        const bool rcp = code < -(1 << 30);
        const int src = code >= 0 ? code : (rcp ? code - baas::kRcpBase : (code <= -2 ? -2 - code : -1));
        if (src >= s->nnz_l) return bad("value source out of range");
        gv[i] = src >= 0 ? (rcp ? 1.0 / tval[src] : tval[src]) : 0.0;
    }
    std::vector<char> ready(n, 0);
    // the column that entry j of row r must read: L rows ascending (diagonal last), U = L^T rows
    // descending (diagonal first)
    const baas::HostSchedule &hs = s->hs;
    auto column = [&](int r, int j) {
        return upper ? s->crow[s->cptr[r + 1] - 1 - j] : hs.l_colidx[hs.l_rowptr[r] + j];
    };
    struct Cta {
        int q = 0, qend = 0;
        std::vector<int> ibuf;
        std::vector<double> vbuf;
        size_t ip = 0, vp = 0;
        bool loaded = false, done = false;
        int expect_nl = -1;  // the row count the previous chunk announced for this one
    };
    std::vector<Cta> cta(P);
    std::vector<std::vector<double>> xs(P, std::vector<double>((size_t)std::max(C.slot_max, 1), 0.0));
    std::vector<std::vector<int>> owner(P, std::vector<int>((size_t)std::max(C.slot_max, 1), -1));
    for (int c = 0; c < P; c++) {
        Cta &K = cta[c];
        K.q = swptr[d][c];
        K.qend = swptr[d][c + 1];
        K.done = K.q == K.qend;
    }
    int remaining = P;
    for (int c = 0; c < P; c++) remaining -= cta[c].done ? 1 : 0;
    while (remaining > 0) {
        bool progress = false;
        for (int c = 0; c < P; c++) {
            Cta &K = cta[c];
            if (K.done) continue;
            if (!K.loaded) {
                const int4 r = rec[d][K.q];
                if (r.x % 8 || r.y % 8 || r.z % 4 || r.w % 4) return bad("window block misaligned");
                if ((long long)r.y * 4 + (long long)r.w * 8 > cap) return bad("window larger than its buffer");
                if (r.x < 0 || r.x + r.y > (int)D.ints.size() || r.z < 0 || r.z + r.w > (int)gv.size())
                    return bad("window outside the plan arrays");
                K.ibuf.assign(D.ints.begin() + r.x, D.ints.begin() + r.x + r.y);
                K.vbuf.assign(gv.begin() + r.z, gv.begin() + r.z + r.w);
                K.ip = K.vp = 0;
                K.loaded = true;
            }
            const int *I = K.ibuf.data() + K.ip;
            const int nl = I[0], E = I[1];
            if (nl < 1 || E < 1) return bad("bad chunk header");
            if (K.expect_nl >= 0 && K.expect_nl != nl) return bad("a chunk header announces the wrong next row count");
            if (K.ip + baas::chunk_nint(nl, E) > K.ibuf.size() || K.vp + baas::chunk_nval(nl, E) > K.vbuf.size())
                return bad("chunk runs past its window");
            const int *rowid = I + baas::kChunkHdr, *slot = rowid + nl, *ne = slot + nl, *kp = ne + nl, *dep = kp + nl;
            const double *V = K.vbuf.data() + K.vp;
            const double *diag = V, *rcp = V + nl, *val = V + 2 * nl;
            const int ns = C.slot_max;
            bool wait = false;
            for (int pos = 0; pos < nl && !wait; pos++) {
                if (ne[pos] < 0 || ne[pos] > E) return bad("row entry count exceeds the chunk stride");
                for (int j = 0; j < ne[pos]; j++) {
                    const int dd = dep[pos * E + j];
                    if (dd < 0) {
                        const int r = -dd - 1;
                        if (r >= n) return bad("remote dependency out of range");
                        if (!ready[r]) wait = true;
                    }
                }
            }
            if (wait) continue;
            // all reads of the step happen before any of its writes (the barrier semantics)
            std::vector<double> outs(nl);
            for (int pos = 0; pos < nl; pos++) {
                const int row = rowid[pos];
                if (row < 0 || row >= n || ready[row]) return bad("row out of range or computed twice");
                if (kp[pos] < 0 || kp[pos] >= C.soff[c + 1] - C.soff[c] || C.srow[C.soff[c] + kp[pos]] != row)
                    return bad("a row's staging position does not name it");
                double sum = 0.0;
                for (int j = 0; j < ne[pos]; j++) {
                    const int dd = dep[pos * E + j];
                    const int col = column(row, j);
                    double xv;
                    if (dd >= 0) {
                        if (dd >= ns) return bad("slot out of range");
                        if (owner[c][dd] != col) return bad("a slot does not hold the column the row needs");
                        xv = xs[c][dd];
                    } else {
                        if (-dd - 1 != col) return bad("a remote dependency names the wrong column");
                        xv = x[-dd - 1];
                    }
                    sum = sum + xv * val[pos * E + j];
                }
                if (rcp[pos] != 1.0 / diag[pos]) return bad("a row's reciprocal slot does not match its diagonal");
                outs[pos] = (b[row] - sum) / diag[pos];
            }
            for (int pos = 0; pos < nl; pos++) {
                const int sl = slot[pos], row = rowid[pos];
                if (sl >= ns) return bad("slot out of range");
                if (sl >= 0) {
                    xs[c][sl] = outs[pos];
                    owner[c][sl] = row;
                }
                x[row] = outs[pos];
                ready[row] = 1;
            }
            K.expect_nl = I[2];
            K.ip += baas::chunk_nint(nl, E);
            K.vp += baas::chunk_nval(nl, E);
            if (K.ip == K.ibuf.size()) {
                K.loaded = false;
                if (++K.q == K.qend) {
                    if (K.expect_nl != 0) return bad("the last chunk announces a successor");
                    K.done = true;
                    remaining--;
                }
            }
            progress = true;
        }
        if (!progress) return bad("no CTA can make progress (the plan would deadlock)");
    }
    for (int i = 0; i < n; i++)
        if (!ready[i]) return bad("a row was never computed");
    return BAAS_OK;
}

baas_status baas_test_emulate_fetch(baas_schedule *s, int parts, int upper, const double *tval, const double *b,
                                    double *x) {
    if (!s || !tval || !b || !x) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    if (s->uploaded) return fail(BAAS_ERR_STATE, "the schedule's plan is resident on a GPU");
    if (s->fault_row >= 0) return fail(BAAS_ERR_STATE, "emulate: the schedule carries an injected fault");
    const int n = s->hs.n;
    const int saved_parts = s->opt.parts;
    if (parts > 0 && s->opt.partition != BAAS_PARTITION_CUSTOM && s->opt.partition != BAAS_PARTITION_BAAS_THREADS)
        s->opt.parts = parts;
    build_plans(s, choose_partition(s, 148), 148);  // plans as for a 148-SM B200
    s->opt.parts = saved_parts;
    const int P = s->P;
    auto bad = [](const std::string &m) { return fail(BAAS_ERR_BAD_ARG, "emulate fetch: " + m); };
    const FetchHost &F = s->fch;
    if (!F.ok) return bad("the plan does not qualify for the fetch walk");
    if (fetch_smem(F, 8, false) > (size_t)kMaxDynSmem) return bad("the sweep plan does not fit shared memory");
    const int d = upper ? 1 : 0;
    const FetchHostDir &D = F.dir[d];
    const ChunkHost &C = s->chk;
    const baas::HostSchedule &hs = s->hs;
    // column of entry j of row r in the reference's order, and the caller's value position
    auto column = [&](int r, int j) { return upper ? s->crow[s->cptr[r + 1] - 1 - j] : hs.l_colidx[hs.l_rowptr[r] + j]; };
    // the caller's upper factor is U = L^T in CSR, i.e. L's columns: positions index crow
    auto tpos = [&](int r, int j) { return upper ? s->cptr[r + 1] - 1 - j : hs.l_rowptr[r] + j; };
    auto nent = [&](int r) { return upper ? s->cptr[r + 1] - s->cptr[r] - 1 : hs.l_rowptr[r + 1] - hs.l_rowptr[r] - 1; };
    auto dpos = [&](int r) { return upper ? s->cptr[r] : hs.l_rowptr[r + 1] - 1; };
    if ((int)D.cblk.size() != P + 1 || (int)D.cfetch.size() != P + 1 || (int)D.code.size() != 4 * n) return bad("table sizes");
    std::vector<char> ready(n, 0);
    struct Cta {
        int step = 0, ns = 0, i0 = 0, nrows = 0, nf0 = 0;
        std::vector<double> slot;
        std::vector<int> owner;  // row whose value a slot holds (-1: none yet)
    };
    std::vector<Cta> cta(P);
    for (int c = 0; c < P; c++) {
        Cta &K = cta[c];
        const int4 cb = D.cblk[c];
        K.ns = cb.z;
        K.i0 = cb.x;
        K.nrows = C.soff[c + 1] - C.soff[c];
        K.nf0 = F.dir[0].cfetch[c + 1] - F.dir[0].cfetch[c];
        const int nf = D.cfetch[c + 1] - D.cfetch[c];
        if (cb.w != C.soff[c]) return bad("a CTA's first record is not its first row");
        if (cb.y != K.ns + 2 + K.nrows || cb.x + cb.y > (int)D.ints.size()) return bad("int block size");
        if (16 * cb.y > 16 * D.ints_max) return bad("int block larger than its shared region");
        if (K.nrows + 1 + K.nf0 + (d ? nf : 0) > F.nslot_max) return bad("slots beyond the shared slot region");
        K.slot.assign((size_t)F.nslot_max, 0.0);
        K.owner.assign((size_t)F.nslot_max, -1);
        for (int k = 0; k < K.nrows; k++) {
            K.slot[k] = b[C.srow[C.soff[c] + k]];
            K.owner[k] = -2;  // staged right-hand side
        }
        K.slot[K.nrows] = -0.0;
    }
    int remaining = 0;
    for (int c = 0; c < P; c++) remaining += cta[c].ns > 0;
    while (remaining > 0) {
        bool progress = false;
        for (int c = 0; c < P; c++) {
            Cta &K = cta[c];
            if (K.step >= K.ns) continue;
            const int4 st = D.ints[K.i0 + K.step];
            const int nl = st.y, rb = K.i0 + K.ns + 2;
            if (nl < 1 || nl > F.ncomp) return bad("step row count out of range");
            if (st.x < 0 || st.x + nl > K.nrows) return bad("step records out of range");
            const int fb = D.cfetch[c], sbase = K.nrows + 1 + (d ? K.nf0 : 0), nf = D.cfetch[c + 1] - fb;
            // a step runs once every staged value it reads has been written by its producer
            bool wait = false;
            for (int q = 0; q < nl && !wait; q++) {
                const int4 r = D.ints[rb + st.x + q];
                const int sl[3] = {r.y, r.z, r.w};
                for (int j = 0; j < 3; j++)
                    if (sl[j] >= sbase) {
                        if (sl[j] >= sbase + nf) return bad("staging slot beyond the fetch list");
                        if (!ready[D.frow[fb + sl[j] - sbase]]) wait = true;
                    }
            }
            if (wait) continue;
            std::vector<double> outs(nl);
            for (int q = 0; q < nl; q++) {
                const int4 r = D.ints[rb + st.x + q];
                if (r.x < 0 || r.x >= K.nrows) return bad("own slot out of range");
                const int row = C.srow[C.soff[c] + r.x];
                if (ready[row]) return bad("a row computed twice");
                const int ne = nent(row);
                const int *code = D.codeT.data() + 4 * (size_t)(C.soff[c] + st.x + q);
                if (code[0] != dpos(row)) return bad("diagonal code does not name the row's diagonal");
                const int sl[3] = {r.y, r.z, r.w};
                double sum = 0.0;
                for (int j = 0; j < 3; j++) {
                    if (j >= ne) {
                        if (sl[j] != K.nrows || code[j + 1] != -1) return bad("an absent entry does not read the zero slot");
                        continue;
                    }
                    const int col = column(row, j);
                    if (code[j + 1] != tpos(row, j)) return bad("entry code does not name the entry");
                    double xv;
                    if (sl[j] < K.nrows) {
                        if (K.owner[sl[j]] != col) return bad("a local slot does not hold the column the row needs");
                        xv = K.slot[sl[j]];
                    } else if (sl[j] >= sbase) {
                        if (D.frow[fb + sl[j] - sbase] != col) return bad("a staging slot names the wrong row");
                        xv = x[col];
                    } else {
                        return bad("a slot between the zero slot and this direction's staging");
                    }
                    sum = sum + xv * tval[code[j + 1]];
                }
                outs[q] = (K.slot[r.x] - sum) / tval[code[0]];
            }
            for (int q = 0; q < nl; q++) {
                const int4 r = D.ints[rb + st.x + q];
                const int row = C.srow[C.soff[c] + r.x];
                K.slot[r.x] = outs[q];
                K.owner[r.x] = row;
                x[row] = outs[q];
                ready[row] = 1;
            }
            if (++K.step == K.ns) {
                remaining--;
                const int4 t0 = D.ints[K.i0 + K.ns], t1 = D.ints[K.i0 + K.ns + 1], tl = D.ints[K.i0 + K.ns - 1];
                if (t0.x != tl.x || t0.y != tl.y || t1.x != tl.x || t1.y != tl.y) return bad("terminal step copies");
            }
            progress = true;
        }
        if (!progress) return bad("no CTA can make progress (the plan would deadlock)");
    }
    for (int i = 0; i < n; i++)
        if (!ready[i]) return bad("a row was never computed");
    return BAAS_OK;
}

// Frees the schedule's device state (plan, workspaces) on its device and returns the schedule to
// its state right after analysis; the host schedule and the batch offsets stay.
static void release_device(baas_schedule *s) {
    if (s->uploaded) {
        int cur = -1;
        cudaGetDevice(&cur);
        if (cur != s->device) cudaSetDevice(s->device);
        s->d_fwd.release();
        s->d_bwd.release();
        s->d_chk.release();
        s->d_fch.release();
        for (auto &kv : s->wins) kv.second.release();
        for (int d = 0; d < 2; d++) {
            if (s->d_gf64[d]) cudaFree(s->d_gf64[d]);
            if (s->d_gf32[d]) cudaFree(s->d_gf32[d]);
            if (s->d_gfT[d]) cudaFree(s->d_gfT[d]);
        }
        if (s->d_dg) cudaFree(s->d_dg);
        for (int d = 0; d < 2; d++) {
            s->d_lv[d].release();
            void *lp[] = {s->d_lv64[d], s->d_ld64[d], s->d_lv32[d], s->d_ld32[d], s->d_lvT[d], s->d_ldT[d]};
            for (void *p : lp)
                if (p) cudaFree(p);
        }
        for (int d = 0; d < 2; d++) {
            if (s->d_gv64[d]) cudaFree(s->d_gv64[d]);
            if (s->d_gv32[d]) cudaFree(s->d_gv32[d]);
            if (s->d_gvT[d]) cudaFree(s->d_gvT[d]);
            void *sp[] = {s->d_sm_lev[d], s->d_sm_rec_t[d], s->d_sm_rec_a[d]};
            for (void *p : sp)
                if (p) cudaFree(p);
        }
        void *smp[] = {s->d_sm_ic_ptr, s->d_sm_ub_col, s->d_sm_ub_pos, s->d_sm_ic_pair, s->d_sm_ut, s->d_sm_lf32,
                       s->d_sm_ut32, s->d_sm_rcp32, s->d_ilu_rec, s->d_ilu_dep, s->d_fbuf[0], s->d_fbuf[1]};
        for (void *p : smp)
            if (p) cudaFree(p);
        void *ptrs[] = {s->d_a_diag, s->d_status, s->d_flags, s->d_bar, s->d_lu, s->d_r, s->d_y, s->d_z, s->d_p,
                        s->d_Ap, s->d_y32, s->d_z32, s->d_part, s->d_iters, s->d_relres, s->d_x0};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        if (s->h_status) cudaFreeHost(s->h_status);
        if (s->d_trace) cudaFree(s->d_trace);
        void *bptrs[] = {s->d_sys_off, s->d_vlo, s->d_sys_lo, s->d_nls, s->d_cta_lo, s->d_cta_hi, s->d_br, s->d_bp,
                         s->d_bAp, s->d_by, s->d_bz, s->d_bpart, s->d_brelres, s->d_blu, s->d_by32, s->d_bz32,
                         s->d_bgv64[0], s->d_bgv64[1], s->d_bgv32[0], s->d_bgv32[1], s->d_biters, s->d_active};
        for (void *p : bptrs)
            if (p) cudaFree(p);
        if (cur >= 0 && cur != s->device) cudaSetDevice(cur);
    }
    baas_schedule fresh;
    fresh.hs = std::move(s->hs);
    fresh.opt = s->opt;
    fresh.nnz_a = s->nnz_a;
    fresh.nnz_l = s->nnz_l;
    fresh.f_ord = std::move(s->f_ord);
    fresh.cptr = std::move(s->cptr);
    fresh.crow = std::move(s->crow);
    fresh.cpos = std::move(s->cpos);
    fresh.fault_row = s->fault_row;
    fresh.sys_off = std::move(s->sys_off);
    fresh.nsys = s->nsys;
    fresh.custom_part = std::move(s->custom_part);
    fresh.sm = std::move(s->sm);
    *s = std::move(fresh);
}

void baas_destroy(baas_schedule *s) {
    if (!s) return;
    release_device(s);
    delete s;
}

baas_status baas_replan(baas_schedule *s, const baas_options *opt) {
    if (!s || !opt) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    if (opt->nthread != s->hs.nthread) return fail(BAAS_ERR_BAD_ARG, "nthread is fixed by the analysis");
    if (opt->mapping != s->opt.mapping) return fail(BAAS_ERR_BAD_ARG, "mapping is fixed by the analysis");
    if (opt->parts < 0 || opt->smem_budget < 0) return fail(BAAS_ERR_BAD_ARG, "parts and smem_budget must be >= 0");
    if (opt->walk < BAAS_WALK_AUTO || opt->walk > BAAS_WALK_SMALL) return fail(BAAS_ERR_BAD_ARG, "unknown walk");
    if (opt->small_cluster != 0 && opt->small_cluster != 1 && opt->small_cluster != 2 && opt->small_cluster != 4 &&
        opt->small_cluster != 8 && opt->small_cluster != 16)
        return fail(BAAS_ERR_BAD_ARG, "small_cluster must be 0, 1, 2, 4, 8 or 16");
    if (opt->partition == BAAS_PARTITION_CUSTOM) {
        if (s->custom_part.empty()) return fail(BAAS_ERR_BAD_ARG, "no custom partition: use baas_replan_custom");
        if (opt->parts != s->opt.parts) return fail(BAAS_ERR_BAD_ARG, "a custom partition fixes parts");
    } else if (opt->partition != BAAS_PARTITION_RANGES && opt->partition != BAAS_PARTITION_BAAS_THREADS &&
               opt->partition != BAAS_PARTITION_BLOCKS && opt->partition != BAAS_PARTITION_AUTO) {
        return fail(BAAS_ERR_BAD_ARG, "unknown partition");
    }
    release_device(s);
    const int analysis = s->opt.analysis, ablation = s->opt.ablation;  // fixed by the analysis
    s->opt = *opt;
    s->opt.analysis = analysis;
    s->opt.ablation = ablation;
    return BAAS_OK;
}

baas_status baas_replan_custom(baas_schedule *s, const int *row_part, int parts, int smem_budget) {
    if (!s || !row_part) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    if (parts < 1) return fail(BAAS_ERR_BAD_ARG, "parts must be >= 1");
    if (smem_budget < 0) return fail(BAAS_ERR_BAD_ARG, "smem_budget must be >= 0");
    const int n = s->hs.n;
    for (int i = 0; i < n; i++)
        if (row_part[i] < 0 || row_part[i] >= parts) return fail(BAAS_ERR_BAD_ARG, "row_part out of [0, parts)");
    release_device(s);
    s->custom_part.assign(row_part, row_part + n);
    s->opt.partition = BAAS_PARTITION_CUSTOM;
    s->opt.parts = parts;
    s->opt.smem_budget = smem_budget;
    return BAAS_OK;
}

baas_status baas_sptrsv(baas_schedule *s, const baas_csr *T, int upper, const double *b, double *x, int nrhs, int ldb,
                        void *stream_) {
    PhaseRange range("trsv");
    if (!s || !b || !x) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    const int n = s->hs.n;
    if (!csr_ok(T, n, s->nnz_l)) return fail(BAAS_ERR_BAD_ARG, "triangular factor does not match the analysed pattern");
    if (nrhs < 1 || ldb < n) return fail(BAAS_ERR_BAD_ARG, "nrhs must be >= 1 and ldb >= n");
    if (x == b) return fail(BAAS_ERR_BAD_ARG, "x must not alias b");
    BAAS_TRY(ensure_device(s));
    cudaStream_t stream = (cudaStream_t)stream_;
    const int d = upper ? 1 : 0;
    int walk = BAAS_WALK_CHUNKED;
    if (nrhs == 1) BAAS_TRY(pick_walk(s, 8, false, walk));
    if (walk == BAAS_WALK_SMALL) {
        BAAS_TRY(upload_small(s, false));
        baas::SmallArgs a = small_args(s, false);
        a.b = b;
        a.x = x;
        const int *tcol = T->colidx;
        const double *tval = T->values;
        void *args[] = {(void *)&a, (void *)&tcol, (void *)&tval};
        s->last_walk = BAAS_WALK_SMALL;
        BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
        BAAS_TRY(launch_small(s, 0, upper != 0, sizeof(double) * (size_t)n, args, stream));
        return read_status(s, stream);
    }
    if (walk == BAAS_WALK_LEVELS) {
        if (!s->d_lv[0].lev) BAAS_TRY(upload_level(s));
        if (!s->d_lvT[d]) {
            BAAS_TRY(dalloc(s->d_lvT[d], (size_t)s->d_lv[d].nent));
            BAAS_TRY(dalloc(s->d_ldT[d], (size_t)s->d_lv[d].npos));
        }
        baas::LevelDir D = s->d_lv[d].view();
        unsigned int spin = s->spin();
        double *v = s->d_lvT[d], *dd = s->d_ldT[d];
        void *args[] = {(void *)&D, (void *)&T->values, (void *)&v, (void *)&dd, (void *)&b, (void *)&x,
                        (void *)&s->d_bar, (void *)&s->d_status, (void *)&spin};
        s->last_walk = BAAS_WALK_LEVELS;
        BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
        BAAS_CUDA(cudaMemsetAsync(s->d_bar, 0, sizeof(unsigned int), stream));
        BAAS_CUDA(cudaLaunchCooperativeKernel((void *)baas::k_sweep_levels, s->P, baas::kStageBlock, args, 0, stream));
        return read_status(s, stream);
    }
    const bool fw = walk == BAAS_WALK_FETCH;
    if (fw) {
        if (!s->d_gfT[d]) BAAS_TRY(dalloc(s->d_gfT[d], (size_t)baas::kFetchVal64 * n));
        baas::FetchPlan fp = fetch_plan(s, 8, false);
        const size_t smem = fetch_smem(s->fch, 8, false);
        unsigned int spin = s->spin();
        double *gv = s->d_gfT[d];
        // the rows' results are published into one of two schedule buffers, which the kernel
        // leaves reset for the next call; after a failed call both are reset here again
        if (!s->d_fbuf[0]) {
            BAAS_TRY(dalloc(s->d_fbuf[0], (size_t)n));
            BAAS_TRY(dalloc(s->d_fbuf[1], (size_t)n));
        }
        if (!s->fbuf_ready) {
            const int fill_blocks = (int)std::min<long long>(4LL * s->num_sms, ((long long)n + 255) / 256);
            for (int k = 0; k < 2; k++)
                baas::k_fill_sentinel<double><<<std::max(fill_blocks, 1), 256, 0, stream>>>(s->d_fbuf[k], n, 1, n);
            BAAS_CUDA(cudaGetLastError());
            s->fbuf_ready = true;
        }
        s->last_walk = BAAS_WALK_FETCH;
        for (int ieee = 0; ieee < 2; ieee++) {
            double *xg = s->d_fbuf[s->fbuf_cur], *xnext = s->d_fbuf[s->fbuf_cur ^ 1];
            void *args[] = {(void *)&fp, (void *)&d, (void *)&T->values, (void *)&gv, (void *)&b, (void *)&x,
                            (void *)&xg, (void *)&xnext, (void *)&s->d_status, (void *)&spin, (void *)&s->d_trace};
            BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
            BAAS_CUDA(cudaLaunchCooperativeKernel(sweep_fetch_kernel(ieee != 0), s->P, baas::kStageBlock, args, smem, stream));
            s->fbuf_cur ^= 1;
            dump_trace(s, upper ? "sptrsv-upper" : "sptrsv-lower", stream);
            const baas_status st = read_status(s, stream);
            if (st != BAAS_OK) s->fbuf_ready = false;
            if (!needs_ieee_repeat(s)) return st;
        }
        return fail(BAAS_ERR_CUDA, "IEEE sweep reported a fast-path division");
    }
    s->last_walk = BAAS_WALK_CHUNKED;
    if (s->opt.walk == BAAS_WALK_FETCH || s->opt.walk == BAAS_WALK_LEVELS || s->opt.walk == BAAS_WALK_SMALL)
        return fail(BAAS_ERR_BAD_ARG, "the fetch, level and single-CTA walks take one right-hand side");
    // right-hand sides walked together: as many as the solution slots leave room for
    const int R = std::min(nrhs, s->rmax64);
    WinCfg *w = nullptr;
    BAAS_TRY(get_windows(s, 8, R, &w));
    if (!s->d_gvT[d]) BAAS_TRY(dalloc(s->d_gvT[d], s->chk.dir[d].vsrcT.size()));
    baas::ChunkPlan pl = chunk_plan(s, *w);
    unsigned int spin = s->spin();
    double *gv = s->d_gvT[d];
    void *args[] = {(void *)&pl, (void *)&d, (void *)&T->values, (void *)&gv, (void *)&b, (void *)&ldb, (void *)&x,
                    (void *)&ldb, (void *)&nrhs, (void *)&R, (void *)&s->d_status, (void *)&spin, (void *)&s->d_trace};
    const bool stg = w->rhs_bytes > 0;
    for (int ieee = 0; ieee < 2; ieee++) {
        BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
        const int fill_blocks = (int)std::min<long long>(4LL * s->num_sms, ((long long)n * nrhs + 255) / 256);
        baas::k_fill_sentinel<double><<<std::max(fill_blocks, 1), 256, 0, stream>>>(x, n, nrhs, ldb);
        BAAS_CUDA(cudaGetLastError());
        BAAS_CUDA(cudaLaunchCooperativeKernel(sweep_kernel(R > 1, stg, ieee != 0), s->P, baas::kStageBlock, args, w->smem,
                                              stream));
        dump_trace(s, upper ? "sptrsv-upper" : "sptrsv-lower", stream);
        const baas_status st = read_status(s, stream);
        if (!needs_ieee_repeat(s)) return st;
    }
    return fail(BAAS_ERR_CUDA, "IEEE sweep reported a fast-path division");
}

static baas_status factor(baas_schedule *s, const baas_csr *A, double *lu, void *stream_, bool ilu) {
    PhaseRange range(ilu ? "ilu" : "ic");
    if (!s || !lu) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    if (s->hs.kind == baas::SchedKind::SpTRSV) return fail(BAAS_ERR_STATE, "a SpTRSV schedule cannot drive a factorisation");
    if (!A || A->n != s->hs.n || A->nnz != s->nnz_a || !A->rowptr || !A->colidx)
        return fail(BAAS_ERR_BAD_ARG, "matrix does not match the analysed pattern");
    BAAS_TRY(ensure_device(s));
    cudaStream_t stream = (cudaStream_t)stream_;
    int walk = BAAS_WALK_CHUNKED;
    if (!ilu && (s->opt.walk == BAAS_WALK_AUTO || s->opt.walk == BAAS_WALK_SMALL)) BAAS_TRY(pick_walk(s, 8, true, walk));
    // ILU0 level by level with grid barriers: asked for, or automatic when the group levels are wide
    // (512 rows or more on average; measured on 7-point convection-diffusion: 48^3 0.91 ms against
    // 0.98 ms for the flag-driven partitioned kernel, 96^3 2.11 ms against 2.68 ms)
    const int nglev = (int)s->hs.exec_level_ptr.size() - 1;
    const bool ilu_levels = ilu && (s->opt.walk == BAAS_WALK_LEVELS ||
                                    (s->opt.walk == BAAS_WALK_AUTO && nglev > 0 && s->hs.n / nglev >= 512));
    if (ilu_levels) {
        if (!s->d_lv[0].lev) BAAS_TRY(upload_level(s));
        if (!s->d_ilu_rec) {
            // per plan position (the level plan's row order): the row's record and its partners'
            // diagonal positions and upper-entry counts (static: they depend on the pattern only)
            LevelHostDir L;
            build_level_dir(s, false, L);
            const baas::HostSchedule &h = s->hs;
            const int np = (int)L.row.size();
            std::vector<int4> rec(np);
            std::vector<int2> dep((size_t)np * baas::kIluLow, int2{0, 0});
            for (int p = 0; p < np; p++) {
                const int i = L.row[p], rb = h.a_rowptr[i], di = h.a_diagptr[i], re = h.a_rowptr[i + 1];
                bool reg = re - rb <= baas::kFacRegs && di - rb <= baas::kIluLow;
                for (int t = 0; reg && t < di - rb; t++) {
                    const int c = h.a_colidx[rb + t];
                    const int nu = h.a_rowptr[c + 1] - h.a_diagptr[c] - 1;
                    if (nu > baas::kIluUp) reg = false;
                    dep[(size_t)p * baas::kIluLow + t] = int2{h.a_diagptr[c], nu};
                }
                rec[p] = reg ? int4{i, rb, re - rb, di - rb} : int4{i, rb, -1, 0};
            }
            BAAS_TRY(upload(s->d_ilu_rec, rec));
            BAAS_TRY(upload(s->d_ilu_dep, dep));
        }
        baas::LevelDir D = s->d_lv[0].view();
        unsigned int spin = s->spin();
        void *args[] = {(void *)&D, (void *)&s->d_ilu_rec, (void *)&s->d_ilu_dep, (void *)&A->rowptr,
                        (void *)&A->colidx, (void *)&s->d_a_diag, (void *)&lu, (void *)&s->d_bar, (void *)&s->d_status,
                        (void *)&spin};
        BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
        BAAS_CUDA(cudaMemsetAsync(s->d_bar, 0, sizeof(unsigned int), stream));
        BAAS_CUDA(cudaLaunchCooperativeKernel((void *)baas::k_ilu0_levels, s->P, baas::kStageBlock, args, 0, stream));
        return read_status(s, stream);
    }
    if (walk == BAAS_WALK_SMALL) {  // IC0 by the cluster walk over the row levels (shared memory: the row scratch only)
        BAAS_TRY(upload_small(s, true));
        baas::SmallArgs a = small_args(s, true);
        a.a_rowptr = A->rowptr;
        a.a_colidx = A->colidx;
        a.lu = lu;
        void *args[] = {(void *)&a};
        BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
        BAAS_TRY(launch_small(s, 2, false, baas::kIcScratch, args, stream));
        return read_status(s, stream);
    }
    BAAS_TRY(next_epoch(s, stream));
    BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
    baas::PartView pv = s->d_fwd.view(s->P);
    unsigned int spin = s->spin();
    void *args[] = {(void *)&pv, (void *)&A->rowptr, (void *)&A->colidx, (void *)&s->d_a_diag, (void *)&lu,
                    (void *)&s->d_flags, (void *)&s->epoch, (void *)&s->d_status, (void *)&spin};
    void *kern = ilu ? (void *)baas::k_factor_part<true> : (void *)baas::k_factor_part<false>;
    BAAS_CUDA(cudaLaunchCooperativeKernel(kern, s->P, baas::kPartBlock, args, 0, stream));
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


// ---------------------------------------------------------------------------------------
// Batched systems (no counterpart in the reference).
// ---------------------------------------------------------------------------------------
int baas_batch_concat(int nsys, const baas_csr *const *sys, int *rowptr, int *colidx, double *values, int *sys_off) {
    if (nsys < 1 || !sys) return -1;
    long long n = 0, nnz = 0;
    for (int k = 0; k < nsys; k++) {
        if (!sys[k] || !sys[k]->rowptr || sys[k]->n <= 0) return -1;
        n += sys[k]->n;
        nnz += sys[k]->rowptr[sys[k]->n];
    }
    if (n > INT_MAX || nnz > INT_MAX) return -1;
    if (!rowptr || !colidx || !sys_off) return (int)nnz;
    int ro = 0, eo = 0;
    rowptr[0] = 0;
    sys_off[0] = 0;
    for (int k = 0; k < nsys; k++) {
        const baas_csr &m = *sys[k];
        for (int i = 0; i < m.n; i++) {
            for (int e = m.rowptr[i]; e < m.rowptr[i + 1]; e++) {
                colidx[eo] = m.colidx[e] + ro;
                if (values && m.values) values[eo] = m.values[e];
                eo++;
            }
            rowptr[ro + i + 1] = eo;
        }
        ro += m.n;
        sys_off[k + 1] = ro;
    }
    return (int)nnz;
}

}  // extern "C"

// Schedule file: "BAASSCH" + format version, the options, the sizes, then every array of the
// analysis (each as a count and its elements), so that loading rebuilds the schedule without
// repeating the analysis. Host byte order; the file is for the machine or cluster that wrote it.
namespace {
constexpr char kSchedMagic[8] = {'B', 'A', 'A', 'S', 'S', 'C', 'H', '1'};

struct SchedWriter {
    FILE *f;
    bool ok = true;
    void raw(const void *p, size_t n) { ok = ok && std::fwrite(p, 1, n, f) == n; }
    template <typename T>
    void val(T v) { raw(&v, sizeof(T)); }
    template <typename T>
    void vec(const std::vector<T> &v) {
        val<long long>((long long)v.size());
        if (!v.empty()) raw(v.data(), sizeof(T) * v.size());
    }
};
struct SchedReader {
    FILE *f;
    bool ok = true;
    void raw(void *p, size_t n) { ok = ok && std::fread(p, 1, n, f) == n; }
    template <typename T>
    T val() {
        T v{};
        raw(&v, sizeof(T));
        return v;
    }
    template <typename T>
    void vec(std::vector<T> &v, long long max_count) {
        const long long n = val<long long>();
        if (!ok || n < 0 || n > max_count) {
            ok = false;
            return;
        }
        v.resize((size_t)n);
        if (n) raw(v.data(), sizeof(T) * (size_t)n);
    }
};

template <class IO, class H, class V>
void sched_arrays(IO &io, H &h, V vec) {
    vec(h.a_rowptr), vec(h.a_colidx), vec(h.a_diagptr), vec(h.l_rowptr), vec(h.l_colidx), vec(h.l_src);
    vec(h.group_ptr), vec(h.group_set), vec(h.level_ptr), vec(h.perm_to_orig), vec(h.node_to_level), vec(h.perm);
    vec(h.exec_level_ptr), vec(h.nthread_per_level), vec(h.thread_boundaries), vec(h.task_boundaries);
    vec(h.thread_cont_to_orig), vec(h.orig_to_thread_cont), vec(h.task_ptr), vec(h.task_set), vec(h.btask_ptr);
    vec(h.btask_set), vec(h.fdag_ptr), vec(h.fdag_set);
    (void)io;
}
}  // namespace

extern "C" {

baas_status baas_schedule_save(const baas_schedule *s, const char *path) {
    if (!s || !path) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(BAAS_ERR_BAD_ARG, std::string("cannot open ") + path + " for writing");
    SchedWriter w{f};
    const baas::HostSchedule &h = s->hs;
    w.raw(kSchedMagic, sizeof(kSchedMagic));
    w.val<int>((int)sizeof(baas_options));
    w.raw(&s->opt, sizeof(baas_options));
    w.val<int>((int)h.kind), w.val<int>(h.n), w.val<int>(h.nthread), w.val<int>(h.ngroups), w.val<int>(h.nlevels);
    w.val<int>(h.ntasks), w.val<int>(s->nnz_a), w.val<int>(s->nnz_l), w.val<int>(s->nsys);
    w.val<double>(h.analysis_ms);
    w.val<int>(h.score.level_window), w.val<double>(h.score.amplify), w.val<double>(h.score.over_gamma);
    w.val<double>(h.score.award_alpha), w.val<double>(h.score.load_beta);
    w.vec(h.cost);
    w.vec(s->sys_off);
    sched_arrays(w, h, [&](const std::vector<int> &v) { w.vec(v); });
    const bool ok = w.ok && std::fclose(f) == 0;
    if (!ok) return fail(BAAS_ERR_BAD_ARG, std::string("writing ") + path + " failed");
    return BAAS_OK;
}

int baas_schedule_info(const baas_schedule *s, int *info) {
    if (!s || !info) return -1;
    info[0] = s->hs.n;
    info[1] = s->nnz_a;
    info[2] = (int)s->hs.kind;
    info[3] = s->hs.nthread;
    info[4] = s->opt.mapping;
    info[5] = s->nsys;
    return 6;
}

baas_status baas_schedule_load(const char *path, baas_schedule **out) {
    if (!path || !out) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    *out = nullptr;
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(BAAS_ERR_BAD_ARG, std::string("cannot open ") + path);
    SchedReader r{f};
    char magic[8];
    r.raw(magic, sizeof(magic));
    if (!r.ok || std::memcmp(magic, kSchedMagic, sizeof(magic)) != 0 || r.val<int>() != (int)sizeof(baas_options)) {
        std::fclose(f);
        return fail(BAAS_ERR_BAD_ARG, std::string(path) + " is not a schedule file of this library version");
    }
    baas_schedule *s = new baas_schedule();
    baas::HostSchedule &h = s->hs;
    r.raw(&s->opt, sizeof(baas_options));
    h.kind = (baas::SchedKind)r.val<int>();
    h.n = r.val<int>(), h.nthread = r.val<int>(), h.ngroups = r.val<int>(), h.nlevels = r.val<int>();
    h.ntasks = r.val<int>(), s->nnz_a = r.val<int>(), s->nnz_l = r.val<int>(), s->nsys = r.val<int>();
    h.analysis_ms = r.val<double>();
    h.score.level_window = r.val<int>(), h.score.amplify = r.val<double>(), h.score.over_gamma = r.val<double>();
    h.score.award_alpha = r.val<double>(), h.score.load_beta = r.val<double>();
    const long long cap = (long long)std::max(s->nnz_a, 0) + 2LL * std::max(h.n, 0) + 16;  // no array is longer
    r.vec(h.cost, cap);
    r.vec(s->sys_off, cap);
    sched_arrays(r, h, [&](std::vector<int> &v) { r.vec(v, cap); });
    std::fclose(f);
    const int n = h.n;
    const bool sane = r.ok && n > 0 && (int)h.a_rowptr.size() == n + 1 && (int)h.a_colidx.size() == s->nnz_a &&
                      (int)h.l_rowptr.size() == n + 1 && (int)h.l_colidx.size() == s->nnz_l &&
                      (int)h.group_ptr.size() == h.ngroups + 1 && (int)h.group_set.size() == n &&
                      (int)h.perm_to_orig.size() == h.ngroups && (int)h.level_ptr.size() == h.nlevels + 1 &&
                      (h.kind >= baas::SchedKind::SpTRSV && h.kind <= baas::SchedKind::ILU0) &&
                      (s->nsys == 0 || (int)s->sys_off.size() == s->nsys + 1);
    if (!sane) {
        delete s;
        return fail(BAAS_ERR_BAD_ARG, std::string(path) + " is truncated or inconsistent");
    }
    build_order(s);
    *out = s;
    return BAAS_OK;
}

baas_status baas_analyze_batch(const baas_csr *A, const int *sys_off, int nsys, const baas_options *opt,
                               baas_schedule **out) {
    if (!A || !sys_off || !out || nsys < 1) return fail(BAAS_ERR_BAD_ARG, "NULL argument or no systems");
    if (!A->rowptr || !A->colidx || A->n <= 0) return fail(BAAS_ERR_BAD_ARG, "empty or NULL pattern");
    if (sys_off[0] != 0 || sys_off[nsys] != A->n) return fail(BAAS_ERR_BAD_ARG, "system offsets must run from 0 to n");
    for (int k = 0; k < nsys; k++) {
        if (sys_off[k + 1] <= sys_off[k]) return fail(BAAS_ERR_BAD_ARG, "every system needs at least one row");
        for (int i = sys_off[k]; i < sys_off[k + 1]; i++)
            for (int e = A->rowptr[i]; e < A->rowptr[i + 1]; e++)
                if (A->colidx[e] < sys_off[k] || A->colidx[e] >= sys_off[k + 1])
                    return fail(BAAS_ERR_BAD_ARG, "an entry couples two systems (the pattern must be block diagonal)");
    }
    const std::vector<int> offsets(sys_off, sys_off + nsys + 1);
    BAAS_TRY(analyze_common(A, BAAS_KERNEL_ICCG, opt, out, &offsets));
    (*out)->sys_off = offsets;
    (*out)->nsys = nsys;
    return BAAS_OK;
}

static baas_status batch_setup(baas_schedule *s, int R) {
    const int n = s->hs.n, P = s->P, ns = s->nsys;
    if (!s->d_sys_off) {
        std::vector<int> vlo(P + 1), sys_lo(P), nls(P), cta_lo(ns, P), cta_hi(ns, -1);
        for (int c = 0; c <= P; c++) vlo[c] = (int)(((long long)n * c) / P);
        int maxls = 1;
        for (int c = 0; c < P; c++) {
            int k = 0;
            while (k + 1 < ns && s->sys_off[k + 1] <= vlo[c]) k++;
            sys_lo[c] = k;
            int cnt = 0;
            for (int q = k; q < ns && s->sys_off[q] < vlo[c + 1]; q++)
                if (s->sys_off[q + 1] > vlo[c]) {
                    cnt++;
                    cta_lo[q] = std::min(cta_lo[q], c);
                    cta_hi[q] = std::max(cta_hi[q], c);
                }
            nls[c] = vlo[c + 1] > vlo[c] ? cnt : 0;
            maxls = std::max(maxls, nls[c]);
        }
        for (int q = 0; q < ns; q++)
            if (cta_hi[q] < 0) return fail(BAAS_ERR_BAD_ARG, "a system has no rows");
        s->maxls = maxls;
        BAAS_TRY(upload(s->d_sys_off, s->sys_off));
        BAAS_TRY(upload(s->d_vlo, vlo));
        BAAS_TRY(upload(s->d_sys_lo, sys_lo));
        BAAS_TRY(upload(s->d_nls, nls));
        BAAS_TRY(upload(s->d_cta_lo, cta_lo));
        BAAS_TRY(upload(s->d_cta_hi, cta_hi));
        BAAS_TRY(dalloc(s->d_active, 1));
        BAAS_TRY(dalloc(s->d_blu, (size_t)s->nnz_a));
        for (int d = 0; d < 2; d++) {
            BAAS_TRY(dalloc(s->d_bgv64[d], s->chk.dir[d].vsrcA.size()));
            BAAS_TRY(dalloc(s->d_bgv32[d], s->chk.dir[d].vsrcA.size()));
        }
    }
    if (s->batch_R < R) {
        double *dp[] = {s->d_br, s->d_bp, s->d_bAp, s->d_by, s->d_bz, s->d_bpart, s->d_brelres};
        for (double *p : dp)
            if (p) cudaFree(p);
        if (s->d_by32) cudaFree(s->d_by32);
        if (s->d_bz32) cudaFree(s->d_bz32);
        if (s->d_biters) cudaFree(s->d_biters);
        const size_t nr = (size_t)n * R;
        BAAS_TRY(dalloc(s->d_br, nr));
        BAAS_TRY(dalloc(s->d_bp, nr));
        BAAS_TRY(dalloc(s->d_bAp, nr));
        BAAS_TRY(dalloc(s->d_by, nr));
        BAAS_TRY(dalloc(s->d_bz, nr));
        BAAS_TRY(dalloc(s->d_by32, nr));
        BAAS_TRY(dalloc(s->d_bz32, nr));
        BAAS_TRY(dalloc(s->d_bpart, (size_t)2 * P * s->maxls * R));
        BAAS_TRY(dalloc(s->d_biters, (size_t)ns * R));
        BAAS_TRY(dalloc(s->d_brelres, (size_t)ns * R));
        s->batch_R = R;
    }
    return BAAS_OK;
}

baas_status baas_iccg_batched(baas_schedule *s, const baas_csr *A, const double *B, double *X, int nrhs, int ldb,
                              double tol, int maxiter, int precision, int *iters, double *relres, void *stream_) {
    PhaseRange range("pcg_batched");
    if (!s || !B || !X || !iters || !relres) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    if (s->nsys < 1) return fail(BAAS_ERR_STATE, "the schedule was not made by baas_analyze_batch");
    if (!csr_ok(A, s->hs.n, s->nnz_a)) return fail(BAAS_ERR_BAD_ARG, "matrix does not match the analysed pattern");
    const int n = s->hs.n;
    if (nrhs < 1 || nrhs > baas::kMaxRhs || ldb < n) return fail(BAAS_ERR_BAD_ARG, "nrhs must be 1..8 and ldb >= n");
    if (maxiter < 0 || !(tol >= 0.0)) return fail(BAAS_ERR_BAD_ARG, "maxiter must be >= 0 and tol >= 0");
    if (precision != BAAS_PREC_FP64 && precision != BAAS_PREC_FP32_FACTORS) return fail(BAAS_ERR_BAD_ARG, "unknown precision");
    BAAS_TRY(ensure_device(s));
    const bool mixed = precision == BAAS_PREC_FP32_FACTORS;
    WinCfg *w = nullptr;
    BAAS_TRY(get_windows(s, mixed ? 4 : 8, nrhs, &w));
    BAAS_TRY(batch_setup(s, nrhs));
    cudaStream_t stream = (cudaStream_t)stream_;
    const int P = s->P;
    const unsigned int active = (unsigned int)(s->nsys * nrhs);
    const size_t xcount = (size_t)(nrhs - 1) * (size_t)ldb + (size_t)n;
    if (!mixed) BAAS_TRY(save_x0(s, X, xcount, stream));

    baas::BatchArgs a{};
    a.n = n;
    a.ldb = ldb;
    a.a_rowptr = A->rowptr;
    a.a_colidx = A->colidx;
    a.a_diag = s->d_a_diag;
    a.a_val = A->values;
    a.B = B;
    a.X = X;
    a.fac = s->d_fwd.view(P);
    a.pl = chunk_plan(s, *w);
    a.bp = baas::BatchPlan{s->nsys, nrhs, s->maxls, s->d_sys_off, s->d_vlo, s->d_sys_lo, s->d_nls, s->d_cta_lo, s->d_cta_hi};
    for (int d = 0; d < 2; d++) {
        a.gv64[d] = s->d_bgv64[d];
        a.gv32[d] = s->d_bgv32[d];
    }
    a.lu = s->d_blu;
    a.gflag = s->d_flags;
    a.r = s->d_br;
    a.p = s->d_bp;
    a.Ap = s->d_bAp;
    a.y = s->d_by;
    a.z = s->d_bz;
    a.y32 = s->d_by32;
    a.z32 = s->d_bz32;
    a.part = s->d_bpart;
    a.bar = s->d_bar;
    a.active = s->d_active;
    a.st = s->d_status;
    a.maxiter = maxiter;
    a.tol = tol;
    a.out_iters = s->d_biters;
    a.out_relres = s->d_brelres;
    a.spin_limit = s->spin();
    a.scal_off = (int)((w->smem + 15) / 16 * 16);
    const size_t smem = (size_t)a.scal_off + (size_t)baas::batch_scal_bytes(s->maxls);
    if (smem > (size_t)kMaxDynSmem) return fail(BAAS_ERR_BAD_ARG, "batched solve: shared memory over budget");
    void *args[] = {(void *)&a};
    const bool mr = nrhs > 1;
    const bool pairs = getenv("BAAS_BATCH_PAIRS") && atoi(getenv("BAAS_BATCH_PAIRS")) > 0;
    const int rw = mixed && (nrhs == 2 || nrhs == 4) && !pairs ? nrhs : 1;
    for (int ieee = 0; ieee < 2; ieee++) {
        if (ieee) BAAS_CUDA(cudaMemcpyAsync(X, s->d_x0, sizeof(double) * xcount, cudaMemcpyDeviceToDevice, stream));
        BAAS_TRY(next_epoch(s, stream));
        a.epoch = s->epoch;
        BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
        BAAS_CUDA(cudaMemsetAsync(s->d_bar, 0, sizeof(unsigned int), stream));
        BAAS_CUDA(cudaMemcpyAsync(s->d_active, &active, sizeof(active), cudaMemcpyHostToDevice, stream));
        BAAS_CUDA(cudaLaunchCooperativeKernel(batched_kernel(mixed, mr, ieee != 0, rw), P, baas::kStageBlock, args, smem,
                                              stream));
        BAAS_CUDA(cudaMemcpyAsync(iters, s->d_biters, sizeof(int) * (size_t)s->nsys * nrhs, cudaMemcpyDeviceToHost, stream));
        BAAS_CUDA(cudaMemcpyAsync(relres, s->d_brelres, sizeof(double) * (size_t)s->nsys * nrhs, cudaMemcpyDeviceToHost,
                                  stream));
        BAAS_TRY(read_status(s, stream));
        if (!needs_ieee_repeat(s)) break;
        if (ieee) return fail(BAAS_ERR_CUDA, "IEEE batched ICCG reported a fast-path division");
    }
    for (int q = 0; q < s->nsys * nrhs; q++)
        if (!(relres[q] < tol)) return fail(BAAS_ERR_NOT_CONVERGED, "maxiter reached before tol for some instance");
    return BAAS_OK;
}

static baas_status iccg_launch(baas_schedule *s, const baas_csr *A, const double *b, double *x, double tol, int maxiter,
                               int precision, int *iters, double *relres, void *stream_, bool reuse, const double *xf,
                               double *grad_a) {
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
            BAAS_TRY(dalloc(s->d_gv64[d], s->chk.dir[d].vsrcA.size()));
            BAAS_TRY(dalloc(s->d_gv32[d], s->chk.dir[d].vsrcA.size()));
        }
        BAAS_TRY(dalloc(s->d_part, (size_t)3 * P));
        BAAS_TRY(dalloc(s->d_iters, 1));
        BAAS_TRY(dalloc(s->d_relres, 1));
        s->ws_ready = true;
    }
    const bool mixed = precision == BAAS_PREC_FP32_FACTORS;
    int walk = BAAS_WALK_CHUNKED;
    BAAS_TRY(pick_walk(s, mixed ? 4 : 8, true, walk));
    if (walk == BAAS_WALK_SMALL) {
        BAAS_TRY(upload_small(s, true));
        baas::SmallArgs a = small_args(s, true);
        a.a_rowptr = A->rowptr;
        a.a_colidx = A->colidx;
        a.a_val = A->values;
        a.lu = s->d_lu;
        a.b = b;
        a.x = x;
        a.r = s->d_r;
        a.Ap = s->d_Ap;
        a.maxiter = maxiter;
        a.tol = tol;
        a.reuse = reuse ? 1 : 0;
        a.out_iters = s->d_iters;
        a.out_relres = s->d_relres;
        a.xf = xf;
        a.grad_a = grad_a;
        void *args[] = {(void *)&a};
        s->last_walk = BAAS_WALK_SMALL;
        BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
        BAAS_TRY(launch_small(s, 1, mixed, std::max((size_t)n * (8 + (mixed ? 4 : 8)), baas::kIcScratch), args, stream));
        int it = 0;
        double rr = 0.0;
        BAAS_CUDA(cudaMemcpyAsync(&it, s->d_iters, sizeof(int), cudaMemcpyDeviceToHost, stream));
        BAAS_CUDA(cudaMemcpyAsync(&rr, s->d_relres, sizeof(double), cudaMemcpyDeviceToHost, stream));
        const baas_status st = read_status(s, stream);
        if (iters) *iters = it;
        if (relres) *relres = rr;
        if (!reuse) s->factor_prec = st == BAAS_OK || st == BAAS_ERR_NOT_CONVERGED ? precision : -1;
        if (st != BAAS_OK) return st;
        if (!(rr < tol)) return fail(BAAS_ERR_NOT_CONVERGED, "maxiter reached before tol");
        return BAAS_OK;
    }
    const bool fw = walk == BAAS_WALK_FETCH, lw = walk == BAAS_WALK_LEVELS;
    if (lw && !s->d_lv[0].lev) BAAS_TRY(upload_level(s));
    if (lw && !s->d_lv64[0]) {
        for (int d = 0; d < 2; d++) {
            BAAS_TRY(dalloc(s->d_lv64[d], (size_t)s->d_lv[d].nent));
            BAAS_TRY(dalloc(s->d_ld64[d], (size_t)s->d_lv[d].npos));
            BAAS_TRY(dalloc(s->d_lv32[d], (size_t)s->d_lv[d].nent));
            BAAS_TRY(dalloc(s->d_ld32[d], (size_t)s->d_lv[d].npos));
        }
    }
    if (fw && !s->d_gf64[0]) {
        for (int d = 0; d < 2; d++) {
            BAAS_TRY(dalloc(s->d_gf64[d], (size_t)baas::kFetchVal64 * n));
            BAAS_TRY(dalloc(s->d_gf32[d], (size_t)baas::kFetchVal32 * n));
        }
        BAAS_TRY(dalloc(s->d_dg, (size_t)n));
    }
    WinCfg *w = nullptr;
    BAAS_TRY(get_windows(s, mixed ? 4 : 8, 1, &w));
    if (!mixed) BAAS_TRY(save_x0(s, x, (size_t)n, stream));
    baas::IccgArgs a{};
    a.n = n;
    a.a_rowptr = A->rowptr;
    a.a_colidx = A->colidx;
    a.a_diag = s->d_a_diag;
    a.a_val = A->values;
    a.b = b;
    a.x = x;
    a.fac = s->d_fwd.view(P);
    a.pl = chunk_plan(s, *w);
    for (int d = 0; d < 2; d++) {
        a.gv64[d] = s->d_gv64[d];
        a.gv32[d] = s->d_gv32[d];
    }
    a.lu = s->d_lu;
    a.gflag = s->d_flags;
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
    a.reuse = reuse ? 1 : 0;
    a.xf = xf;
    a.grad_a = grad_a;
    size_t smem = w->smem;
    if (fw) {
        a.fp = fetch_plan(s, mixed ? 4 : 8, true);
        for (int d = 0; d < 2; d++) {
            a.gf64[d] = s->d_gf64[d];
            a.gf32[d] = s->d_gf32[d];
        }
        smem = fetch_smem(s->fch, mixed ? 4 : 8, true);
        // IC0 by the fetch walk when no entry's dot product has a column match
        a.fac_fetch = s->fwd.mpair.empty() ? 1 : 0;
        a.dg = s->d_dg;
    }
    if (lw) {
        for (int d = 0; d < 2; d++) {
            a.lv[d] = s->d_lv[d].view();
            a.lv64[d] = s->d_lv64[d];
            a.ld64[d] = s->d_ld64[d];
            a.lv32[d] = s->d_lv32[d];
            a.ld32[d] = s->d_ld32[d];
        }
        smem = 0;
    }
    s->last_walk = walk;
    void *args[] = {(void *)&a};
    const bool stg = w->rhs_bytes > 0;
    int it = 0;
    double rr = 0.0;
    baas_status st = BAAS_OK;
    for (int ieee = 0; ieee < 2; ieee++) {
        if (ieee) BAAS_CUDA(cudaMemcpyAsync(x, s->d_x0, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, stream));
        BAAS_TRY(next_epoch(s, stream));
        a.epoch = s->epoch;
        BAAS_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(DevStatus), stream));
        BAAS_CUDA(cudaMemsetAsync(s->d_bar, 0, sizeof(unsigned int), stream));
        BAAS_CUDA(cudaLaunchCooperativeKernel(iccg_kernel(mixed, (fw || lw) ? false : stg, ieee != 0, walk), P,
                                              baas::kStageBlock, args, smem, stream));
        BAAS_CUDA(cudaMemcpyAsync(&it, s->d_iters, sizeof(int), cudaMemcpyDeviceToHost, stream));
        BAAS_CUDA(cudaMemcpyAsync(&rr, s->d_relres, sizeof(double), cudaMemcpyDeviceToHost, stream));
        dump_trace(s, "iccg", stream);
        st = read_status(s, stream);
        if (!needs_ieee_repeat(s)) break;
        if (ieee) return fail(BAAS_ERR_CUDA, "IEEE ICCG reported a fast-path division");
    }
    if (iters) *iters = it;
    if (relres) *relres = rr;
    if (!reuse) s->factor_prec = st == BAAS_OK || st == BAAS_ERR_NOT_CONVERGED ? precision : -1;
    if (st != BAAS_OK) return st;
    if (!(rr < tol)) return fail(BAAS_ERR_NOT_CONVERGED, "maxiter reached before tol");
    return BAAS_OK;
}

baas_status baas_iccg(baas_schedule *s, const baas_csr *A, const double *b, double *x, double tol, int maxiter,
                      int precision, int *iters, double *relres, void *stream) {
    PhaseRange range("pcg");
    return iccg_launch(s, A, b, x, tol, maxiter, precision, iters, relres, stream, false, nullptr, nullptr);
}

// Adjoint solve: A^T lambda = g with the IC0 factors of the previous baas_iccg (A is symmetric,
// so the transposed sweeps L^-T, L^-1 of the preconditioner are the forward ones), from
// lambda = 0; with x and grad_a, the pattern gradient grad_a[e] = -lambda_i x_j in the same launch.
baas_status baas_iccg_adjoint(baas_schedule *s, const baas_csr *A, const double *g, double *lambda, const double *x,
                              double *grad_a, double tol, int maxiter, int precision, int *iters, double *relres,
                              void *stream_) {
    PhaseRange range("pcg_adjoint");
    if (!s || !g || !lambda) return fail(BAAS_ERR_BAD_ARG, "NULL argument");
    if ((x == nullptr) != (grad_a == nullptr)) return fail(BAAS_ERR_BAD_ARG, "x and grad_a go together");
    if (s->factor_prec != precision)
        return fail(BAAS_ERR_STATE, "no IC0 factors of this precision: run baas_iccg on this schedule first");
    cudaStream_t stream = (cudaStream_t)stream_;
    BAAS_CUDA(cudaMemsetAsync(lambda, 0, sizeof(double) * (size_t)s->hs.n, stream));
    return iccg_launch(s, A, g, lambda, tol, maxiter, precision, iters, relres, stream_, true, x, grad_a);
}

}  // extern "C"
