// Device stages of the schedule analysis: the data-parallel integer stages of the pipeline run on
// the GPU, with outputs identical to the host stages' (schedule.cpp), while the serial BFS
// coarsenings and the mappings stay on the host. The stages (reference file:line of the behaviour):
//   transpose    CSR <-> CSC with rows ascending in each column (spm/CSR.cpp:914-950, the
//                per-column quicksort at :945-949; spm/DAG.cpp:481-564 for the inverse DAG)
//   two_hop      the two-hop transitive reduction (DAG::partialSparsification_CSC,
//                spm/DAG.cpp:295-344, cliqueSimplification off)
//   group_dag    the DAG between groups, sorted and unique (merge/Coarsen.cpp:748-801)
//   levels       Kahn levels with the self-counting in-degree, nodes ascending inside each level
//                (DAG_levelSet_CSC, spm/DAG.cpp:572-629)
// Determinism: atomics only count; every order that reaches an output comes from a stable radix
// sort (CUB) of entries generated in a fixed order, so the result does not depend on scheduling.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "schedule.hpp"

namespace baas {
namespace {

constexpr int kAnBlock = 256;

int grid_for(long long work) {
    return (int)std::max<long long>(1, std::min<long long>(148 * 16, (work + kAnBlock - 1) / kAnBlock));
}

int nbits(unsigned long long x) {  // smallest b with x < 2^b (at least 1)
    int b = 1;
    while (b < 64 && (x >> b) != 0) b++;
    return b;
}

// row of every entry: the row r with ptr[r] <= e < ptr[r + 1] (rows may be empty)
__global__ void k_entry_rows(const int *__restrict__ ptr, int n, int m, int *rows) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        int lo = 0, hi = n;  // last r with ptr[r] <= e
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (ptr[mid] <= e)
                lo = mid;
            else
                hi = mid;
        }
        rows[e] = lo;
    }
}

__global__ void k_count(const int *__restrict__ idx, int m, int *cnt) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) atomicAdd(cnt + idx[e], 1);
}

// Two-hop reduction on a CSC DAG (each column: the node itself first, then its children
// ascending): the edge i -> j is dead when a child k of i also has j as a child. A thread per node
// marks only its own column's entries and counts the survivors.
__global__ void k_two_hop(const int *__restrict__ ptr, const int *__restrict__ idx, int n, unsigned char *keep,
                          int *alive) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int cb = ptr[i] + 1, ce = ptr[i + 1], nk = ce - cb;
        for (int e = ptr[i]; e < ce; e++) keep[e] = 1;
        if (nk >= 2)
            for (int a = 0; a < nk; a++) {
                const int k = idx[cb + a];
                for (int e = ptr[k] + 1; e < ptr[k + 1]; e++) {
                    const int j = idx[e];
                    int lo = 0, hi = nk;  // lower bound of j among i's children
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (idx[cb + mid] < j)
                            lo = mid + 1;
                        else
                            hi = mid;
                    }
                    if (lo < nk && idx[cb + lo] == j) keep[cb + lo] = 0;
                }
            }
        int c = 0;
        for (int e = ptr[i]; e < ce; e++) c += keep[e];
        alive[i] = c;
    }
}

// group of every node: owner[set[e]] = the group k with gptr[k] <= e < gptr[k + 1]
__global__ void k_owner(const int *__restrict__ gptr, const int *__restrict__ gset, int ng, int n, int *owner) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        int lo = 0, hi = ng;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (gptr[mid] <= e)
                lo = mid;
            else
                hi = mid;
        }
        owner[gset[e]] = lo;
    }
}

// one key per DAG entry: (group of the node) * ng + (group of the entry's node)
__global__ void k_pair_keys(const int *__restrict__ rows, const int *__restrict__ idx, const int *__restrict__ owner,
                            int m, unsigned long long ng, unsigned long long *keys) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x)
        keys[e] = (unsigned long long)owner[rows[e]] * ng + (unsigned long long)owner[idx[e]];
}

__global__ void k_split_keys(const unsigned long long *__restrict__ keys, const int *__restrict__ nkeys,
                             unsigned long long ng, int *idx, int *cnt) {
    const int m = *nkeys;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        idx[e] = (int)(keys[e] % ng);
        atomicAdd(cnt + (int)(keys[e] / ng), 1);
    }
}

// Kahn levels with the queue on the device. Level l's nodes sit in order[lo[l] .. lo[l] + lc[l]);
// the round for level l releases their children (the node's own entry skipped) and a child whose
// count drops to 1 (its own entry) is appended to level l + 1. Each round also writes lo[l + 1],
// so the rounds need no host round trip; a round past the last level finds lc[l] = 0 and returns.
__global__ void k_kahn_start(const int *__restrict__ indeg, int n, int *order, int *lc, int *level) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (indeg[i] == 1) {
            order[atomicAdd(lc + 1, 1)] = i;
            level[i] = 1;
        }
}

__global__ void k_kahn_round(const int *__restrict__ ptr, const int *__restrict__ idx, int *order, int *lo, int *lc,
                             int *indeg, int *level, int lvl) {
    const int start = lo[lvl], nf = lc[lvl];
    if (blockIdx.x == 0 && threadIdx.x == 0) lo[lvl + 1] = start + nf;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nf; q += gridDim.x * blockDim.x) {
        const int cur = order[start + q];
        for (int e = ptr[cur]; e < ptr[cur + 1]; e++) {
            const int c = idx[e];
            if (c == cur) continue;
            if (atomicSub(indeg + c, 1) == 2) {
                order[start + nf + atomicAdd(lc + lvl + 1, 1)] = c;
                level[c] = lvl + 1;
            }
        }
    }
}

__global__ void k_iota(int *v, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

}  // namespace

// Buffers come from a stream-ordered pool of this analysis's own (cudaMallocFromPoolAsync): a
// release returns memory to the pool without synchronising, and the pool keeps it for the next
// stage; destroying the pool at the end hands everything back.
struct DeviceStages::Impl {
    cudaStream_t st = nullptr;
    cudaMemPool_t pool = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
};

DeviceStages::DeviceStages() : impl_(new Impl()) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaStreamCreateWithFlags(&impl_->st, cudaStreamNonBlocking) != cudaSuccess) {
        fail("no CUDA device for the device analysis");
        return;
    }
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    unsigned long long keep = ~0ull;
    if (cudaMemPoolCreate(&impl_->pool, &props) != cudaSuccess ||
        cudaMemPoolSetAttribute(impl_->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess)
        fail("memory pool");
}

DeviceStages::~DeviceStages() {
    if (impl_->st) cudaStreamSynchronize(impl_->st);
    if (impl_->pool) cudaMemPoolDestroy(impl_->pool);  // frees every buffer still allocated from it
    if (impl_->st) cudaStreamDestroy(impl_->st);
    delete impl_;
}

bool DeviceStages::fail(const char *what) {
    if (err.empty()) {
        const cudaError_t e = cudaGetLastError();
        err = std::string("device analysis: ") + what + (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : "");
    }
    return false;
}

bool DeviceStages::check(const char *what) {
    if (!ok()) return false;
    const cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? true : fail(what);
}

void *DeviceStages::alloc(size_t bytes) {
    if (!ok()) return nullptr;
    void *p = nullptr;
    if (cudaMallocFromPoolAsync(&p, bytes ? bytes : 4, impl_->pool, impl_->st) != cudaSuccess) {
        fail("device allocation");
        return nullptr;
    }
    return p;
}

void DeviceStages::release(void *p) {
    if (p && impl_->st) cudaFreeAsync(p, impl_->st);
}

void DeviceStages::release(Graph &g) {
    release(g.ptr);
    release(g.idx);
    g = Graph();
}

void *DeviceStages::scratch(size_t bytes) {
    if (!ok()) return nullptr;
    if (bytes > impl_->tmp_bytes) {
        release(impl_->tmp);  // stream-ordered: the work queued before still sees the old buffer
        impl_->tmp = alloc(bytes);
        impl_->tmp_bytes = impl_->tmp ? bytes : 0;
    }
    return impl_->tmp;
}

// ptr[0..n] = exclusive scan of cnt[0..n) with cnt[n] = 0 (so ptr[n] = the total)
bool DeviceStages::scan(int *cnt, int *ptr, int n) {
    if (!ok()) return false;
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt, ptr, n + 1, impl_->st);
    void *t = scratch(bytes);
    if (!t) return false;
    cub::DeviceScan::ExclusiveSum(t, bytes, cnt, ptr, n + 1, impl_->st);
    return check("scan");
}

DeviceStages::Graph DeviceStages::upload(const std::vector<int> &ptr, const std::vector<int> &idx) {
    Graph g;
    g.n = (int)ptr.size() - 1;
    g.m = (int)idx.size();
    g.ptr = (int *)alloc(sizeof(int) * ptr.size());
    g.idx = (int *)alloc(sizeof(int) * (size_t)g.m);
    if (!ok()) return Graph();
    if (cudaMemcpyAsync(g.ptr, ptr.data(), sizeof(int) * ptr.size(), cudaMemcpyHostToDevice, impl_->st) != cudaSuccess ||
        (g.m && cudaMemcpyAsync(g.idx, idx.data(), sizeof(int) * (size_t)g.m, cudaMemcpyHostToDevice, impl_->st) != cudaSuccess))
        fail("upload");
    return g;
}

bool DeviceStages::download(const Graph &g, std::vector<int> &ptr, std::vector<int> &idx) {
    if (!ok()) return false;
    ptr.resize((size_t)g.n + 1);
    idx.resize((size_t)g.m);
    if (cudaMemcpyAsync(ptr.data(), g.ptr, sizeof(int) * ptr.size(), cudaMemcpyDeviceToHost, impl_->st) != cudaSuccess ||
        (g.m && cudaMemcpyAsync(idx.data(), g.idx, sizeof(int) * (size_t)g.m, cudaMemcpyDeviceToHost, impl_->st) != cudaSuccess) ||
        cudaStreamSynchronize(impl_->st) != cudaSuccess)
        return fail("download");
    return true;
}

// Transpose of a square pattern: a stable sort of the entries (in row-major order) by column puts
// each column's rows in ascending order, as the host's scatter in increasing row order does.
DeviceStages::Graph DeviceStages::transpose(const Graph &g) {
    Graph t;
    const int n = g.n, m = g.m;
    int *rows = (int *)alloc(sizeof(int) * (size_t)m), *keys = (int *)alloc(sizeof(int) * (size_t)m);
    int *cnt = (int *)alloc(sizeof(int) * ((size_t)n + 1));
    t.n = n;
    t.m = m;
    t.ptr = (int *)alloc(sizeof(int) * ((size_t)n + 1));
    t.idx = (int *)alloc(sizeof(int) * (size_t)m);
    if (!ok()) return Graph();
    cudaStream_t st = impl_->st;
    cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)n + 1), st);
    if (m > 0) {
        k_entry_rows<<<grid_for(m), kAnBlock, 0, st>>>(g.ptr, n, m, rows);
        k_count<<<grid_for(m), kAnBlock, 0, st>>>(g.idx, m, cnt);
        size_t bytes = 0;
        const int eb = nbits((unsigned long long)std::max(n - 1, 1));
        cub::DeviceRadixSort::SortPairs(nullptr, bytes, g.idx, keys, rows, t.idx, m, 0, eb, st);
        void *tmp = scratch(bytes);
        if (!tmp) return Graph();
        cub::DeviceRadixSort::SortPairs(tmp, bytes, g.idx, keys, rows, t.idx, m, 0, eb, st);
    }
    scan(cnt, t.ptr, n);
    release(rows);
    release(keys);
    release(cnt);
    if (!check("transpose")) return Graph();
    return t;
}

DeviceStages::Graph DeviceStages::two_hop(const Graph &dag) {
    Graph r;
    const int n = dag.n, m = dag.m;
    unsigned char *keep = (unsigned char *)alloc((size_t)m);
    int *alive = (int *)alloc(sizeof(int) * ((size_t)n + 1)), *nsel = (int *)alloc(sizeof(int));
    r.n = n;
    r.ptr = (int *)alloc(sizeof(int) * ((size_t)n + 1));
    r.idx = (int *)alloc(sizeof(int) * (size_t)m);
    if (!ok()) return Graph();
    cudaStream_t st = impl_->st;
    cudaMemsetAsync(alive, 0, sizeof(int) * ((size_t)n + 1), st);
    k_two_hop<<<grid_for(n), kAnBlock, 0, st>>>(dag.ptr, dag.idx, n, keep, alive);
    scan(alive, r.ptr, n);
    size_t bytes = 0;
    cub::DeviceSelect::Flagged(nullptr, bytes, dag.idx, keep, r.idx, nsel, m, st);
    void *tmp = scratch(bytes);
    if (!tmp) return Graph();
    cub::DeviceSelect::Flagged(tmp, bytes, dag.idx, keep, r.idx, nsel, m, st);
    if (cudaMemcpyAsync(&r.m, r.ptr + n, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        fail("two-hop reduction");
    release(keep);
    release(alive);
    release(nsel);
    if (!check("two-hop reduction")) return Graph();
    return r;
}

DeviceStages::Graph DeviceStages::group_dag(const Graph &dag, const std::vector<int> &gptr, const std::vector<int> &gset) {
    Graph out;
    const int n = dag.n, m = dag.m, ng = (int)gptr.size() - 1;
    if ((int)gset.size() != n || ng < 1) {
        fail("group_dag: the grouping does not cover the DAG's nodes");
        return out;
    }
    Graph grp = upload(gptr, gset);
    int *owner = (int *)alloc(sizeof(int) * (size_t)n), *rows = (int *)alloc(sizeof(int) * (size_t)m);
    unsigned long long *keys = (unsigned long long *)alloc(sizeof(unsigned long long) * (size_t)m);
    unsigned long long *sorted = (unsigned long long *)alloc(sizeof(unsigned long long) * (size_t)m);
    unsigned long long *uniq = (unsigned long long *)alloc(sizeof(unsigned long long) * (size_t)m);
    int *nuniq = (int *)alloc(sizeof(int)), *cnt = (int *)alloc(sizeof(int) * ((size_t)ng + 1));
    out.n = ng;
    out.ptr = (int *)alloc(sizeof(int) * ((size_t)ng + 1));
    if (!ok()) return Graph();
    cudaStream_t st = impl_->st;
    const unsigned long long NG = (unsigned long long)ng;
    k_owner<<<grid_for(n), kAnBlock, 0, st>>>(grp.ptr, grp.idx, ng, n, owner);
    k_entry_rows<<<grid_for(m), kAnBlock, 0, st>>>(dag.ptr, n, m, rows);
    k_pair_keys<<<grid_for(m), kAnBlock, 0, st>>>(rows, dag.idx, owner, m, NG, keys);
    const int eb = nbits(NG * NG - 1);
    size_t b1 = 0, b2 = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, b1, keys, sorted, m, 0, eb, st);
    cub::DeviceSelect::Unique(nullptr, b2, sorted, uniq, nuniq, m, st);
    void *tmp = scratch(std::max(b1, b2));
    if (!tmp) return Graph();
    cub::DeviceRadixSort::SortKeys(tmp, b1, keys, sorted, m, 0, eb, st);
    cub::DeviceSelect::Unique(tmp, b2, sorted, uniq, nuniq, m, st);
    int mu = 0;
    if (cudaMemcpyAsync(&mu, nuniq, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        fail("group DAG");
        return Graph();
    }
    out.m = mu;
    out.idx = (int *)alloc(sizeof(int) * (size_t)mu);
    if (!ok()) return Graph();
    cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)ng + 1), st);
    k_split_keys<<<grid_for(mu), kAnBlock, 0, st>>>(uniq, nuniq, NG, out.idx, cnt);
    scan(cnt, out.ptr, ng);
    release(grp);
    for (void *p : {(void *)owner, (void *)rows, (void *)keys, (void *)sorted, (void *)uniq, (void *)nuniq, (void *)cnt})
        release(p);
    if (!check("group DAG")) return Graph();
    return out;
}

int DeviceStages::levels(const Graph &dag, std::vector<int> &node_to_level, std::vector<int> &perm_to_orig,
                         std::vector<int> &level_ptr) {
    constexpr int kRoundsPerCheck = 16;  // rounds queued between two reads of the frontier size
    const int n = dag.n, m = dag.m;
    const size_t nl = (size_t)n + kRoundsPerCheck + 2;  // levels <= n, plus the rounds past the end
    int *indeg = (int *)alloc(sizeof(int) * (size_t)n), *lev = (int *)alloc(sizeof(int) * (size_t)n);
    int *order = (int *)alloc(sizeof(int) * (size_t)n), *lo = (int *)alloc(sizeof(int) * nl);
    int *lc = (int *)alloc(sizeof(int) * nl), *nodes = (int *)alloc(sizeof(int) * (size_t)n);
    int *lsorted = (int *)alloc(sizeof(int) * (size_t)n), *perm = (int *)alloc(sizeof(int) * (size_t)n);
    if (!ok()) return 0;
    cudaStream_t st = impl_->st;
    cudaMemsetAsync(indeg, 0, sizeof(int) * (size_t)n, st);
    cudaMemsetAsync(lev, 0, sizeof(int) * (size_t)n, st);
    cudaMemsetAsync(lo, 0, sizeof(int) * nl, st);
    cudaMemsetAsync(lc, 0, sizeof(int) * nl, st);
    k_count<<<grid_for(m), kAnBlock, 0, st>>>(dag.idx, m, indeg);
    k_kahn_start<<<grid_for(n), kAnBlock, 0, st>>>(indeg, n, order, lc, lev);
    const int grid = grid_for(n);
    int lvl = 1, last = 0;
    std::vector<int> counts(kRoundsPerCheck);
    while (ok()) {
        for (int r = 0; r < kRoundsPerCheck; r++)
            k_kahn_round<<<grid, kAnBlock, 0, st>>>(dag.ptr, dag.idx, order, lo, lc, indeg, lev, lvl + r);
        // sizes of levels lvl+1 .. lvl+16: the last non-empty one so far, and whether any is empty
        if (cudaMemcpyAsync(counts.data(), lc + lvl + 1, sizeof(int) * kRoundsPerCheck, cudaMemcpyDeviceToHost, st) !=
                cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            fail("levels");
            return 0;
        }
        bool end = false;
        for (int r = 0; r < kRoundsPerCheck && !end; r++) {
            if (counts[r] == 0)
                end = true;
            else
                last = lvl + r + 1;
        }
        if (lvl == 1) last = std::max(last, 1);
        lvl += kRoundsPerCheck;
        if (end) break;
        if (lvl > n + 1) {
            fail("levels: more levels than nodes");
            return 0;
        }
    }
    if (!ok()) return 0;
    const int nlev = last;
    // nodes ascending inside each level: a stable sort of 0..n-1 by level
    k_iota<<<grid_for(n), kAnBlock, 0, st>>>(nodes, n);
    size_t bytes = 0;
    const int eb = nbits((unsigned long long)nlev);
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, lev, lsorted, nodes, perm, n, 0, eb, st);
    void *tmp = scratch(bytes);
    if (!tmp) return 0;
    cub::DeviceRadixSort::SortPairs(tmp, bytes, lev, lsorted, nodes, perm, n, 0, eb, st);
    node_to_level.resize(n);
    perm_to_orig.resize(n);
    if (cudaMemcpyAsync(node_to_level.data(), lev, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(perm_to_orig.data(), perm, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        fail("levels");
        return 0;
    }
    level_ptr.assign((size_t)nlev + 1, 0);
    for (int i = 0; i < n; i++) {
        const int l = node_to_level[i];
        if (l < 1 || l > nlev) {  // a node no round released: the DAG has a cycle
            fail("levels: the DAG has a cycle");
            return 0;
        }
        level_ptr[l]++;
    }
    for (int l = 0; l < nlev; l++) level_ptr[l + 1] += level_ptr[l];
    for (void *p : {(void *)indeg, (void *)lev, (void *)order, (void *)lo, (void *)lc, (void *)nodes, (void *)lsorted,
                    (void *)perm})
        release(p);
    return nlev;
}

}  // namespace baas
