// Host-side BAAS schedule (see schedule.hpp for the stage list and reference citations).
//
// Data structures are flat CSR-like vectors; the reference's std::list queues become FIFO
// vectors with a read cursor (same visiting order). Where the reference's output depends on
// the library's algorithm choice (std::nth_element tie order, merge/LevelTask.cpp:2482) the
// same standard-library call is made on the same inputs.
#include "schedule.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstdint>
#include <limits>
#include <memory>
#include <numeric>
#include <thread>
#include <unordered_set>

namespace baas {
namespace {


struct Csx {  // compressed sparse rows or columns
    std::vector<int> ptr, idx;
    int n() const { return (int)ptr.size() - 1; }
    int len(int i) const { return ptr[i + 1] - ptr[i]; }
};

// Transpose of an n x n pattern. Entries are scattered in increasing source order, so every
// output row comes out ascending -- what DAG::inverseDAG's per-row quicksort and dcsr2csc's
// per-column quicksort produce for duplicate-free rows (spm/DAG.cpp:481-564, spm/CSR.cpp:914-950).
Csx transpose(const Csx &a) {
    const int n = a.n();
    Csx t;
    t.ptr.assign(n + 1, 0);
    t.idx.resize(a.idx.size());
    for (int v : a.idx) t.ptr[v + 1]++;
    for (int i = 0; i < n; i++) t.ptr[i + 1] += t.ptr[i];
    std::vector<int> cur(t.ptr.begin(), t.ptr.end() - 1);
    for (int i = 0; i < n; i++)
        for (int e = a.ptr[i]; e < a.ptr[i + 1]; e++) t.idx[cur[a.idx[e]]++] = i;
    return t;
}

// Stage 2: drop edge i->j when a child k of i also has j as a child (one hop through the
// unpruned DAG). Column i's own entry (first, the diagonal) is never dropped.
Csx two_hop_reduce(const Csx &dag) {
    const int n = dag.n();
    std::vector<uint8_t> dead(dag.idx.size(), 0);
    for (int i = 0; i < n; i++) {
        const int cb = dag.ptr[i] + 1, ce = dag.ptr[i + 1];
        if (ce - cb < 2) continue;  // a single child cannot be reached through a sibling
        const int *kids = dag.idx.data() + cb;
        const int nk = ce - cb;
        for (int a = 0; a < nk; a++) {
            const int k = kids[a];
            for (int e = dag.ptr[k] + 1; e < dag.ptr[k + 1]; e++) {
                const int j = dag.idx[e];
                const int *hit = std::lower_bound(kids, kids + nk, j);
                if (hit != kids + nk && *hit == j) dead[cb + (hit - kids)] = 1;
            }
        }
    }
    Csx out;
    out.ptr.assign(n + 1, 0);
    out.idx.reserve(dag.idx.size());
    for (int i = 0; i < n; i++) {
        for (int e = dag.ptr[i]; e < dag.ptr[i + 1]; e++)
            if (!dead[e]) out.idx.push_back(dag.idx[e]);
        out.ptr[i + 1] = (int)out.idx.size();
    }
    return out;
}

struct Grouping {
    int ngroups = 0;
    std::vector<int> ptr, set;
};

// Counting-sort relabel of BFS groups by a representative node (max for reverse trees, min for
// forward trees); nodes keep their BFS order inside a group (merge/Coarsen.cpp:345-398, :176-224).
void relabel_groups(int n, Grouping &g, bool by_max) {
    std::vector<int> gid(n, 0), cnt(n + 1, 0);
    for (int k = 0; k < g.ngroups; k++) {
        int id = by_max ? 0 : n;
        for (int e = g.ptr[k]; e < g.ptr[k + 1]; e++) {
            const int v = g.set[e];
            if (by_max ? (v > id) : (v < id)) id = v;
        }
        cnt[id + 1] = g.ptr[k + 1] - g.ptr[k];
        for (int e = g.ptr[k]; e < g.ptr[k + 1]; e++) gid[g.set[e]] = id;
    }
    for (int i = 1; i < n; i++) cnt[i + 1] += cnt[i];
    std::vector<int> ptr;
    ptr.reserve(g.ngroups + 1);
    ptr.push_back(0);
    for (int i = 0; i < n; i++)
        if (cnt[i + 1] != cnt[i]) ptr.push_back(cnt[i + 1]);
    std::vector<int> set(n);
    for (int i = 0; i < n; i++) set[cnt[gid[g.set[i]]]++] = g.set[i];
    g.ptr.swap(ptr);
    g.set.swap(set);
}

// Stages 3 and 5: BFS tree coarsening. `reverse` grows groups from sinks towards parents that
// have exactly one child; otherwise from sources towards children that have exactly one parent.
// `inv_pre`: dag's transpose when the caller has it already (the device stages make it).
Grouping tree_coarsen(const Csx &dag, bool reverse, const Csx *inv_pre = nullptr) {
    const int n = dag.n();
    Csx inv_own;
    if (!inv_pre) inv_own = transpose(dag);
    const Csx &inv = inv_pre ? *inv_pre : inv_own;
    const Csx &up = reverse ? inv : dag;    // where the next tree members come from
    const Csx &down = reverse ? dag : inv;  // whose length decides "single edge" (self + 1)

    std::vector<int> roots;
    roots.reserve(n);
    for (int i = 0; i < n; i++)
        if ((reverse ? dag.len(i) : inv.len(i)) == 1) roots.push_back(i);
    size_t rhead = 0;

    Grouping g;
    g.set.resize(n);
    g.ptr.reserve(n + 1);
    std::vector<uint8_t> visited(n, 0);
    std::vector<int> fifo;
    fifo.reserve(n);
    std::vector<int> found;
    int cnt = 0;
    while (rhead < roots.size()) {
        int head = roots[rhead++];
        visited[head] = 1;
        fifo.clear();
        fifo.push_back(head);
        size_t fhead = 0;
        g.ptr.push_back(cnt);
        g.ngroups++;
        while (fhead < fifo.size()) {
            head = fifo[fhead++];
            g.set[cnt++] = head;
            found.clear();
            bool tree = true;
            // parents of head = its inverse row without the trailing self entry; children of
            // head = its CSC column without the leading self entry
            const int b = reverse ? up.ptr[head] : up.ptr[head] + 1;
            const int e = reverse ? up.ptr[head + 1] - 1 : up.ptr[head + 1];
            for (int q = b; q < e; q++) {
                const int v = up.idx[q];
                if (visited[v]) continue;
                visited[v] = 1;
                found.push_back(v);
                if (down.len(v) != 2) tree = false;
            }
            if (tree)
                fifo.insert(fifo.end(), found.begin(), found.end());
            else
                roots.insert(roots.end(), found.begin(), found.end());
        }
    }
    if (g.ptr.empty() || g.ptr.back() != cnt) g.ptr.push_back(cnt);
    relabel_groups(n, g, /*by_max=*/reverse);
    return g;
}

// Stage 4: DAG between groups: every child of every member, mapped to its group, sorted, unique.
Csx group_dag(int n, const Grouping &g, const Csx &dag) {
    std::vector<int> owner(n);
    for (int k = 0; k < g.ngroups; k++)
        for (int e = g.ptr[k]; e < g.ptr[k + 1]; e++) owner[g.set[e]] = k;
    Csx out;
    out.ptr.assign(g.ngroups + 1, 0);
    std::vector<int> tmp;
    for (int k = 0; k < g.ngroups; k++) {
        tmp.clear();
        for (int e = g.ptr[k]; e < g.ptr[k + 1]; e++) {
            const int v = g.set[e];
            for (int q = dag.ptr[v]; q < dag.ptr[v + 1]; q++) tmp.push_back(owner[dag.idx[q]]);
        }
        std::sort(tmp.begin(), tmp.end());
        tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
        out.idx.insert(out.idx.end(), tmp.begin(), tmp.end());
        out.ptr[k + 1] = (int)out.idx.size();
    }
    return out;
}

// Stage 7: Kahn BFS levels where a node is ready at in-degree 1 (its own diagonal entry).
void level_sets(const Csx &dag, HostSchedule &s) {
    const int n = dag.n();
    std::vector<int> indeg(n, 0);
    for (int v : dag.idx) indeg[v]++;
    std::vector<int> q(n);
    int rear = 0;
    for (int i = 0; i < n; i++)
        if (indeg[i] == 1) q[rear++] = i;
    std::vector<int> lptr(n + 1, 0);
    s.node_to_level.assign(n, 1);
    int front = 0, lvl = 0;
    while (front < rear) {
        const int stop = rear;
        lvl++;
        while (front < stop) {
            const int cur = q[front++];
            s.node_to_level[cur] = lvl;
            for (int e = dag.ptr[cur]; e < dag.ptr[cur + 1]; e++) {
                const int c = dag.idx[e];
                if (c == cur) continue;
                if (--indeg[c] == 1) q[rear++] = c;
            }
        }
        lptr[lvl] = front;
    }
    s.nlevels = lvl;
    s.level_ptr.assign(lptr.begin(), lptr.begin() + lvl + 1);
    s.exec_level_ptr = s.level_ptr;
    for (int l = 0; l < lvl; l++) std::sort(q.begin() + s.level_ptr[l], q.begin() + s.level_ptr[l + 1]);
    s.perm_to_orig.assign(q.begin(), q.begin() + n);
    s.perm.assign(n, 0);
    for (int i = 0; i < n; i++) s.perm[s.perm_to_orig[i]] = i;
}

// Stages 2-7 of a block-diagonal pattern (systems at rows off[q] .. off[q + 1]), system by system on
// host threads, concatenated into s (groups, their rows, the final group DAG, the level set) and
// fdag. No DAG edge joins two systems, so every stage restricted to one system is that system's own:
// a tree grows from a root of its system, and each system's roots are visited in the same relative
// order as in the whole pattern's BFS (initial roots ascending, then appended roots in discovery
// order); relabel_groups orders groups by a representative row, which keeps the systems in row
// order; the Kahn levels of independent DAGs are the unions of their levels, nodes ascending. The
// concatenation is therefore identical to the whole pattern's stages 2-7.
void split_stages(HostSchedule &s, const std::vector<int> &off, Csx &fdag) {
    const int ns = (int)off.size() - 1;
    struct Part {
        std::vector<int> gptr, gset;
        Csx fdag;
        HostSchedule lv;
    };
    std::vector<Part> parts(ns);
    auto work = [&](int q) {
        const int r0 = off[q], m = off[q + 1] - off[q];
        const int e0 = s.l_rowptr[r0];
        Csx lower;
        lower.ptr.resize(m + 1);
        for (int i = 0; i <= m; i++) lower.ptr[i] = s.l_rowptr[r0 + i] - e0;
        lower.idx.resize(lower.ptr[m]);
        for (int e = 0; e < lower.ptr[m]; e++) lower.idx[e] = s.l_colidx[e0 + e] - r0;
        const Csx dag = two_hop_reduce(transpose(lower));
        const Grouping rev = tree_coarsen(dag, true);
        const Csx gdag = group_dag(m, rev, dag);
        const Grouping fwd = tree_coarsen(gdag, false);
        Part &P = parts[q];
        P.gptr.assign(1, 0);
        for (int f = 0; f < fwd.ngroups; f++) {
            for (int t = fwd.ptr[f]; t < fwd.ptr[f + 1]; t++) {
                const int g = fwd.set[t];
                for (int e = rev.ptr[g]; e < rev.ptr[g + 1]; e++) P.gset.push_back(rev.set[e] + r0);
            }
            P.gptr.push_back((int)P.gset.size());
        }
        P.fdag = group_dag(rev.ngroups, fwd, gdag);
        level_sets(P.fdag, P.lv);
    };
    const int nt = std::max(1, std::min<int>(ns, (int)std::thread::hardware_concurrency()));
    std::atomic<int> next(0);
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; t++)
        pool.emplace_back([&] {
            for (int q = next++; q < ns; q = next++) work(q);
        });
    for (auto &t : pool) t.join();

    std::vector<int> goff(ns + 1, 0);
    int nlev = 0;
    for (int q = 0; q < ns; q++) {
        goff[q + 1] = goff[q] + (int)parts[q].gptr.size() - 1;
        nlev = std::max(nlev, parts[q].lv.nlevels);
    }
    const int ng = goff[ns];
    s.ngroups = ng;
    s.group_ptr.assign(1, 0);
    s.group_set.clear();
    fdag.ptr.assign(1, 0);
    fdag.idx.clear();
    s.node_to_level.clear();
    for (int q = 0; q < ns; q++) {
        const Part &P = parts[q];
        const int base = (int)s.group_set.size();
        for (size_t g = 1; g < P.gptr.size(); g++) s.group_ptr.push_back(base + P.gptr[g]);
        s.group_set.insert(s.group_set.end(), P.gset.begin(), P.gset.end());
        for (int g = 0; g + 1 < (int)P.fdag.ptr.size(); g++) {
            for (int e = P.fdag.ptr[g]; e < P.fdag.ptr[g + 1]; e++) fdag.idx.push_back(P.fdag.idx[e] + goff[q]);
            fdag.ptr.push_back((int)fdag.idx.size());
        }
        s.node_to_level.insert(s.node_to_level.end(), P.lv.node_to_level.begin(), P.lv.node_to_level.end());
    }
    s.nlevels = nlev;
    s.level_ptr.assign(nlev + 1, 0);
    s.perm_to_orig.clear();
    s.perm_to_orig.reserve(ng);
    for (int l = 0; l < nlev; l++) {
        for (int q = 0; q < ns; q++) {
            const HostSchedule &L = parts[q].lv;
            if (l >= L.nlevels) continue;
            for (int p = L.level_ptr[l]; p < L.level_ptr[l + 1]; p++) s.perm_to_orig.push_back(L.perm_to_orig[p] + goff[q]);
        }
        s.level_ptr[l + 1] = (int)s.perm_to_orig.size();
    }
    s.exec_level_ptr = s.level_ptr;
    s.perm.assign(ng, 0);
    for (int i = 0; i < ng; i++) s.perm[s.perm_to_orig[i]] = i;
}

// Stage 8: merge/LevelMerge.cpp:118-262.
void threads_per_level(HostSchedule &s) {
    const int nl = s.nlevels, nc = s.nthread;
    s.nthread_per_level.assign(nl, 1);
    if (nl == 1) {
        s.nthread_per_level[0] = std::min(s.level_ptr[1] - s.level_ptr[0], nc);
        return;
    }
    for (int l = 0; l < nl; l++) {
        const int groups = s.level_ptr[l + 1] - s.level_ptr[l];
        int rows = 0;
        long long nnz = 0;
        for (int p = s.level_ptr[l]; p < s.level_ptr[l + 1]; p++) {
            const int g = s.perm_to_orig[p];
            rows += s.group_ptr[g + 1] - s.group_ptr[g];
            if (s.kind == SchedKind::SpTRSV || s.kind == SchedKind::ICCG)
                for (int e = s.group_ptr[g]; e < s.group_ptr[g + 1]; e++) {
                    const int r = s.group_set[e];
                    nnz += s.a_rowptr[r + 1] - s.a_rowptr[r];
                }
        }
        int t;
        if (s.kind == SchedKind::SpTRSV || s.kind == SchedKind::ICCG) {
            const int inz = (int)nnz;
            if (rows < 16 || groups <= 4 || inz < 32) {
                t = 1;
            } else {
                const int avg = (rows + 7) / 8;
                t = std::min(std::min(std::max(inz / 32, avg), groups), nc);
            }
        } else {  // IC0 and ILU0 share one rule
            if (rows < 4 || groups <= 2) {
                t = 1;
            } else {
                const int avg = (rows + 1) / 2;
                t = std::min(std::min(avg, groups), nc);
            }
        }
        s.nthread_per_level[l] = t;
    }
}

// The level merge of level_merge_group / level_merge_group_TRSV (merge/LevelMerge.cpp:313-421) on
// per-level thread counts `t`: consecutive single-thread levels are merged by the reference's
// two-pointer scan, and the merged levels number their groups from 0 (constructLevelMerge
// :423-452).
void merge_levels(HostSchedule &s, std::vector<int> t) {
    const int nl = s.nlevels;
    const std::vector<int> lp = s.level_ptr;
    std::vector<int> mptr(nl + 1, 0);
    int m = 0;
    for (int i = 1; i < nl;) {
        if (t[i] == 1 && t[i] == t[m]) {
            i++;
        } else {
            m++;
            t[m] = t[i];
            mptr[m] = lp[i];
            i++;
        }
    }
    m++;
    mptr[m] = lp[nl];
    s.nlevels = m;
    s.level_ptr.assign(mptr.begin(), mptr.begin() + m + 1);
    s.nthread_per_level.assign(t.begin(), t.begin() + m);
    for (int l = 0; l < m; l++)
        for (int j = s.level_ptr[l]; j < s.level_ptr[l + 1]; j++) s.node_to_level[s.perm_to_orig[j]] = l;
}

// Stages 8-9 of the cost-split mapping, the Scheduler's P2P algorithm (test/Schedule.hpp:233-240,
// 263-265): level_merge_group (merge/LevelMerge.cpp:367-421) with threads per level by
// level_nthreads_group (:282-311; rule :102-114: one thread below 40 rows or at most 12 groups,
// else max(ceil(rows / 10), groups) capped by the thread count; a single level gets
// min(groups, threads)).
void merge_levels_group(HostSchedule &s) {
    const int nl = s.nlevels, nc = s.nthread;
    const std::vector<int> &lp = s.level_ptr;
    std::vector<int> t(nl, 1);
    if (nl == 1) {
        t[0] = std::min(lp[1] - lp[0], nc);
    } else {
        for (int l = 0; l < nl; l++) {
            const int groups = lp[l + 1] - lp[l];
            int rows = 0;
            for (int p = lp[l]; p < lp[l + 1]; p++) {
                const int g = s.perm_to_orig[p];
                rows += s.group_ptr[g + 1] - s.group_ptr[g];
            }
            t[l] = (rows < 40 || groups <= 12) ? 1 : std::min(std::max((rows + 9) / 10, groups), nc);
        }
    }
    merge_levels(s, std::move(t));
}

// level_nthreads_base (merge/LevelMerge.cpp:265-279): as many threads as groups, at most nthread.
void threads_per_level_base(HostSchedule &s) {
    s.nthread_per_level.assign(s.nlevels, 1);
    for (int l = 0; l < s.nlevels; l++)
        s.nthread_per_level[l] = std::min(s.level_ptr[l + 1] - s.level_ptr[l], s.nthread);
}

// Task::constructTask (merge/LevelTask.cpp:42-196): each level's groups are cut into up to
// nthread_per_level contiguous ranges of about equal cost (a lower_bound on the level's running
// cost for multiples of ceil-divided load; a search that starts past the level's end finds
// nothing, as std::lower_bound does on an empty range), one task per non-empty range of a thread
// (barrier: one task per level and thread, empty or not).
void cost_split_map(HostSchedule &s, bool barrier) {
    const int nl = s.nlevels, nt = s.nthread, nodes = s.ngroups;
    const int *lp = s.level_ptr.data();
    const int *p2o = s.perm_to_orig.data();
    std::vector<std::pair<int, int>> rows((size_t)nl * nt);
    std::vector<double> cb((size_t)nodes + nt, 0.0);
    for (int l = 0; l < nl; l++) {
        const int exec = s.nthread_per_level[l], lb = lp[l], le = lp[l + 1];
        double load = 0;
        for (int i = lb; i < le; i++) {
            cb[i] = load;
            load += s.cost[p2o[i]];
        }
        const double per = (load + exec - 1) / exec;
        int pre = lb, r = lb, t;
        for (t = 0; t < exec; t++) {
            const int nr = r <= le ? (int)(std::lower_bound(cb.begin() + r, cb.begin() + le, (t + 1) * per) - cb.begin()) : r;
            r = nr;
            const int b = pre, e = std::min(r, le);
            pre = e;
            rows[(size_t)t * nl + l] = {b, e};
            ++r;
        }
        for (t = exec; t < nt; t++) rows[(size_t)t * nl + l] = {le, le};
    }
    std::vector<int> rsum(nt + 1, 0);
    s.thread_boundaries.assign(nt + 1, 0);
    for (int tid = 0; tid < nt; tid++) {
        int sum = 0, cnt = 0;
        for (int l = 0; l < nl; l++) {
            const int d = rows[(size_t)tid * nl + l].second - rows[(size_t)tid * nl + l].first;
            sum += d;
            if (barrier || d) cnt++;
        }
        rsum[tid + 1] = sum;
        s.thread_boundaries[tid + 1] = cnt;
    }
    for (int tid = 0; tid < nt; tid++) {
        rsum[tid + 1] += rsum[tid];
        s.thread_boundaries[tid + 1] += s.thread_boundaries[tid];
    }
    s.ntasks = s.thread_boundaries[nt];
    s.task_boundaries.assign(s.ntasks + 1, 0);
    s.thread_cont_to_orig.assign(nodes, 0);
    s.orig_to_thread_cont.assign(nodes, 0);
    for (int tid = 0; tid < nt; tid++) {
        int off = rsum[tid], task = s.thread_boundaries[tid];
        for (int l = 0; l < nl; l++) {
            const auto &rg = rows[(size_t)tid * nl + l];
            if (!barrier && rg.second <= rg.first) continue;
            s.task_boundaries[task++] = off;
            for (int j = rg.first; j < rg.second; j++) {
                s.orig_to_thread_cont[p2o[j]] = off;
                s.thread_cont_to_orig[off] = p2o[j];
                off++;
            }
        }
    }
    s.task_boundaries[s.ntasks] = nodes;
}

// The common end of the level-by-level mappers (four-rule, finish-time): runs of consecutive
// single-thread levels merge into the run's first task (merge/LevelTask.cpp:2646-2676, the same
// scan at :1858-1894), then taskMapToBoundaries (:198-304, non-barrier form) turns the per-level
// thread ranges of by_level_thread into thread/task boundaries and both permutations.
void finish_mapping(HostSchedule &s, std::vector<std::pair<int, int>> &task_rows, const std::vector<int> &by_level_thread,
                    std::vector<int> level_single) {
    const int nl = s.nlevels, nt = s.nthread, nodes = s.ngroups;
    {
        std::vector<int> run_start(nl + 1, 0), ntpl(s.nthread_per_level);
        int m = 0;
        for (int lvl = 1; lvl < nl;) {
            if (ntpl[lvl] == 1 && ntpl[m] == 1) {
                auto &pre = task_rows[(size_t)level_single[m] * nl + run_start[m]];
                auto &post = task_rows[(size_t)level_single[lvl] * nl + lvl];
                pre.second = post.second;
                post = {0, 0};
                lvl++;
            } else {
                m++;
                ntpl[m] = ntpl[lvl];
                level_single[m] = level_single[lvl];
                run_start[m] = lvl;
                lvl++;
            }
        }
    }

    // taskMapToBoundaries, non-barrier form (merge/LevelTask.cpp:198-304)
    std::vector<int> rows_before(nt + 1, 0);
    s.thread_boundaries.assign(nt + 1, 0);
    for (int t = 0; t < nt; t++) {
        int sum = 0, cnt = 0;
        for (int l = 0; l < nl; l++) {
            const auto &tr = task_rows[(size_t)t * nl + l];
            const int d = tr.second - tr.first;
            sum += d;
            if (d) ++cnt;
        }
        rows_before[t + 1] = sum;
        s.thread_boundaries[t + 1] = cnt;
    }
    for (int t = 0; t < nt; t++) {
        rows_before[t + 1] += rows_before[t];
        s.thread_boundaries[t + 1] += s.thread_boundaries[t];
    }
    s.ntasks = s.thread_boundaries[nt];
    s.task_boundaries.assign(s.ntasks + 1, 0);
    s.orig_to_thread_cont.assign(nodes, 0);
    s.thread_cont_to_orig.assign(nodes, 0);
    for (int t = 0; t < nt; t++) {
        int row = rows_before[t], task = s.thread_boundaries[t];
        for (int l = 0; l < nl; l++) {
            const auto &tr = task_rows[(size_t)t * nl + l];
            if (tr.second > tr.first) {
                s.task_boundaries[task++] = row;
                for (int j = tr.first; j < tr.second; j++) {
                    s.orig_to_thread_cont[by_level_thread[j]] = row;
                    s.thread_cont_to_orig[row] = by_level_thread[j];
                    row++;
                }
            }
        }
    }
    s.task_boundaries[s.ntasks] = nodes;
}


// Stage 9: four-rule mapping of groups to virtual threads, then the merge of consecutive
// single-thread levels and the conversion to thread/task boundaries.
//
// The reference computes the per-thread vote sums inside an OpenMP region whose threads split
// each level into ceil(width / nthread)-sized node ranges, then the master thread adds the
// per-range partial sums in range order (merge/LevelTask.cpp:2386-2469). That order is
// reproduced exactly; all-zero partials are skipped, which cannot change a sum of positive
// votes.
void four_rule_map(HostSchedule &s, const Csx &dag_csr) {
    const int nl = s.nlevels, nt = s.nthread, nodes = s.ngroups;
    const int *lp = s.level_ptr.data();
    const int *p2o = s.perm_to_orig.data();

    std::vector<int> by_level_thread(nodes);  // nodeByLevelThreadTask
    std::vector<int> node_thread(nodes, -1);  // origNodeToThread
    std::vector<std::pair<int, int>> task_rows((size_t)nl * nt);
    std::vector<int> level_single(nl, -1);    // levelThreadOne

    // level 0: cost-balanced contiguous split (merge/LevelTask.cpp:2325-2371)
    {
        const int et = s.nthread_per_level[0];
        const int lb = lp[0], le = lp[1];
        std::vector<double> pre(le - lb + 1);
        double load = 0.0;
        for (int i = lb; i < le; i++) {
            pre[i - lb] = load;
            load += s.cost[p2o[i]];
        }
        const double per = (load + et - 1) / et;
        int prev_end = lb, r = lb;
        if (et == 1) level_single[0] = 0;
        for (int t = 0; t < et; t++) {
            // lower_bound over [r, le); an empty or inverted range returns r
            int nr = r;
            if (r < le) nr = lb + (int)(std::lower_bound(pre.begin() + (r - lb), pre.begin() + (le - lb), (t + 1) * per) - pre.begin());
            r = nr;
            const int b = prev_end, e = std::min(r, le);
            prev_end = e;
            task_rows[(size_t)t * nl + 0] = {b, e};
            for (int k = b; k < e; k++) {
                by_level_thread[k] = p2o[k];
                node_thread[p2o[k]] = t;
            }
            ++r;
        }
        for (int t = et; t < nt; t++) task_rows[(size_t)t * nl + 0] = {le, le};
    }

    std::vector<double> sel(nt), part(nt), penalty(nt), local_load(nt), score(nt);
    std::vector<int> touched, idx(nt);
    std::vector<uint8_t> chosen(nt), in_touched(nt);
    std::vector<std::vector<int>> thread_nodes(nt);
    // per-node affinity towards each parent thread: (thread, sum) in first-seen order
    std::vector<int> aff_ptr;
    std::vector<int> aff_thr;
    std::vector<double> aff_val, aff_total;
    const ScoreParams &sp = s.score;
    const double pen0 = sp.load_beta * std::log(1.0 + (1.0 - 0.0));
    // the vote's two logarithms, computed once per group and per level distance (the same calls
    // on the same arguments give the same values)
    std::vector<double> log_size(nodes);
    for (int g = 0; g < nodes; g++) log_size[g] = std::log2(1.0 * (s.group_ptr[g + 1] - s.group_ptr[g] + 1));
    std::vector<double> log_diff(std::max(sp.level_window, 0) + 1);
    for (int d = 0; d <= std::max(sp.level_window, 0); d++) log_diff[d] = std::log2(d + 1);

    for (int lvl = 1; lvl < nl; lvl++) {
        const int lb = lp[lvl], le = lp[lvl + 1];
        const int et = s.nthread_per_level[lvl];
        const int width = le - lb;
        std::fill(sel.begin(), sel.end(), 0.0);
        std::fill(penalty.begin(), penalty.end(), pen0);
        std::fill(local_load.begin(), local_load.end(), 0.0);
        for (int t = 0; t < nt; t++) {
            idx[t] = t;
            thread_nodes[t].clear();
        }

        // votes, split into the reference's per-OpenMP-thread node ranges
        const int chunk = (width + nt - 1) / nt;
        aff_ptr.assign(width + 1, 0);
        aff_thr.clear();
        aff_val.clear();
        aff_total.assign(width, 0.0);
        double level_load = 0.0;
        for (int tid = 0; tid < nt; tid++) {
            const int rb = std::min(lb + chunk * tid, le);
            const int re = std::min(lb + chunk * (tid + 1), le);
            if (rb >= re) continue;
            touched.clear();
            for (int i = rb; i < re; i++) {
                const int node = p2o[i];
                const int nlev = s.node_to_level[node];
                level_load += s.cost[node];
                const int abeg = (int)aff_thr.size();
                for (int q = dag_csr.ptr[node]; q < dag_csr.ptr[node + 1] - 1; q++) {
                    const int par = dag_csr.idx[q];
                    const int rt = node_thread[par];
                    const int diff = nlev - s.node_to_level[par];
                    if (diff > sp.level_window) continue;
                    const double vote = sp.amplify * log_size[par] / log_diff[diff];
                    if (!in_touched[rt]) {
                        in_touched[rt] = 1;
                        part[rt] = 0.0;
                        touched.push_back(rt);
                    }
                    part[rt] += vote;
                    aff_total[i - lb] += vote;
                    int a = abeg;
                    while (a < (int)aff_thr.size() && aff_thr[a] != rt) a++;
                    if (a == (int)aff_thr.size()) {
                        aff_thr.push_back(rt);
                        aff_val.push_back(0.0);
                    }
                    aff_val[a] += vote;
                }
                aff_ptr[i - lb + 1] = (int)aff_thr.size();
            }
            for (int t : touched) {
                sel[t] += part[t];
                in_touched[t] = 0;
            }
        }
        // level_load is a sum of integer-valued costs, exact in any order
        const double avg = level_load / et;

        std::nth_element(idx.begin(), idx.begin() + et, idx.end(),
                         [&sel](int a, int b) { return sel[a] > sel[b]; });
        if (et == 1) level_single[lvl] = idx[0];
        std::fill(chosen.begin(), chosen.end(), 0);
        for (int k = 0; k < et; k++) chosen[idx[k]] = 1;

        for (int i = lb; i < le; i++) {
            const int node = p2o[i];
            const double total = aff_total[i - lb];
            const int ab = aff_ptr[i - lb], ae = aff_ptr[i - lb + 1];
            double best = std::numeric_limits<double>::lowest();
            int target = -1;
            for (int t = 0; t < nt; t++) {
                if (!chosen[t]) continue;
                double a = 0.0;
                for (int q = ab; q < ae; q++)
                    if (aff_thr[q] == t) {
                        a = aff_val[q];
                        break;
                    }
                score[t] = sp.award_alpha * (a / total) + penalty[t];
                if (score[t] > best) {
                    best = score[t];
                    target = t;
                }
            }
            thread_nodes[target].push_back(node);
            local_load[target] += s.cost[node];
            const double util = local_load[target] / avg;
            double pen;
            if (util < 1.0)
                pen = sp.load_beta * std::log(1.0 + (1.0 - util));
            else if (util > 1.05)
                pen = std::numeric_limits<double>::lowest();
            else
                pen = -sp.over_gamma * (std::exp(10 * (util - 1)) - 1);
            penalty[target] = pen;
        }

        int pos = lb;
        for (int t = 0; t < nt; t++) {
            auto &tr = task_rows[(size_t)t * nl + lvl];
            if (chosen[t]) {
                tr = {pos, pos + (int)thread_nodes[t].size()};
                for (int v : thread_nodes[t]) {
                    by_level_thread[pos++] = v;
                    node_thread[v] = t;
                }
            } else {
                tr = {pos, pos};
            }
        }
    }

    finish_mapping(s, task_rows, by_level_thread, level_single);
}

// Stage 9 of the finish-time mapping, the Scheduler's P2P_TIME algorithm
// (Task::constructMappingByFinishTime, merge/LevelTask.cpp:1647-1910). Level 0 is split by cost as
// in the four-rule mapping, and each thread accumulates its busy time. On every later level the
// nthread_per_level[l] threads that finish first are chosen (std::nth_element), every group's
// earliest start is the latest finish among its parents (held in an int, as the reference
// holds it), the groups are sorted by that start (std::sort) and each goes, in that order, to
// the chosen thread that finishes first (std::min_element), which advances that thread's time.
// The same standard-library calls on the same sequences give the reference's order also among
// ties.
void finish_time_map(HostSchedule &s, const Csx &dag_csr) {
    const int nl = s.nlevels, nt = s.nthread, nodes = s.ngroups;
    const int *lp = s.level_ptr.data();
    const int *p2o = s.perm_to_orig.data();
    std::vector<int> by_level_thread(nodes);
    std::vector<std::pair<int, int>> task_rows((size_t)nl * nt);
    std::vector<int> level_single(nl, -1);
    std::vector<double> finish(nodes, 0.0), ttime(nt, 0.0);
    {
        const int et = s.nthread_per_level[0];
        const int lb = lp[0], le = lp[1];
        std::vector<double> pre(le - lb + 1);
        double load = 0.0;
        for (int i = lb; i < le; i++) {
            pre[i - lb] = load;
            load += s.cost[p2o[i]];
        }
        const double per = (load + et - 1) / et;
        int prev_end = lb, r = lb;
        if (et == 1) level_single[0] = 0;
        for (int t = 0; t < et; t++) {
            int nr = r;
            if (r < le) nr = lb + (int)(std::lower_bound(pre.begin() + (r - lb), pre.begin() + (le - lb), (t + 1) * per) - pre.begin());
            r = nr;
            const int b = prev_end, e = std::min(r, le);
            prev_end = e;
            task_rows[(size_t)t * nl + 0] = {b, e};
            for (int k = b; k < e; k++) {
                const int node = p2o[k];
                by_level_thread[k] = node;
                ttime[t] += s.cost[node];
                finish[node] = ttime[t];
            }
            ++r;
        }
        for (int t = et; t < nt; t++) task_rows[(size_t)t * nl + 0] = {le, le};
    }
    std::vector<int> tidx(nt), order;
    std::vector<std::vector<int>> tnodes(nt);
    std::vector<uint8_t> chosen(nt);
    for (int lvl = 1; lvl < nl; lvl++) {
        const int lb = lp[lvl], le = lp[lvl + 1];
        const int et = s.nthread_per_level[lvl];
        for (auto &v : tnodes) v.clear();
        std::iota(tidx.begin(), tidx.end(), 0);
        std::nth_element(tidx.begin(), tidx.begin() + et, tidx.end(), [&](int a, int b) { return ttime[a] < ttime[b]; });
        if (et == 1) level_single[lvl] = tidx[0];
        for (int i = lb; i < le; i++) {
            const int node = p2o[i];
            int start = 0;
            for (int q = dag_csr.ptr[node]; q < dag_csr.ptr[node + 1] - 1; q++) {
                const int par = dag_csr.idx[q];
                start = start < finish[par] ? (int)finish[par] : start;
            }
            finish[node] = start;
        }
        order.assign(p2o + lb, p2o + le);
        std::sort(order.begin(), order.end(), [&](int a, int b) { return finish[a] < finish[b]; });
        for (int node : order) {
            const int t = *std::min_element(tidx.begin(), tidx.begin() + et, [&](int a, int b) { return ttime[a] < ttime[b]; });
            finish[node] = ttime[t] + s.cost[node];
            ttime[t] = finish[node];
            tnodes[t].push_back(node);
        }
        std::fill(chosen.begin(), chosen.end(), 0);
        for (int q = 0; q < et; q++) chosen[tidx[q]] = 1;
        int pos = lb;
        for (int t = 0; t < nt; t++) {
            auto &tr = task_rows[(size_t)t * nl + lvl];
            if (chosen[t]) {
                tr = {pos, pos + (int)tnodes[t].size()};
                for (int v : tnodes[t]) by_level_thread[pos++] = v;
            } else {
                tr = {pos, pos};
            }
        }
    }
    finish_mapping(s, task_rows, by_level_thread, level_single);
}

// Stage 9 of the affinity mapping, the Scheduler's P2P_MAPPING algorithm
// (Task::constructMappingMergeSerial, merge/LevelTask.cpp:1206-1645). Level 0 is split by cost.
// On every later level each group scores the threads of its parents within the level window
// (`< LEVEL_WINDOW_SIZE` here, unlike the four-rule mapping's `<=`) and keeps its top
// ceil(sqrt(min(exec, nthread))) threads; the threads with the highest total share execute.
// Groups go to their top thread when it executes (costs summed as ints, as the reference sums
// them there). Overloaded threads give back groups from their end. The given-back and
// unplaced groups then try their next-best threads, and finally fill the threads still under
// the average. The reference iterates two std::unordered_set<int>, so the same containers and the
// same sequence of reserve / clear / insert / erase calls are used here: under the same standard
// library they iterate in the same order. False if the reference's scan would drop a group (its
// leftover loop falls back to thread 0 when no executing thread is still filling).
bool affinity_map(HostSchedule &s, const Csx &dag_csr) {
    struct NodeScore {
        int node;
        int thread;
        double score;
    };
    const int nl = s.nlevels, nt = s.nthread, nodes = s.ngroups;
    const int *lp = s.level_ptr.data();
    const int *p2o = s.perm_to_orig.data();
    const int *o2p = s.perm.data();
    const int *n2l = s.node_to_level.data();
    std::vector<int> by_level_thread(nodes, -1), node_thread(nodes, -1);
    std::vector<std::pair<int, int>> task_rows((size_t)nl * nt);
    std::vector<int> level_single(nl, -1);
    {
        const int et = s.nthread_per_level[0];
        const int lb = lp[0], le = lp[1];
        std::vector<double> pre(le - lb + 1);
        double load = 0.0;
        for (int i = lb; i < le; i++) {
            pre[i - lb] = load;
            load += s.cost[p2o[i]];
        }
        const double per = (load + et - 1) / et;
        int prev_end = lb, r = lb;
        if (et == 1) level_single[0] = 0;
        for (int t = 0; t < et; t++) {
            int nr = r;
            if (r < le) nr = lb + (int)(std::lower_bound(pre.begin() + (r - lb), pre.begin() + (le - lb), (t + 1) * per) - pre.begin());
            r = nr;
            const int b = prev_end, e = std::min(r, le);
            prev_end = e;
            task_rows[(size_t)t * nl + 0] = {b, e};
            for (int k = b; k < e; k++) {
                by_level_thread[k] = p2o[k];
                node_thread[p2o[k]] = t;
            }
            ++r;
        }
        for (int t = et; t < nt; t++) task_rows[(size_t)t * nl + 0] = {le, le};
    }
    std::vector<double> node_score(nt), thread_load(nt), thread_score(nt);
    std::vector<int> tidx(nt), thread_order(nt), disperse;
    std::vector<std::vector<int>> tnodes(nt);
    std::unordered_set<int> allocating;
    std::unordered_set<int> chosen;
    chosen.reserve(nt);
    allocating.reserve(nt);
    disperse.reserve(nodes);
    const double alpha = 1.2;
    for (int lvl = 1; lvl < nl; lvl++) {
        const int lb = lp[lvl], le = lp[lvl + 1];
        const int et = s.nthread_per_level[lvl];
        const int width = le - lb;
        chosen.clear();
        disperse.clear();
        allocating.clear();
        std::fill(thread_load.begin(), thread_load.end(), 0.0);
        std::fill(thread_score.begin(), thread_score.end(), 0.0);
        std::iota(thread_order.begin(), thread_order.end(), 0);
        for (auto &v : tnodes) v.clear();
        const int sw = (int)std::ceil(std::sqrt((double)std::min(et, nt)));
        std::vector<NodeScore> table((size_t)sw * width);
        for (int i = lb; i < le; i++) {
            std::fill(node_score.begin(), node_score.end(), 0.0);
            const int node = p2o[i];
            const int nlev = n2l[node];
            for (int q = dag_csr.ptr[node]; q < dag_csr.ptr[node + 1] - 1; q++) {
                const int par = dag_csr.idx[q];
                const int diff = nlev - n2l[par];
                if (diff < s.score.level_window)
                    node_score[node_thread[par]] +=
                        s.score.amplify * std::log2(1.0 * (s.group_ptr[par + 1] - s.group_ptr[par] + 1)) / std::log2(1.0 * (diff + 1));
            }
            std::iota(tidx.begin(), tidx.end(), 0);
            std::partial_sort(tidx.begin(), tidx.begin() + sw, tidx.end(), [&](int a, int b) { return node_score[a] > node_score[b]; });
            double total = 0.0;
            for (int m = 0; m < sw; m++) {
                const int t = tidx[m];
                auto &en = table[(size_t)(i - lb) + (size_t)m * width];
                en.node = node;
                en.thread = t;
                en.score = node_score[t];
                total += node_score[t] * std::exp(-alpha * (m + 1));
            }
            for (int m = 0; m < sw; m++) {
                const int t = tidx[m];
                thread_score[t] += node_score[t] * std::exp(-alpha * (m + 1)) / total;
            }
        }
        std::sort(table.begin(), table.begin() + width, [](NodeScore &a, NodeScore &b) {
            if (a.thread != b.thread) return a.thread < b.thread;
            return a.score > b.score;
        });
        std::sort(thread_order.begin(), thread_order.end(), [&](int a, int b) { return thread_score[a] > thread_score[b]; });
        chosen.insert(thread_order.begin(), thread_order.begin() + et);
        if (et == 1) level_single[lvl] = thread_order[0];
        double level_load = 0;
        for (int i = 0; i < width; i++) {
            const NodeScore &it = table[i];
            const int c = (int)s.cost[it.node];
            level_load += c;
            if (chosen.find(it.thread) != chosen.end()) {
                tnodes[it.thread].push_back(it.node);
                thread_load[it.thread] += c;
            } else {
                disperse.push_back(it.node);
            }
        }
        const double avg = (level_load + et - 1) / et;
        for (auto &t : chosen) {
            if (thread_load[t] >= avg) {
                int node = tnodes[t].back();
                while (thread_load[t] - s.cost[node] >= avg) {
                    disperse.push_back(node);
                    tnodes[t].pop_back();
                    thread_load[t] -= s.cost[node];
                    node = tnodes[t].back();
                }
            } else {
                allocating.insert(t);
            }
        }
        int ndisp = 0;
        for (size_t i = 0; i < disperse.size(); i++) {
            const int node = disperse[i];
            bool placed = false;
            for (int w = 1; w < sw; w++) {
                const int p = table[(size_t)w * width + (size_t)(o2p[node] - lb)].thread;
                if (allocating.find(p) != allocating.end()) {
                    thread_load[p] += s.cost[node];
                    tnodes[p].push_back(node);
                    if (thread_load[p] >= avg) allocating.erase(p);
                    placed = true;
                    break;
                }
            }
            if (!placed) disperse[ndisp++] = node;
        }
        auto iter = allocating.begin();
        int ai = 0, t = 0;
        while (ai < ndisp && iter != allocating.end()) {
            t = *iter;
            while (thread_load[t] <= avg && ai < ndisp) {
                const int node = disperse[ai++];
                thread_load[t] += s.cost[node];
                tnodes[t].push_back(node);
            }
            iter++;
        }
        while (ai < ndisp) tnodes[t].push_back(disperse[ai++]);
        int pos = lb;
        for (int th = 0; th < nt; th++) {
            auto &tr = task_rows[(size_t)th * nl + lvl];
            if (chosen.find(th) != chosen.end()) {
                tr = {pos, pos + (int)tnodes[th].size()};
                for (int v : tnodes[th]) {
                    if (pos >= le) return false;
                    by_level_thread[pos++] = v;
                    node_thread[v] = th;
                }
            } else {
                tr = {pos, pos};
            }
        }
        if (pos != le) return false;  // a group was left on a thread that does not execute
    }
    finish_mapping(s, task_rows, by_level_thread, level_single);
    return true;
}

// Stage 10: for every task, the sorted set of tasks on other threads that own a parent group.
void task_dags(HostSchedule &s, const Csx &dag_csr) {
    const int nt = s.nthread, ntask = s.ntasks;
    std::vector<int> owner(s.ngroups);
    for (int t = 0; t < ntask; t++)
        for (int r = s.task_boundaries[t]; r < s.task_boundaries[t + 1]; r++) owner[s.thread_cont_to_orig[r]] = t;
    s.task_ptr.assign(ntask + 1, 0);
    s.task_set.clear();
    std::vector<int> dep;
    for (int th = 0; th < nt; th++) {
        const int tb = s.thread_boundaries[th], te = s.thread_boundaries[th + 1];
        for (int t = tb; t < te; t++) {
            dep.clear();
            for (int r = s.task_boundaries[t]; r < s.task_boundaries[t + 1]; r++) {
                const int g = s.thread_cont_to_orig[r];
                for (int q = dag_csr.ptr[g]; q < dag_csr.ptr[g + 1]; q++) {
                    const int v = owner[dag_csr.idx[q]];
                    if (v < tb || v >= te) dep.push_back(v);
                }
            }
            std::sort(dep.begin(), dep.end());
            dep.erase(std::unique(dep.begin(), dep.end()), dep.end());
            s.task_set.insert(s.task_set.end(), dep.begin(), dep.end());
            s.task_ptr[t + 1] = (int)s.task_set.size();
        }
    }
    Csx td{s.task_ptr, s.task_set};
    Csx bt = transpose(td);
    s.btask_ptr = std::move(bt.ptr);
    s.btask_set = std::move(bt.idx);
}

}  // namespace

const char *validate_pattern(int n, const int *rowptr, const int *colidx, SchedKind kind) {
    if (n <= 0) return "n must be positive";
    if (!rowptr || !colidx) return "rowptr/colidx must not be NULL";
    if (rowptr[0] != 0) return "rowptr[0] must be 0 (0-based CSR)";
    for (int i = 0; i < n; i++) {
        if (rowptr[i + 1] < rowptr[i]) return "rowptr must be non-decreasing";
        bool diag = false;
        for (int e = rowptr[i]; e < rowptr[i + 1]; e++) {
            const int c = colidx[e];
            if (c < 0 || c >= n) return "column index out of range";
            if (e > rowptr[i] && colidx[e - 1] >= c) return "column indices must be strictly ascending in each row";
            if (c == i) diag = true;
            if (kind == SchedKind::SpTRSV && c > i) return "SpTRSV analysis takes the lower triangle only";
        }
        if (!diag) return "every row needs its diagonal entry";
    }
    return "";
}

bool build_schedule(HostSchedule &s, int n, const int *rowptr, const int *colidx, SchedKind kind, int nthread,
                    Mapping mapping, Ablation ablation, bool device, std::string &why, const std::vector<int> *sys_off,
                    const ScoreParams &score) {
    // BAASWOA and BAASWOAS leave the rows ungrouped: one group per row on the two-hop DAG
    const bool aggregate = ablation == Ablation::None || ablation == Ablation::WOS;
    // a block-diagonal batch: stages 2-7 system by system on host threads
    const bool split = sys_off && sys_off->size() > 2 && !device && aggregate;
    auto t0 = std::chrono::steady_clock::now();
    // BAAS_ANALYSIS_TRACE=1: stage times of the analysis on stderr
    const bool trace = getenv("BAAS_ANALYSIS_TRACE") && atoi(getenv("BAAS_ANALYSIS_TRACE")) > 0;
    auto tl = t0;
    auto stage = [&](const char *name) {
        if (!trace) return;
        const auto t = std::chrono::steady_clock::now();
        fprintf(stderr, "[baas analysis] %s %.2f ms\n", name, std::chrono::duration<double, std::milli>(t - tl).count());
        tl = t;
    };
    s = HostSchedule();
    s.kind = kind;
    s.score = score;
    s.n = n;
    s.nthread = nthread;
    const int nnz = rowptr[n];
    s.a_rowptr.assign(rowptr, rowptr + n + 1);
    s.a_colidx.assign(colidx, colidx + nnz);
    s.a_diagptr.assign(n, 0);
    for (int i = 0; i < n; i++) {
        int e = rowptr[i];
        while (e < rowptr[i + 1] && colidx[e] < i) e++;
        s.a_diagptr[i] = e;
    }

    // Stage 1: lower triangle incl. diagonal (test/Schedule.hpp:134-154) and its CSC
    s.l_rowptr.assign(n + 1, 0);
    for (int i = 0; i < n; i++) s.l_rowptr[i + 1] = s.l_rowptr[i] + s.a_diagptr[i] - rowptr[i] + 1;
    s.l_colidx.resize(s.l_rowptr[n]);
    s.l_src.resize(s.l_rowptr[n]);
    for (int i = 0; i < n; i++)
        for (int e = rowptr[i]; e <= s.a_diagptr[i]; e++) {
            s.l_colidx[s.l_rowptr[i] + e - rowptr[i]] = colidx[e];
            s.l_src[s.l_rowptr[i] + e - rowptr[i]] = e;
        }
    // With `device`, the transposes, the two-hop reduction, the group DAGs and the level sets run
    // on the GPU (DeviceStages), the DAGs staying resident there between the stages; the BFS
    // coarsenings, the mappings and the task DAGs run here on the host in both cases.
    std::unique_ptr<DeviceStages> D;
    DeviceStages::Graph dL, d0, dd, dinv, dg, dginv, df, dfcsr;
    auto dev_failed = [&]() {
        why = D->err;
        return false;
    };
    Csx dag, inv, gdag, fdag, dag_csr;
    Grouping rev, fwd;
    if (device) {
        D.reset(new DeviceStages());
        dL = D->upload(s.l_rowptr, s.l_colidx);
        d0 = D->transpose(dL);  // column j: j itself, then the rows that depend on j
        D->release(dL);
        stage("lower triangle + CSC (device)");
        dd = D->two_hop(d0);  // stage 2
        D->release(d0);
        dinv = D->transpose(dd);
        D->download(dd, dag.ptr, dag.idx);
        D->download(dinv, inv.ptr, inv.idx);
        D->release(dinv);
        if (!D->ok()) return dev_failed();
        stage("two-hop reduction + inverse (device)");
    }
    if (device && !aggregate) {
        df = dd;
        dd = DeviceStages::Graph();
        fdag = dag;
        dag_csr = std::move(inv);
    } else if (device) {
        rev = tree_coarsen(dag, true, &inv);  // stage 3
        stage("reverse-tree coarsening (host)");
        dg = D->group_dag(dd, rev.ptr, rev.set);  // stage 4
        D->release(dd);
        dginv = D->transpose(dg);
        Csx ginv;
        D->download(dg, gdag.ptr, gdag.idx);
        D->download(dginv, ginv.ptr, ginv.idx);
        D->release(dginv);
        if (!D->ok()) return dev_failed();
        stage("group DAG + inverse (device)");
        fwd = tree_coarsen(gdag, false, &ginv);  // stage 5
        stage("forward-tree coarsening (host)");
        df = D->group_dag(dg, fwd.ptr, fwd.set);
        D->release(dg);
        D->download(df, fdag.ptr, fdag.idx);
        if (!D->ok()) return dev_failed();
        stage("group DAG of the forward groups (device)");
    } else if (split) {
        split_stages(s, *sys_off, fdag);
        stage("stages 2-7 per system (host threads)");
    } else {
        Csx lower{s.l_rowptr, s.l_colidx};
        Csx dag0 = transpose(lower);  // column j: j itself, then the rows that depend on j
        stage("lower triangle + CSC");
        dag = two_hop_reduce(dag0);  // stage 2
        stage("two-hop reduction");
        if (aggregate) {
            rev = tree_coarsen(dag, true);    // stage 3
            gdag = group_dag(n, rev, dag);    // stage 4
            fwd = tree_coarsen(gdag, false);  // stage 5
            stage("tree coarsening + group DAGs");
        } else {
            fdag = dag;
        }
    }
    if (split) {
        // groups, group DAG and level set already concatenated
    } else if (aggregate) {
        // remap forward groups (of reverse groups) onto rows (merge/Coarsen.cpp:896-928)
        s.ngroups = fwd.ngroups;
        s.group_ptr.assign(1, 0);
        s.group_ptr.reserve(fwd.ngroups + 1);
        s.group_set.clear();
        s.group_set.reserve(n);
        for (int f = 0; f < fwd.ngroups; f++) {
            for (int q = fwd.ptr[f]; q < fwd.ptr[f + 1]; q++) {
                const int g = fwd.set[q];
                s.group_set.insert(s.group_set.end(), rev.set.begin() + rev.ptr[g], rev.set.begin() + rev.ptr[g + 1]);
            }
            s.group_ptr.push_back((int)s.group_set.size());
        }
        if (!device) fdag = group_dag(rev.ngroups, fwd, gdag);
    } else {  // one group per row (test/SpTRSVRuntime.hpp:925-932, :1148-1156)
        s.ngroups = n;
        s.group_ptr.resize(n + 1);
        s.group_set.resize(n);
        for (int i = 0; i < n; i++) {
            s.group_ptr[i + 1] = i + 1;
            s.group_set[i] = i;
        }
        s.group_ptr[0] = 0;
    }

    // Stage 6: cost = rows' lower-triangle lengths summed over the group (merge/Coarsen.cpp:854-891)
    s.cost.assign(s.ngroups, 0.0);
    for (int g = 0; g < s.ngroups; g++)
        for (int e = s.group_ptr[g]; e < s.group_ptr[g + 1]; e++) {
            const int r = s.group_set[e];
            s.cost[g] += 1 * (s.l_rowptr[r + 1] - s.l_rowptr[r]);
        }

    stage("remap + group DAG + cost");
    if (device) {  // stage 7 on the device; the dependency-order DAG for the mapping with it
        s.nlevels = D->levels(df, s.node_to_level, s.perm_to_orig, s.level_ptr);
        if (aggregate) {
            dfcsr = D->transpose(df);
            D->download(dfcsr, dag_csr.ptr, dag_csr.idx);
            D->release(dfcsr);
        }
        D->release(df);
        if (!D->ok()) return dev_failed();
        s.exec_level_ptr = s.level_ptr;
        s.perm.assign(s.ngroups, 0);
        for (int i = 0; i < s.ngroups; i++) s.perm[s.perm_to_orig[i]] = i;
        D.reset();
        stage("level sets + inverse DAG (device)");
    } else if (!split) {
        level_sets(fdag, s);  // stage 7
        stage("level sets");
    }
    if (ablation == Ablation::WOAS) {
        threads_per_level_base(s);
    } else if (ablation == Ablation::WOS) {  // level_merge_group_TRSV (merge/LevelMerge.cpp:313-365)
        threads_per_level(s);
        merge_levels(s, s.nthread_per_level);
    } else if (mapping == Mapping::FourRule || mapping == Mapping::FinishTime || mapping == Mapping::Affinity) {
        threads_per_level(s);  // stage 8
    } else {
        merge_levels_group(s);
    }
    for (int g = 0; g < s.ngroups; g++)  // test/Schedule.hpp:72-79
        std::sort(s.group_set.begin() + s.group_ptr[g], s.group_set.begin() + s.group_ptr[g + 1]);
    if (!device) dag_csr = transpose(fdag);  // parents of each group, then the group itself
    stage("threads per level + group sort + inverse DAG");
    if (ablation == Ablation::WOS || ablation == Ablation::WOAS)
        cost_split_map(s, false);  // Task::constructTask
    else if (mapping == Mapping::FourRule)
        four_rule_map(s, dag_csr);  // stage 9
    else if (mapping == Mapping::FinishTime)
        finish_time_map(s, dag_csr);
    else if (mapping == Mapping::Affinity) {
        if (!affinity_map(s, dag_csr)) {
            why = "the P2P_MAPPING scan left a group on a thread that does not execute";
            return false;
        }
    }
    else
        cost_split_map(s, mapping == Mapping::CostSplitBarrier);
    stage("mapping");
    task_dags(s, dag_csr);          // stage 10
    stage("task DAGs");
    s.fdag_ptr = std::move(fdag.ptr);
    s.fdag_set = std::move(fdag.idx);
    auto t1 = std::chrono::steady_clock::now();
    s.analysis_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return true;
}

}  // namespace baas
