// Host-side BAAS schedule: the integer graph pipeline that precedes every numeric kernel.
//
// Stages (reference file:line of the behaviour each stage reproduces):
//   1. lower-triangle DAG in CSC form            test/Schedule.hpp:134-154, spm/CSR.cpp:914-950
//   2. two-hop transitive reduction              spm/DAG.cpp:295-344 (cliqueSimplification=false)
//   3. reverse-tree coarsening (BFS)             merge/Coarsen.cpp:234-403, :43-71
//   4. group DAG                                 merge/Coarsen.cpp:748-801
//   5. forward-tree coarsening + remap           merge/Coarsen.cpp:73-229, :12-40, :896-928
//   6. group cost                                merge/Coarsen.cpp:854-891
//   7. level sets (Kahn BFS, self-counting)      spm/DAG.cpp:348-392, :572-629
//   8. threads per level                         merge/LevelMerge.cpp:118-262
//   9. four-rule affinity mapping + 1-thread level merge
//                                                merge/LevelTask.cpp:2295-2684, :198-304
//  10. task DAG and backward task DAG            merge/LevelTask.cpp:487-672, :3126-3184
// The result is bit-identical to the reference's arrays for the same nthread (the reference
// must run with OMP threads == nthread; see stage 9).
#pragma once

#include <string>
#include <vector>

namespace baas {

enum class SchedKind { SpTRSV = 0, ICCG = 1, IC0 = 2, ILU0 = 3 };

// The four-rule mapper's scoring constants, the reference's compile-time macros
// (merge/include/MergeMarco.hpp:5-23: LEVEL_WINDOW_SIZE, AMPLIFY_FACTOR, OVER_REGULARIZATION_GMMA,
// AWARD_ALPHA, LOAD_REGULARIZATION_BETA); the defaults are the reference's values. The affinity
// mapping (P2P_MAPPING) reads the window and the amplification too.
struct ScoreParams {
    int level_window = 6;
    double amplify = 2.0;
    double over_gamma = 6.0;
    double award_alpha = 1.0;
    double load_beta = 0.1;
};

struct HostSchedule {
    SchedKind kind = SchedKind::ICCG;
    ScoreParams score;
    int n = 0;
    int nthread = 1;

    // analysed matrix pattern (full A, or L for SchedKind::SpTRSV)
    std::vector<int> a_rowptr, a_colidx, a_diagptr;
    // lower triangle incl. diagonal (diagonal last), CSR; index map into A's entries
    std::vector<int> l_rowptr, l_colidx, l_src;

    // reference-visible schedule
    int ngroups = 0;
    int nlevels = 0;
    int ntasks = 0;
    std::vector<int> group_ptr, group_set;            // rows ascending inside each group
    std::vector<int> level_ptr, perm_to_orig, node_to_level, perm;  // LevelSet
    // the dependency levels of the group DAG (Kahn levels, before any merge): the GPU plans run
    // a level's groups in parallel, so they follow these even when the exported level set is
    // the merged one (the cost-split mapping's merged levels chain dependent groups)
    std::vector<int> exec_level_ptr;
    std::vector<int> nthread_per_level;
    std::vector<int> thread_boundaries, task_boundaries;
    std::vector<int> thread_cont_to_orig, orig_to_thread_cont;
    std::vector<int> task_ptr, task_set;              // parents of each task (other threads)
    std::vector<int> btask_ptr, btask_set;            // children of each task (backward parents)
    std::vector<double> cost;
    std::vector<int> fdag_ptr, fdag_set;              // final group DAG (CSC, self first)

    double analysis_ms = 0.0;
};

// Validates A's pattern for `kind` (square, sorted, diagonal present, lower-only for SpTRSV).
// Returns an empty string when valid, else the reason.
const char *validate_pattern(int n, const int *rowptr, const int *colidx, SchedKind kind);

// How groups are mapped to virtual threads: the BAAS four-rule mapping (P2P_RULE); the
// Scheduler's P2P algorithm -- level merge plus a cost-balanced contiguous split per level
// (Task::constructTask), with one task per non-empty range or, in barrier mode, one per level
// and thread; P2P_TIME, earliest-finishing threads take the earliest-startable groups; or
// P2P_MAPPING, parent-thread affinity scores with load rebalancing.
enum class Mapping { FourRule = 0, CostSplit = 1, CostSplitBarrier = 2, FinishTime = 3, Affinity = 4 };

// The SpTRSV runtime's ablation classes (test/SpTRSV_level_merge.cpp:156-299): None is BAAS; WOS
// keeps the coarsening and replaces the four-rule mapping by a TRSV level merge and the
// cost-balanced split (SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P); WOA keeps the four-rule mapping on
// ungrouped rows (...MapFourRuleAblationWOAggregation); WOAS does neither: ungrouped rows, as
// many threads per level as rows (level_nthreads_base), the cost-balanced split
// (...MapFourRuleAblationBase).
enum class Ablation { None = 0, WOS = 1, WOA = 2, WOAS = 3 };

// The data-parallel integer stages on the current CUDA device (analysis.cu): transposes, the
// two-hop reduction (stage 2), the group DAGs (stage 4 and the one after stage 5) and the level
// sets (stage 7). Patterns stay resident on the device between stages; every output equals the
// host stage's. After a CUDA error every call is a no-op and `err` holds the reason.
class DeviceStages {
public:
    struct Graph {  // square pattern on the device: n rows (or columns), m entries
        int n = 0, m = 0;
        int *ptr = nullptr, *idx = nullptr;
    };
    DeviceStages();
    ~DeviceStages();
    DeviceStages(const DeviceStages &) = delete;
    DeviceStages &operator=(const DeviceStages &) = delete;
    bool ok() const { return err.empty(); }
    std::string err;

    Graph upload(const std::vector<int> &ptr, const std::vector<int> &idx);
    bool download(const Graph &g, std::vector<int> &ptr, std::vector<int> &idx);
    Graph transpose(const Graph &g);  // each output row's entries ascending
    Graph two_hop(const Graph &dag);   // CSC DAG, each column's own node first
    // DAG between the groups (gptr, gset) of dag's nodes: every entry of every member mapped to
    // its group, sorted and unique per group
    Graph group_dag(const Graph &dag, const std::vector<int> &gptr, const std::vector<int> &gset);
    // Kahn levels (1-based per node), nodes ascending inside each level; returns the level count
    int levels(const Graph &dag, std::vector<int> &node_to_level, std::vector<int> &perm_to_orig,
               std::vector<int> &level_ptr);
    void release(Graph &g);

private:
    struct Impl;
    Impl *impl_;
    bool fail(const char *what);
    bool check(const char *what);
    void *alloc(size_t bytes);
    void release(void *p);
    void *scratch(size_t bytes);
    bool scan(int *cnt, int *ptr, int n);
};

// Runs stages 1-10. `rowptr`/`colidx` are host arrays of the analysed matrix. With `device`, the
// stages DeviceStages covers run on the current CUDA device; the schedule is the same. With
// `sys_off` (the row offsets of a block-diagonal batch, no entry coupling two systems), stages 2-7
// run system by system on host threads; the schedule is again the same. False with `why` set when
// the affinity mapping would leave a group unmapped (the reference's P2P_MAPPING scan can) or a
// device stage failed.
bool build_schedule(HostSchedule &s, int n, const int *rowptr, const int *colidx, SchedKind kind, int nthread,
                    Mapping mapping, Ablation ablation, bool device, std::string &why,
                    const std::vector<int> *sys_off = nullptr, const ScoreParams &score = ScoreParams());

}  // namespace baas
