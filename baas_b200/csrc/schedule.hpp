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

#include <vector>

namespace baas {

enum class SchedKind { SpTRSV = 0, ICCG = 1, IC0 = 2, ILU0 = 3 };

struct HostSchedule {
    SchedKind kind = SchedKind::ICCG;
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

// Runs stages 1-10. `rowptr`/`colidx` are host arrays of the analysed matrix. False when the
// affinity mapping would leave a group unmapped (the reference's P2P_MAPPING scan can).
bool build_schedule(HostSchedule &s, int n, const int *rowptr, const int *colidx, SchedKind kind, int nthread,
                    Mapping mapping = Mapping::FourRule);

}  // namespace baas
