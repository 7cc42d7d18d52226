/*
 * baas_b200.h -- C ABI of the B200-native BAAS sparse hot path.
 *
 * The path is the one the reference drives from pcg_opt (test/iccg_level_merge.cpp:380-533):
 * schedule construction (transitive reduction, bidirectional tree coarsening, level sets,
 * per-level thread counts, four-rule affinity mapping, task DAG), then IC0 / ILU0 and the
 * forward / backward triangular sweeps driven by that schedule, then the ICCG loop.
 *
 * Conventions
 *  - Every function returns a baas_status; nothing aborts the process.
 *  - Indices are int32, values FP64 (as in the reference's SPM::CSR, spm/include/CSR.hpp:16-31).
 *  - baas_analyze works on HOST arrays and needs no GPU. Every other compute call takes CUDA
 *    DEVICE pointers owned by the caller and a cudaStream_t passed as `void *stream`
 *    (NULL = legacy default stream). Calls are stream-ordered; a call returns after its work
 *    is enqueued unless it has to read a status or a scalar back (it then synchronises that
 *    stream and says so below).
 *  - A baas_schedule owns all of its host and device memory. It is not re-entrant: calls on
 *    one schedule must not overlap in time (the reference's single taskFinsished array per
 *    schedule has the same restriction, merge/include/LevelTask.hpp:177).
 *  - Device waits are bounded: a wait that exceeds baas_options.spin_limit polls ends the
 *    kernel with BAAS_ERR_TIMEOUT instead of hanging (the reference spins forever,
 *    merge/include/SpTRSV.hpp:16-23).
 */
#ifndef BAAS_B200_H
#define BAAS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum baas_status {
    BAAS_OK = 0,
    BAAS_ERR_BAD_ARG = 1,       /* NULL pointer, size mismatch, pattern the path cannot take */
    BAAS_ERR_CUDA = 2,          /* a CUDA runtime call failed (see baas_last_error_string) */
    BAAS_ERR_TIMEOUT = 3,       /* a bounded device wait ran out (schedule or input is inconsistent) */
    BAAS_ERR_ZERO_PIVOT = 4,    /* IC0 met a pivot <= 0 (left unchanged, as merge/IC.cpp:371-378 does)
                                   or ILU0 met a zero pivot; the factor is still written */
    BAAS_ERR_NOT_CONVERGED = 5, /* ICCG hit maxiter before the tolerance */
    BAAS_ERR_NO_DEVICE = 6,     /* the compute call needs a CUDA device and none is usable */
    BAAS_ERR_STATE = 7          /* call order violated (e.g. a sweep before the factor exists) */
} baas_status;

/* Which reference driver's schedule to reproduce. */
typedef enum baas_kernel {
    /* SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRule (test/SpTRSVRuntime.hpp:617-852): the input
     * is the lower triangle L (diagonal last in each row); level thread counts from
     * level_nthreads_group_TRSV over L (merge/LevelMerge.cpp:164-200). */
    BAAS_KERNEL_SPTRSV = 0,
    /* Schedule::Scheduler(A, isSymmetric=true, isTRSVPerm=false, P2P_RULE, nthread)
     * (test/Schedule.hpp:117-296): the input is the full SPD matrix A; thread counts from
     * level_nthreads_group_TRSV over the FULL A (test/Schedule.hpp:248); also builds the
     * backward (inverse) task schedule. Used by ICCG. */
    BAAS_KERNEL_ICCG = 1,
    /* IC_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRule (test/ICRuntime.hpp:353-583). */
    BAAS_KERNEL_IC0 = 2,
    /* ILU_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRule (test/ILURuntime.hpp:207-436); the pattern
     * must be structurally symmetric, as the reference assumes. */
    BAAS_KERNEL_ILU0 = 3
} baas_kernel;

/* Schedule arrays exported for parity checks (names of the reference's members). */
typedef enum baas_field {
    BAAS_FIELD_NGROUPS = 0,            /* scalar: groups after both coarsenings */
    BAAS_FIELD_NLEVELS = 1,            /* scalar: levels of the group DAG */
    BAAS_FIELD_NTASKS = 2,             /* scalar */
    BAAS_FIELD_GROUP_PTR = 3,          /* group_ptr[ngroups+1] */
    BAAS_FIELD_GROUP_SET = 4,          /* group_set[n], rows ascending within a group */
    BAAS_FIELD_LEVEL_PTR = 5,          /* LevelSet::level_ptr[nlevels+1] */
    BAAS_FIELD_PERM_TO_ORIG = 6,       /* LevelSet::permToOrig[ngroups] */
    BAAS_FIELD_NODE_TO_LEVEL = 7,      /* LevelSet::nodeToLevel[ngroups], 1-based */
    BAAS_FIELD_NTHREAD_PER_LEVEL = 8,  /* nthread_per_level[nlevels] */
    BAAS_FIELD_THREAD_BOUNDARIES = 9,  /* Task::threadBoundaries[nthread+1] */
    BAAS_FIELD_TASK_BOUNDARIES = 10,   /* Task::taskBoundaries[ntasks+1] */
    BAAS_FIELD_THREAD_CONT_TO_ORIG = 11, /* Task::threadContToOrigPerm[ngroups] */
    BAAS_FIELD_ORIG_TO_THREAD_CONT = 12, /* Task::origToThreadContPerm[ngroups] */
    BAAS_FIELD_TASK_PTR = 13,          /* task DAG (parents), CSR ptr[ntasks+1] */
    BAAS_FIELD_TASK_SET = 14,          /* task DAG parents */
    BAAS_FIELD_BTASK_PTR = 15,         /* backward (inverse) task DAG ptr[ntasks+1] */
    BAAS_FIELD_BTASK_SET = 16,         /* backward parents */
    BAAS_FIELD_COST = 17,              /* Coarsen::costComputation cost[ngroups] (integer-valued) */
    BAAS_FIELD_GROUP_DAG_PTR = 18,     /* DAG between the final groups, CSC ptr[ngroups+1] */
    BAAS_FIELD_GROUP_DAG_SET = 19      /* each group's column: its children groups and itself, ascending */
} baas_field;

typedef enum baas_precision {
    BAAS_PREC_FP64 = 0,           /* factors and sweeps in FP64 */
    BAAS_PREC_FP32_FACTORS = 1    /* factor computed in FP64, stored and applied in FP32 with FP32
                                     accumulation; CG recurrence and dots stay FP64 */
} baas_precision;

/* CSR matrix, 0-based, column indices strictly ascending in each row. For baas_analyze the
 * arrays are host memory; for the compute calls they are device memory. `values` may be NULL
 * for baas_analyze. */
typedef struct baas_csr {
    int n;               /* rows == columns */
    int nnz;             /* rowptr[n] */
    const int *rowptr;   /* n + 1 */
    const int *colidx;   /* nnz */
    const double *values;/* nnz */
} baas_csr;

typedef struct baas_options {
    int nthread;      /* the reference's num_thread: virtual threads of the schedule (>= 1) */
    int spin_limit;   /* polls before a device wait gives up (0 = library default) */
    int parts;        /* CTAs that own rows in the partitioned kernels (0 = automatic: about one
                         per 2,048 rows, at most one per SM) */
    int partition;    /* BAAS_PARTITION_AUTO (default), BAAS_PARTITION_RANGES, BAAS_PARTITION_BLOCKS,
                         BAAS_PARTITION_BAAS_THREADS, or BAAS_PARTITION_CUSTOM (set by
                         baas_replan_custom only) */
    int smem_budget;  /* bytes of shared memory per CTA for solution slots and the two plan
                         window buffers (0 = library default, 220 KiB; at most 224 KiB) */
    int mapping;      /* BAAS_MAPPING_FOUR_RULE (default) or, for BAAS_KERNEL_ICCG, one of the
                         Scheduler's other mappings; fixed by the analysis */
    int walk;         /* BAAS_WALK_AUTO (default), BAAS_WALK_CHUNKED, BAAS_WALK_FETCH,
                         BAAS_WALK_LEVELS or BAAS_WALK_SMALL: which triangular-sweep kernel the
                         single-right-hand-side sweeps and ICCG use */
    int analysis;     /* BAAS_ANALYSIS_HOST (default) or BAAS_ANALYSIS_DEVICE: where the analysis's
                         data-parallel stages run; the schedule is identical either way */
    int ablation;     /* BAAS_ABLATION_NONE (default) or, for BAAS_KERNEL_SPTRSV with the four-rule
                         mapping, one of the SpTRSV runtime's ablation schedules */
    int small_cluster; /* CTAs of BAAS_WALK_SMALL's thread-block cluster: 0 = automatic (16 from
                         8,192 rows up where the device holds such a cluster, else 8; 8 from 2,048
                         rows up; else 1), or 1, 2, 4, 8 or 16 (16: a non-portable cluster size,
                         refused where the device cannot hold one) */
    /* The four-rule mapping's scoring constants, the reference's compile-time macros
     * (merge/include/MergeMarco.hpp:5-23); baas_options_default sets the reference's values.
     * The affinity mapping (BAAS_MAPPING_AFFINITY) reads level_window and amplify. */
    int level_window;   /* LEVEL_WINDOW_SIZE: parents more levels up than this do not vote (6) */
    double amplify;     /* AMPLIFY_FACTOR: weight of a parent group's size in its vote (2.0) */
    double over_gamma;  /* OVER_REGULARIZATION_GMMA: penalty slope past the load average (6.0) */
    double award_alpha; /* AWARD_ALPHA: weight of the affinity award (1.0) */
    double load_beta;   /* LOAD_REGULARIZATION_BETA: weight of the under-load bonus (0.1) */
} baas_options;

/* The SpTRSV runtime's ablation classes (test/SpTRSV_level_merge.cpp:156-299), kind
 * BAAS_KERNEL_SPTRSV only. NONE: BAAS (SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRule). WOS
 * (BAASWOS, SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P, test/SpTRSVRuntime.hpp:448-535): both coarsenings,
 * then level_merge_group_TRSV and the cost-balanced split (Task::constructTask) instead of the
 * four-rule mapping. WOA (BAASWOA, ...MapFourRuleAblationWOAggregation, :1114-1190): no coarsening
 * (one group per row of the two-hop DAG), the four-rule mapping. WOAS (BAASWOAS,
 * ...MapFourRuleAblationBase, :913-975): no coarsening, min(rows, nthread) threads per level
 * (level_nthreads_base), the cost-balanced split. The GPU sweep runs any of them. */
enum { BAAS_ABLATION_NONE = 0, BAAS_ABLATION_WOS = 1, BAAS_ABLATION_WOA = 2, BAAS_ABLATION_WOAS = 3 };

/* Where baas_analyze runs the schedule's data-parallel integer stages: the transposes of the
 * lower triangle and of the DAGs (dcsr2csc, spm/CSR.cpp:914-950), the two-hop reduction
 * (partialSparsification_CSC, spm/DAG.cpp:295-344), the group DAGs (merge/Coarsen.cpp:748-801)
 * and the level sets (DAG_levelSet_CSC, spm/DAG.cpp:572-629). HOST: all on the calling thread.
 * DEVICE: those stages on the current CUDA device (stable radix sorts, frontier rounds), the BFS
 * coarsenings and the mappings on the host; every exported field is identical to HOST's. DEVICE
 * without a usable device fails with BAAS_ERR_NO_DEVICE. */
enum { BAAS_ANALYSIS_HOST = 0, BAAS_ANALYSIS_DEVICE = 1 };

/* Triangular-sweep kernels. CHUNKED: the plan streamed through shared memory in windows, any row
 * width, up to 8 right-hand sides walked together. FETCH: rows of at most 3 off-diagonal entries
 * (stencil matrices) and one right-hand side; the compute warps read every dependency from shared
 * memory while the CTA's last warp brings other CTAs' results in. LEVELS: one right-hand side;
 * every thread of the launch takes groups of a level and a grid barrier ends the level -- for
 * shallow group DAGs (unstructured or permuted patterns: a few dozen wide levels). SMALL: one
 * right-hand side, one thread-block cluster of 8 or 16 CTAs (one CTA below 2,048 rows), each holding the
 * whole solution in shared memory (8 bytes a row; ICCG adds p, and z is 8 or 4 bytes); rows by row
 * level, a row's result stored into every CTA's copy, a cluster barrier per level, the next
 * level's entries loaded while the current one computes -- for systems of up to about 26,000 rows
 * (sweeps) or 13,000 (FP64 ICCG) / 17,000 (FP32 factors); baas_ic0 takes it at any size. AUTO: FETCH wherever
 * the plan qualifies and fits shared memory, else SMALL when the system fits it and its row DAG
 * has at most 64 levels each way, else LEVELS when the group DAG has at most 64 levels, else
 * CHUNKED. Sweeps and factors are bit-identical between the walks. */
enum { BAAS_WALK_AUTO = 0, BAAS_WALK_CHUNKED = 1, BAAS_WALK_FETCH = 2, BAAS_WALK_LEVELS = 3, BAAS_WALK_SMALL = 4 };

/* How the analysis maps groups to the reference's virtual threads (Schedule::ALG_SCHEDULE,
 * test/Schedule.hpp:31-37, 263-281). FOUR_RULE: P2P_RULE, the BAAS four-rule mapping
 * (merge/LevelTask.cpp:2295-2684). COST_SPLIT: P2P -- level merge (merge/LevelMerge.cpp:372-421)
 * and a cost-balanced contiguous split of every merged level (Task::constructTask,
 * merge/LevelTask.cpp:42-196), one task per non-empty range. COST_SPLIT_BARRIER: the same split
 * with the barrier-mode task layout (Task(ngroups, true): one task per level and thread).
 * FINISH_TIME: P2P_TIME (Task::constructMappingByFinishTime, merge/LevelTask.cpp:1647-1910): on
 * each level the threads that finish first take the groups that can start first. AFFINITY:
 * P2P_MAPPING (Task::constructMappingMergeSerial, merge/LevelTask.cpp:1206-1645): groups score
 * their parents' threads, the best-scoring threads execute, loads are rebalanced. All but
 * FOUR_RULE are the Scheduler's (kind BAAS_KERNEL_ICCG only). The GPU plan does not depend on the
 * mapping except through BAAS_PARTITION_BAAS_THREADS. */
enum {
    BAAS_MAPPING_FOUR_RULE = 0,
    BAAS_MAPPING_COST_SPLIT = 1,
    BAAS_MAPPING_COST_SPLIT_BARRIER = 2,
    BAAS_MAPPING_FINISH_TIME = 3,
    BAAS_MAPPING_AFFINITY = 4
};

/* How rows are given to CTAs. RANGES: contiguous row-index ranges, so every cross-CTA
 * dependency of the lower sweep points to an earlier CTA. BAAS_THREADS: CTA t runs the groups the
 * four-rule mapping gives virtual thread t (requires parts == nthread or parts == 0). CUSTOM: a
 * caller's row-to-CTA map (baas_replan_custom). BLOCKS: when the pattern is a 1-, 2- or 3-D
 * stencil in natural ordering (the off-diagonal offsets of L are {1, n1, n1*n2}), boxes of the
 * grid of at most 2,048 rows, shaped to keep the sweeps' critical path inside few boxes; other
 * patterns get RANGES. AUTO (the default): BLOCKS when the pattern is such a grid, its rows hold
 * at most 3 off-diagonal entries, parts == 0 and the fetch walk may run (the combination it is
 * fastest on), else RANGES. Any partition is deadlock-free (every CTA walks its rows in level
 * order and a row only waits on rows of lower levels) and gives bit-identical sweeps and factors;
 * the ICCG sums its dot products CTA by CTA, so its iterates differ between partitions in the
 * last bits. */
enum {
    BAAS_PARTITION_RANGES = 0,
    BAAS_PARTITION_BAAS_THREADS = 1,
    BAAS_PARTITION_CUSTOM = 2,
    BAAS_PARTITION_BLOCKS = 3,
    BAAS_PARTITION_AUTO = 4
};

typedef struct baas_schedule baas_schedule;

/* Fills *opt with the defaults (nthread = 8, library-chosen GPU parameters). */
void baas_options_default(baas_options *opt);

/* Builds the reference-identical BAAS schedule for `kind` from A's pattern (host arrays),
 * plus this library's device execution plan (uploaded on first GPU use). Replaces
 * Scheduler::Scheduler + Scheduler::preprocessing (test/Schedule.hpp:117-155, 181-296) and the
 * runtime classes' buildset() (test/SpTRSVRuntime.hpp:675-775, test/ICRuntime.hpp:408-520,
 * test/ILURuntime.hpp:265-385). Needs no GPU. */
baas_status baas_analyze(const baas_csr *A, baas_kernel kind, const baas_options *opt, baas_schedule **out);

/* Copies schedule array `field` into out (if out != NULL) and returns its length (-1 for an
 * unknown field). Host only. */
int baas_schedule_export(const baas_schedule *s, int field, int *out);

/* Wall time of baas_analyze in milliseconds (the reference's Scheduling_Time,
 * test/SpTRSV_level_merge.cpp:70). */
double baas_schedule_analysis_ms(const baas_schedule *s);

/* The sweep kernel (BAAS_WALK_CHUNKED or BAAS_WALK_FETCH) of the schedule's last baas_sptrsv or
 * baas_iccg call; 0 before the first. No counterpart in the reference. */
int baas_schedule_last_walk(const baas_schedule *s);

/* CTAs of the schedule's current device plan (0 before one is built: at the first GPU call, or by
 * a plan test hook). With box != NULL, writes the grid box shape and the box counts per axis
 * (6 ints; zeros unless the plan uses grid boxes). No counterpart in the reference. */
int baas_plan_parts(const baas_schedule *s, int *box);

/* Frees the schedule and its device memory. */
void baas_destroy(baas_schedule *s);

/* Writes the analysed schedule (its options, the pattern it was built for and every array of the
 * analysis) to a file, and reads one back, so that a later process skips the analysis; the loaded
 * schedule behaves as the one saved (its device plan is built at its first GPU call). No
 * counterpart in the reference, which re-analyses on every run. The file is in this host's byte
 * order and this library version's layout; a file of another version, or a truncated or
 * inconsistent one, is refused with BAAS_ERR_BAD_ARG. */
baas_status baas_schedule_save(const baas_schedule *s, const char *path);
baas_status baas_schedule_load(const char *path, baas_schedule **out);

/* What a schedule was analysed for, into info[0..5]: rows, nnz of the analysed matrix, kind
 * (baas_kernel), nthread, mapping, systems of a batch (0 otherwise). Returns 6 (-1 on NULL). */
int baas_schedule_info(const baas_schedule *s, int *info);

/* MatrixMarket ingestion. Replaces SPM::CSR(const char *fileName) (spm/CSR.cpp:90-112), which
 * reads through loadMatrixMarket_mmio_highlevel_coo (spm/COO.cpp:322-338), mmio_allinone_coo
 * (spm/mmio_highlevel.cpp:748-921) and dcoo2csr (spm/COO.cpp:222-317). Reads a coordinate
 * MatrixMarket file (real, integer or pattern values; general, symmetric or hermitian storage,
 * the latter two expanded to both triangles) into a host CSR with each row sorted by column.
 * The arrays match the reference reader's for every file without repeated (row, column)
 * entries; a repeated entry is BAAS_ERR_BAD_ARG here (the reference's order for it is
 * unspecified). The library allocates the arrays: release them with baas_csr_free. */
baas_status baas_csr_read_mtx(const char *path, baas_csr *out);
void baas_csr_free(baas_csr *mat);

/* Rebuilds the schedule's device execution plan with other options (parts, partition,
 * smem_budget, spin_limit; nthread must stay as analysed) without repeating the analysis: the
 * device plan and workspaces are freed and built again at the next GPU call. Used by the
 * autotuner (baas_b200/autotune.py). No counterpart in the reference. */
baas_status baas_replan(baas_schedule *s, const baas_options *opt);

/* Alternate mapper (no counterpart in the reference, whose OpenMP threads are its partition):
 * rebuilds the device plan with row i owned by CTA row_part[i], 0 <= row_part[i] < parts; a
 * coarsened group goes with the CTA of its first row. parts must not exceed the device's SMs
 * (checked at the next GPU call). smem_budget as in baas_options. Like baas_replan, frees the
 * device plan; later baas_replan calls keep the map while partition stays CUSTOM. */
baas_status baas_replan_custom(baas_schedule *s, const int *row_part, int parts, int smem_budget);

/* Failure-detection test hook (no counterpart in the reference, whose waits never end):
 * makes the forward sweep's row `row` wait on a value that nothing ever writes, so the next
 * forward sweep on this schedule ends with BAAS_ERR_TIMEOUT after spin_limit polls while every
 * memory access stays in bounds and the CUDA context stays usable. Must be called before the
 * schedule's first GPU call; `row` needs an off-diagonal entry in L. */
baas_status baas_test_inject_unsatisfiable_wait(baas_schedule *s, int row);

/* Plan test hook (no counterpart in the reference): builds the chunked sweep plan for `parts`
 * CTAs (0 = automatic, assuming 148 SMs) and a shared-memory budget of `smem_budget` bytes (0 =
 * default), then runs it on the host -- CTA by CTA, each step only once all its cross-CTA
 * dependencies are written -- checking every offset, size and index against the layout the
 * kernels read, and writes x (host arrays; tval are the triangular factor's values, upper as
 * in baas_sptrsv). Returns BAAS_ERR_BAD_ARG with a description on any inconsistency, and
 * BAAS_ERR_STATE once the schedule's plan is resident on a GPU. */
baas_status baas_test_emulate_sweep(baas_schedule *s, int parts, int smem_budget, int upper, const double *tval,
                                    const double *b, double *x);

/* Plan test hook (no counterpart in the reference): builds the fetch-walk plan (BAAS_WALK_FETCH)
 * for `parts` CTAs (0 = automatic, assuming 148 SMs) and runs it on the host, step by step and
 * each step only once its staged values' producers are written, checking every record, slot,
 * fetch-list entry and value code against the pattern, and writes x (host arrays; tval as for
 * baas_test_emulate_sweep). BAAS_ERR_BAD_ARG names the first violation, or that the pattern does
 * not qualify. Must run before the schedule's first GPU call. */
baas_status baas_test_emulate_fetch(baas_schedule *s, int parts, int upper, const double *tval, const double *b,
                                    double *x);

/* Division test hook (no counterpart in the reference), on device arrays a, b, q of n doubles.
 * mode 0: q[i] = a[i] / b[i] as the FP64 sweeps compute it -- Markstein's correction on the stored
 * reciprocal of b[i] where that is proven exact, else the IEEE division (the sweeps get the latter
 * by repeating the launch with IEEE divisions); mode 1: the IEEE correctly rounded division;
 * mode 2: q[i] = 1 where the fast path declines (a repeat would follow), else 0.
 * Synchronises `stream` to read the status. */
baas_status baas_test_divide(const double *a, const double *b, double *q, long long n, int mode, void *stream);

/* Forward sweep x = L^-1 b (upper = 0; L is the analysed lower triangle, diagonal LAST in each
 * row) or backward sweep x = U^-1 b (upper = 1; U has the transposed pattern, diagonal FIRST).
 * Replaces Scheduler::runForwardTRSVNoPerm / runBackwardTRSVNoPerm (test/Schedule.hpp:332-347),
 * i.e. sptrsv_p2p_csr_group_merge_no_perm_alloc (merge/SpTRSV.cpp:421-478) and
 * sptrsv_backward_p2p_csr_group_merge_no_perm_alloc (:601-660); results are bit-identical to
 * them. b and x hold nrhs column-major right-hand sides with leading dimension ldb >= n;
 * x must not alias b. Synchronises `stream` to read the status. */
baas_status baas_sptrsv(baas_schedule *s, const baas_csr *T, int upper, const double *b, double *x,
                        int nrhs, int ldb, void *stream);

/* IC0 in place on lu (device, pre-filled with A.values), A the analysed full SPD matrix.
 * Replaces Scheduler::runIC0 (test/Schedule.hpp:316-322) =
 * spic0_csr_uL_p2p_group_merge_no_perm (merge/IC.cpp:296-393); bit-identical factor.
 * Synchronises `stream` to read the status. */
baas_status baas_ic0(baas_schedule *s, const baas_csr *A, double *lu, void *stream);

/* IC0 that allocates no memory, for callers that cannot call cudaMalloc at the moment they
 * factor: a hot loop of a real-time or latency-bound application that reserved all of its
 * memory up front, a plug-in whose host application forbids device allocation after start-up,
 * or a host framework whose device memory belongs to its own allocator.
 * No counterpart in the reference (its CPU routines malloc freely).
 *
 * Same arguments, arithmetic and result as baas_ic0 (bit-identical factor). Its scratch -- one
 * ready flag per row and a status word -- is a static device array of fixed size inside this
 * library, so it takes at most 2,097,152 rows (BAAS_ERR_BAD_ARG beyond), and every GPU that
 * loads the library holds that 8 MB until the process exits.
 *  - The schedule's device plan must already be resident: make one ordinary GPU call on the
 *    schedule (e.g. baas_ic0) during set-up; otherwise this returns BAAS_ERR_STATE.
 *  - Its first call on a device looks up that device's address of the static array (with the
 *    device current) and keeps it for the process; after a device reset (cudaDeviceReset) or a
 *    rebuilt primary context that address is stale, so do not call it again after one.
 *  - All calls share the one array (it keeps the last call's contents; each call clears what
 *    must start at zero): calls that overlap on the GPU -- on two streams, or on two schedules
 *    at once -- race and must not be issued.
 * Synchronises `stream` to read the status. */
baas_status baas_ic0_noalloc(baas_schedule *s, const baas_csr *A, double *lu, void *stream);

/* ILU0 in place on lu (device, pre-filled with A.values). Replaces
 * ilu0_p2p_csr_group_merge_no_perm_alloc (merge/ILU.cpp:638-720); bit-identical factor.
 * Synchronises `stream` to read the status. */
baas_status baas_ilu0(baas_schedule *s, const baas_csr *A, double *lu, void *stream);

/* IC0-preconditioned CG on A x = b (device arrays; x holds the initial guess and receives the
 * solution), stopping once ||r_k|| / ||r_0|| < tol or after maxiter iterations. One persistent
 * kernel runs the factorisation and the whole iteration loop. Follows pcg_opt
 * (test/iccg_level_merge.cpp:380-533) with a break at tol. Writes the iteration count and the
 * final relative residual; synchronises `stream`. Requires a schedule of kind
 * BAAS_KERNEL_ICCG. */
baas_status baas_iccg(baas_schedule *s, const baas_csr *A, const double *b, double *x, double tol,
                      int maxiter, int precision, int *iters, double *relres, void *stream);

/* Adjoint of baas_iccg (no counterpart in the reference). For x = A^-1 b and a loss L(x), with
 * g = dL/dx: solves A^T lambda = g (lambda starts at 0) by the same preconditioned CG, reusing
 * the IC0 factors that the previous baas_iccg call on this schedule computed -- A must hold the
 * same values and `precision` must match that call, else BAAS_ERR_STATE. A is symmetric, so
 * the transposed preconditioner sweeps are the forward ones. Then dL/db = lambda, and if x and
 * grad_a are given (both or neither), the same launch writes the gradient on A's sparsity
 * pattern, grad_a[e] = -lambda_i * x_j for every entry e = (i, j) of A (nnz doubles). All
 * arrays are device arrays; synchronises `stream`. */
baas_status baas_iccg_adjoint(baas_schedule *s, const baas_csr *A, const double *g, double *lambda, const double *x,
                              double *grad_a, double tol, int maxiter, int precision, int *iters, double *relres,
                              void *stream);

/* Batched systems (no counterpart in the reference, which solves one system per call).
 * baas_batch_concat (host arrays) concatenates nsys CSR matrices into one block-diagonal
 * pattern: rowptr (sum n + 1), colidx and values (sum nnz; values may be NULL) and the row
 * offsets of the systems, sys_off (nsys + 1). Returns the total nnz; with rowptr, colidx or
 * sys_off NULL it only returns the total (for sizing); -1 on bad input. */
int baas_batch_concat(int nsys, const baas_csr *const *sys, int *rowptr, int *colidx, double *values, int *sys_off);

/* Analyses a block-diagonal SPD pattern (host arrays) of nsys systems with row offsets sys_off
 * as one ICCG schedule: the systems' level sets merge, so one launch serves them all. Rejects a
 * pattern with an entry between two systems. */
baas_status baas_analyze_batch(const baas_csr *A, const int *sys_off, int nsys, const baas_options *opt,
                               baas_schedule **out);

/* Solves every system of a batch schedule for nrhs right-hand sides (1..8) with IC0-PCG in one
 * persistent launch: A is the block-diagonal matrix (device), B and X are n x nrhs column-major
 * device arrays (leading dimension ldb; X holds the initial guesses). Each (system, right-hand
 * side) pair is its own CG instance, stopping once its ||r_k|| / ||r_0|| < tol; the launch ends
 * when all have stopped or after maxiter iterations. Writes per instance (index s * nrhs + r)
 * the iterations and the final relative residual into the HOST arrays iters and relres;
 * BAAS_ERR_NOT_CONVERGED if any instance missed tol. precision as for baas_iccg. */
baas_status baas_iccg_batched(baas_schedule *s, const baas_csr *A, const double *B, double *X, int nrhs, int ldb,
                              double tol, int maxiter, int precision, int *iters, double *relres, void *stream);

/* Human-readable text for the last error on this thread (never NULL). */
const char *baas_last_error_string(void);

/* Library version string. */
const char *baas_version(void);

#ifdef __cplusplus
}
#endif

#endif /* BAAS_B200_H */
