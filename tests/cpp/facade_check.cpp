// Drives the C++ facade (include/baas_b200.hpp) the way the reference's ICCG driver drives
// Schedule::Scheduler (test/iccg_level_merge.cpp): preprocessing, runIC0, forward and backward
// sweeps on host arrays -- and the runtime classes' evaluate() -- and checks every result bit
// for bit against the oracle (oracle/baas_oracle.c). "--analysis-only" stops before the GPU.
#include <cstdio>
#include <cstring>
#include <vector>

#include "baas_b200.hpp"
extern "C" {
#include "baas_oracle.h"
}

// The members of the reference's SPM::CSR that the facade reads (spm/include/CSR.hpp:16-30).
struct CSR {
    int m = 0, n = 0;
    int *rowptr = nullptr, *colidx = nullptr;
    double *values = nullptr;
    std::vector<int> rp, ci;
    std::vector<double> va;
    void bind() {
        rowptr = rp.data();
        colidx = ci.data();
        values = va.data();
        m = n = (int)rp.size() - 1;
    }
};

// 7-point Laplacian on k^3 plus shift*I, natural order, columns ascending.
static CSR laplace3d(int k, double shift) {
    CSR A;
    const int n = k * k * k;
    A.rp.push_back(0);
    for (int z = 0; z < k; z++)
        for (int y = 0; y < k; y++)
            for (int x = 0; x < k; x++) {
                const int i = (z * k + y) * k + x;
                auto add = [&](int c, double v) {
                    A.ci.push_back(c);
                    A.va.push_back(v);
                };
                if (z > 0) add(i - k * k, -1.0);
                if (y > 0) add(i - k, -1.0);
                if (x > 0) add(i - 1, -1.0);
                add(i, 6.0 + shift);
                if (x < k - 1) add(i + 1, -1.0);
                if (y < k - 1) add(i + k, -1.0);
                if (z < k - 1) add(i + k * k, -1.0);
                A.rp.push_back((int)A.ci.size());
            }
    (void)n;
    A.bind();
    return A;
}

// L = lower triangle of lu (diagonal last), U = L^T (diagonal first).
static void split(const CSR &A, const std::vector<double> &lu, CSR &L, CSR &U) {
    const int n = A.m;
    L.rp.assign(1, 0);
    for (int i = 0; i < n; i++) {
        for (int e = A.rp[i]; e < A.rp[i + 1]; e++)
            if (A.ci[e] <= i) {
                L.ci.push_back(A.ci[e]);
                L.va.push_back(lu[e]);
            }
        L.rp.push_back((int)L.ci.size());
    }
    std::vector<int> cnt(n + 1, 0);
    for (int c : L.ci) cnt[c + 1]++;
    for (int i = 0; i < n; i++) cnt[i + 1] += cnt[i];
    U.rp = cnt;
    U.ci.resize(L.ci.size());
    U.va.resize(L.va.size());
    std::vector<int> cur(cnt.begin(), cnt.end() - 1);
    for (int i = 0; i < n; i++)
        for (int e = L.rp[i]; e < L.rp[i + 1]; e++) {
            const int c = L.ci[e];
            U.ci[cur[c]] = i;
            U.va[cur[c]] = L.va[e];
            cur[c]++;
        }
    L.bind();
    U.bind();
}

static int fail(const char *what) {
    std::printf("FAIL %s\n", what);
    return 1;
}

int main(int argc, char **argv) {
    const bool analysis_only = argc > 1 && std::strcmp(argv[1], "--analysis-only") == 0;
    CSR A = laplace3d(12, 1e-3);
    const int n = A.m, nnz = A.rp[n];
    baas_b200::Scheduler<CSR> sch(&A, true, false, baas_b200::P2P_RULE, 8);
    sch.preprocessing();
    int ngroups = 0;
    baas_schedule_export(sch.handle(), BAAS_FIELD_NGROUPS, &ngroups);
    if (ngroups <= 0 || ngroups > n) return fail("schedule");
    try {
        baas_b200::Scheduler<CSR> bad(&A, true, true, baas_b200::P2P_RULE, 8);
        return fail("isTRSVPerm accepted");
    } catch (const std::runtime_error &) {
    }
    // the P2P algorithm (level merge + cost split): a different task layout on the same groups
    baas_b200::Scheduler<CSR> p2p(&A, true, false, baas_b200::P2P, 8);
    p2p.preprocessing();
    int ntasks_rule = 0, ntasks_p2p = 0, ngroups_p2p = 0;
    baas_schedule_export(sch.handle(), BAAS_FIELD_NTASKS, &ntasks_rule);
    baas_schedule_export(p2p.handle(), BAAS_FIELD_NTASKS, &ntasks_p2p);
    baas_schedule_export(p2p.handle(), BAAS_FIELD_NGROUPS, &ngroups_p2p);
    if (ngroups_p2p != ngroups || ntasks_p2p <= 0 || ntasks_p2p == ntasks_rule) return fail("P2P schedule");
    if (analysis_only) {
        std::printf("OK analysis ngroups=%d\n", ngroups);
        return 0;
    }

    // IC0 on host arrays, against the oracle
    std::vector<int> diag(n);
    for (int i = 0; i < n; i++) {
        int e = A.rp[i];
        while (A.ci[e] < i) e++;
        diag[i] = e;
    }
    std::vector<double> lu(A.va), want(A.va);
    sch.runIC0(&A, lu.data());
    if (orc_ic0(n, A.rowptr, A.colidx, diag.data(), want.data()) != 0) return fail("oracle pivots");
    if (std::memcmp(lu.data(), want.data(), sizeof(double) * nnz) != 0) return fail("runIC0");
    std::vector<double> lu2(A.va);
    p2p.runIC0(&A, lu2.data());
    if (std::memcmp(lu2.data(), want.data(), sizeof(double) * nnz) != 0) return fail("runIC0 (P2P)");

    CSR L, U;
    split(A, lu, L, U);
    std::vector<double> b(n), y(n), z(n), yw(n), zw(n);
    for (int i = 0; i < n; i++) b[i] = 1.0 - 2.0 * ((i * 7919) % 1000) / 1000.0;
    sch.runForwardTRSVNoPerm(&L, y.data(), b.data());
    orc_lower_solve(n, L.rowptr, L.colidx, L.values, b.data(), yw.data());
    if (std::memcmp(y.data(), yw.data(), sizeof(double) * n) != 0) return fail("runForwardTRSVNoPerm");
    sch.runBackwardTRSVNoPerm(&U, z.data(), y.data());
    orc_upper_solve_desc(n, U.rowptr, U.colidx, U.values, yw.data(), zw.data());
    if (std::memcmp(z.data(), zw.data(), sizeof(double) * n) != 0) return fail("runBackwardTRSVNoPerm");
    // isSymmetric = false: the forward schedule only (test/Schedule.hpp:289-292)
    baas_b200::Scheduler<CSR> fwd_only(&A, false, false, baas_b200::P2P_RULE, 8);
    std::vector<double> y2(n);
    fwd_only.runForwardTRSVNoPerm(&L, y2.data(), b.data());
    if (std::memcmp(y2.data(), yw.data(), sizeof(double) * n) != 0) return fail("forward sweep (isSymmetric = false)");
    try {
        fwd_only.runBackwardTRSVNoPerm(&U, z.data(), y.data());
        return fail("backward sweep without a backward schedule accepted");
    } catch (const std::runtime_error &) {
    }

    // runtime classes
    std::vector<double> xtrue(n);
    for (int i = 0; i < n; i++) xtrue[i] = 0.5 + 0.25 * std::sin(0.1 * i);
    baas_b200::SpTRSVRuntime<CSR> sp(&L, xtrue.data(), n, L.rp[n], 1.0, "BAAS-B200-SpTRSV", 8);
    sp.set_num_test(3);
    sp.evaluate();
    if (!(sp.getMaxError() < 1e-10)) return fail("SpTRSVRuntime");
    // the reference's ablation classes: their schedules, the same sweep result
    baas_b200::SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P<CSR> wos(&L, xtrue.data(), n, L.rp[n], 1.0, "BAASWOS", 8);
    baas_b200::SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRuleAblationWOAggregation<CSR> woa(&L, xtrue.data(), n, L.rp[n],
                                                                                          1.0, "BAASWOA", 8);
    baas_b200::SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRuleAblationBase<CSR> woas(&L, xtrue.data(), n, L.rp[n], 1.0,
                                                                                  "BAASWOAS", 8);
    baas_b200::SpTRSVRuntime<CSR> *abl[3] = {&wos, &woa, &woas};
    for (auto *r : abl) {
        r->set_num_test(2);
        r->evaluate();
        if (!(r->getMaxError() < 1e-10)) return fail(r->getAlgName().c_str());
        for (int i = 0; i < n; i++)
            if (r->getSolution()[i] != sp.getSolution()[i]) return fail("ablation sweep differs from BAAS's");
    }
    baas_b200::ICRuntime<CSR> ic(&A, want.data(), n, nnz, "BAAS-B200-IC0", 8);
    ic.set_num_test(3);
    ic.evaluate();
    if (ic.getMaxError() != 0.0) return fail("ICRuntime");
    std::printf("OK gpu ngroups=%d sptrsv_ms=%.4f ic0_ms=%.4f\n", ngroups, sp.getElaspedTime(), ic.getElaspedTime());
    return 0;
}
