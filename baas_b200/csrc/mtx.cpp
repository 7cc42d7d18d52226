// MatrixMarket ingestion: a coordinate MatrixMarket file into a host CSR.
//
// Follows the reference's reader chain SPM::CSR(const char *fileName) (spm/CSR.cpp:90-112) ->
// loadMatrixMarket_mmio_highlevel_coo (spm/COO.cpp:322-338) -> mmio_allinone_coo
// (spm/mmio_highlevel.cpp:748-921) -> dcoo2csr with sorting (spm/COO.cpp:222-317):
//   - entries are read in file order, 1-based indices made 0-based; `pattern` entries get the
//     value 1 and `integer` entries their integer value;
//   - symmetric and hermitian files keep the stored entries first and then append, in file
//     order, the mirror (col, row) of every stored off-diagonal entry;
//   - a counting sort by row keeps that order within each row, then each row is sorted by
//     column index.
// The reference sorts rows with its own unstable quicksort, so a repeated (row, column) entry
// would land in an unspecified order there; this reader rejects repeated entries instead. For
// every other file the arrays are identical to the reference's.
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>

#include "../../include/baas_b200.h"

namespace baas {
// set by the C-ABI layer (capi.cu)
baas_status set_error(baas_status code, const std::string &msg);
}

namespace {

bool lower_eq(const std::string &a, const char *b) {
    if (a.size() != strlen(b)) return false;
    for (size_t i = 0; i < a.size(); i++)
        if (tolower((unsigned char)a[i]) != b[i]) return false;
    return true;
}

baas_status bad(const std::string &why) { return baas::set_error(BAAS_ERR_BAD_ARG, "read_mtx: " + why); }

}  // namespace

extern "C" baas_status baas_csr_read_mtx(const char *path, baas_csr *out) {
    if (!path || !out) return bad("NULL argument");
    *out = baas_csr{0, 0, nullptr, nullptr, nullptr};
    FILE *f = fopen(path, "r");
    if (!f) return bad(std::string("cannot open ") + path + ": " + strerror(errno));
    std::vector<char> line(1 << 16);
    auto next_line = [&](bool skip_comments) -> bool {
        while (fgets(line.data(), (int)line.size(), f)) {
            if (skip_comments && line[0] == '%') continue;
            const char *p = line.data();
            while (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n') p++;
            if (skip_comments && *p == 0) continue;
            return true;
        }
        return false;
    };
    // banner: %%MatrixMarket matrix coordinate <field> <symmetry>
    if (!next_line(false)) {
        fclose(f);
        return bad("empty file");
    }
    char w[5][64] = {};
    if (sscanf(line.data(), "%63s %63s %63s %63s %63s", w[0], w[1], w[2], w[3], w[4]) != 5 ||
        !lower_eq(w[0], "%%matrixmarket") || !lower_eq(w[1], "matrix")) {
        fclose(f);
        return bad("not a MatrixMarket matrix banner");
    }
    if (!lower_eq(w[2], "coordinate")) {
        fclose(f);
        return bad("only the coordinate (sparse) format is read");
    }
    const std::string field = w[3], sym = w[4];
    const bool real = lower_eq(field, "real") || lower_eq(field, "double");
    const bool integer = lower_eq(field, "integer"), pattern = lower_eq(field, "pattern");
    if (!real && !integer && !pattern) {
        fclose(f);
        return bad("field '" + field + "' is not read (real, integer or pattern)");
    }
    const bool symmetric = lower_eq(sym, "symmetric") || lower_eq(sym, "hermitian");
    if (!symmetric && !lower_eq(sym, "general")) {
        fclose(f);
        return bad("symmetry '" + sym + "' is not read (general, symmetric or hermitian)");
    }
    long long m = 0, n = 0, nz = 0;
    if (!next_line(true) || sscanf(line.data(), "%lld %lld %lld", &m, &n, &nz) != 3) {
        fclose(f);
        return bad("missing size line");
    }
    if (m != n || m <= 0 || nz < 0 || m > 0x7fffffffLL || nz > 0x3fffffffLL) {
        fclose(f);
        return bad("the matrix must be square with 0 < n < 2^31 and at most 2^30 stored entries");
    }
    std::vector<int> ri, ci;
    std::vector<double> va;
    ri.reserve((size_t)(symmetric ? 2 * nz : nz));
    ci.reserve(ri.capacity());
    va.reserve(ri.capacity());
    for (long long k = 0; k < nz; k++) {
        if (!next_line(true)) {
            fclose(f);
            return bad("fewer entries than the size line declares");
        }
        char *p = line.data(), *e = nullptr;
        const long long i = strtoll(p, &e, 10);
        if (e == p) break;
        p = e;
        const long long j = strtoll(p, &e, 10);
        if (e == p) {
            fclose(f);
            return bad("malformed entry line");
        }
        p = e;
        double v = 1.0;
        if (real) {
            v = strtod(p, &e);
            if (e == p) {
                fclose(f);
                return bad("malformed entry value");
            }
        } else if (integer) {
            const long long iv = strtoll(p, &e, 10);
            if (e == p) {
                fclose(f);
                return bad("malformed entry value");
            }
            v = (double)iv;
        }
        if (i < 1 || i > m || j < 1 || j > n) {
            fclose(f);
            return bad("entry index out of range");
        }
        ri.push_back((int)(i - 1));
        ci.push_back((int)(j - 1));
        va.push_back(v);
    }
    fclose(f);
    if ((long long)ri.size() != nz) return bad("fewer entries than the size line declares");
    if (symmetric) {
        const size_t stored = ri.size();
        for (size_t k = 0; k < stored; k++)
            if (ri[k] != ci[k]) {
                ri.push_back(ci[k]);
                ci.push_back(ri[k]);
                va.push_back(va[k]);
            }
    }
    const int N = (int)n;
    const size_t nnz = ri.size();
    if (nnz > 0x7fffffffULL) return bad("too many entries");
    int *rowptr = (int *)malloc(sizeof(int) * ((size_t)N + 1));
    int *colidx = (int *)malloc(sizeof(int) * std::max<size_t>(nnz, 1));
    double *values = (double *)malloc(sizeof(double) * std::max<size_t>(nnz, 1));
    if (!rowptr || !colidx || !values) {
        free(rowptr);
        free(colidx);
        free(values);
        return baas::set_error(BAAS_ERR_CUDA, "read_mtx: out of host memory");
    }
    // counting sort by row (file order kept within a row), then each row by column
    std::vector<int> next((size_t)N + 1, 0);
    for (size_t k = 0; k < nnz; k++) next[(size_t)ri[k] + 1]++;
    for (int r = 0; r < N; r++) next[(size_t)r + 1] += next[r];
    for (int r = 0; r <= N; r++) rowptr[r] = next[r];
    for (size_t k = 0; k < nnz; k++) {
        const int q = next[ri[k]]++;
        colidx[q] = ci[k];
        values[q] = va[k];
    }
    std::vector<std::pair<int, double>> row;
    for (int r = 0; r < N; r++) {
        const int b = rowptr[r], e = rowptr[r + 1];
        row.clear();
        for (int q = b; q < e; q++) row.push_back({colidx[q], values[q]});
        std::stable_sort(row.begin(), row.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
        for (int q = b; q < e; q++) {
            colidx[q] = row[q - b].first;
            values[q] = row[q - b].second;
            if (q > b && colidx[q] == colidx[q - 1]) {
                free(rowptr);
                free(colidx);
                free(values);
                return bad("repeated entry (" + std::to_string(r + 1) + ", " + std::to_string(colidx[q] + 1) + ")");
            }
        }
    }
    out->n = N;
    out->nnz = (int)nnz;
    out->rowptr = rowptr;
    out->colidx = colidx;
    out->values = values;
    return BAAS_OK;
}

extern "C" void baas_csr_free(baas_csr *mat) {
    if (!mat) return;
    free(const_cast<int *>(mat->rowptr));
    free(const_cast<int *>(mat->colidx));
    free(const_cast<double *>(mat->values));
    *mat = baas_csr{0, 0, nullptr, nullptr, nullptr};
}
