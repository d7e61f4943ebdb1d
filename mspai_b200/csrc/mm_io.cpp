// Matrix Market input/output and problem assembly (host side).
#include "host_util.h"
#include "mspai_b200_io.h"

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

namespace {

int io_fail(char* msg, int len, int code, const std::string& text)
{
    if (msg && len > 0) {
        std::strncpy(msg, text.c_str(), static_cast<size_t>(len) - 1);
        msg[len - 1] = '\0';
    }
    return code;
}

struct Triplet {
    int32_t r, c;
    double v;
};

// Sorted CSC from triplets (duplicates summed) into an owned mspai_matrix.
int triplets_to_csc(int nrows, int ncols, std::vector<Triplet>& t, bool values, mspai_matrix* out)
{
    std::sort(t.begin(), t.end(), [](const Triplet& a, const Triplet& b) {
        return a.c != b.c ? a.c < b.c : a.r < b.r;
    });
    size_t w = 0;
    for (size_t i = 0; i < t.size(); i++) {
        if (w > 0 && t[w - 1].r == t[i].r && t[w - 1].c == t[i].c)
            t[w - 1].v += t[i].v;
        else
            t[w++] = t[i];
    }
    t.resize(w);
    out->nrows = nrows;
    out->ncols = ncols;
    out->nnz = static_cast<int64_t>(w);
    out->colptr = static_cast<int64_t*>(std::calloc(static_cast<size_t>(ncols) + 1, sizeof(int64_t)));
    out->rowidx = static_cast<int32_t*>(std::malloc(std::max<size_t>(w, 1) * sizeof(int32_t)));
    out->values = values ? static_cast<double*>(std::malloc(std::max<size_t>(w, 1) * sizeof(double)))
                         : nullptr;
    if (!out->colptr || !out->rowidx || (values && !out->values))
        return MSPAI_ERR_ALLOC;
    for (size_t i = 0; i < w; i++) {
        out->colptr[t[i].c + 1]++;
        out->rowidx[i] = t[i].r;
        if (values)
            out->values[i] = t[i].v;
    }
    for (int c = 0; c < ncols; c++)
        out->colptr[c + 1] += out->colptr[c];
    return MSPAI_OK;
}

}  // namespace

extern "C" {

mspai_csc mspai_matrix_view(const mspai_matrix* m)
{
    mspai_csc v;
    v.nrows = m->nrows;
    v.ncols = m->ncols;
    v.nnz = m->nnz;
    v.colptr = m->colptr;
    v.rowidx = m->rowidx;
    v.values = m->values;
    v.mem = MSPAI_MEM_HOST;
    return v;
}

void mspai_matrix_free(mspai_matrix* m)
{
    if (!m)
        return;
    std::free(m->colptr);
    std::free(m->rowidx);
    std::free(m->values);
    m->colptr = nullptr;
    m->rowidx = nullptr;
    m->values = nullptr;
    m->nnz = 0;
}

int mspai_mm_read(const char* path, mspai_matrix* out, char* msg, int32_t len)
{
    std::memset(out, 0, sizeof(*out));
    FILE* f = std::fopen(path, "r");
    if (!f)
        return io_fail(msg, len, MSPAI_ERR_IO,
                       std::string("Could not open file ") + path + " for read access!");
    char line[4096];
    if (!std::fgets(line, sizeof(line), f)) {
        std::fclose(f);
        return io_fail(msg, len, MSPAI_ERR_INPUT, "Empty Matrix Market file");
    }
    char banner[64] = {0}, obj[64] = {0}, fmt[64] = {0}, field[64] = {0}, sym[64] = {0};
    if (std::sscanf(line, "%63s %63s %63s %63s %63s", banner, obj, fmt, field, sym) != 5 ||
        std::strcmp(banner, "%%MatrixMarket") != 0) {
        std::fclose(f);
        return io_fail(msg, len, MSPAI_ERR_INPUT, "Missing %%MatrixMarket banner");
    }
    for (char* p : {obj, fmt, field, sym})
        for (; *p; ++p)
            *p = static_cast<char>(std::tolower(static_cast<unsigned char>(*p)));
    if (std::strcmp(obj, "matrix") != 0 || std::strcmp(fmt, "coordinate") != 0) {
        std::fclose(f);
        return io_fail(msg, len, MSPAI_ERR_INPUT, "Only 'matrix coordinate' files are supported");
    }
    const bool pattern = std::strcmp(field, "pattern") == 0;
    if (!pattern && std::strcmp(field, "real") != 0 && std::strcmp(field, "integer") != 0 &&
        std::strcmp(field, "double") != 0) {
        std::fclose(f);
        return io_fail(msg, len, MSPAI_ERR_INPUT,
                       std::string("Unsupported Matrix Market field: ") + field);
    }
    const bool symmetric = std::strcmp(sym, "symmetric") == 0;
    if (!symmetric && std::strcmp(sym, "general") != 0) {
        std::fclose(f);
        return io_fail(msg, len, MSPAI_ERR_INPUT, std::string("Unsupported symmetry: ") + sym);
    }
    do {
        if (!std::fgets(line, sizeof(line), f)) {
            std::fclose(f);
            return io_fail(msg, len, MSPAI_ERR_INPUT,
                           "Could not read matrix size and nnz's properly!");
        }
    } while (line[0] == '%');
    long long m = 0, n = 0, nz = 0;
    if (std::sscanf(line, "%lld %lld %lld", &m, &n, &nz) != 3 || m < 0 || n < 0 || nz < 0 ||
        m > 0x7fffffff || n > 0x7fffffff) {
        std::fclose(f);
        return io_fail(msg, len, MSPAI_ERR_INPUT,
                       "Could not read matrix size and nnz's properly! Second line must be "
                       "m n nnz");
    }
    std::vector<Triplet> t;
    t.reserve(static_cast<size_t>(symmetric ? 2 * nz : nz));
    for (long long i = 0; i < nz; i++) {
        if (!std::fgets(line, sizeof(line), f)) {
            std::fclose(f);
            return io_fail(msg, len, MSPAI_ERR_INPUT, "Truncated Matrix Market file");
        }
        for (char* p = line; *p; ++p)  // the reference accepts ',' separators
            if (*p == ',')
                *p = ' ';
        char* e = nullptr;
        const long long r = std::strtoll(line, &e, 10);
        char* e2 = nullptr;
        const long long c = std::strtoll(e, &e2, 10);
        if (e == line || e2 == e || r < 1 || r > m || c < 1 || c > n) {
            std::fclose(f);
            return io_fail(msg, len, MSPAI_ERR_INPUT,
                           "Bad entry on line " + std::to_string(i + 3) + " of " + path);
        }
        double v = 1.0;
        if (!pattern) {
            char* e3 = nullptr;
            v = std::strtod(e2, &e3);
            if (e3 == e2) {
                std::fclose(f);
                return io_fail(msg, len, MSPAI_ERR_INPUT,
                               "Missing value on line " + std::to_string(i + 3) + " of " + path);
            }
        }
        t.push_back({static_cast<int32_t>(r - 1), static_cast<int32_t>(c - 1), v});
        if (symmetric && r != c)
            t.push_back({static_cast<int32_t>(c - 1), static_cast<int32_t>(r - 1), v});
    }
    std::fclose(f);
    int rc = triplets_to_csc(static_cast<int>(m), static_cast<int>(n), t, !pattern, out);
    out->symmetric = symmetric ? 1 : 0;
    if (rc != MSPAI_OK)
        return io_fail(msg, len, rc, "Out of host memory");
    return MSPAI_OK;
}

int mspai_mm_write(const char* path, const mspai_csc* M, char* msg, int32_t len)
{
    if (!M || M->mem != MSPAI_MEM_HOST)
        return io_fail(msg, len, MSPAI_ERR_PARAM, "mspai_mm_write needs a host matrix");
    FILE* f = std::fopen(path, "w");
    if (!f)
        return io_fail(msg, len, MSPAI_ERR_IO,
                       std::string("Failed writing preconditioner to file ") + path +
                           "\nCheck your access rights!");
    std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n");
    std::fprintf(f, "%d %d %lld\n", M->nrows, M->ncols, static_cast<long long>(M->nnz));
    for (int c = 0; c < M->ncols; c++)
        for (int64_t p = M->colptr[c]; p < M->colptr[c + 1]; p++) {
            const double v = M->values ? M->values[p] : 1.0;
            std::fprintf(f, "%d %d%s%.13e\n", M->rowidx[p] + 1, c + 1, v < 0.0 ? " " : "  ", v);
        }
    const int bad = std::ferror(f);
    std::fclose(f);
    if (bad)
        return io_fail(msg, len, MSPAI_ERR_IO, std::string("Write error on ") + path);
    return MSPAI_OK;
}

int mspai_probing_assemble(const mspai_csc* A, const mspai_csc* Ce, const mspai_csc* Be,
                           double rho, mspai_matrix* C_out, mspai_matrix* B_out, char* msg,
                           int32_t len)
{
    std::memset(C_out, 0, sizeof(*C_out));
    std::memset(B_out, 0, sizeof(*B_out));
    if (!A || A->mem != MSPAI_MEM_HOST || !A->values)
        return io_fail(msg, len, MSPAI_ERR_PARAM, "A must be a host matrix with values");
    if (A->nrows != A->ncols)
        return io_fail(msg, len, MSPAI_ERR_INPUT, "Matrix must be square");
    const int n = A->ncols;
    if ((Ce == nullptr) != (Be == nullptr))
        return io_fail(msg, len, MSPAI_ERR_PARAM,
                       "Only one probing condition defined!\nPlease set a probing condition "
                       "for C (-Ce)\nand a probing condition for B (-Be)!");
    int p = 0;
    if (Ce) {
        if (Ce->ncols != n || Be->ncols != n)
            return io_fail(msg, len, MSPAI_ERR_INPUT,
                           "Mismatch in matrix and probing dimensions!\nProbing matrix and "
                           "system/target matrix must\nhave the same number of columns.");
        if (Ce->nrows != Be->nrows)
            return io_fail(msg, len, MSPAI_ERR_INPUT,
                           "Mismatch in probing dimensions!\nProbing matrix Ce and probing "
                           "matrix Be\nmust have the same number of rows!");
        if (!Ce->values || !Be->values || Ce->mem != MSPAI_MEM_HOST || Be->mem != MSPAI_MEM_HOST)
            return io_fail(msg, len, MSPAI_ERR_PARAM, "probing matrices must be host with values");
        p = Ce->nrows;
    }
    std::vector<Triplet> tc, tb;
    tc.reserve(static_cast<size_t>(A->nnz) + (Ce ? static_cast<size_t>(Ce->nnz) : 0));
    for (int c = 0; c < n; c++)
        for (int64_t q = A->colptr[c]; q < A->colptr[c + 1]; q++)
            tc.push_back({A->rowidx[q], c, A->values[q]});
    for (int c = 0; c < n; c++)
        tb.push_back({c, c, 1.0});
    if (Ce) {
        for (int c = 0; c < n; c++) {
            for (int64_t q = Ce->colptr[c]; q < Ce->colptr[c + 1]; q++)
                tc.push_back({n + Ce->rowidx[q], c, Ce->values[q] * rho});
            for (int64_t q = Be->colptr[c]; q < Be->colptr[c + 1]; q++)
                tb.push_back({n + Be->rowidx[q], c, Be->values[q] * rho});
        }
    }
    int rc = triplets_to_csc(n + p, n, tc, true, C_out);
    if (rc == MSPAI_OK)
        rc = triplets_to_csc(n + p, n, tb, true, B_out);
    if (rc != MSPAI_OK)
        return io_fail(msg, len, rc, "Out of host memory");
    return MSPAI_OK;
}

int mspai_pattern_generate(const mspai_csc* C, int32_t kind, mspai_matrix* P_out)
{
    std::memset(P_out, 0, sizeof(*P_out));
    if (!C || C->mem != MSPAI_MEM_HOST)
        return MSPAI_ERR_PARAM;
    const int n = C->ncols;
    std::vector<Triplet> t;
    if (kind == 1) {
        for (int c = 0; c < n; c++)
            t.push_back({c, c, 1.0});
    }
    else if (kind == 2) {
        for (int c = 0; c < n; c++)
            for (int64_t q = C->colptr[c]; q < C->colptr[c + 1]; q++) {
                if (C->rowidx[q] >= n)
                    break;  // probing rows are not part of P(A)
                t.push_back({C->rowidx[q], c, 1.0});
            }
    }
    else {
        return MSPAI_ERR_PARAM;
    }
    return triplets_to_csc(n, n, t, false, P_out);
}

int mspai_block_pattern_generate(const mspai_csc* C, int32_t bs, int32_t kind,
                                 mspai_matrix* P_out)
{
    std::memset(P_out, 0, sizeof(*P_out));
    if (!C || C->mem != MSPAI_MEM_HOST || bs < 1 || C->ncols % bs != 0)
        return MSPAI_ERR_PARAM;
    const int n = C->ncols, nb = n / bs;
    std::vector<Triplet> t;
    if (kind == 1) {
        for (int c = 0; c < nb; c++)
            t.push_back({c, c, 1.0});
    }
    else if (kind == 2) {
        for (int c = 0; c < n; c++)
            for (int64_t q = C->colptr[c]; q < C->colptr[c + 1]; q++) {
                if (C->rowidx[q] >= n)
                    break;
                t.push_back({C->rowidx[q] / bs, c / bs, 1.0});
            }
    }
    else {
        return MSPAI_ERR_PARAM;
    }
    for (auto& x : t)
        x.v = 0.0;  // duplicates are summed: keep a pattern
    int rc = triplets_to_csc(nb, nb, t, false, P_out);
    return rc;
}

int mspai_row_structure(const mspai_csc* C, int32_t nrows_keep, mspai_matrix* R_out)
{
    std::memset(R_out, 0, sizeof(*R_out));
    if (!C || C->mem != MSPAI_MEM_HOST)
        return MSPAI_ERR_PARAM;
    std::vector<int64_t> rp;
    std::vector<int32_t> rc;
    mspai_host::csc_row_structure(C->ncols, C->colptr, C->rowidx, nrows_keep, rp, rc);
    R_out->nrows = C->ncols;
    R_out->ncols = nrows_keep;
    R_out->nnz = static_cast<int64_t>(rc.size());
    R_out->colptr = static_cast<int64_t*>(std::malloc(rp.size() * sizeof(int64_t)));
    R_out->rowidx = static_cast<int32_t*>(std::malloc(std::max<size_t>(rc.size(), 1) * sizeof(int32_t)));
    if (!R_out->colptr || !R_out->rowidx)
        return MSPAI_ERR_ALLOC;
    std::memcpy(R_out->colptr, rp.data(), rp.size() * sizeof(int64_t));
    if (!rc.empty())
        std::memcpy(R_out->rowidx, rc.data(), rc.size() * sizeof(int32_t));
    return MSPAI_OK;
}

}  // extern "C"
