// Options: reference defaults and the reference's option checks.
//
// Defaults follow Command_Line::Parameters (reference src/Command_Line.cpp:
// 192-225); the checks and their messages follow
// PC_MSPAI::PCSetFromOptions_SPAI (src/imspai.cpp:238-480) and the parameter
// dependencies of the user documentation (doc/mspai-1.2.pdf section 2.4).
#include "host_util.h"
#include "mspai_b200.h"

#include <algorithm>
#include <cstdio>
#include <cstring>

extern "C" void mspai_default_params(mspai_params* p)
{
    std::memset(p, 0, sizeof(*p));
    p->ep = 0.4;
    p->mn = 5;
    p->ns = 5;
    p->um = 1;
    p->hs = 6;
    p->cs = 0;
    p->qr = 0;
    p->ch = 0;
    p->fg = 0.3;
    p->pk = 0;
    p->pm = 0;
    p->schur = 0;
    p->rho = 1.0;
    p->bs = 1;
    p->target = 1;
    p->probing = 0;
    p->prec = MSPAI_PREC_MIXED;
    p->refine = 4;
    p->batched = 1;
    p->verbose = 0;
    p->col_begin = 0;
    p->col_end = 0;
    p->keep_factors = 0;
    p->reuse_factors = 0;
}

static int fail(char* msg, int len, const char* text)
{
    if (msg && len > 0) {
        std::strncpy(msg, text, static_cast<size_t>(len) - 1);
        msg[len - 1] = '\0';
    }
    return MSPAI_ERR_PARAM;
}

extern "C" int mspai_validate_params(const mspai_params* p, char* msg, int32_t len)
{
    char buf[512];
    if (msg && len > 0)
        msg[0] = '\0';
    if (!p)
        return fail(msg, len, "null parameters");
    if (p->ns < 0) {
        std::snprintf(buf, sizeof(buf),
                      "Illegal number of improvement steps: %d\nAllowed are positive values.",
                      p->ns);
        return fail(msg, len, buf);
    }
    if (p->ep < 0) {
        std::snprintf(buf, sizeof(buf), "Illegal epsilon: %g\nAllowed are positive values.", p->ep);
        return fail(msg, len, buf);
    }
    if (p->mn < 0) {
        std::snprintf(buf, sizeof(buf), "Illegal maximum number of new candidates: %d", p->mn);
        return fail(msg, len, buf);
    }
    if (p->hs < 0 || p->hs > 6) {
        std::snprintf(buf, sizeof(buf),
                      "Illegal hash table size parameter: %d\nAllowed are 0..6 (default 6).",
                      p->hs);
        return fail(msg, len, buf);
    }
    if (p->cs < 0 || p->cs > 10000000) {
        std::snprintf(buf, sizeof(buf),
                      "Illegal cache size parameter: %d\nAllowed are positiv values smaller "
                      "than 1e+7.",
                      p->cs);
        return fail(msg, len, buf);
    }
    if (p->ch < 0 || p->ch > 1) {
        std::snprintf(buf, sizeof(buf),
                      "Illegal hash size parameter: %d\nPlease use 1 for using a hashtable and "
                      "0 for not using a hashtable.",
                      p->ch);
        return fail(msg, len, buf);
    }
    if (p->cs > 0 && p->ch > 0)
        return fail(msg, len,
                    "Caching and Hashing cannot be used simultaneously\nPlease use either "
                    "caching OR hashing algorithm.");
    if (p->cs > 0 && p->qr > 0)
        return fail(msg, len,
                    "QR-Updates and Caching optimization cannot\nbe used simultaneously!");
    if (p->ch > 0 && p->qr > 0)
        return fail(msg, len,
                    "QR-Updates and Hashing optimization cannot\nbe used simultaneously!");
    if (p->qr < 0 || p->qr > 5) {
        std::snprintf(buf, sizeof(buf), "Illegal parameter for qr: %d\nAllowed are 0..5.", p->qr);
        return fail(msg, len, buf);
    }
    if (p->fg < 0.0 || p->fg > 1.0) {
        std::snprintf(buf, sizeof(buf),
                      "Illegal parameter for fg: %g\nAllowed are:\n0.0 <= fg <= 1.0", p->fg);
        return fail(msg, len, buf);
    }
    if (p->rho < 0.0) {
        std::snprintf(buf, sizeof(buf),
                      "Illegal parameter for rho: %g\nAllowed are:\n0.0 <= rho", p->rho);
        return fail(msg, len, buf);
    }
    if (p->um < 0 || p->um > 1) {
        std::snprintf(buf, sizeof(buf), "Illegal value for using mean value: %d", p->um);
        return fail(msg, len, buf);
    }
    if (p->schur < 0 || p->schur > 1) {
        std::snprintf(buf, sizeof(buf), "Illegal value for using schur value: %d", p->schur);
        return fail(msg, len, buf);
    }
    if (p->schur && !p->target)
        return fail(msg, len,
                    "Arbitrary target matrices are not\nallowed when using schur probing!");
    if (p->schur && !p->probing)
        return fail(msg, len,
                    "No probing condition defined but schur \nprobing requested!");
    if (p->pk < 0) {
        std::snprintf(buf, sizeof(buf), "Illegal number of prerequesting columns k: %d", p->pk);
        return fail(msg, len, buf);
    }
    if (p->pm < 0 || p->pm > 1) {
        std::snprintf(buf, sizeof(buf),
                      "Illegal parameter for prerequesting maximum columns: %d", p->pm);
        return fail(msg, len, buf);
    }
    if ((p->probing || !p->target) && (p->ns > 0 || p->qr > 0))
        return fail(msg, len,
                    "Probing constraints and/or target matrix approximations\nare only "
                    "supported in static MSPAI yet!\nPlease set the number of improvement "
                    "steps to 0.");
    if (p->bs < 1) {
        std::snprintf(buf, sizeof(buf), "Illegal block size: %d", p->bs);
        return fail(msg, len, buf);
    }
    if (p->prec != MSPAI_PREC_FP64 && p->prec != MSPAI_PREC_MIXED) {
        std::snprintf(buf, sizeof(buf), "Illegal precision: %d", p->prec);
        return fail(msg, len, buf);
    }
    if (p->reuse_factors < 0 || p->reuse_factors > 64) {
        std::snprintf(buf, sizeof(buf), "Illegal number of re-setup refinement steps: %d",
                      p->reuse_factors);
        return fail(msg, len, buf);
    }
    if (p->refine < 0 || p->refine > 16) {
        std::snprintf(buf, sizeof(buf), "Illegal number of refinement steps: %d", p->refine);
        return fail(msg, len, buf);
    }
    return MSPAI_OK;
}

namespace mspai_host {

void csc_row_structure(int ncols, const int64_t* colptr, const int32_t* rowidx, int nrows_keep,
                       std::vector<int64_t>& rptr, std::vector<int32_t>& rcol)
{
    rptr.assign(static_cast<size_t>(nrows_keep) + 1, 0);
    for (int c = 0; c < ncols; c++)
        for (int64_t p = colptr[c]; p < colptr[c + 1]; p++)
            if (rowidx[p] < nrows_keep)
                rptr[rowidx[p] + 1]++;
    for (int r = 0; r < nrows_keep; r++)
        rptr[r + 1] += rptr[r];
    rcol.assign(static_cast<size_t>(rptr[nrows_keep]), 0);
    std::vector<int64_t> fill(rptr.begin(), rptr.end() - 1);
    for (int c = 0; c < ncols; c++)  // ascending c keeps each row's list sorted
        for (int64_t p = colptr[c]; p < colptr[c + 1]; p++)
            if (rowidx[p] < nrows_keep)
                rcol[fill[rowidx[p]]++] = c;
}

}  // namespace mspai_host
