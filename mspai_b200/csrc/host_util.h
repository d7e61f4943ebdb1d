// Host-side helpers shared by the engine, the Matrix Market layer and the CLI.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace mspai_host {

// Row structure (CSR column lists) of the first `nrows_keep` rows of a CSC
// matrix: for every row r < nrows_keep the sorted column indices j with
// C(r, j) != 0.  This is the row_idcs structure the reference keeps for
// non-symmetric input (src/Compressed_Lines.h:53-101).
void csc_row_structure(int ncols, const int64_t* colptr, const int32_t* rowidx, int nrows_keep,
                       std::vector<int64_t>& rptr, std::vector<int32_t>& rcol);

}  // namespace mspai_host
