/*
 * mspai_b200 -- Matrix Market input/output and problem assembly (host, C ABI).
 *
 * These replace the reference's file layer: Read_mm_Matrix::Read_Matrix_File
 * / Read_Target_File (src/Read_mm_Matrix.cpp:115-420), Pattern::
 * Arbitrary_Pattern / Diagonal_Pattern / Matrix::To_Pattern
 * (src/Pattern.cpp:75-139, 378-423, src/Matrix.imp:286-356) and
 * Matrix::Write_Matrix_To_File (src/Matrix.cpp:251-340).
 */
#ifndef MSPAI_B200_IO_H
#define MSPAI_B200_IO_H

#include "mspai_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A host CSC matrix owned by the library (free with mspai_matrix_free). */
typedef struct {
    int32_t nrows, ncols;
    int64_t nnz;
    int64_t* colptr;
    int32_t* rowidx;
    double* values;  /* NULL for a pattern file */
    int32_t symmetric; /* the file was stored symmetric (expanded on read) */
} mspai_matrix;

/* View of an owned matrix as a mspai_csc (host memory). */
mspai_csc mspai_matrix_view(const mspai_matrix* m);

void mspai_matrix_free(mspai_matrix* m);

/*
 * Reads a Matrix Market coordinate file (real, integer or pattern; general or
 * symmetric; symmetric files are expanded).  Entries are sorted by column and
 * row; duplicate entries are summed.  Returns MSPAI_ERR_IO / MSPAI_ERR_INPUT
 * with a message in msg on failure.
 */
int mspai_mm_read(const char* path, mspai_matrix* out, char* msg, int32_t msg_len);

/*
 * Writes M in the reference's output format: "%%MatrixMarket matrix
 * coordinate real general", "m n nnz", then one "row col<sp>value" line per
 * entry, 1-based, value "%.13e" preceded by one space if negative and two
 * otherwise (src/Matrix.cpp:290-312).
 */
int mspai_mm_write(const char* path, const mspai_csc* M, char* msg, int32_t msg_len);

/*
 * Builds C = [A; rho * Ce] (probing rows appended at n..n+p-1, values
 * scaled by rho as src/Read_mm_Matrix.cpp:566-577) and the target
 * B = [I; rho * Be] (src/Read_mm_Matrix.cpp:601-667).  Ce and Be are p x n;
 * either may be NULL (no probing: C = A and B = I).  Outputs are owned.
 */
int mspai_probing_assemble(const mspai_csc* A, const mspai_csc* Ce, const mspai_csc* Be,
                           double rho, mspai_matrix* C_out, mspai_matrix* B_out, char* msg,
                           int32_t msg_len);

/*
 * Start patterns: kind 1 = diagonal (Diagonal_Pattern), kind 2 = the pattern
 * of the first n rows of C (To_Pattern with probing rows omitted).
 */
int mspai_pattern_generate(const mspai_csc* C, int32_t kind, mspai_matrix* P_out);

/*
 * Block start patterns for constant block size bs (n / bs block columns):
 * kind 1 = diagonal blocks, kind 2 = the block pattern of C's first n rows
 * (a block is present when any of its entries is stored), as the reference's
 * Diagonal_Pattern / To_Pattern on the block matrix of
 * Matrix::Convert_Block_Matrix (src/Matrix.imp:1280-1360).
 */
int mspai_block_pattern_generate(const mspai_csc* C, int32_t bs, int32_t kind,
                                 mspai_matrix* P_out);

/*
 * The reference's power pattern with its count-based sparsification
 * (To_Pattern_Powers, src/Matrix.imp:359-470, there through PETSc): with
 * S = Sparsify(|A|), then nb_pw times { S = Sparsify(S) (from the second
 * time on); S = S S }, then S = Sparsify(S), P = pattern(S).  Sparsify
 * (src/Matrix.imp:471-620) keeps in column k the lfill_k = nnz(A(:, k))
 * largest entries by magnitude, every entry equal in magnitude to the
 * smallest kept one, and the diagonal (which takes the place of the smallest
 * kept entry when it is not among them; value 0 when absent).  Equal
 * magnitudes are ordered by row (a stable sort of the row-ordered column).
 * A square on the host with values, 0 <= nb_pw <= 4; computed on GPU
 * `device`; P_out owned (mspai_matrix_free), its values the magnitudes of S.
 * A column may hold at most 8192 products or entries, else
 * MSPAI_ERR_CAPACITY.
 */
int mspai_pattern_powers(const mspai_csc* A, int32_t nb_pw, int32_t device, mspai_matrix* P_out,
                         char* msg, int32_t msg_len);

/*
 * Start pattern from the square of A (the first n rows of C), computed on
 * GPU `device`: P(:, k) = { i : |(A^2)(i, k)| >= drop * max_i |(A^2)(i, k)| }
 * (drop = 0 keeps the whole pattern of A^2).  The family of the reference's
 * power patterns (To_Pattern_Powers / To_Pattern_Power,
 * src/Matrix.imp:359-470, src/Matrix.cpp:602-636, there through PETSc
 * MatMatMult and a count-based Sparsify); here a relative drop tolerance.
 * C on the host with values; P_out owned (mspai_matrix_free).  A column of
 * A^2 may gather at most 8192 products A(i, l) A(l, k), else
 * MSPAI_ERR_CAPACITY.
 */
int mspai_pattern_power2(const mspai_csc* C, double drop, int32_t device, mspai_matrix* P_out,
                         char* msg, int32_t msg_len);

/* CSR row structure of the first nrows_keep rows of C, as a CSC of C^T. */
int mspai_row_structure(const mspai_csc* C, int32_t nrows_keep, mspai_matrix* R_out);

#ifdef __cplusplus
}
#endif

#endif /* MSPAI_B200_IO_H */
