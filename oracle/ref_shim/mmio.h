/*
 * mmio.h -- a small Matrix Market reader/writer with the function names the
 * culip reference's libs/test/test.impl.h calls (the NIST mmio library it
 * was written against is not installed here).  Written from the Matrix
 * Market exchange format: a banner line "%%MatrixMarket matrix
 * <coordinate|array> <real|integer|pattern> <general|symmetric|...>",
 * comment lines starting with '%', a size line, then the entries (1-based
 * "i j [v]" for coordinate, one value per line in column order for array).
 *
 * TEST INFRASTRUCTURE ONLY (reference build, oracle/build_ref.py).
 *
 * MM_typecode holds four characters: [0] 'M' (matrix), [1] 'C' coordinate /
 * 'A' array, [2] 'R' real / 'I' integer / 'P' pattern, [3] 'G' general /
 * 'S' symmetric / 'K' skew-symmetric.
 */
#pragma once

#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef char MM_typecode[4];

int mm_read_banner(FILE* f, MM_typecode* code);
int mm_read_mtx_crd_size(FILE* f, int* m, int* n, int* nnz);
int mm_read_mtx_array_size(FILE* f, int* m, int* n);
/* reads nnz entries (1-based indices as in the file; pattern entries get 1.0) */
int mm_read_mtx_crd_data(FILE* f, int m, int n, int nnz, int* ii, int* jj, double* val, const char* code);
int mm_write_banner(FILE* f, const char* code);
int mm_write_mtx_crd_size(FILE* f, int m, int n, int nnz);
int mm_write_mtx_array_size(FILE* f, int m, int n);

static inline int mm_is_matrix(const char* c) { return c[0] == 'M'; }
static inline int mm_is_sparse(const char* c) { return c[1] == 'C'; }
static inline int mm_is_array(const char* c) { return c[1] == 'A'; }
static inline int mm_is_real(const char* c) { return c[2] == 'R'; }
static inline int mm_is_pattern(const char* c) { return c[2] == 'P'; }
static inline int mm_is_symmetric(const char* c) { return c[3] == 'S'; }
static inline int mm_is_general(const char* c) { return c[3] == 'G'; }
static inline void mm_initialize_typecode(MM_typecode* c) { (*c)[0] = ' '; (*c)[1] = ' '; (*c)[2] = ' '; (*c)[3] = 'G'; }
static inline void mm_set_matrix(MM_typecode* c) { (*c)[0] = 'M'; }
static inline void mm_set_sparse(MM_typecode* c) { (*c)[1] = 'C'; }
static inline void mm_set_coordinate(MM_typecode* c) { (*c)[1] = 'C'; }
static inline void mm_set_array(MM_typecode* c) { (*c)[1] = 'A'; }
static inline void mm_set_dense(MM_typecode* c) { (*c)[1] = 'A'; }
static inline void mm_set_real(MM_typecode* c) { (*c)[2] = 'R'; }
static inline void mm_set_integer(MM_typecode* c) { (*c)[2] = 'I'; }
static inline void mm_set_pattern(MM_typecode* c) { (*c)[2] = 'P'; }
static inline void mm_set_general(MM_typecode* c) { (*c)[3] = 'G'; }
static inline void mm_set_symmetric(MM_typecode* c) { (*c)[3] = 'S'; }

#ifdef __cplusplus
}
#endif
