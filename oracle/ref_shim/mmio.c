/*
 * mmio.c -- the Matrix Market reader/writer declared in mmio.h (own code,
 * written from the format description there).  TEST INFRASTRUCTURE ONLY.
 */
#include "mmio.h"

#include <ctype.h>
#include <string.h>

static void lower(char* s)
{
    for (; *s; ++s) *s = (char)tolower((unsigned char)*s);
}

int mm_read_banner(FILE* f, MM_typecode* code)
{
    char line[1024], banner[64], obj[64], fmt[64], field[64], sym[64];
    mm_initialize_typecode(code);
    if (!fgets(line, sizeof line, f)) return 1;
    if (sscanf(line, "%63s %63s %63s %63s %63s", banner, obj, fmt, field, sym) != 5) return 2;
    if (strcmp(banner, "%%MatrixMarket") != 0) return 3;
    lower(obj); lower(fmt); lower(field); lower(sym);
    if (strcmp(obj, "matrix") != 0) return 4;
    mm_set_matrix(code);
    if (strcmp(fmt, "coordinate") == 0) mm_set_coordinate(code);
    else if (strcmp(fmt, "array") == 0) mm_set_array(code);
    else return 5;
    if (strcmp(field, "real") == 0 || strcmp(field, "double") == 0) mm_set_real(code);
    else if (strcmp(field, "integer") == 0) mm_set_integer(code);
    else if (strcmp(field, "pattern") == 0) mm_set_pattern(code);
    else return 6;
    if (strcmp(sym, "general") == 0) mm_set_general(code);
    else if (strcmp(sym, "symmetric") == 0) mm_set_symmetric(code);
    else if (strcmp(sym, "skew-symmetric") == 0) (*code)[3] = 'K';
    else return 7;
    return 0;
}

/* next line that is neither a comment nor blank */
static int next_data_line(FILE* f, char* line, int cap)
{
    while (fgets(line, cap, f)) {
        const char* p = line;
        while (*p == ' ' || *p == '\t') ++p;
        if (*p == '%' || *p == '\n' || *p == '\r' || *p == 0) continue;
        return 1;
    }
    return 0;
}

int mm_read_mtx_crd_size(FILE* f, int* m, int* n, int* nnz)
{
    char line[1024];
    *m = *n = *nnz = 0;
    if (!next_data_line(f, line, sizeof line)) return 1;
    return sscanf(line, "%d %d %d", m, n, nnz) == 3 ? 0 : 2;
}

int mm_read_mtx_array_size(FILE* f, int* m, int* n)
{
    char line[1024];
    *m = *n = 0;
    if (!next_data_line(f, line, sizeof line)) return 1;
    return sscanf(line, "%d %d", m, n) == 2 ? 0 : 2;
}

int mm_read_mtx_crd_data(FILE* f, int m, int n, int nnz, int* ii, int* jj, double* val, const char* code)
{
    (void)m; (void)n;
    for (int k = 0; k < nnz; ++k) {
        if (mm_is_pattern(code)) {
            if (fscanf(f, "%d %d", &ii[k], &jj[k]) != 2) return 1;
            val[k] = 1.0;
        } else {
            if (fscanf(f, "%d %d %lg", &ii[k], &jj[k], &val[k]) != 3) return 1;
        }
    }
    return 0;
}

int mm_write_banner(FILE* f, const char* code)
{
    const char* fmt = mm_is_array(code) ? "array" : "coordinate";
    const char* field = code[2] == 'I' ? "integer" : code[2] == 'P' ? "pattern" : "real";
    const char* sym = code[3] == 'S' ? "symmetric" : code[3] == 'K' ? "skew-symmetric" : "general";
    return fprintf(f, "%%%%MatrixMarket matrix %s %s %s\n", fmt, field, sym) > 0 ? 0 : 1;
}

int mm_write_mtx_crd_size(FILE* f, int m, int n, int nnz)
{
    return fprintf(f, "%d %d %d\n", m, n, nnz) > 0 ? 0 : 1;
}

int mm_write_mtx_array_size(FILE* f, int m, int n)
{
    return fprintf(f, "%d %d\n", m, n) > 0 ? 0 : 1;
}
