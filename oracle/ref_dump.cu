/*
 * ref_dump.cu -- runs the culip reference's own BlockiLDLt / CSRMatrixSPMV /
 * SQMR (compiled from its sources by oracle/build_ref.py) on one input and
 * writes what they computed, so the tests can compare culip_b200 with the
 * reference itself.
 *
 * TEST INFRASTRUCTURE ONLY: built into oracle/_ref/ref_dump, run by the
 * tests as the checker, never by the product.
 *
 * The steps follow apps/block_ildlt/block_ildlt_invariants.h:73-196
 * (bildlt_fun): K and the pivot starts go to the BlockiLDLt constructor, the
 * factorization runs, the solve analysis for the chosen algorithm, then
 * SQMR(K, tol, max_it, preconditioner).  Differences: the system comes
 * from a binary file instead of MatrixMarket files, the permutation is the
 * identity (host_permute with the identity returns K unchanged), b is
 * given instead of K * ones, and compute() is run as its steps
 * (block_ildlt.impl.cuh:107-145, same order) so that the numeric
 * factorization is timed apart from the host symbolic phase.
 *
 * usage: ref_dump <in.bin> <out.bin> <precision 0=float 1=double>
 *                 <pivot 0=static 1=BK 2=Rook> <fill_level> <fill_factor>
 *                 <threshold> <tol> <max_it> <solve_algorithm 0..3>
 *                 <jacobi_sweeps> <solve_repeats>
 *
 * in.bin (little endian): int32 n, int32 num_blocks, int64 nnz,
 *   int32 rowptr[n+1], int32 colidx[nnz], float64 val[nnz],
 *   int32 block_starts[num_blocks+1], int32 is_piv[n], float64 b[n]
 * out.bin: records {char name[16], int32 kind (0 int32, 1 float32,
 *   2 float64, 3 int64), int64 count, data}; see the names written below.
 */
#include <libs/utils/types.cuh>
#include <libs/la/preconditioner/block_ildlt.cuh>
#include <libs/la/spmv.cuh>
#include <libs/la/iterative_solvers/sqmr.cuh>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace NS_CULIP;
using namespace NS_CULIP::NS_LA;

namespace {

struct Input {
    int n = 0, num_blocks = 0;
    int64_t nnz = 0;
    std::vector<int> rowptr, colidx, block_starts, is_piv;
    std::vector<double> val, b;
};

template <class V>
bool read_into(FILE* f, V& v, size_t count)
{
    v.resize(count);
    return count == 0 || fread(v.data(), sizeof(v[0]), count, f) == count;
}

bool read_input(const char* path, Input& in)
{
    FILE* f = fopen(path, "rb");
    if (!f) return false;
    bool ok = fread(&in.n, 4, 1, f) == 1 && fread(&in.num_blocks, 4, 1, f) == 1 && fread(&in.nnz, 8, 1, f) == 1;
    ok = ok && in.n > 0 && in.num_blocks > 0 && in.nnz > 0 && in.nnz < (int64_t)INT32_MAX;
    ok = ok && read_into(f, in.rowptr, in.n + 1) && read_into(f, in.colidx, in.nnz) && read_into(f, in.val, in.nnz);
    ok = ok && read_into(f, in.block_starts, in.num_blocks + 1) && read_into(f, in.is_piv, in.n);
    ok = ok && read_into(f, in.b, in.n);
    fclose(f);
    return ok && in.rowptr[in.n] == in.nnz && in.block_starts[in.num_blocks] == in.n;
}

struct Writer {
    FILE* f;
    template <class T>
    void put(const char* name, const T* p, int64_t count)
    {
        char tag[16] = {};
        strncpy(tag, name, 15);
        int32_t kind = std::is_same<T, int32_t>::value ? 0 : std::is_same<T, float>::value ? 1
                       : std::is_same<T, double>::value ? 2 : 3;
        fwrite(tag, 1, 16, f);
        fwrite(&kind, 4, 1, f);
        fwrite(&count, 8, 1, f);
        if (count) fwrite(p, sizeof(T), count, f);
    }
    template <class T>
    void put(const char* name, const std::vector<T>& v) { put(name, v.data(), (int64_t)v.size()); }
    template <class T>
    void put1(const char* name, T v) { put(name, &v, 1); }
};

template <class T>
std::vector<T> to_host(const dense_vector_t<T>* d)
{
    dense_vector_ptr<T> h = make_managed_dense_vector_ptr<T>(false);
    *h = d;
    return std::vector<T>(h->dense_val, h->dense_val + h->m);
}

template <class T>
dense_vector_ptr<T> to_device(const std::vector<double>& v)
{
    dense_vector_ptr<T> h = make_managed_dense_vector_ptr<T>((mat_size_t)v.size(), false);
    for (size_t i = 0; i < v.size(); ++i) h->dense_val[i] = (T)v[i];
    dense_vector_ptr<T> d = make_managed_dense_vector_ptr<T>(true);
    *d = h.get();
    return d;
}

double seconds_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// BlockiLDLt with access to its protected state for the dump
template <typename T, bool BK, bool Rook>
class Dumper : public BlockiLDLt<T, BK, Rook> {
public:
    using Base = BlockiLDLt<T, BK, Rook>;
    using Base::Base;

    double symbolic_s = 0, upload_s = 0, factor_s = 0;

    // the steps of BlockiLDLt::compute (block_ildlt.impl.cuh:107-145), timed
    void compute_timed(mat_int_t fill_level, T fill_factor, T threshold)
    {
        dense_vector_ptr<mat_int_t> A_block_nnz, U_block_nnz;
        auto t0 = std::chrono::steady_clock::now();
        this->build_initial_coarse(A_block_nnz);
        this->determine_coarse_level_fill_and_diag(fill_level, A_block_nnz->dense_val, U_block_nnz);
        this->build_block_csc();
        this->find_level_sets();
        this->build_blocks(fill_factor, U_block_nnz->dense_val);
        symbolic_s = seconds_since(t0);
        // upload_data sizes the in-flight tile store as the int product
        // m_max_level_blocks * 32 * 32 (block_ildlt.impl.cuh:1343-1345) and the
        // kernels index it with int offsets: refuse levels whose tiles would
        // overflow it instead of running into out-of-bounds writes
        if ((int64_t)this->m_max_level_blocks * 1024 >= (int64_t)INT32_MAX) {
            fprintf(stderr, "ref_dump: %d blocks in one level exceed the reference's int32 tile store\n",
                    this->m_max_level_blocks);
            std::exit(3);
        }
        t0 = std::chrono::steady_clock::now();
        this->upload_data();
        upload_s = seconds_since(t0);
        CHECK_CUDA(cudaDeviceSynchronize());
        t0 = std::chrono::steady_clock::now();
        this->factorize(threshold);
        CHECK_CUDA(cudaDeviceSynchronize());
        factor_s = seconds_since(t0);
        this->download_data();
        this->eval_results();
    }

    static void put_list(Writer& w, const char* off, const char* idx, const compressed_block_list& l)
    {
        w.put(off, l.offsets->dense_val, (int64_t)l.offsets->m);
        w.put(idx, l.indices->dense_val, (int64_t)l.indices->m);
    }

    void dump(Writer& w)
    {
        const matrix_block* blk = this->m_h_blocks->dense_val;
        const int64_t nb = (int64_t)this->m_h_blocks->m;
        std::vector<int32_t> desc((size_t)nb * 9);
        for (int64_t i = 0; i < nb; ++i) {
            int32_t* d = &desc[(size_t)i * 9];
            d[0] = blk[i].id; d[1] = (int32_t)blk[i].format; d[2] = blk[i].nnz; d[3] = blk[i].max_nnz;
            d[4] = blk[i].got_extra; d[5] = blk[i].block_row; d[6] = blk[i].block_col;
            d[7] = blk[i].col_ptr; d[8] = blk[i].val_ptr;
        }
        w.put("blocks", desc);
        w.put("val_store", this->m_h_block_val_store->dense_val, (int64_t)this->m_h_block_val_store->m);
        w.put("ix_store", this->m_h_block_ix_store->dense_val, (int64_t)this->m_h_block_ix_store->m);
        w.put("tri", this->m_h_tridiagonal->dense_val, (int64_t)this->m_h_tridiagonal->m);
        w.put("perm", this->m_h_permutation->dense_val, (int64_t)this->m_h_permutation->m);
        w.put("is_piv", to_host<mat_int_t>(this->m_d_ispiv.get()));
        w.put("block_starts", this->m_h_block_starts->dense_val, (int64_t)this->m_h_block_starts->m);
        put_list(w, "coarse_off", "coarse_col", this->m_h_coarse_csr);
        put_list(w, "csc_off", "csc_blk", this->m_h_coarse_csc);
        put_list(w, "level_off", "level_rows", this->m_h_levels);
        put_list(w, "lblk_off", "lblk", this->m_h_levels_blocks);
        w.put1<int32_t>("max_level_blks", this->m_max_level_blocks);
    }
};

template <typename T, bool BK, bool Rook>
int run(const Input& in, Writer& w, char** argv)
{
    const mat_int_t fill_level = atoi(argv[5]);
    const T fill_factor = (T)std::max(1.0, atof(argv[6]));
    const T threshold = (T)atof(argv[7]);
    const T tol = (T)atof(argv[8]);
    const mat_int_t max_it = atoi(argv[9]);
    const int algo = atoi(argv[10]);
    const mat_int_t sweeps = atoi(argv[11]);
    const int repeats = std::max(1, atoi(argv[12]));
    const int n = in.n;

    gpu_handle_ptr handle(new gpu_handle_t);

    // host K in T (the reference driver reads doubles and casts, test.impl.h:66)
    csr_matrix_ptr<T> h_K = make_csr_matrix_ptr<T>(n, n, in.nnz, false);
    std::copy(in.rowptr.begin(), in.rowptr.end(), h_K->csr_row);
    std::copy(in.colidx.begin(), in.colidx.end(), h_K->csr_col);
    for (int64_t k = 0; k < in.nnz; ++k) h_K->csr_val[k] = (T)in.val[k];

    // pivot starts from the 0/1 pivot vector, as bildlt_fun builds them
    std::vector<mat_int_t> piv_starts;
    for (int i = 0; i < n; ++i)
        if (in.is_piv[i] == 1) piv_starts.push_back(i);
    piv_starts.push_back(n);

    Dumper<T, BK, Rook> prec(handle, h_K.get(), (mat_int_t)piv_starts.size() - 1, piv_starts.data(),
                             in.num_blocks, in.block_starts.data());
    prec.compute_timed(fill_level, fill_factor, threshold);
    prec.dump(w);

    prec.set_solve_algorithm((SOLVE_ALGORITHM)algo, sweeps);
    auto t0 = std::chrono::steady_clock::now();
    prec.solve_analysis();
    const double analysis_s = seconds_since(t0);

    // the three preconditioner stages applied to b on their own
    dense_vector_ptr<T> d_b = to_device<T>(in.b);
    dense_vector_ptr<T> d_y = make_managed_dense_vector_ptr<T>(n, true);
    prec.solve_left(d_b.get(), d_y.get());
    w.put("apply_left", to_host<T>(d_y.get()));
    prec.solve_middle(d_b.get(), d_y.get());
    w.put("apply_middle", to_host<T>(d_y.get()));
    prec.solve_right(d_b.get(), d_y.get());
    w.put("apply_right", to_host<T>(d_y.get()));

    // SQMR with the reference's CSR operator
    csr_matrix_ptr<T> d_K = make_csr_matrix_ptr<T>(true);
    *d_K = h_K.get();
    CSRMatrixSPMV<T> spmv(handle, d_K.get());
    SQMR<T> sqmr(handle, (SPMV<T>*)&spmv, tol, max_it, (Preconditioner<T>*)&prec);
    dense_vector_ptr<T> d_x = make_managed_dense_vector_ptr<T>(n, true);
    T residual = 0;
    mat_int_t iterations = 0;
    double best = 1e300;
    for (int r = 0; r < repeats; ++r) {
        CHECK_CUDA(cudaDeviceSynchronize());
        t0 = std::chrono::steady_clock::now();
        sqmr.solve(d_b.get(), d_x.get(), residual, iterations);
        CHECK_CUDA(cudaDeviceSynchronize());
        best = std::min(best, seconds_since(t0));
    }
    const std::vector<T> x = to_host<T>(d_x.get());

    // true relative residual ||b - K x|| / ||b|| in double on the host
    double rr = 0, bb = 0;
    for (int i = 0; i < n; ++i) {
        double s = in.b[i];
        for (int k = in.rowptr[i]; k < in.rowptr[i + 1]; ++k) s -= in.val[k] * (double)x[in.colidx[k]];
        rr += s * s;
        bb += in.b[i] * in.b[i];
    }
    w.put("x", x);
    w.put1<double>("residual", (double)residual);
    w.put1<int32_t>("iterations", iterations);
    w.put1<double>("true_relres", std::sqrt(rr) / std::sqrt(bb));
    w.put1<double>("symbolic_s", prec.symbolic_s);
    w.put1<double>("upload_s", prec.upload_s);
    w.put1<double>("factor_s", prec.factor_s);
    w.put1<double>("analysis_s", analysis_s);
    w.put1<double>("sqmr_s", best);
    printf("ref_dump: n=%d factor %.3f ms, sqmr %.3f ms, %d iterations, residual %g, true relres %g\n", n,
           prec.factor_s * 1e3, best * 1e3, iterations, (double)residual, std::sqrt(rr) / std::sqrt(bb));
    return 0;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc != 13) {
        fprintf(stderr, "usage: %s in.bin out.bin precision pivot fill_level fill_factor threshold tol max_it "
                        "solve_algorithm jacobi_sweeps solve_repeats\n", argv[0]);
        return 2;
    }
    Input in;
    if (!read_input(argv[1], in)) {
        fprintf(stderr, "ref_dump: cannot read %s\n", argv[1]);
        return 2;
    }
    const int prec = atoi(argv[3]), pivot = atoi(argv[4]);
    if (pivot == 2) {
        // the reference's Rook search (block_ildlt_kernels.impl.cuh:886-945) has no iteration bound
        fprintf(stderr, "ref_dump: Rook pivoting is not run here\n");
        return 2;
    }
    FILE* f = fopen(argv[2], "wb");
    if (!f) return 2;
    Writer w{f};
    int rc;
    if (prec == 1) rc = pivot == 1 ? run<double, true, false>(in, w, argv) : run<double, false, false>(in, w, argv);
    else rc = pivot == 1 ? run<float, true, false>(in, w, argv) : run<float, false, false>(in, w, argv);
    fclose(f);
    GlobalMemPool().cleanup();
    return rc;
}
