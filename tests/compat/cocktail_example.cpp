// cocktail_example.cpp — the reference's y = A^k x example (src/eval.cpp:19-72)
// written against the compat headers and linked with libclspmv_b200.so.
//
//   cocktail_example <matrix.mtx> <iterations>
//
// Partitions the matrix with analyze_matrix (tables from $CLSPMVPATH), runs
// the iterations on the GPU through init_mat_kernels / do_spmv /
// cpy_vector_from_gpu, the same iterations on the host with coo_spmv, and
// compares. Exit 0 when every entry agrees to 1e-4 relative to the largest
// magnitude, then runs evaluate() once.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "analyze.h"
#include "fileio.h"
#include "spmv_cocktail.h"
#include "spmv_serial.h"
#include "util.h"

int main(int argc, char** argv)
{
    if (argc < 3) return 2;
    coo_matrix<int, float> coomat;
    init_coo_matrix(coomat);
    ReadMMF(argv[1], &coomat);
    const int iterations = atoi(argv[2]);
    const int n = coomat.matinfo.width, m = coomat.matinfo.height;
    if (coomat.matinfo.nnz == 0 || n != m) return 3;
    std::vector<float> vec(n), res(m, 0.0f);
    for (int i = 0; i < n; i++) vec[i] = (float)((i % 5) - 2) * 0.25f;

    cocktail<int, int, float> mat;
    init_cocktail(mat);
    analyze_matrix(coomat, mat);

    cocktail_gpu gpumat;
    cocktail_kernels kernels;
    init_mat_kernels(mat, vec.data(), res.data(), gpumat, kernels, true);
    if (cocktail_last_status()) return 4;
    cpy_result_from_cpu(gpumat, kernels.context, kernels.cmdQueue, res.data(), m);
    for (int i = 0; i < iterations; i++) {
        do_spmv(kernels, kernels.context, kernels.cmdQueue, 1);
        cpy_vector_from_gpu(gpumat, kernels.context, kernels.cmdQueue, gpumat.res, m);
    }
    std::vector<float> gpures(m);
    cpy_result_to_cpu(gpumat, kernels.context, kernels.cmdQueue, gpures.data(), m);
    if (cocktail_last_status()) return 5;
    free_mat_kernels(gpumat, kernels);

    std::vector<float> cpuvec(vec), cpures(res);
    for (int i = 0; i < iterations; i++) {
        coo_spmv<int, float>(&coomat, cpuvec.data(), cpures.data(), n);
        memcpy(cpuvec.data(), cpures.data(), sizeof(float) * n);
    }
    two_vec_compare(cpures.data(), gpures.data(), m);
    double big = 0.0, worst = 0.0;
    for (int i = 0; i < m; i++) big = fmax(big, fabs(cpures[i]));
    for (int i = 0; i < m; i++) worst = fmax(worst, fabs((double)cpures[i] - (double)gpures[i]));
    printf("A^%d x: largest |y| %g, largest difference %g\n", iterations, big, worst);
    const bool ok = worst <= 1e-4 * (big > 0 ? big : 1.0);

    std::vector<float> coores(m);
    spmv_only(&coomat, vec.data(), coores.data());
    std::vector<float> zero(m, 0.0f);
    evaluate(mat, vec.data(), zero.data(), coores.data());
    const int st = cocktail_last_status();
    free_cocktail(mat);
    free_coo_matrix(coomat);
    return ok && st == 0 ? 0 : 6;
}
