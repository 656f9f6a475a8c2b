/*
 * analyze.h — Cocktail partitioning of a COO matrix into up to nine
 * storage formats, source-compatible with clSpMV's header of the same name
 * (include/analyze.h:1-260 of the reference): the benchmark-table entry
 * types, the `cocktail<>` result struct with its member order, and
 * analyze_matrix() with the same arguments and defaults.
 *
 * analyze_matrix() reads the benchmark tables from $CLSPMVPATH/benchmark/
 * (<fmt>.ben, the reference's text formats, src/analyze.cpp:16-174) as the
 * reference does. analyze_matrix_tables() takes the tables explicitly, and
 * read_bench_tables() reports missing or empty tables instead of crashing
 * (the reference segfaults on the empty tables it ships).
 */
#ifndef __ANALYZE__H__
#define __ANALYZE__H__

#include <vector>

#include "constant.h"
#include "matrix_storage.h"

struct overhead_entry {
    unsigned int groupnum;
    unsigned int threadnum;
    double microsec;
};

class basic_entry {
public:
    unsigned int dimension;
    unsigned int width;
};

class block_entry {
public:
    unsigned int bheight;
    unsigned int bwidth;
    unsigned int dimension;
    unsigned int blocknum;
};

class bdia_entry : public basic_entry { public: double bdia_gflops[BDIA_IMP_NUM]; };
class dia_entry : public basic_entry { public: double dia_gflops[DIA_IMP_NUM]; };
class sbell_entry : public block_entry { public: double sbell_gflops[SBELL_IMP_NUM]; };
class bell_entry : public block_entry { public: double bell_gflops[BELL_IMP_NUM]; };
class bcsr_entry : public block_entry { public: double bcsr_gflops[BCSR_IMP_NUM]; };
class sell_entry : public basic_entry { public: double sell_gflops[SELL_IMP_NUM]; };
class ell_entry : public basic_entry { public: double ell_gflops[ELL_IMP_NUM]; };
class csr_entry : public basic_entry { public: unsigned int csr_groupnum; double csr_gflops[CSR_IMP_NUM]; };
class coo_entry : public basic_entry { public: unsigned int coo_groupnum; double coo_gflops[COO_IMP_NUM]; };

struct benchmark_all {
    std::vector<overhead_entry> overhead;
    std::vector<bdia_entry> bdia;
    std::vector<dia_entry> dia;
    std::vector<sbell_entry> sbell;
    std::vector<bell_entry> bell;
    std::vector<bcsr_entry> bcsr;
    std::vector<sell_entry> sell;
    std::vector<ell_entry> ell;
    std::vector<csr_entry> csr;
    std::vector<coo_entry> coo;
};

/* cocktail<>: include/analyze.h:105-144 of the reference (member order kept) */
template <class dimType, class offsetType, class dataType>
struct cocktail {
    bool ifusebdia;
    bool ifusedia;
    bool ifusesbell;
    bool ifusebell;
    bool ifusebcsr;
    bool ifusesell;
    bool ifuseell;
    bool ifusecsr;
    bool ifusecoo;

    int bdia_meth_num;
    int dia_meth_num;
    int sbell_meth_num;
    int bell_meth_num;
    int bcsr_meth_num;
    int sell_meth_num;
    int ell_meth_num;
    int csr_meth_num;
    int coo_meth_num;

    int csr_group_num;
    int coo_group_num;

    int mat_width;
    int mat_height;
    int mat_nnz;

    bdia_matrix<dimType, offsetType, dataType> bdia;
    dia_matrix<dimType, offsetType, dataType> dia;
    sbell_matrix<dimType, dataType> sbell;
    b4ell_matrix<dimType, dataType> bell;
    b4csr_matrix<dimType, dataType> bcsr;
    sell_matrix<dimType, dataType> sell;
    ell_matrix<dimType, dataType> ell;
    csr_matrix<dimType, dataType> csr;
    coo_matrix<dimType, dataType> coo;
};

/* init_cocktail: include/analyze.h:146-181 */
template <class dimType, class offsetType, class dataType>
void init_cocktail(cocktail<dimType, offsetType, dataType>& mat)
{
    mat.ifusebdia = mat.ifusedia = mat.ifusesbell = mat.ifusebell = mat.ifusebcsr = false;
    mat.ifusesell = mat.ifuseell = mat.ifusecsr = mat.ifusecoo = false;
    mat.bdia_meth_num = mat.dia_meth_num = mat.sbell_meth_num = mat.bell_meth_num = mat.bcsr_meth_num = 0;
    mat.sell_meth_num = mat.ell_meth_num = mat.csr_meth_num = mat.coo_meth_num = 0;
    mat.csr_group_num = mat.coo_group_num = 0;
    mat.mat_width = mat.mat_height = mat.mat_nnz = 0;
    init_bdia_matrix(mat.bdia);
    init_dia_matrix(mat.dia);
    init_sbell_matrix(mat.sbell);
    init_b4ell_matrix(mat.bell);
    init_b4csr_matrix(mat.bcsr);
    init_sell_matrix(mat.sell);
    init_ell_matrix(mat.ell);
    init_csr_matrix(mat.csr);
    init_coo_matrix(mat.coo);
}

/* free_cocktail: include/analyze.h:183-205 */
template <class dimType, class offsetType, class dataType>
void free_cocktail(cocktail<dimType, offsetType, dataType>& mat)
{
    mat.ifusebdia = mat.ifusedia = mat.ifusesbell = mat.ifusebell = mat.ifusebcsr = false;
    mat.ifusesell = mat.ifuseell = mat.ifusecsr = mat.ifusecoo = false;
    free_bdia_matrix(mat.bdia);
    free_dia_matrix(mat.dia);
    free_sbell_matrix(mat.sbell);
    free_b4ell_matrix(mat.bell);
    free_b4csr_matrix(mat.bcsr);
    free_sell_matrix(mat.sell);
    free_ell_matrix(mat.ell);
    free_csr_matrix(mat.csr);
    free_coo_matrix(mat.coo);
}

struct maxflop_info {
    int bdia_meth_num;
    double bdia_max_flop;
    int dia_meth_num;
    double dia_max_flop;
    /* 1x4, 2x4, 4x4, 8x4, 1x8, 2x8, 4x8, 8x8 */
    int sbell_meth_num[8];
    double sbell_max_flop[8];
    int bell_meth_num[8];
    double bell_max_flop[8];
    int bcsr_meth_num[8];
    double bcsr_max_flop[8];
    int sell_meth_num;
    double sell_max_flop;
    int ell_meth_num;
    double ell_max_flop;
    int csr_meth_num;
    int csr_groupnum;
    double csr_max_flop;
    int coo_meth_num;
    int coo_groupnum;
    double coo_max_flop;
    double max_dia_base_flop;
    double max_block_base_flop;
    double max_flat_base_flop;
};

struct four_index {
    unsigned int dim_s_wid_s;
    unsigned int dim_s_wid_l;
    unsigned int dim_l_wid_s;
    unsigned int dim_l_wid_l;
};

/* ReadBench (src/analyze.cpp:177-210) from <dir>/benchmark/<fmt>.ben.
 * Returns 0 when every table was read and is non-empty; otherwise a
 * negative number and `bench` holds what could be read. */
int read_bench_tables(const char* dir, benchmark_all& bench);

/* analyze_matrix: src/analyze.cpp:3714-3900. Tables from $CLSPMVPATH. */
void analyze_matrix(coo_matrix<int, float>& coomat, cocktail<int, int, float>& mat, float dia_priority_multiplier = 1.0,
                    bool estimate_flat_partial = true, bool estimate_flat_full = false);

/* The same partitioning with tables already in memory. `coomat` must be
 * sorted by (row, col). */
void analyze_matrix_tables(const benchmark_all& bench, coo_matrix<int, float>& coomat, cocktail<int, int, float>& mat,
                           float dia_priority_multiplier = 1.0, bool estimate_flat_partial = true,
                           bool estimate_flat_full = false);

#endif
