// ref_shim.cpp — extern "C" wrappers around clSpMV's own serial code, compiled
// from the reference sources in place (oracle/Makefile, target `ref`) into
// oracle/_ref/libclspmv_ref.so. TEST INFRASTRUCTURE ONLY: the parity tests
// use it to pin the C oracle and to compare the library's converters byte
// for byte; bench.py may time its csr_spmv as the reference CPU baseline.
//
// The reference templates are instantiated with <int, float> / <int, int,
// float>; the C structs of clspmv_b200.h are layout-identical to them (the
// library checks this with static_asserts), so pointers are reinterpreted.
// Headers come from the reference tree only (-I<reference>/include); the
// plain C ABI header is included by relative path.
#include "matrix_storage.h"
#include "spmv_serial.h"
#include "util.h"
#include "analyze.h"
#include "fileio.h"
#include "../include/clspmv_b200.h"

typedef coo_matrix<int, float> coo_t;
typedef csr_matrix<int, float> csr_t;
typedef dia_matrix<int, int, float> dia_t;
typedef bdia_matrix<int, int, float> bdia_t;
typedef ell_matrix<int, float> ell_t;
typedef sell_matrix<int, float> sell_t;
typedef bcsr_matrix<int, float> bcsr_t;
typedef bell_matrix<int, float> bell_t;
typedef b4csr_matrix<int, float> b4csr_t;
typedef b4ell_matrix<int, float> b4ell_t;
typedef sbell_matrix<int, float> sbell_t;

static_assert(sizeof(clspmv_coo_f32) == sizeof(coo_t), "coo");
static_assert(sizeof(clspmv_csr_f32) == sizeof(csr_t), "csr");
static_assert(sizeof(clspmv_dia_f32) == sizeof(dia_t), "dia");
static_assert(sizeof(clspmv_bdia_f32) == sizeof(bdia_t), "bdia");
static_assert(sizeof(clspmv_ell_f32) == sizeof(ell_t), "ell");
static_assert(sizeof(clspmv_sell_f32) == sizeof(sell_t), "sell");
static_assert(sizeof(clspmv_bcsr_f32) == sizeof(bcsr_t), "bcsr");
static_assert(sizeof(clspmv_bell_f32) == sizeof(bell_t), "bell");
static_assert(sizeof(clspmv_b4csr_f32) == sizeof(b4csr_t), "b4csr");
static_assert(sizeof(clspmv_b4ell_f32) == sizeof(b4ell_t), "b4ell");
static_assert(sizeof(clspmv_sbell_f32) == sizeof(sbell_t), "sbell");

template <class T, class C> static T* R(C* p) { return reinterpret_cast<T*>(p); }

extern "C" {

void ref_free(void* p) { free(p); }

int ref_sort_coo(clspmv_coo_f32* m) { return sort_coo(R<coo_t>(m)) ? 1 : 0; }
int ref_if_sorted_coo(clspmv_coo_f32* m) { return if_sorted_coo(R<coo_t>(m)) ? 1 : 0; }
void ref_coo2csr(clspmv_coo_f32* s, clspmv_csr_f32* d) { coo2csr(R<coo_t>(s), R<csr_t>(d)); }
void ref_pad_csr(clspmv_csr_f32* s, clspmv_csr_f32* d, int alignment) { pad_csr(R<csr_t>(s), R<csr_t>(d), alignment); }
int ref_coo2dia(clspmv_coo_f32* s, clspmv_dia_f32* d, int alignment) { return coo2dia<int, int, float>(R<coo_t>(s), R<dia_t>(d), alignment) ? 1 : 0; }
int ref_coo2bdia(clspmv_coo_f32* s, clspmv_bdia_f32* d, int alignment) { return coo2bdia<int, int, float>(R<coo_t>(s), R<bdia_t>(d), alignment) ? 1 : 0; }
void ref_coo2ell(clspmv_coo_f32* s, clspmv_ell_f32* d, int alignment, int ellnum) { coo2ell(R<coo_t>(s), R<ell_t>(d), alignment, ellnum); }
void ref_coo2sell(clspmv_coo_f32* s, clspmv_sell_f32* d, unsigned sh) { coo2sell(R<coo_t>(s), R<sell_t>(d), sh); }
void ref_coo2bcsr(clspmv_coo_f32* s, clspmv_bcsr_f32* d, unsigned bw, unsigned bh, int alignment) { coo2bcsr(R<coo_t>(s), R<bcsr_t>(d), bw, bh, alignment); }
int ref_coo2b4csr(clspmv_coo_f32* s, clspmv_b4csr_f32* d, unsigned bw, unsigned bh, int alignment) { return coo2b4csr(R<coo_t>(s), R<b4csr_t>(d), bw, bh, alignment) ? 1 : 0; }
void ref_coo2bell(clspmv_coo_f32* s, clspmv_bell_f32* d, unsigned bw, unsigned bh, int alignment, int ellnum) { coo2bell(R<coo_t>(s), R<bell_t>(d), bw, bh, alignment, ellnum); }
int ref_coo2b4ell(clspmv_coo_f32* s, clspmv_b4ell_f32* d, unsigned bw, unsigned bh, int alignment, int ellnum) { return coo2b4ell(R<coo_t>(s), R<b4ell_t>(d), bw, bh, alignment, ellnum) ? 1 : 0; }
int ref_coo2sbell(clspmv_coo_f32* s, clspmv_sbell_f32* d, unsigned bw, unsigned bh, unsigned sh) { return coo2sbell(R<coo_t>(s), R<sbell_t>(d), bw, bh, sh) ? 1 : 0; }

void ref_dia2coo(clspmv_dia_f32* s, clspmv_coo_f32* d) { dia2coo(R<dia_t>(s), R<coo_t>(d)); }
void ref_bdia2coo(clspmv_bdia_f32* s, clspmv_coo_f32* d) { bdia2coo(R<bdia_t>(s), R<coo_t>(d)); }
void ref_ell2coo(clspmv_ell_f32* s, clspmv_coo_f32* d) { ell2coo(R<ell_t>(s), R<coo_t>(d)); }
void ref_bcsr2coo(clspmv_bcsr_f32* s, clspmv_coo_f32* d) { bcsr2coo(R<bcsr_t>(s), R<coo_t>(d)); }
void ref_bell2coo(clspmv_bell_f32* s, clspmv_coo_f32* d) { bell2coo(R<bell_t>(s), R<coo_t>(d)); }

void ref_coo_spmv(clspmv_coo_f32* m, float* x, float* y, int n) { coo_spmv(R<coo_t>(m), x, y, n); }
void ref_csr_spmv(clspmv_csr_f32* m, float* x, float* y, int n) { csr_spmv(R<csr_t>(m), x, y, n); }
void ref_dia_spmv(clspmv_dia_f32* m, float* x, float* y, int n) { dia_spmv(R<dia_t>(m), x, y, n); }
void ref_bdia_spmv(clspmv_bdia_f32* m, float* x, float* y, int n) { bdia_spmv(R<bdia_t>(m), x, y, n); }
void ref_ell_spmv(clspmv_ell_f32* m, float* x, float* y, int n) { ell_spmv(R<ell_t>(m), x, y, n); }
void ref_sell_spmv(clspmv_sell_f32* m, float* x, float* y, int n) { sell_spmv(R<sell_t>(m), x, y, n); }
void ref_sbell_spmv(clspmv_sbell_f32* m, float* x, float* y, int n) { sbell_spmv(R<sbell_t>(m), x, y, n); }
void ref_bcsr_spmv(clspmv_bcsr_f32* m, float* x, float* y, int n) { bcsr_spmv(R<bcsr_t>(m), x, y, n); }
void ref_bell_spmv(clspmv_bell_f32* m, float* x, float* y, int n) { bell_spmv(R<bell_t>(m), x, y, n); }
// analyze_matrix (src/analyze.cpp:3714-3900) with CLSPMVPATH pointing at
// `table_root` (it reads <table_root>/benchmark/*.ben).
void ref_analyze_matrix(clspmv_coo_f32* m, clspmv_cocktail_f32* out, const char* table_root, float mult, int partial, int full)
{
    setenv("CLSPMVPATH", table_root, 1);
    cocktail<int, int, float>* c = reinterpret_cast<cocktail<int, int, float>*>(out);
    init_cocktail(*c);
    analyze_matrix(*R<coo_t>(m), *c, mult, partial != 0, full != 0);
}
static_assert(sizeof(clspmv_cocktail_f32) == sizeof(cocktail<int, int, float>), "cocktail");
// spmv_only: src/util.cpp:85-91 (zeroes y, then coo_spmv)
void ref_spmv_only(clspmv_coo_f32* m, float* x, float* y) { spmv_only(R<coo_t>(m), x, y); }
// ReadMMF: src/fileio.cpp:10-109 (arrays malloc'ed; release with ref_free)
void ref_read_mmf(const char* path, clspmv_coo_f32* out) { ReadMMF(const_cast<char*>(path), R<coo_t>(out)); }

}  // extern "C"
