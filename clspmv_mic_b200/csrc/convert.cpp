// convert.cpp — extern "C" converter entry points of libclspmv_b200.so.
//
// Each wrapper reinterprets the plain C struct of clspmv_b200.h as the
// matching matrix_storage.h template (layout identity is checked below) and
// calls the template converter. The reference converters these replace are
// cited in clspmv_b200.h next to each declaration.
#include <cstddef>
#include <new>
#include <cstring>
#include <cstdlib>
#include "clspmv_b200.h"
#include "matrix_storage.h"

#define LAYOUT_SAME(C, T)                                                      \
    static_assert(sizeof(C) == sizeof(T), #C " size differs from " #T);        \
    static_assert(alignof(C) == alignof(T), #C " alignment differs from " #T)

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

LAYOUT_SAME(clspmv_coo_f32, coo_t);
LAYOUT_SAME(clspmv_csr_f32, csr_t);
LAYOUT_SAME(clspmv_dia_f32, dia_t);
LAYOUT_SAME(clspmv_bdia_f32, bdia_t);
LAYOUT_SAME(clspmv_ell_f32, ell_t);
LAYOUT_SAME(clspmv_sell_f32, sell_t);
LAYOUT_SAME(clspmv_bcsr_f32, bcsr_t);
LAYOUT_SAME(clspmv_bell_f32, bell_t);
LAYOUT_SAME(clspmv_b4csr_f32, b4csr_t);
LAYOUT_SAME(clspmv_b4ell_f32, b4ell_t);
LAYOUT_SAME(clspmv_sbell_f32, sbell_t);
static_assert(offsetof(clspmv_b4ell_f32, b4ell_col_id) == offsetof(b4ell_t, b4ell_col_id), "b4ell layout");
static_assert(offsetof(clspmv_sbell_f32, sbell_slice_ptr) == offsetof(sbell_t, sbell_slice_ptr), "sbell layout");
static_assert(offsetof(clspmv_bdia_f32, bdia_data) == offsetof(bdia_t, bdia_data), "bdia layout");
static_assert(offsetof(clspmv_sell_f32, sell_slice_ptr) == offsetof(sell_t, sell_slice_ptr), "sell layout");

namespace {

template <class T, class C> T* as_tmpl(C* p) { return reinterpret_cast<T*>(p); }
template <class T, class C> const T* as_tmpl(const C* p) { return reinterpret_cast<const T*>(p); }

bool coo_ok(const clspmv_coo_f32* m)
{
    if (!m || m->matinfo.width < 0 || m->matinfo.height < 0 || m->matinfo.nnz < 0) return false;
    if (m->matinfo.nnz > 0 && (!m->coo_row_id || !m->coo_col_id || !m->coo_data)) return false;
    return true;
}

// Bounds of every index, so that no converter writes outside its arrays.
bool coo_in_range(const clspmv_coo_f32* m)
{
    for (int i = 0; i < m->matinfo.nnz; i++) {
        int r = m->coo_row_id[i], c = m->coo_col_id[i];
        if (r < 0 || r >= m->matinfo.height || c < 0 || c >= m->matinfo.width) return false;
    }
    return true;
}

bool block_shape_ok(unsigned int bw, unsigned int bh)
{
    return (bw == 4 || bw == 8) && (bh == 1 || bh == 2 || bh == 4 || bh == 8);
}

template <class F> int guarded(F&& f)
{
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return CLSPMV_ERR_ALLOC;
    } catch (...) {
        return CLSPMV_ERR_ARG;
    }
}

}  // namespace

extern "C" {

int clspmv_sort_coo_f32(clspmv_coo_f32* mat)
{
    if (!coo_ok(mat)) return CLSPMV_ERR_ARG;
    return guarded([&] { sort_coo(as_tmpl<coo_t>(mat)); return (int)CLSPMV_OK; });
}

int clspmv_is_sorted_coo_f32(const clspmv_coo_f32* mat)
{
    if (!coo_ok(mat)) return 0;
    return if_sorted_coo(const_cast<coo_t*>(as_tmpl<coo_t>(mat))) ? 1 : 0;
}

int clspmv_coo2csr_f32(const clspmv_coo_f32* src, clspmv_csr_f32* dst)
{
    if (!coo_ok(src) || !dst || !coo_in_range(src)) return CLSPMV_ERR_ARG;
    if (!clspmv_is_sorted_coo_f32(src)) return CLSPMV_ERR_NOT_SORTED;
    return guarded([&] {
        coo2csr(const_cast<coo_t*>(as_tmpl<coo_t>(src)), as_tmpl<csr_t>(dst));
        return (int)CLSPMV_OK;
    });
}

int clspmv_pad_csr_f32(const clspmv_csr_f32* src, clspmv_csr_f32* dst, int alignment)
{
    if (!src || !dst || alignment <= 0 || !src->csr_row_ptr) return CLSPMV_ERR_ARG;
    return guarded([&] {
        pad_csr(const_cast<csr_t*>(as_tmpl<csr_t>(src)), as_tmpl<csr_t>(dst), alignment);
        return (int)CLSPMV_OK;
    });
}

// The reference's coo2dia (include/matrix_storage.h:936-1014) sizes every
// diagonal at aligned(min(w, h)) and writes the value of row r at index r,
// so a taller-than-wide matrix with an entry at or below that row would
// write past its arrays; such input is rejected (CLSPMV_ERR_ARG). Taller
// matrices whose entries all sit above it convert exactly as there.
static bool rows_fit_diagonals(const clspmv_coo_f32* src, int alignment)
{
    const int w = src->matinfo.width, h = src->matinfo.height;
    if (h <= w) return true;
    const long long len = aligned_length<long long>(w, alignment);
    for (int i = 0; i < src->matinfo.nnz; i++)
        if (src->coo_row_id[i] >= len) return false;
    return true;
}

int clspmv_coo2dia_f32(const clspmv_coo_f32* src, clspmv_dia_f32* dst, int alignment)
{
    if (!coo_ok(src) || !dst || alignment <= 0 || !coo_in_range(src)) return CLSPMV_ERR_ARG;
    if (!rows_fit_diagonals(src, alignment)) return CLSPMV_ERR_ARG;
    return guarded([&] {
        bool ok = coo2dia<int, int, float>(const_cast<coo_t*>(as_tmpl<coo_t>(src)), as_tmpl<dia_t>(dst), alignment);
        return ok ? (int)CLSPMV_OK : (int)CLSPMV_ERR_REFUSED;
    });
}

int clspmv_coo2bdia_f32(const clspmv_coo_f32* src, clspmv_bdia_f32* dst, int alignment)
{
    if (!coo_ok(src) || !dst || alignment <= 0 || !coo_in_range(src)) return CLSPMV_ERR_ARG;
    if (!rows_fit_diagonals(src, alignment)) return CLSPMV_ERR_ARG;
    return guarded([&] {
        bool ok = coo2bdia<int, int, float>(const_cast<coo_t*>(as_tmpl<coo_t>(src)), as_tmpl<bdia_t>(dst), alignment);
        return ok ? (int)CLSPMV_OK : (int)CLSPMV_ERR_REFUSED;
    });
}

int clspmv_coo2ell_f32(const clspmv_coo_f32* src, clspmv_ell_f32* dst, int alignment, int ellnum)
{
    if (!coo_ok(src) || !dst || alignment <= 0 || ellnum < 0 || !coo_in_range(src)) return CLSPMV_ERR_ARG;
    if (!clspmv_is_sorted_coo_f32(src)) return CLSPMV_ERR_NOT_SORTED;
    return guarded([&] {
        coo_t* s = const_cast<coo_t*>(as_tmpl<coo_t>(src));
        bool ok = coo2ell(s, as_tmpl<ell_t>(dst), alignment, ellnum);
        if (ok) return (int)CLSPMV_OK;
        // distinguish "row longer than ellnum" (bad argument) from overflow
        if (ellnum > 0) {
            int maxlen = 0, run = 0;
            for (int i = 0; i < s->matinfo.nnz; i++) {
                run = (i > 0 && s->coo_row_id[i] == s->coo_row_id[i - 1]) ? run + 1 : 1;
                if (run > maxlen) maxlen = run;
            }
            if (maxlen > ellnum) return (int)CLSPMV_ERR_ARG;
        }
        return (int)CLSPMV_ERR_REFUSED;
    });
}

int clspmv_coo2sell_f32(const clspmv_coo_f32* src, clspmv_sell_f32* dst, unsigned int slice_height)
{
    if (!coo_ok(src) || !dst || slice_height == 0 || !coo_in_range(src)) return CLSPMV_ERR_ARG;
    if (!clspmv_is_sorted_coo_f32(src)) return CLSPMV_ERR_NOT_SORTED;
    return guarded([&] {
        coo2sell(const_cast<coo_t*>(as_tmpl<coo_t>(src)), as_tmpl<sell_t>(dst), slice_height);
        return (int)CLSPMV_OK;
    });
}

int clspmv_coo2bcsr_f32(const clspmv_coo_f32* src, clspmv_bcsr_f32* dst, unsigned int bwidth, unsigned int bheight, int alignment)
{
    if (!coo_ok(src) || !dst || bwidth == 0 || bheight == 0 || alignment <= 0 || !coo_in_range(src)) return CLSPMV_ERR_ARG;
    if (!clspmv_is_sorted_coo_f32(src)) return CLSPMV_ERR_NOT_SORTED;
    return guarded([&] {
        coo2bcsr(const_cast<coo_t*>(as_tmpl<coo_t>(src)), as_tmpl<bcsr_t>(dst), bwidth, bheight, alignment);
        return (int)CLSPMV_OK;
    });
}

int clspmv_coo2b4csr_f32(const clspmv_coo_f32* src, clspmv_b4csr_f32* dst, unsigned int bwidth, unsigned int bheight, int alignment)
{
    if (!coo_ok(src) || !dst || alignment <= 0 || !coo_in_range(src)) return CLSPMV_ERR_ARG;
    if (!block_shape_ok(bwidth, bheight)) return CLSPMV_ERR_UNSUPPORTED;
    if (!clspmv_is_sorted_coo_f32(src)) return CLSPMV_ERR_NOT_SORTED;
    return guarded([&] {
        bool ok = coo2b4csr(const_cast<coo_t*>(as_tmpl<coo_t>(src)), as_tmpl<b4csr_t>(dst), bwidth, bheight, alignment);
        return ok ? (int)CLSPMV_OK : (int)CLSPMV_ERR_REFUSED;
    });
}

int clspmv_coo2bell_f32(const clspmv_coo_f32* src, clspmv_bell_f32* dst, unsigned int bwidth, unsigned int bheight, int alignment, int ellnum)
{
    if (!coo_ok(src) || !dst || bwidth == 0 || bheight == 0 || alignment <= 0 || ellnum < 0 || !coo_in_range(src)) return CLSPMV_ERR_ARG;
    if (!clspmv_is_sorted_coo_f32(src)) return CLSPMV_ERR_NOT_SORTED;
    return guarded([&] {
        bool ok = coo2bell(const_cast<coo_t*>(as_tmpl<coo_t>(src)), as_tmpl<bell_t>(dst), bwidth, bheight, alignment, ellnum);
        return ok ? (int)CLSPMV_OK : (int)CLSPMV_ERR_ARG;
    });
}

int clspmv_coo2b4ell_f32(const clspmv_coo_f32* src, clspmv_b4ell_f32* dst, unsigned int bwidth, unsigned int bheight, int alignment, int ellnum)
{
    if (!coo_ok(src) || !dst || alignment <= 0 || ellnum < 0 || !coo_in_range(src)) return CLSPMV_ERR_ARG;
    if (!block_shape_ok(bwidth, bheight)) return CLSPMV_ERR_UNSUPPORTED;
    if (!clspmv_is_sorted_coo_f32(src)) return CLSPMV_ERR_NOT_SORTED;
    return guarded([&] {
        bool ok = coo2b4ell(const_cast<coo_t*>(as_tmpl<coo_t>(src)), as_tmpl<b4ell_t>(dst), bwidth, bheight, alignment, ellnum);
        return ok ? (int)CLSPMV_OK : (int)CLSPMV_ERR_REFUSED;
    });
}

int clspmv_coo2sbell_f32(const clspmv_coo_f32* src, clspmv_sbell_f32* dst, unsigned int bwidth, unsigned int bheight, unsigned int slice_height)
{
    if (!coo_ok(src) || !dst || slice_height == 0 || !coo_in_range(src)) return CLSPMV_ERR_ARG;
    if (!block_shape_ok(bwidth, bheight)) return CLSPMV_ERR_UNSUPPORTED;
    if (!clspmv_is_sorted_coo_f32(src)) return CLSPMV_ERR_NOT_SORTED;
    return guarded([&] {
        bool ok = coo2sbell(const_cast<coo_t*>(as_tmpl<coo_t>(src)), as_tmpl<sbell_t>(dst), bwidth, bheight, slice_height);
        return ok ? (int)CLSPMV_OK : (int)CLSPMV_ERR_REFUSED;
    });
}

#define INVERSE(NAME, CT, TT, CALL)                                           \
    int NAME(const CT* src, clspmv_coo_f32* dst)                              \
    {                                                                         \
        if (!src || !dst) return CLSPMV_ERR_ARG;                              \
        return guarded([&] {                                                  \
            CALL(const_cast<TT*>(as_tmpl<TT>(src)), as_tmpl<coo_t>(dst));     \
            return (int)CLSPMV_OK;                                            \
        });                                                                   \
    }

INVERSE(clspmv_csr2coo_f32, clspmv_csr_f32, csr_t, csr2coo)
INVERSE(clspmv_dia2coo_f32, clspmv_dia_f32, dia_t, dia2coo)
INVERSE(clspmv_bdia2coo_f32, clspmv_bdia_f32, bdia_t, bdia2coo)
INVERSE(clspmv_ell2coo_f32, clspmv_ell_f32, ell_t, ell2coo)
INVERSE(clspmv_bcsr2coo_f32, clspmv_bcsr_f32, bcsr_t, bcsr2coo)
INVERSE(clspmv_bell2coo_f32, clspmv_bell_f32, bell_t, bell2coo)
INVERSE(clspmv_sell2coo_f32, clspmv_sell_f32, sell_t, sell2coo)
INVERSE(clspmv_b4csr2coo_f32, clspmv_b4csr_f32, b4csr_t, b4csr2coo)
INVERSE(clspmv_b4ell2coo_f32, clspmv_b4ell_f32, b4ell_t, b4ell2coo)
INVERSE(clspmv_sbell2coo_f32, clspmv_sbell_f32, sbell_t, sbell2coo)
#undef INVERSE

int clspmv_coo2coo_f32(const clspmv_coo_f32* src, clspmv_coo_f32* dst)
{
    if (!coo_ok(src) || !dst) return CLSPMV_ERR_ARG;
    const size_t n = (size_t)src->matinfo.nnz;
    dst->matinfo = src->matinfo;
    dst->coo_row_id = (int*)malloc(sizeof(int) * (n ? n : 1));
    dst->coo_col_id = (int*)malloc(sizeof(int) * (n ? n : 1));
    dst->coo_data = (float*)malloc(sizeof(float) * (n ? n : 1));
    if (!dst->coo_row_id || !dst->coo_col_id || !dst->coo_data) {
        clspmv_free_coo_f32(dst);
        return CLSPMV_ERR_ALLOC;
    }
    if (n) {
        memcpy(dst->coo_row_id, src->coo_row_id, n * sizeof(int));
        memcpy(dst->coo_col_id, src->coo_col_id, n * sizeof(int));
        memcpy(dst->coo_data, src->coo_data, n * sizeof(float));
    }
    return CLSPMV_OK;
}

void clspmv_free_coo_f32(clspmv_coo_f32* m) { if (m) free_coo_matrix(*as_tmpl<coo_t>(m)); }
void clspmv_free_csr_f32(clspmv_csr_f32* m) { if (m) free_csr_matrix(*as_tmpl<csr_t>(m)); }
void clspmv_free_dia_f32(clspmv_dia_f32* m) { if (m) free_dia_matrix(*as_tmpl<dia_t>(m)); }
void clspmv_free_bdia_f32(clspmv_bdia_f32* m) { if (m) free_bdia_matrix(*as_tmpl<bdia_t>(m)); }
void clspmv_free_ell_f32(clspmv_ell_f32* m) { if (m) free_ell_matrix(*as_tmpl<ell_t>(m)); }
void clspmv_free_sell_f32(clspmv_sell_f32* m) { if (m) free_sell_matrix(*as_tmpl<sell_t>(m)); }
void clspmv_free_bcsr_f32(clspmv_bcsr_f32* m) { if (m) free_bcsr_matrix(*as_tmpl<bcsr_t>(m)); }
void clspmv_free_bell_f32(clspmv_bell_f32* m) { if (m) free_bell_matrix(*as_tmpl<bell_t>(m)); }
void clspmv_free_b4csr_f32(clspmv_b4csr_f32* m) { if (m) free_b4csr_matrix(*as_tmpl<b4csr_t>(m)); }
void clspmv_free_b4ell_f32(clspmv_b4ell_f32* m) { if (m) free_b4ell_matrix(*as_tmpl<b4ell_t>(m)); }
void clspmv_free_sbell_f32(clspmv_sbell_f32* m) { if (m) free_sbell_matrix(*as_tmpl<sbell_t>(m)); }

}  // extern "C"
