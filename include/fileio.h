/*
 * fileio.h — Matrix Market input, source-compatible with include/fileio.h
 * of clSpMV (src/fileio.cpp:10-109). Implemented in libclspmv_b200.
 */
#ifndef CLSPMV_FILEIO_H
#define CLSPMV_FILEIO_H

#include "matrix_storage.h"

/* Reads a coordinate Matrix Market file into a row-sorted COO matrix:
 * 1-based indices become 0-based, pattern entries read as 1.0, and a
 * "symmetric" file gets the mirror of every off-diagonal entry. Prints a
 * message and leaves `mat` empty (nnz 0, NULL arrays) when the file cannot
 * be read; clspmv_read_mmf_f32 returns the status instead. */
void ReadMMF(char* filename, coo_matrix<int, float>* mat);

#endif /* CLSPMV_FILEIO_H */
