#ifndef CUSZP_INCLUDE_CUSZP_CUSZP_ENTRY_1D_F64_H
#define CUSZP_INCLUDE_CUSZP_CUSZP_ENTRY_1D_F64_H

// Per-mode 1D f64 entry points, same C++ signatures (and so the same mangled
// symbols) as the reference's include/cuSZp/cuSZp_entry_1D_f64.h:6-11; each
// replaces the launcher of the same name in src/cuSZp_entry_1D_f64.cu.
// Device pointers in and out; compress returns the stream length in *cmpSize
// after the stream has completed, decompress returns after the output is written.

#include <cuda_runtime.h>
#include <cstddef>

void cuSZp_compress_1D_fixed_f64(double* d_oriData, unsigned char* d_cmpBytes, size_t nbEle, size_t* cmpSize, double errorBound, cudaStream_t stream = 0);
void cuSZp_decompress_1D_fixed_f64(double* d_decData, unsigned char* d_cmpBytes, size_t nbEle, size_t cmpSize, double errorBound, cudaStream_t stream = 0);
void cuSZp_compress_1D_plain_f64(double* d_oriData, unsigned char* d_cmpBytes, size_t nbEle, size_t* cmpSize, double errorBound, cudaStream_t stream = 0);
void cuSZp_decompress_1D_plain_f64(double* d_decData, unsigned char* d_cmpBytes, size_t nbEle, size_t cmpSize, double errorBound, cudaStream_t stream = 0);
void cuSZp_compress_1D_outlier_f64(double* d_oriData, unsigned char* d_cmpBytes, size_t nbEle, size_t* cmpSize, double errorBound, cudaStream_t stream = 0);
void cuSZp_decompress_1D_outlier_f64(double* d_decData, unsigned char* d_cmpBytes, size_t nbEle, size_t cmpSize, double errorBound, cudaStream_t stream = 0);

#endif // CUSZP_INCLUDE_CUSZP_CUSZP_ENTRY_1D_F64_H
