// Complex GEMM on the fifth-generation tensor cores (tcgen05, kind::tf32) in
// 3xTF32: every FP64 operand is split into a TF32 high part and a TF32 low
// part, and each real product is formed as hi*hi + hi*lo + lo*hi with FP32
// accumulation in tensor memory (about 21 significant bits).
#pragma once
#include "linalg.cuh"

// D = alpha*A*B + beta*C + gammaI*I for every batch item (A, B not transposed,
// no diagonal scaling).  Every A and B is scaled by a power of two that brings
// its largest entry below 1 before the split (FP32 range), and the product is
// scaled back exactly; scale_ws is device scratch of 2*batch ints.  err
// (device int) is set to 1 if a tensor-core completion wait runs out; the
// affected tile is then not written.
// tile_n: columns of D per CTA, 128 (two CTAs per SM) or 256 (one CTA per SM,
// every converted A slab serves twice the columns).  With planes (device
// scratch of zgemm_tf32x3_planes_bytes) and tile_n = 128, A and B are first
// split into TF32 planes once (not once per output tile) and the product
// kernel moves them into shared memory with bulk copies.
cudaError_t zgemm_tf32x3_batched(const GemmArgs& g, int* scale_ws, int* err, cudaStream_t st, int tile_n = 128,
                                 float* planes = nullptr, size_t planes_bytes = 0);
// Scratch bytes of the pre-split planes of a batched M x N x K product.
size_t zgemm_tf32x3_planes_bytes(int M, int N, int K, int batch);
