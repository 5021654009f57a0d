// Generic batched device operations used around the H_eff apply: grouped FP64
// GEMM (DMMA) with transpose flags, sub-matrix copies (reshapes between left /
// right / both pairing), and the vector algebra of the Davidson solver.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "device.hpp"

namespace qcm {

// C[c_off] (M x N, ldc) = alpha * op(A)[a_off] * op(B)[b_off] + beta * C
// op(A) = A (lda, column-major) or A^T; same for B.
// Row-blocked operands (arb / crb > 0): rows m of op(A) / C come in blocks of arb / crb rows,
// block j starting at a_off + j*a_bs / c_off + j*c_bs (a stack of matrices with their own
// layout, as a boundary's MPO-index blocks are stored); M must be a multiple of the block.
struct GemmJob {
    uint64_t a_off, b_off, c_off;
    uint32_t M, N, K, lda, ldb, ldc;
    uint32_t ta, tb;
    double alpha, beta;
    uint32_t arb = 0, crb = 0;
    uint64_t a_bs = 0, c_bs = 0;
};

// dst[dst_off + i + j*dst_ld] = src[src_off + i + j*src_ld] (i < rows, j < cols);
// with trans: dst[dst_off + j + i*dst_ld] = src[...] (transposed copy);
// with rev: source column j is read from column cols - 1 - j (reversed column order)
struct CopyJob {
    uint64_t src_off, dst_off;
    uint32_t rows, cols, src_ld, dst_ld, trans, rev;
};

// Runs a list of GEMM jobs (all operands addressed from the three base pointers, whose
// lengths in doubles are a_len, b_len, c_len: every job is checked against them on the
// host before the launch).  Jobs are uploaded to `jobbuf` (reused, grown as needed) and
// launched on stream s.
void batched_gemm(const std::vector<GemmJob>& jobs, const double* A, uint64_t a_len, const double* B, uint64_t b_len,
                  double* C, uint64_t c_len, DBuf<GemmJob>& jobbuf, DBuf<uint32_t>& tilebuf, cudaStream_t s);
void batched_copy(const std::vector<CopyJob>& jobs, const double* src, uint64_t src_len, double* dst, uint64_t dst_len,
                  DBuf<CopyJob>& jobbuf, cudaStream_t s);
// throws unless the rows x cols column-major sub-matrix at off (leading dimension ld) lies in [0, len)
void check_extent(uint64_t off, uint64_t rows, uint64_t cols, uint64_t ld, uint64_t len, const char* what);

// Vector algebra (length n): out[j] = <V_j, w> for j < m (V_j at V + j*ldv), written to device out.
// Two passes: DOT_PARTS partial sums per product over a fixed strided partition of [0, n), then
// a fixed-order tree over the partials, so the result is reproducible and does not depend on
// the device; scratch holds m * DOT_PARTS doubles.
constexpr unsigned DOT_PARTS = 256;
void dev_dots(const double* V, uint64_t ldv, uint32_t m, const double* w, uint64_t n, double* out, double* scratch,
              cudaStream_t s);
// y = sum_j c[j] * V_j  (c on device, m <= 64), or y += ...
void dev_lincomb(const double* V, uint64_t ldv, uint32_t m, const double* c, uint64_t n, double* y, bool accumulate,
                 cudaStream_t s);
// y = a*x + b*y (a, b host scalars)
void dev_axpby(double a, const double* x, double b, double* y, uint64_t n, cudaStream_t s);
// y += sa * (*a_dev) * x  (scalar read on the device: no host round trip)
void dev_axpy_dscalar(const double* a_dev, double sa, const double* x, double* y, uint64_t n, cudaStream_t s);
// p[i] = v
void dev_fill(double* p, uint64_t n, double v, cudaStream_t s);
// scale rows (row_scale) or columns of a column-major block: A(i,j) *= d[i] or d[j]
void dev_scale_rows(double* A, uint32_t rows, uint32_t cols, uint32_t lda, const double* d, cudaStream_t s);
void dev_scale_cols(double* A, uint32_t rows, uint32_t cols, uint32_t lda, const double* d, cudaStream_t s);

}  // namespace qcm
