// Standalone transpose: element (r, c) of a rows x cols array, read at
// in[r * row_is + c * col_is], written at out[r * row_os + c * col_os] -- the
// problem of the reference's transpose solver (core/solvers/transpose_solver.c:
// 97-141: dims[0] = columns, dims[1] = rows, real or complex, float or double).
//
// B200 form: 32 x 32 element tiles through shared memory (one pad column, so
// both the row-wise fill and the column-wise drain hit 32 distinct banks for
// 4-byte elements and stay conflict-free per 8-byte / 16-byte quarter-warp
// phase for wider ones). The fill reads a tile row by row along the input's
// column stride, the drain writes it column by column along the output's row
// stride: with col_is = 1 and row_os = 1 (a plain transpose) both are
// coalesced. Elements are moved as raw 4 / 8 / 16-byte words, so the result is
// bit-exact. In place, a square transpose swaps tile pairs (t_r, t_c) /
// (t_c, t_r) inside one CTA; the host routes other in-place layouts through a
// dense temporary.
#include <cstdint>

#include "fftz_kernels.h"

namespace fftz {

template <int EB> struct Word;
template <> struct Word<4> { typedef uint32_t type; };
template <> struct Word<8> { typedef uint2 type; };
template <> struct Word<16> { typedef uint4 type; };

constexpr int kTile = 32, kRows = 8;  // 32 x 8 threads move a 32 x 32 tile

template <int EB>
__global__ void __launch_bounds__(kTile * kRows) transpose_kernel(const unsigned char *__restrict__ in,
                                                                   unsigned char *__restrict__ out, int64_t rows,
                                                                   int64_t cols, int64_t row_is, int64_t col_is,
                                                                   int64_t row_os, int64_t col_os) {
  typedef typename Word<EB>::type W;
  __shared__ W tile[kTile][kTile + 1];
  const W *src = (const W *)in;
  W *dst = (W *)out;
  const int64_t r0 = (int64_t)blockIdx.y * kTile, c0 = (int64_t)blockIdx.x * kTile;
  const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
  for (int j = 0; j < kTile; j += kRows) {
    const int64_t r = r0 + ty + j, c = c0 + tx;
    if (r < rows && c < cols) tile[ty + j][tx] = src[r * row_is + c * col_is];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kTile; j += kRows) {
    const int64_t r = r0 + tx, c = c0 + ty + j;
    if (r < rows && c < cols) dst[r * row_os + c * col_os] = tile[tx][ty + j];
  }
}

// In place, square n x n with out strides = in strides swapped: CTA (bx, by)
// with bx >= by exchanges tiles (by, bx) and (bx, by); the others exit.
template <int EB>
__global__ void __launch_bounds__(kTile * kRows) transpose_square_inplace_kernel(unsigned char *data, int64_t n,
                                                                                  int64_t row_s, int64_t col_s) {
  typedef typename Word<EB>::type W;
  __shared__ W ta[kTile][kTile + 1];
  __shared__ W tb[kTile][kTile + 1];
  if (blockIdx.x < blockIdx.y) return;
  W *d = (W *)data;
  const int64_t ra = (int64_t)blockIdx.y * kTile, ca = (int64_t)blockIdx.x * kTile;  // tile A, its mirror B
  const int tx = threadIdx.x, ty = threadIdx.y;
  const bool diag = blockIdx.x == blockIdx.y;
#pragma unroll
  for (int j = 0; j < kTile; j += kRows) {
    int64_t r = ra + ty + j, c = ca + tx;
    if (r < n && c < n) ta[ty + j][tx] = d[r * row_s + c * col_s];
    r = ca + ty + j;
    c = ra + tx;
    if (!diag && r < n && c < n) tb[ty + j][tx] = d[r * row_s + c * col_s];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kTile; j += kRows) {
    // element (ra + tx, ca + ty + j) of A goes to (ca + ty + j, ra + tx)
    int64_t r = ca + ty + j, c = ra + tx;
    if (r < n && c < n) d[r * row_s + c * col_s] = ta[tx][ty + j];
    r = ra + ty + j;
    c = ca + tx;
    if (!diag && r < n && c < n) d[r * row_s + c * col_s] = tb[tx][ty + j];
  }
}

}  // namespace fftz

extern "C" {

int fftz_launch_transpose(const void *in, void *out, int64_t rows, int64_t cols, int64_t row_is, int64_t col_is,
                          int64_t row_os, int64_t col_os, int elem_bytes, void *stream) {
  const int64_t tr = (rows + fftz::kTile - 1) / fftz::kTile, tc = (cols + fftz::kTile - 1) / fftz::kTile;
  if (tr > 65535 || tc > 0x7fffffffLL) return (int)cudaErrorInvalidConfiguration;
  const dim3 grid((unsigned)tc, (unsigned)tr), block(fftz::kTile, fftz::kRows);
  const unsigned char *i = (const unsigned char *)in;
  unsigned char *o = (unsigned char *)out;
  cudaStream_t st = (cudaStream_t)stream;
  switch (elem_bytes) {
    case 4: fftz::transpose_kernel<4><<<grid, block, 0, st>>>(i, o, rows, cols, row_is, col_is, row_os, col_os); break;
    case 8: fftz::transpose_kernel<8><<<grid, block, 0, st>>>(i, o, rows, cols, row_is, col_is, row_os, col_os); break;
    case 16:
      fftz::transpose_kernel<16><<<grid, block, 0, st>>>(i, o, rows, cols, row_is, col_is, row_os, col_os);
      break;
    default: return (int)cudaErrorInvalidValue;
  }
  return (int)cudaGetLastError();
}

int fftz_launch_transpose_square_inplace(void *data, int64_t n, int64_t row_s, int64_t col_s, int elem_bytes,
                                         void *stream) {
  const int64_t t = (n + fftz::kTile - 1) / fftz::kTile;
  if (t > 65535) return (int)cudaErrorInvalidConfiguration;
  const dim3 grid((unsigned)t, (unsigned)t), block(fftz::kTile, fftz::kRows);
  unsigned char *d = (unsigned char *)data;
  cudaStream_t st = (cudaStream_t)stream;
  switch (elem_bytes) {
    case 4: fftz::transpose_square_inplace_kernel<4><<<grid, block, 0, st>>>(d, n, row_s, col_s); break;
    case 8: fftz::transpose_square_inplace_kernel<8><<<grid, block, 0, st>>>(d, n, row_s, col_s); break;
    case 16: fftz::transpose_square_inplace_kernel<16><<<grid, block, 0, st>>>(d, n, row_s, col_s); break;
    default: return (int)cudaErrorInvalidValue;
  }
  return (int)cudaGetLastError();
}

}  // extern "C"
