// f32.cu -- element conversions for LHLWorkspace{Float32} (F:703-705: the reference's
// element type T = Float32).  A Float32 workspace keeps its arrays in FP64 storage holding
// float values: J is rounded to float on the way in, the reduction's factors and Ht are
// rounded to float, the shift LU runs in float arithmetic (shift.cu), and float vectors are
// widened for the solve and rounded back.
#include "internal.cuh"

namespace lhl {

// dst[c, r] = (double)src[c, r] over a rows x cols column-major block
__global__ void f32_to_f64_kernel(const float* __restrict__ src, int lds, double* __restrict__ dst, int ldd, int rows,
                                  int cols)
{
    const size_t total = (size_t)rows * cols;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e / rows), r = (int)(e - (size_t)c * rows);
        dst[(size_t)c * ldd + r] = (double)src[(size_t)c * lds + r];
    }
}

// dst[c, r] = src[c, r] rounded to float, kept as double (in place when dst == src)
__global__ void round_f32_kernel(const double* src, int lds, double* dst, int ldd, int rows, int cols)
{
    const size_t total = (size_t)rows * cols;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e / rows), r = (int)(e - (size_t)c * rows);
        dst[(size_t)c * ldd + r] = (double)(float)src[(size_t)c * lds + r];
    }
}

// dst[c, r] = (float)src[c, r]
__global__ void f64_to_f32_kernel(const double* __restrict__ src, int lds, float* __restrict__ dst, int ldd, int rows,
                                  int cols)
{
    const size_t total = (size_t)rows * cols;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e / rows), r = (int)(e - (size_t)c * rows);
        dst[(size_t)c * ldd + r] = (float)src[(size_t)c * lds + r];
    }
}

// complex columns <-> pairs of real columns: column c of the interleaved complex block X (ld
// ldx complex elements) is real column 2c (real parts) and 2c + 1 (imaginary parts) of R (ld n)
__global__ void split_complex_kernel(const double* __restrict__ X, int ldx, double* __restrict__ R, int n, int cols)
{
    const size_t total = (size_t)n * cols * 2;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int rc = (int)(e / n), r = (int)(e - (size_t)rc * n);  // real column rc = 2c + p
        R[(size_t)rc * n + r] = X[2 * ((size_t)(rc >> 1) * ldx + r) + (rc & 1)];
    }
}

__global__ void join_complex_kernel(const double* __restrict__ R, int n, double* __restrict__ X, int ldx, int cols)
{
    const size_t total = (size_t)n * cols * 2;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int rc = (int)(e / n), r = (int)(e - (size_t)rc * n);
        X[2 * ((size_t)(rc >> 1) * ldx + r) + (rc & 1)] = R[(size_t)rc * n + r];
    }
}

static unsigned conv_grid(size_t total)
{
    const size_t b = (total + 255) / 256;
    return (unsigned)(b < 4096 ? (b ? b : 1) : 4096);
}

cudaError_t launch_f32_to_f64(const float* src, int lds, double* dst, int ldd, int rows, int cols, cudaStream_t st)
{
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    f32_to_f64_kernel<<<conv_grid((size_t)rows * cols), 256, 0, st>>>(src, lds, dst, ldd, rows, cols);
    return cudaGetLastError();
}

cudaError_t launch_round_f32(const double* src, int lds, double* dst, int ldd, int rows, int cols, cudaStream_t st)
{
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    round_f32_kernel<<<conv_grid((size_t)rows * cols), 256, 0, st>>>(src, lds, dst, ldd, rows, cols);
    return cudaGetLastError();
}

cudaError_t launch_f64_to_f32(const double* src, int lds, float* dst, int ldd, int rows, int cols, cudaStream_t st)
{
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    f64_to_f32_kernel<<<conv_grid((size_t)rows * cols), 256, 0, st>>>(src, lds, dst, ldd, rows, cols);
    return cudaGetLastError();
}

cudaError_t launch_split_complex(const double* X, int ldx, double* R, int n, int cols, cudaStream_t st)
{
    if (n <= 0 || cols <= 0) return cudaSuccess;
    split_complex_kernel<<<conv_grid((size_t)n * cols * 2), 256, 0, st>>>(X, ldx, R, n, cols);
    return cudaGetLastError();
}

cudaError_t launch_join_complex(const double* R, int n, double* X, int ldx, int cols, cudaStream_t st)
{
    if (n <= 0 || cols <= 0) return cudaSuccess;
    join_complex_kernel<<<conv_grid((size_t)n * cols * 2), 256, 0, st>>>(R, n, X, ldx, cols);
    return cudaGetLastError();
}

}  // namespace lhl
