// noalloc.cu -- lhl_reduce_noalloc: the reduction of lhl_reduce for callers that cannot
// allocate device memory.
//
// Who needs it: a caller whose device memory is fully owned by someone else -- a host
// application that hands this library a fixed memory budget, a Julia session whose GPU
// pool (CUDA.jl) must stay the only allocator, or code that runs where cudaMalloc is not
// allowed or would synchronize the device.  lhl_ws_create allocates the workspace with
// cudaMalloc; this entry point instead takes every input and output from the caller and
// keeps the reduction's scratch (panel copies, GEMV partials, pivot candidates, barrier
// counter, ...) in one file-scope device array of fixed size, reserved when the library
// is loaded and held by every GPU that loads it until the process exits.
//
// Limits and rules:
//  - n <= LHL_NOALLOC_NMAX (1024); larger n is rejected with LHL_ERR_DIM.
//  - The first call on a device looks up the array's device address on that device
//    (cudaGetSymbolAddress, with that device current) and caches it; make that first call
//    before any stream capture.
//  - Every call on a device shares the one array.  Two calls whose work overlaps on the GPU
//    (different streams, or different host threads) race on it and corrupt each other.
//  - The array keeps the last call's contents; each call clears what must start at zero
//    (the grid-barrier counter, the error flag) with cudaMemsetAsync, which allocates
//    nothing.
//  - A bounded wait that expires inside the reduction leaves LHL_ERR_TIMEOUT in the array's
//    error word; lhl_reduce_noalloc_check reads it back (and clears it) once the stream is
//    done, as lhl_ws_check does for a workspace.  Read it before the next call, which
//    clears it.
//  - dJ must not overlap the outputs: the first thing a call queues is the copy of J into
//    dfactors.
// No cudaMalloc, cudaFree or allocating library routine is called on this path.
#include <string.h>

#include "internal.cuh"

namespace {

constexpr int NMAX = LHL_NOALLOC_NMAX;
constexpr int NCAND = 1024;                        // >= CTAs of the persistent reduction grid
constexpr size_t OFF_B0 = 0;                                       // NMAX x 17
constexpr size_t OFF_TSNAP = OFF_B0 + (size_t)NMAX * 17;           // NMAX x 17
constexpr size_t OFF_PART = OFF_TSNAP + (size_t)NMAX * 17;         // (NMAX/64) x NMAX
constexpr size_t OFF_BUF2 = OFF_PART + (size_t)(NMAX / 64) * NMAX; // 499 x 499 (unblocked path)
constexpr size_t OFF_BSUM = OFF_BUF2 + (size_t)499 * 499;          // 2 NMAX
constexpr size_t OFF_BFAC = OFF_BSUM + 2 * (size_t)NMAX;           // NMAX
constexpr size_t OFF_CANDV = OFF_BFAC + (size_t)NMAX;              // NCAND
constexpr size_t OFF_CANDS = OFF_CANDV + NCAND;                    // NCAND
constexpr size_t OFF_TAB = OFF_CANDS + NCAND;                      // step table (<= 512 doubles)
constexpr size_t OFF_INTS = OFF_TAB + 512;                         // ints: cand_i, flags, barrier
constexpr size_t NDOUBLE = OFF_INTS + (NCAND + 64) / 2 + 1;

// The scratch: one static device array, 256-byte aligned.
static __device__ __align__(256) double g_noalloc_scratch[NDOUBLE];

constexpr int MAXDEV = 64;
static double* g_scratch_ptr[MAXDEV];  // device address of g_noalloc_scratch, per device
constexpr size_t ERR_OFFSET_BYTES = OFF_INTS * sizeof(double) + (NCAND + 4) * sizeof(int);
constexpr unsigned long long DEFAULT_LIMIT_NS = 2000000000ull;
static unsigned long long g_limit_ns = DEFAULT_LIMIT_NS;  // every bounded wait of these calls

// The device address of the scratch array on the current device, looked up once per device.
static double* scratch_base(int* status)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAXDEV) {
        *status = LHL_ERR_CUDA;
        return nullptr;
    }
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            *status = LHL_ERR_CUDA;
            return nullptr;
        }
        g_scratch_ptr[dev] = (double*)p;
    }
    *status = LHL_OK;
    return g_scratch_ptr[dev];
}

static bool overlaps(const void* a, size_t abytes, const void* b, size_t bbytes)
{
    const char* x = (const char*)a;
    const char* y = (const char*)b;
    return x < y + bbytes && y < x + abytes;
}

}  // namespace

extern "C" int lhl_reduce_noalloc(int64_t n, const double* dJ, int64_t ldj, int balance, double* dfactors,
                                  double* dHt, int64_t* dipiv, int64_t* dperm, int64_t* diperm, double* dscale,
                                  double* discale, void* stream)
{
    if (n < 0) return LHL_ERR_DIM;
    if (n > NMAX) return LHL_ERR_DIM;
    if (n == 0) return LHL_OK;
    if (!dJ || !dfactors || !dHt || !dperm || !diperm || !dscale || !discale || (n > 2 && !dipiv)) return LHL_ERR_ARG;
    if (ldj < n) return LHL_ERR_DIM;
    // J is read while dfactors is written: the caller's J may share no byte with an output
    const size_t jbytes = ((size_t)(ldj) * (size_t)(n - 1) + (size_t)n) * sizeof(double);
    const size_t nnbytes = (size_t)n * (size_t)n * sizeof(double);
    if (overlaps(dJ, jbytes, dfactors, nnbytes) || overlaps(dJ, jbytes, dHt, nnbytes) ||
        overlaps(dfactors, nnbytes, dHt, nnbytes))
        return LHL_ERR_ARG;
    // the fixed scratch must hold this build's grid and step table; checked before any work is queued
    if (lhl::reduce_grid_size() > NCAND || lhl::stepTabBytes() > 512 * sizeof(double)) return LHL_ERR_CUDA;
    int status = LHL_OK;
    double* base = scratch_base(&status);
    if (!base) return status;
    int* ints = (int*)(base + OFF_INTS);
    cudaStream_t st = (cudaStream_t)stream;

    cudaError_t e = cudaMemcpy2DAsync(dfactors, n * sizeof(double), dJ, ldj * sizeof(double), n * sizeof(double), n,
                                      cudaMemcpyDeviceToDevice, st);
    // barrier counter, error flag and balancing flag start at zero on every call
    if (e == cudaSuccess) e = cudaMemsetAsync(ints + NCAND, 0, 64 * sizeof(int), st);
    if (e != cudaSuccess) return LHL_ERR_CUDA;

    lhl::RedArgs a;
    memset(&a, 0, sizeof(a));
    a.n = (int)n;
    a.nb = 16;
    a.A = dfactors;
    a.ipiv = dipiv;
    a.B0 = base + OFF_B0;
    a.tsnap = base + OFF_TSNAP;
    a.part = base + OFF_PART;
    a.buf2 = base + OFF_BUF2;
    a.bsum = base + OFF_BSUM;
    a.bfac = base + OFF_BFAC;
    a.cand_v = base + OFF_CANDV;
    a.cand_s = base + OFF_CANDS;
    a.tab = base + OFF_TAB;
    a.cand_i = ints;
    a.bflag = ints + NCAND;
    a.err = ints + NCAND + 4;
    a.bar = (unsigned int*)(ints + NCAND + 8);
    a.scale = dscale;
    a.iscale = discale;
    a.limit_ns = g_limit_ns;
    a.ptimes = nullptr;
    a.use_tma = (n % 2 == 0) ? 1 : 0;
    const int mode = n <= 2 ? 0 : (n < 500 ? 1 : 2);
    if (!balance) {
        e = lhl::launch_fill_ones(dscale, discale, (int)n, st);
        if (e != cudaSuccess) return LHL_ERR_CUDA;
    }
    e = lhl::launch_reduce(a, balance ? 1 : 0, mode, st);
    if (e != cudaSuccess) return LHL_ERR_CUDA;
    if (mode == 1) {
        e = lhl::launch_unblocked_assemble((int)n, dfactors, a.buf2, dipiv, st);
        if (e != cudaSuccess) return LHL_ERR_CUDA;
    }
    e = lhl::launch_ht_perm((int)n, dfactors, dHt, dipiv, dperm, diperm, st);
    return e == cudaSuccess ? LHL_OK : LHL_ERR_CUDA;
}

extern "C" int lhl_reduce_noalloc_check(void* stream)
{
    int status = LHL_OK;
    double* base = scratch_base(&status);
    if (!base) return status;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaStreamSynchronize(st) != cudaSuccess) return LHL_ERR_CUDA;
    int err = 0;
    // a copy out of the static array into the caller's stack: no allocation
    if (cudaMemcpyFromSymbol(&err, g_noalloc_scratch, sizeof(int), ERR_OFFSET_BYTES, cudaMemcpyDeviceToHost) !=
        cudaSuccess)
        return LHL_ERR_CUDA;
    if (err) {
        const int zero = 0;
        if (cudaMemcpyToSymbol(g_noalloc_scratch, &zero, sizeof(int), ERR_OFFSET_BYTES, cudaMemcpyHostToDevice) !=
            cudaSuccess)
            return LHL_ERR_CUDA;
    }
    return err ? err : LHL_OK;
}

extern "C" int lhl_reduce_noalloc_set_barrier_limit_ns(uint64_t limit_ns)
{
    g_limit_ns = limit_ns ? (unsigned long long)limit_ns : DEFAULT_LIMIT_NS;
    return LHL_OK;
}
