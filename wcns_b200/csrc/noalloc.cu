// noalloc.cu -- wcns_residual_noalloc: the residual norms of wcns_residual
// for caller-owned device arrays, with no device allocation at all.
//
// Some callers cannot allocate device memory at the moment they need the
// residual: a host code that hands all GPU memory management to its own
// pool allocator (and forbids cudaMalloc/cudaFree outside it), a code running
// inside another library's callback, or one whose memory budget is already
// fully committed.  For them the per-CTA partial sums live in one file-scope
// device array of fixed size instead of context-allocated scratch.
//
// The kernels restate the two residual kernels of k_misc.cu with the same
// launch shape (32 CTAs of 256 threads per block), the same per-point
// arithmetic and the same reduction order, so the results are bitwise those
// of wcns_residual on the same fields.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/wcns_b200.h"
#include "wcns_dev.cuh"

namespace wcns {
void set_last_error(const std::string &msg);  // capi.cu
}

namespace {

constexpr int NA_CTAS = 32;       // partial sums per block (as wcns_residual)
constexpr int NA_THREADS = 256;

struct NaBlock {
    const double *f[7];  // dq1..dq5, dtdt, vol (ghosted layout)
    int ni, nj, nk, pad;
};

// Layout of the scratch array: the block table, the partial sums (sum and
// max per CTA), the outputs (res[nb], resmax[nb], rms).
constexpr size_t NA_TAB_BYTES = sizeof(NaBlock) * WCNS_NOALLOC_MAX_BLOCKS;
constexpr size_t NA_PART_BYTES = sizeof(double) * 2 * NA_CTAS * WCNS_NOALLOC_MAX_BLOCKS;
constexpr size_t NA_OUT_BYTES = sizeof(double) * (2 * WCNS_NOALLOC_MAX_BLOCKS + 1);
constexpr size_t NA_BYTES = (NA_TAB_BYTES + NA_PART_BYTES + NA_OUT_BYTES + 255) / 256 * 256;
static_assert(NA_TAB_BYTES % 16 == 0 && NA_PART_BYTES % 16 == 0, "scratch carving keeps 16-byte alignment");

// Shared by every call on a device and kept until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

__device__ __forceinline__ long long na_idx(const NaBlock &B, int i, int j, int k) {
    return (long long)(k + 2) * ((long long)(B.nj + 6) * (B.ni + 6)) + (long long)(j + 2) * (B.ni + 6) + (i + 2);
}

// residual_curve (PostProcess.f90:1195-1347): per block sum and max of
// (|dq| / (dtdt * vol))^2 over the points 2..n-1 of every direction
__global__ void __launch_bounds__(NA_THREADS) k_na_partial(const NaBlock *__restrict__ tab, double *partial) {
    const int bi = blockIdx.y;
    const NaBlock B = tab[bi];
    const int mi = B.ni - 2, mj = B.nj - 2, mk = B.nk - 2;
    const long long np = (mi > 0 && mj > 0 && mk > 0) ? (long long)mi * mj * mk : 0;
    double s = 0.0, mx = 0.0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < np; q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (q < 0x7fffffffLL) {  // 32-bit divisions where they suffice
            const int qq = (int)q, r = qq / mi;
            i = qq - r * mi + 2;
            j = r % mj + 2;
            k = r / mj + 2;
        } else {
            i = (int)(q % mi) + 2;
            j = (int)((q / mi) % mj) + 2;
            k = (int)(q / ((long long)mi * mj)) + 2;
        }
        const long long id = na_idx(B, i, j, k);
        const double dtime1 = 1.0 / (B.f[5][id] * B.f[6][id]);
#pragma unroll
        for (int m = 0; m < 5; m++) {
            const double d = fabs(B.f[m][id]) * dtime1;
            s = s + d * d;
            mx = d > mx ? d : mx;
        }
    }
    __shared__ double ss[NA_THREADS], sm[NA_THREADS];
    ss[threadIdx.x] = s;
    sm[threadIdx.x] = mx;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            ss[threadIdx.x] = ss[threadIdx.x] + ss[threadIdx.x + w];
            sm[threadIdx.x] = sm[threadIdx.x + w] > sm[threadIdx.x] ? sm[threadIdx.x + w] : sm[threadIdx.x];
        }
        __syncthreads();
    }
    // every CTA rewrites its two slots on every call (also when it saw no
    // point), so nothing from an earlier call is read
    if (threadIdx.x == 0) {
        partial[2 * ((long long)bi * gridDim.x + blockIdx.x)] = ss[0];
        partial[2 * ((long long)bi * gridDim.x + blockIdx.x) + 1] = sm[0];
    }
}

__global__ void k_na_final(const NaBlock *__restrict__ tab, int nblocks, const double *partial, double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double total = 0.0;
    long long np = 0;
    for (int b = 0; b < nblocks; b++) {
        double s = 0.0, mx = 0.0;
        for (int c = 0; c < NA_CTAS; c++) {
            s = s + partial[2 * ((long long)b * NA_CTAS + c)];
            const double m = partial[2 * ((long long)b * NA_CTAS + c) + 1];
            mx = m > mx ? m : mx;
        }
        total = total + s;
        const long long npb = (long long)(tab[b].ni - 2) * (tab[b].nj - 2) * (tab[b].nk - 2) * 5;
        out[b] = s / (double)npb;
        out[nblocks + b] = mx;
        np += npb;
    }
    out[2 * nblocks] = sqrt(total / (double)np);
}

// Device address of the scratch array, looked up once per device with that
// device current (the array's name is only a host-side stand-in).
constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mutex;
unsigned char *g_na_addr[NA_MAX_DEVICES] = {};

int na_scratch(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        wcns::set_last_error(std::string("wcns_residual_noalloc: no CUDA device: ") + cudaGetErrorString(e));
        return WCNS_ERR_CUDA;
    }
    if (dev < 0 || dev >= NA_MAX_DEVICES) {
        wcns::set_last_error("wcns_residual_noalloc: device ordinal beyond the supported 64");
        return WCNS_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            wcns::set_last_error(std::string("wcns_residual_noalloc: cudaGetSymbolAddress failed: ") +
                                 cudaGetErrorString(e));
            return WCNS_ERR_CUDA;
        }
        g_na_addr[dev] = (unsigned char *)p;
    }
    *out = g_na_addr[dev];
    return 0;
}

}  // namespace

extern "C" int wcns_residual_noalloc(int nblocks, const int *dims, const double *const *fields, double *res_per_block,
                                     double *resmax_per_block, double *rms, void *stream) {
    if (nblocks < 1 || !dims || !fields) {
        wcns::set_last_error("wcns_residual_noalloc: invalid argument");
        return WCNS_ERR_ARGUMENT;
    }
    if (nblocks > WCNS_NOALLOC_MAX_BLOCKS) {
        wcns::set_last_error("wcns_residual_noalloc: " + std::to_string(nblocks) + " blocks exceed the maximum of " +
                             std::to_string(WCNS_NOALLOC_MAX_BLOCKS));
        return WCNS_ERR_ARGUMENT;
    }
    NaBlock tab[WCNS_NOALLOC_MAX_BLOCKS];
    for (int b = 0; b < nblocks; b++) {
        NaBlock &B = tab[b];
        B.ni = dims[3 * b];
        B.nj = dims[3 * b + 1];
        B.nk = dims[3 * b + 2];
        B.pad = 0;
        if (B.ni < 3 || B.nj < 3 || B.nk < 3) {
            wcns::set_last_error("wcns_residual_noalloc: block dimensions must be >= 3");
            return WCNS_ERR_ARGUMENT;
        }
        for (int f = 0; f < 7; f++) {
            B.f[f] = fields[7 * b + f];
            if (!B.f[f]) {
                wcns::set_last_error("wcns_residual_noalloc: null field pointer");
                return WCNS_ERR_ARGUMENT;
            }
        }
    }
    unsigned char *base = nullptr;
    int rc = na_scratch(&base);
    if (rc) return rc;
    NaBlock *dtab = (NaBlock *)base;
    double *partial = (double *)(base + NA_TAB_BYTES);
    double *out = (double *)(base + NA_TAB_BYTES + NA_PART_BYTES);
    cudaStream_t st = (cudaStream_t)stream;
    double h[2 * WCNS_NOALLOC_MAX_BLOCKS + 1];
    cudaError_t e = cudaMemcpyAsync(dtab, tab, sizeof(NaBlock) * nblocks, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_na_partial<<<dim3(NA_CTAS, nblocks), NA_THREADS, 0, st>>>(dtab, partial);
        k_na_final<<<1, 32, 0, st>>>(dtab, nblocks, partial, out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, out, sizeof(double) * (2 * nblocks + 1), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        wcns::set_last_error(std::string("wcns_residual_noalloc: CUDA error: ") + cudaGetErrorString(e));
        return WCNS_ERR_CUDA;
    }
    for (int b = 0; b < nblocks; b++) {
        if (res_per_block) res_per_block[b] = h[b];
        if (resmax_per_block) resmax_per_block[b] = h[nblocks + b];
    }
    if (rms) *rms = h[2 * nblocks];
    return 0;
}
