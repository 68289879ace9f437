/*
 * vh_noalloc.cu -- Cornelius surface elements of caller-owned device cubes
 * without any device allocation by the library.
 *
 * Some callers cannot let a library call cudaMalloc: host frameworks that
 * reserve the whole device up front for their own pool allocator (a raw
 * cudaMalloc then fails or fragments their pool), and per-event loops that run
 * next to other work on the same GPU, where cudaMalloc/cudaFree synchronise
 * the device and stall every other stream.  vh_cornelius_surfaces_noalloc
 * serves them: the caller passes device buffers for the input cubes and for
 * all outputs, and the only working memory -- the per-cube element counts,
 * their prefix-sum block totals and a small header -- lives in the
 * file-scope device array g_noalloc_scratch below, sized for
 * VH_NOALLOC_MAX_CUBES cubes.  Every GPU that loads the library holds that
 * array (about 1 MiB) until the process exits.
 *
 * Host code must not use the array's name as an address (on the host it is a
 * stand-in symbol); the device address is looked up once per device with
 * cudaGetSymbolAddress, with that device current, on the first call made on
 * it (and again if that device's context was destroyed and re-created since).
 * That first call should therefore come before any stream capture.
 *
 * If the elements do not fit in cap_elements, the first cap_elements of them
 * (in cube order) are written and *d_n_elements still receives the full total,
 * so a caller detects truncation by comparing it with cap_elements.
 * Every call on a device shares the one array and leaves its contents behind;
 * each call re-zeroes what must start at zero, and calls whose work overlaps
 * on the GPU (different streams, no ordering between them) race on it.
 */
#include <cuda_runtime.h>
#include <mutex>

#include "vh_b200.h"
#include "vh_internal.h"
#include "vh_kernels.h"
#include "vh_cornelius.cuh"

namespace vh {

constexpr long long kNoAllocBlocks = (VH_NOALLOC_MAX_CUBES + 1 + kScanChunk - 1) / kScanChunk + 1;
/* [0, MAX+1): element counts, then offsets; [MAX+1, +nb): scan block sums;
 * last 4: header -- [0] element total, [1] error flag */
constexpr long long kNoAllocInts = VH_NOALLOC_MAX_CUBES + 1 + kNoAllocBlocks + 4;

static __device__ __align__(256) int g_noalloc_scratch[kNoAllocInts];

__global__ void noalloc_reset_kernel()
{
    int *hdr = g_noalloc_scratch + (kNoAllocInts - 4);
    hdr[0] = 0;
    hdr[1] = 0;
}

__device__ __forceinline__ int noalloc_cube(int dim, const double *cubes, int c, double v0, double d0, double d1,
                                            double d2, double d3, cor::Work &w, double cen[][4], double nor[][4])
{
    if (dim == 3) {
        double cb[2][2][2];
        for (int i = 0; i < 8; i++) (&cb[0][0][0])[i] = cubes[8LL * c + i];
        const double dx3[3] = {d0, d1, d2};
        return cor::surface_3d(w, cb, v0, dx3, cen, nor);
    }
    double h[2][2][2][2];
    for (int i = 0; i < 16; i++) (&h[0][0][0][0])[i] = cubes[16LL * c + i];
    const double dx[4] = {d0, d1, d2, d3};
    return cor::surface_4d(w, h, v0, dx, cen, nor);
}

__global__ void __launch_bounds__(128) noalloc_count_kernel(int dim, const double *cubes, int n, double v0, double d0,
                                                            double d1, double d2, double d3, int *counts_out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    cor::Work w;
    double cen[cor::kMaxHedra][4], nor[cor::kMaxHedra][4];
    int ne = noalloc_cube(dim, cubes, c, v0, d0, d1, d2, d3, w, cen, nor);
    if (ne < 0) { atomicExch(g_noalloc_scratch + (kNoAllocInts - 3), 1); ne = 0; }
    g_noalloc_scratch[c] = ne;
    counts_out[c] = ne;
}

__global__ void __launch_bounds__(128) noalloc_emit_kernel(int dim, const double *cubes, int n, double v0, double d0,
                                                           double d1, double d2, double d3, double *elements, int cap)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    cor::Work w;
    double cen[cor::kMaxHedra][4], nor[cor::kMaxHedra][4];
    const int ne = noalloc_cube(dim, cubes, c, v0, d0, d1, d2, d3, w, cen, nor);
    const long long off = g_noalloc_scratch[c];
    for (int k = 0; k < ne; k++) {
        if (off + k >= cap) return;
        double *o = elements + (off + k) * 2 * dim;
        for (int j = 0; j < dim; j++) o[j] = cen[k][j + 4 - dim];
        for (int j = 0; j < dim; j++) o[dim + j] = nor[k][j + 4 - dim];
    }
}

__global__ void noalloc_finish_kernel(int *n_elements)
{
    const int *hdr = g_noalloc_scratch + (kNoAllocInts - 4);
    *n_elements = hdr[1] ? -1 : hdr[0];
}

/* device address of g_noalloc_scratch, looked up once per device and
 * context: a context that is torn down and created again (cudaDeviceReset,
 * or a primary context released by its last user) may load the module at
 * another address, so the cached address is tied to the context it was
 * looked up in.  The current context comes from the driver's
 * cuCtxGetCurrent, reached through the runtime so that the library does not
 * link the driver library. */
typedef int (*CtxGetCurrentFn)(void **);
static std::mutex g_sym_mu;
static int *g_sym_addr[64];
static void *g_sym_ctx[64];

static void *current_context()
{
    static CtxGetCurrentFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return (CtxGetCurrentFn)p;
    }();
    void *ctx = nullptr;
    if (fn && fn(&ctx) != 0) ctx = nullptr;
    return ctx;
}

static cudaError_t scratch_address(int dev, int **out)
{
    std::lock_guard<std::mutex> lk(g_sym_mu);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    void *ctx = current_context();
    if (!g_sym_addr[dev] || g_sym_ctx[dev] != ctx) {
        int *p = nullptr;
        cudaError_t rc = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
        if (rc != cudaSuccess) return rc;
        g_sym_addr[dev] = p;
        g_sym_ctx[dev] = current_context();   /* the lookup made the primary context current if none was */
    }
    *out = g_sym_addr[dev];
    return cudaSuccess;
}

} // namespace vh

extern "C" int vh_cornelius_surfaces_noalloc(int dim, const double *d_cubes, int n_cubes, double value0,
                                             const double *dx, double *d_elements, int cap_elements,
                                             int *d_counts, int *d_n_elements, void *stream)
{
    if ((dim != 3 && dim != 4) || n_cubes < 0 || (n_cubes > 0 && (!d_cubes || !d_counts)) || !dx || !d_n_elements ||
        (cap_elements > 0 && !d_elements) || cap_elements < 0)
        return vh::set_error(VH_ERR_ARG, "vh_cornelius_surfaces_noalloc: bad argument");
    if (n_cubes > VH_NOALLOC_MAX_CUBES)
        return vh::set_error(VH_ERR_ARG, "vh_cornelius_surfaces_noalloc: n_cubes exceeds VH_NOALLOC_MAX_CUBES "
                                         "(262144); split the batch or use vh_cornelius_surfaces");
    int dev = 0;
    cudaError_t rc = cudaGetDevice(&dev);
    int *base = nullptr;
    if (rc == cudaSuccess) rc = vh::scratch_address(dev, &base);
    if (rc != cudaSuccess)
        return vh::set_error(VH_ERR_CUDA, std::string("vh_cornelius_surfaces_noalloc: ") + cudaGetErrorString(rc));
    cudaStream_t st = (cudaStream_t)stream;
    const double d3 = dim == 4 ? dx[3] : 0.0;
    const unsigned grid = (unsigned)((n_cubes + 127) / 128);
    int *counts = base;
    int *bsum = base + VH_NOALLOC_MAX_CUBES + 1;
    int *hdr = base + (vh::kNoAllocInts - 4);
    vh::noalloc_reset_kernel<<<1, 1, 0, st>>>();
    if (n_cubes > 0) {
        vh::noalloc_count_kernel<<<grid, 128, 0, st>>>(dim, d_cubes, n_cubes, value0, dx[0], dx[1], dx[2], d3, d_counts);
        vh::exclusive_scan(counts, n_cubes, bsum, hdr, st);
        if (cap_elements > 0)
            vh::noalloc_emit_kernel<<<grid, 128, 0, st>>>(dim, d_cubes, n_cubes, value0, dx[0], dx[1], dx[2], d3,
                                                          d_elements, cap_elements);
    }
    vh::noalloc_finish_kernel<<<1, 1, 0, st>>>(d_n_elements);
    rc = cudaGetLastError();
    if (rc != cudaSuccess)
        return vh::set_error(VH_ERR_CUDA, std::string("vh_cornelius_surfaces_noalloc: ") + cudaGetErrorString(rc));
    return VH_OK;
}
