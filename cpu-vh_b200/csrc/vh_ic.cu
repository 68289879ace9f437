/*
 * vh_ic.cu -- initial conditions generated on the device, into an event's
 * interior staging planes (e, p, u), so that a served event does not wait for
 * a host generator:
 *
 *  - optical Glauber (the reference's GlauberModel.cpp:26-108 geometry with
 *    the longitudinal plateau of InitialConditions.cpp:1046-1063): one thread
 *    per transverse cell integrates both Woods-Saxon thickness functions by
 *    Simpson's rule along z (601 points), the participant density's maximum
 *    is reduced with an atomic max on its bit pattern, and a second kernel
 *    writes e, p(e), u = (1, 0, 0, 0) for every cell;
 *  - lumpy hotspots: the random centres and amplitudes are drawn on the host
 *    (the same counter-based stream as the host generator) and one thread per
 *    cell sums the Gaussians.
 *
 * The arithmetic follows the host generators (vh_host.cpp) operation for
 * operation; exp comes from the device math library, so values may differ
 * from the host generator's in the last bits.
 */
#include <cuda_runtime.h>
#include "vh_kernels.h"

namespace vh {

__device__ __forceinline__ double ws_thickness_dev(double r2, double R, double a)
{
    const double n0 = 0.17;
    const double zmax = R + 15. * a;
    const int nzq = 600;
    const double hz = 2. * zmax / nzq;
    double sum = 0.;
    for (int k = 0; k <= nzq; ++k) {
        double z = -zmax + k * hz;
        double rr = sqrt(r2 + z * z);
        double f = n0 / (1. + exp((rr - R) / a));
        double wgt = (k == 0 || k == nzq) ? 1. : (k % 2 ? 4. : 2.);
        sum += wgt * f;
    }
    return sum * hz / 3.;
}

__global__ void glauber_npart_kernel(const __grid_constant__ GlauberArgs G, double *npart, unsigned long long *mx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= G.nx || j >= G.ny) return;
    const double x = (i - (G.nx - 1) / 2.) * G.dx, y = (j - (G.ny - 1) / 2.) * G.dy;
    const double TA = ws_thickness_dev((x + G.b / 2) * (x + G.b / 2) + y * y, G.R, G.a);
    const double TB = ws_thickness_dev((x - G.b / 2) * (x - G.b / 2) + y * y, G.R, G.a);
    const double np = TA * (1. - exp(-G.sigma_nn * TB)) + TB * (1. - exp(-G.sigma_nn * TA));
    npart[i + (long long)G.nx * j] = np;
    /* np >= 0: its bit pattern orders like its value */
    atomicMax(mx, (unsigned long long)__double_as_longlong(np));
}

template <int EOS>
__global__ void glauber_fill_kernel(const __grid_constant__ GlauberArgs G, const double *npart,
                                    const unsigned long long *mx, double *e, double *p, double *u)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= G.nx || j >= G.ny) return;
    const long long N = (long long)G.nx * G.ny * G.nz;
    const long long m = i + (long long)G.nx * (j + (long long)G.ny * k);
    const double npmax = __longlong_as_double((long long)*mx);
    const double var = G.eta_sigma * G.eta_sigma;
    const double eta = (k - (G.nz - 1) / 2) * G.dz;       /* integer (nz - 1) / 2 */
    const double sc = fabs(eta) - G.eta_flat / 2;
    const double L = sc > 0 ? exp(-sc * sc / var / 2) : 1.0;
    const double ed = G.e0 * (npart[i + (long long)G.nx * j] / npmax) * L + 1.e-3;
    e[m] = ed;
    p[m] = eos_p<EOS>(G.eos, ed);
    u[m] = 1.0; u[N + m] = 0.0; u[2 * N + m] = 0.0; u[3 * N + m] = 0.0;
}

template <int EOS>
__global__ void hotspot_fill_kernel(const __grid_constant__ HotspotArgs H, double *e, double *p, double *u)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= H.nx || j >= H.ny) return;
    const long long N = (long long)H.nx * H.ny;
    const long long m = i + (long long)H.nx * j;
    const double x = (i - (H.nx - 1) / 2.) * H.dx, y = (j - (H.ny - 1) / 2.) * H.dy;
    const double inv2w2 = 1. / (2. * H.w * H.w);
    double ed = 1.e-3;
    for (int s = 0; s < H.nspots; ++s) {
        const double dx = x - __ldg(H.spots + s), dy = y - __ldg(H.spots + H.nspots + s);
        const double r2 = dx * dx + dy * dy;
        if (r2 < 50. * H.w * H.w) ed += __ldg(H.spots + 2 * H.nspots + s) * exp(-r2 * inv2w2);
    }
    e[m] = ed;
    p[m] = eos_p<EOS>(H.eos, ed);
    u[m] = 1.0; u[N + m] = 0.0; u[2 * N + m] = 0.0; u[3 * N + m] = 0.0;
}

void launch_glauber_ic(const GlauberArgs &g, double *npart, unsigned long long *mx, double *e, double *p, double *u,
                       cudaStream_t s)
{
    dim3 block(32, 4, 1);
    dim3 g2((g.nx + 31) / 32, (g.ny + 3) / 4, 1), g3((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz);
    cudaMemsetAsync(mx, 0, sizeof(unsigned long long), s);
    glauber_npart_kernel<<<g2, block, 0, s>>>(g, npart, mx);
    if (g.eos_kind == 1) glauber_fill_kernel<1><<<g3, block, 0, s>>>(g, npart, mx, e, p, u);
    else glauber_fill_kernel<0><<<g3, block, 0, s>>>(g, npart, mx, e, p, u);
}

void launch_hotspot_ic(const HotspotArgs &h, double *e, double *p, double *u, cudaStream_t s)
{
    dim3 block(32, 4, 1);
    dim3 g2((h.nx + 31) / 32, (h.ny + 3) / 4, 1);
    if (h.eos_kind == 1) hotspot_fill_kernel<1><<<g2, block, 0, s>>>(h, e, p, u);
    else hotspot_fill_kernel<0><<<g2, block, 0, s>>>(h, e, p, u);
}

} // namespace vh
