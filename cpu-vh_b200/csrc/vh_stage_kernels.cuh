/*
 * vh_stage_kernels.cuh -- the single-event stage kernels and their launcher,
 * templated on the precision mode.  vh_kt.cu instantiates the FP64 form
 * (MIXED = false, bit-exact), vh_mixed.cu the mixed-precision form; the two
 * translation units are compiled with different floating-point flags.
 */
#ifndef VH_STAGE_KERNELS_CUH
#define VH_STAGE_KERNELS_CUH

#include <cstdlib>
#include "vh_stage.cuh"

namespace vh {

#ifndef VH_STAGE_MIN_BLOCKS
#define VH_STAGE_MIN_BLOCKS 4   /* 128 registers: 16 warps/SM; measured faster than 2-3 blocks at 168-255
                                   (the source kernel, which spills 224 bytes at 128: 0.78 ms per launch
                                   against 0.89 at 3 blocks and 168 registers) */
#endif

/* interior cell (i, j, k) of this thread, at padded index s */
__device__ __forceinline__ bool stage_cell(const StageArgs &A, int &i, int &j, int &k, long long &s)
{
    i = blockIdx.x * blockDim.x + threadIdx.x + 2;
    j = blockIdx.y * blockDim.y + threadIdx.y + 2;
    k = blockIdx.z + 2;
    if (i >= A.nx + 2 || j >= A.ny + 2) return false;
    s = i + (long long)A.ncx * j + (long long)A.ncx * A.ncy * k;
    return true;
}

/* the same for a 1-D grid over all nx*ny*nz interior cells, x fastest: no
 * lane idles at the end of a row (the per-cell phases need no tile) */
__device__ __forceinline__ bool stage_cell_flat(const StageArgs &A, int &i, int &j, int &k, long long &s)
{
    /* 32-bit index arithmetic: an event's cell count is far below 2^31 */
    const unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned nxy = (unsigned)A.nx * (unsigned)A.ny;
    if (c >= nxy * (unsigned)A.nz) return false;
    k = (int)(c / nxy);
    const int r = (int)(c - (unsigned)k * nxy);
    j = r / A.nx;
    i = r - j * A.nx + 2;
    j += 2;
    k += 2;
    s = i + (long long)A.ncx * j + (long long)A.ncx * A.ncy * k;
    return true;
}

template <int NQ, int EOS, bool HAS_Z, bool STAGE2, bool MIXED>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_stage_kernel(const __grid_constant__ StageArgs A)
{
    int i, j, k;
    long long s;
    if (!stage_cell(A, i, j, k, s)) return;
    stage_phase<NQ, EOS, HAS_Z, STAGE2, MIXED>(A, i, j, k, s);
}

/* Phase-split form of the same stage: five short kernels instead of one long
 * one.  Each phase's code is a fraction of the fused kernel's and fits the
 * instruction cache: the fused kernel spends most of its stall time waiting
 * for instruction fetch on large lattices. */
template <int NQ, int EOS, bool MIXED>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_source_kernel(const __grid_constant__ StageArgs A)
{
    pdl_wait();       /* reads the previous stage's results: wait, then let the flux start */
    pdl_trigger();
    int i, j, k;
    long long s;
    if (!stage_cell_flat(A, i, j, k, s)) return;
    source_phase<NQ, EOS, MIXED>(A, s);
}

template <int NQ, int EOS, int DIR, bool MIXED>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_flux_kernel(const __grid_constant__ StageArgs A)
{
    int i, j, k;
    long long s;
    if (!stage_cell(A, i, j, k, s)) return;
    flux_phase<NQ, EOS, DIR, MIXED>(A, s);
}

/* face-parallel fused stage (small lattices): 32 cells of one row per block,
 * 1 + 2 ndir threads per cell */
constexpr int kFacesTX = 32;

template <int NQ, int EOS, bool HAS_Z, bool STAGE2, bool MIXED>
__global__ void __launch_bounds__(kFacesTX * 7, 2) kt_stage_faces_kernel(const __grid_constant__ StageArgs A)
{
    constexpr int ND = HAS_Z ? 3 : 2;
    __shared__ double sm[2 * ND * NQ * kFacesTX];
    const int i = blockIdx.x * kFacesTX + threadIdx.x + 2;
    const int j = blockIdx.y + 2;
    const int k = blockIdx.z + 2;
    stage_faces_cell<NQ, EOS, HAS_Z, STAGE2, MIXED>(A, i, j, k, i < A.nx + 2, sm, kFacesTX);
}

/* face-parallel (default) or one-thread-per-cell fused stage: VH_STAGE_FACES=0
 * selects the latter */
static inline bool stage_faces()
{
    static int on = [] {
        const char *e = getenv("VH_STAGE_FACES");
        return (e && e[0] == '0') ? 0 : 1;
    }();
    return on == 1;
}

/* FP64 flux with the stencil tile staged in shared memory (cp.async): the
 * block's 32 x 4 cells and their 2-cell halo along DIR, all components */
template <int NQ, int EOS, int DIR>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_flux_staged_kernel(const __grid_constant__ StageArgs A)
{
    constexpr int TX = 32, TY = 4;
    __shared__ double sm[NQ * (TX + (DIR == 1 ? 4 : 0)) * (TY + (DIR == 1 ? 0 : 4))];
    const int i0 = blockIdx.x * TX;
    int j0, k0;
    if (DIR == 3) { j0 = blockIdx.y; k0 = blockIdx.z * TY; } else { j0 = blockIdx.y * TY; k0 = blockIdx.z; }
    flux_staged_tile<NQ, EOS, DIR, TX, TY>(A, i0, j0, k0, sm);
}

/* the same tile with every half slope computed once (flux_slopes_tile);
 * dynamic shared memory: FluxTile::kDoubles(NQ) doubles, up to 53.8 KB */
template <int NQ, int EOS, int DIR>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_flux_slopes_kernel(const __grid_constant__ StageArgs A)
{
    constexpr int TX = 32, TY = 4;
    extern __shared__ double smd[];
    const int i0 = blockIdx.x * TX;
    int j0, k0;
    if (DIR == 3) { j0 = blockIdx.y; k0 = blockIdx.z * TY; } else { j0 = blockIdx.y * TY; k0 = blockIdx.z; }
    flux_slopes_tile<NQ, EOS, DIR, TX, TY>(A, i0, j0, k0, smd);
}

/* The phase-split stage's kernels go out with programmatic dependent
 * launch: each flux kernel starts its staging and root solves while the
 * previous phase drains and waits only before adding to the accumulator
 * (flux_lines_block); the source and finalize kernels wait at their start.
 * VH_PDL=0 launches them in plain stream order. */
static inline bool pdl_enabled()
{
    static int on = [] {
        const char *e = getenv("VH_PDL");
        return (e && e[0] == '0') ? 0 : 1;
    }();
    return on == 1;
}

template <typename... P>
static void launch_pdl(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, const StageArgs &a)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, a);
}

template <int NQ, int EOS, int DIR>
static void launch_flux_slopes(const StageArgs &a, dim3 grid, dim3 block, cudaStream_t s)
{
    constexpr size_t bytes = sizeof(double) * FluxTile<DIR, 32, 4>::kDoubles(NQ);
    static const bool attr = [] {
        cudaFuncSetAttribute(kt_flux_slopes_kernel<NQ, EOS, DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)bytes);
        cudaFuncSetAttribute(kt_flux_slopes_kernel<NQ, EOS, DIR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)((VH_STAGE_MIN_BLOCKS * (bytes + 1024) * 100 + 228 * 1024 - 1) / (228 * 1024)));
        return true;
    }();
    (void)attr;
    kt_flux_slopes_kernel<NQ, EOS, DIR><<<grid, block, bytes, s>>>(a);
}

/* the flux over line pieces (flux_lines_block): a 1-D grid of 128-thread
 * blocks, dynamic shared memory 2 * NQ * FluxLines::plane(nd) doubles */
template <int NQ, int EOS, int DIR, int MB, int UNR>
__global__ void __launch_bounds__(128, MB) kt_flux_lines_kernel(const __grid_constant__ StageArgs A)
{
    extern __shared__ double smd[];
    flux_lines_block<NQ, EOS, DIR, UNR, true>(A, smd, blockIdx.x);
}

template <int NQ, int EOS, int DIR, int MB, int UNR = 1>
static void launch_flux_lines(const StageArgs &a, cudaStream_t s)
{
    using G = FluxLines<DIR>;
    const int nd = (DIR == 1) ? a.nx : (DIR == 2) ? a.ny : a.nz;
    const size_t bytes = sizeof(double) * 2 * NQ * (size_t)G::plane(nd);
    static size_t attr_bytes = 0;
    if (bytes > attr_bytes) {
        cudaFuncSetAttribute(kt_flux_lines_kernel<NQ, EOS, DIR, MB, UNR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)bytes);
        /* shared memory for MB resident blocks (1 KB reserved per block) out
         * of 228 KB, and the rest of the SM's 256 KB left to L1, which holds
         * the EoS table of the root solves; VH_CARVEOUT overrides (percent) */
        int pct = (int)((MB * (bytes + 1024) * 100 + 228 * 1024 - 1) / (228 * 1024));
        if (pct > 100) pct = 100;
        if (const char *e = getenv("VH_CARVEOUT")) pct = atoi(e);
        cudaFuncSetAttribute(kt_flux_lines_kernel<NQ, EOS, DIR, MB, UNR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             pct);
        attr_bytes = bytes;
    }
    const long long runs = (long long)nd * G::bundles(a.nx, a.ny, a.nz);
    const unsigned blocks = (unsigned)((runs + G::PB - 1) / G::PB);
    launch_pdl(kt_flux_lines_kernel<NQ, EOS, DIR, MB, UNR>, dim3(blocks), dim3(128), bytes, s, a);
}

/* FP64 flux form of the phase-split stage: VH_FLUX_FORM=lines (default:
 * line pieces, 5 blocks per SM at 96 registers, the component loop unrolled
 * by 3), lines4 (4 blocks per SM, up to 128 registers, loop rolled), slopes
 * (32 x 4 tiles with shared half slopes) or staged (32 x 4 tiles, every cell
 * computing its own slopes).  Measured on the 131x131x61 Glauber event (ms
 * per step of the x/y/eta launches, two each): lines 0.74/0.77/0.78 (0.74/
 * 0.85/0.87 with the shared-memory carveout at its maximum, which left L1
 * 28 KB for the EoS table and the loads; 0.75/0.86/0.87 with the loop
 * rolled), lines4 0.89/0.98/0.99, slopes 0.98/1.00/1.03, staged
 * 1.10/1.09/1.12. */
static inline int flux_form()
{
    static int f = [] {
        const char *e = getenv("VH_FLUX_FORM");
        if (!e) return 3;
        if (e[0] == 'l') return e[5] == '4' ? 2 : 3;
        return (e[0] == 's' && e[1] == 't') ? 0 : 1;
    }();
    return f;
}

/* staged flux on (default) or off: VH_FLUX_STAGED=0 selects the kernel that
 * reads the stencil straight from device memory */
static inline bool flux_staged()
{
    static int on = [] {
        const char *e = getenv("VH_FLUX_STAGED");
        return (e && e[0] == '0') ? 0 : 1;
    }();
    return on == 1;
}

/* face-once flux (mixed precision): 32 x 8 threads, each face computed once
 * and shared with both adjacent cells through shared memory */
constexpr int kFaceTX = 32, kFaceTY = 8;

template <int NQ, int EOS, int DIR>
__global__ void __launch_bounds__(kFaceTX * kFaceTY, 2) kt_flux_face_kernel(const __grid_constant__ StageArgs A)
{
    __shared__ double sm[NQ * kFaceTX * kFaceTY];
    int i0, j0, k0;
    if (DIR == 1) { i0 = blockIdx.x * (kFaceTX - 1); j0 = blockIdx.y * kFaceTY; k0 = blockIdx.z; }
    else if (DIR == 2) { i0 = blockIdx.x * kFaceTX; j0 = blockIdx.y * (kFaceTY - 1); k0 = blockIdx.z; }
    else { i0 = blockIdx.x * kFaceTX; j0 = blockIdx.y; k0 = blockIdx.z * (kFaceTY - 1); }
    flux_faces_tile<NQ, EOS, DIR, kFaceTX, kFaceTY, true>(A, i0, j0, k0, sm);
}

/* the face-once flux over line pieces (flux_faces_lines), 128 threads */
template <int NQ, int EOS, int DIR, int MB>
__global__ void __launch_bounds__(128, MB) kt_flux_face_lines_kernel(const __grid_constant__ StageArgs A)
{
    __shared__ double sm[NQ * 128];
    flux_faces_lines<NQ, EOS, DIR, true>(A, sm, blockIdx.x);
}

template <int NQ, int EOS, int DIR, int MB>
static void launch_flux_face_lines(const StageArgs &a, cudaStream_t s)
{
    using G = FaceLinesG<DIR>;
    const int nd = (DIR == 1) ? a.nx : (DIR == 2) ? a.ny : a.nz;
    const long long faces = (long long)(nd + 1) * G::bundles(a.nx, a.ny, a.nz);
    const unsigned blocks = (unsigned)((faces + G::PB - 2) / (G::PB - 1));
    launch_pdl(kt_flux_face_lines_kernel<NQ, EOS, DIR, MB>, dim3(blocks), dim3(128), 0, s, a);
}

/* mixed-precision flux form of the phase-split stage: VH_FACE_FORM=lines
 * (default: faces over line pieces along y and eta, 32 x 8 face tiles along
 * x, where a warp passes each face to the next lane by shuffle) or tiles
 * (32 x 8 face tiles along every axis).  131x131x61 Glauber event, ms per
 * step x/y/eta: lines 0.646/0.658/0.715, tiles 0.646/0.723/0.747; along x
 * line pieces measured 0.712 (a block barrier for the next face where the
 * tile's warp uses a shuffle), at 3 blocks per SM y/eta 0.744/0.803 */
static inline int face_form()
{
    static int f = [] {
        const char *e = getenv("VH_FACE_FORM");
        return (e && e[0] == 't') ? 0 : 4;
    }();
    return f;
}

template <int DIR>
static inline dim3 face_grid(const StageArgs &a)
{
    if (DIR == 1) return dim3((a.nx + kFaceTX - 2) / (kFaceTX - 1), (a.ny + kFaceTY - 1) / kFaceTY, a.nz);
    if (DIR == 2) return dim3((a.nx + kFaceTX - 1) / kFaceTX, (a.ny + kFaceTY - 2) / (kFaceTY - 1), a.nz);
    return dim3((a.nx + kFaceTX - 1) / kFaceTX, a.ny, (a.nz + kFaceTY - 2) / (kFaceTY - 1));
}

/* MIXED is part of the kernel's name although the body is the same: the
 * FP64 and the mixed translation units compile it with different
 * floating-point flags, and one name for two different device functions
 * would leave it to the runtime which of the two a launch runs */
template <int NQ, int EOS, bool HAS_Z, bool STAGE2, bool MIXED>
__global__ void __launch_bounds__(128, VH_STAGE_MIN_BLOCKS) kt_final_kernel(const __grid_constant__ StageArgs A)
{
    pdl_wait();       /* reads the accumulated update */
    pdl_trigger();
    int i, j, k;
    long long s;
    if (!stage_cell_flat(A, i, j, k, s)) return;
    final_body<NQ, EOS, HAS_Z, STAGE2>(A, i, j, k, s);
}

/* Fused (face-parallel) for small lattices, which are latency-bound;
 * phase-split from 2^15 interior cells up.  Measured on B200 (FP64, table EoS,
 * ms/step fused vs split): 101^2 0.095 vs 0.253; 201^2 0.309 vs 0.285; 41^3
 * 1.07 vs 0.62; 131x131x61 12.98 vs 5.18.  VH_STAGE_MODE=fused|split
 * overrides. */
static inline bool use_split(const StageArgs &a)
{
    static int forced = [] {
        const char *e = getenv("VH_STAGE_MODE");
        return !e ? -1 : (e[0] == 'f' ? 0 : 1);
    }();
    if (forced >= 0) return forced == 1;
    return (long long)a.nx * a.ny * a.nz >= (1LL << 15);
}

template <int NQ, int EOS, bool MIXED>
static void launch_stage_t(const StageArgs &a, cudaStream_t s, StageMarks *m)
{
    dim3 block(32, 4, 1);
    dim3 grid((a.nx + 31) / 32, (a.ny + 3) / 4, a.nz);
    const bool z = a.nz > 1, st2 = a.qbase != nullptr;
    if (m) { m->n = 0; cudaEventRecord(m->ev[0], s); }
    auto mark = [&](int phase) {
        if (!m) return;
        m->phase[m->n] = phase;
        cudaEventRecord(m->ev[++m->n], s);
    };
    if (!use_split(a) && stage_faces()) {
        const dim3 gf((a.nx + kFacesTX - 1) / kFacesTX, a.ny, a.nz);
        const dim3 bf(kFacesTX, z ? 7 : 5, 1);
        if (z && st2) kt_stage_faces_kernel<NQ, EOS, true, true, MIXED><<<gf, bf, 0, s>>>(a);
        else if (z) kt_stage_faces_kernel<NQ, EOS, true, false, MIXED><<<gf, bf, 0, s>>>(a);
        else if (st2) kt_stage_faces_kernel<NQ, EOS, false, true, MIXED><<<gf, bf, 0, s>>>(a);
        else kt_stage_faces_kernel<NQ, EOS, false, false, MIXED><<<gf, bf, 0, s>>>(a);
        mark(5);
        return;
    }
    if (!use_split(a)) {
        if (z && st2) kt_stage_kernel<NQ, EOS, true, true, MIXED><<<grid, block, 0, s>>>(a);
        else if (z) kt_stage_kernel<NQ, EOS, true, false, MIXED><<<grid, block, 0, s>>>(a);
        else if (st2) kt_stage_kernel<NQ, EOS, false, true, MIXED><<<grid, block, 0, s>>>(a);
        else kt_stage_kernel<NQ, EOS, false, false, MIXED><<<grid, block, 0, s>>>(a);
        mark(5);
        return;
    }
    const dim3 gflat((unsigned)(((long long)a.nx * a.ny * a.nz + 127) / 128));
    launch_pdl(kt_source_kernel<NQ, EOS, MIXED>, gflat, dim3(128), 0, s, a);
    mark(0);
    if constexpr (MIXED) {
        if (face_form() != 0) {
            const dim3 fb(kFaceTX, kFaceTY, 1);
            launch_pdl(kt_flux_face_kernel<NQ, EOS, 1>, face_grid<1>(a), fb, 0, s, a);
            mark(1);
            launch_flux_face_lines<NQ, EOS, 2, 4>(a, s);
            mark(2);
            if (z) { launch_flux_face_lines<NQ, EOS, 3, 4>(a, s); mark(3); }
        } else {
            const dim3 fb(kFaceTX, kFaceTY, 1);
            launch_pdl(kt_flux_face_kernel<NQ, EOS, 1>, face_grid<1>(a), fb, 0, s, a);
            mark(1);
            launch_pdl(kt_flux_face_kernel<NQ, EOS, 2>, face_grid<2>(a), fb, 0, s, a);
            mark(2);
            if (z) { launch_pdl(kt_flux_face_kernel<NQ, EOS, 3>, face_grid<3>(a), fb, 0, s, a); mark(3); }
        }
    } else if (flux_staged() && flux_form() != 0) {
        const dim3 g3((a.nx + 31) / 32, a.ny, (a.nz + 3) / 4);
        if (flux_form() == 2) {
            launch_flux_lines<NQ, EOS, 1, 4>(a, s);
            mark(1);
            launch_flux_lines<NQ, EOS, 2, 4>(a, s);
            mark(2);
            if (z) { launch_flux_lines<NQ, EOS, 3, 4>(a, s); mark(3); }
        } else if (flux_form() == 3) {
            launch_flux_lines<NQ, EOS, 1, 5, 3>(a, s);
            mark(1);
            launch_flux_lines<NQ, EOS, 2, 5, 3>(a, s);
            mark(2);
            if (z) { launch_flux_lines<NQ, EOS, 3, 5, 3>(a, s); mark(3); }
        } else {
            launch_flux_slopes<NQ, EOS, 1>(a, grid, block, s);
            mark(1);
            launch_flux_slopes<NQ, EOS, 2>(a, grid, block, s);
            mark(2);
            if (z) { launch_flux_slopes<NQ, EOS, 3>(a, g3, block, s); mark(3); }
        }
    } else if (flux_staged()) {
        const dim3 g3((a.nx + 31) / 32, a.ny, (a.nz + 3) / 4);
        kt_flux_staged_kernel<NQ, EOS, 1><<<grid, block, 0, s>>>(a);
        mark(1);
        kt_flux_staged_kernel<NQ, EOS, 2><<<grid, block, 0, s>>>(a);
        mark(2);
        if (z) { kt_flux_staged_kernel<NQ, EOS, 3><<<g3, block, 0, s>>>(a); mark(3); }
    } else {
        kt_flux_kernel<NQ, EOS, 1, MIXED><<<grid, block, 0, s>>>(a);
        mark(1);
        kt_flux_kernel<NQ, EOS, 2, MIXED><<<grid, block, 0, s>>>(a);
        mark(2);
        if (z) { kt_flux_kernel<NQ, EOS, 3, MIXED><<<grid, block, 0, s>>>(a); mark(3); }
    }
    if (z && st2) launch_pdl(kt_final_kernel<NQ, EOS, true, true, MIXED>, gflat, dim3(128), 0, s, a);
    else if (z) launch_pdl(kt_final_kernel<NQ, EOS, true, false, MIXED>, gflat, dim3(128), 0, s, a);
    else if (st2) launch_pdl(kt_final_kernel<NQ, EOS, false, true, MIXED>, gflat, dim3(128), 0, s, a);
    else launch_pdl(kt_final_kernel<NQ, EOS, false, false, MIXED>, gflat, dim3(128), 0, s, a);
    mark(4);
}

} // namespace vh

#endif
