/*
 * vh_batch_kernels.cuh -- the batched phase kernel: one launch covers every
 * member of a batch through a tile table (member, i0, j0, k), each block
 * staging its member's stage arguments in shared memory and running the same
 * per-cell bodies as the single-event kernels.  Templated on the precision
 * mode; vh_batch.cu instantiates the FP64 form, vh_mixed.cu the mixed one.
 */
#ifndef VH_BATCH_KERNELS_CUH
#define VH_BATCH_KERNELS_CUH

#include "vh_stage.cuh"

namespace vh {

static_assert(sizeof(StageArgs) % 8 == 0, "StageArgs is staged to shared memory in 8-byte words");


/* phase 0 source, 1-3 x/y/eta flux, 4 finalize, 5 fused stage; ZM (phases 4
 * and 5): 0 every member 2+1D, 1 every member 3+1D, 2 mixed (per member) */
template <int NQ, int EOS, int PHASE, bool STAGE2, int ZM, bool MIXED>
__global__ void __launch_bounds__(128, 4) kt_batch_kernel(const __grid_constant__ BatchLaunch B)
{
    __shared__ __align__(16) StageArgs sA;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nthr = blockDim.x * blockDim.y;
    int cur = -1;
    for (int t = blockIdx.x; t < B.ntiles; t += gridDim.x) {
        const int4 tile = __ldg(B.tiles + t);
        if (tile.x != cur) {           /* uniform over the block */
            __syncthreads();
            const unsigned long long *src = reinterpret_cast<const unsigned long long *>(B.args + tile.x);
            unsigned long long *dst = reinterpret_cast<unsigned long long *>(&sA);
            for (int w = tid; w < (int)(sizeof(StageArgs) / 8); w += nthr) dst[w] = src[w];
            __syncthreads();
            cur = tile.x;
        }
        const int i = tile.y + threadIdx.x + 2, j = tile.z + threadIdx.y + 2, k = tile.w + 2;
        if (i >= sA.nx + 2 || j >= sA.ny + 2) continue;
        const long long s = i + (long long)sA.ncx * j + (long long)sA.ncx * sA.ncy * k;
        if constexpr (PHASE == 0) {
            source_phase<NQ, EOS, MIXED>(sA, s);
        } else if constexpr (PHASE >= 1 && PHASE <= 3) {
            flux_phase<NQ, EOS, PHASE, MIXED>(sA, s);
        } else if constexpr (PHASE == 4) {
            if (ZM == 1 || (ZM == 2 && sA.nz > 1)) final_body<NQ, EOS, true, STAGE2>(sA, i, j, k, s);
            else final_body<NQ, EOS, false, STAGE2>(sA, i, j, k, s);
        } else {
            if (ZM == 1 || (ZM == 2 && sA.nz > 1)) stage_phase<NQ, EOS, true, STAGE2, MIXED>(sA, i, j, k, s);
            else stage_phase<NQ, EOS, false, STAGE2, MIXED>(sA, i, j, k, s);
        }
    }
}

/* Mixed precision: the face-once flux of one axis over the batch, one block
 * of 32 x 8 faces per tile (member, i0, j0, k0) -- flux_faces_tile, as the
 * single-event kt_flux_face_kernel runs it, so a member's fluxes equal its
 * single-event ones.  Tiles step by 31 cells along x for DIR 1 and by 7 along
 * y (DIR 2) or eta (DIR 3): the last face of a tile row only feeds the cell
 * below it. */
constexpr int kBatchFaceTX = 32, kBatchFaceTY = 8;

template <int NQ, int EOS, int DIR>
__global__ void __launch_bounds__(kBatchFaceTX * kBatchFaceTY, 2) kt_batch_face_kernel(const __grid_constant__ BatchLaunch B)
{
    __shared__ __align__(16) StageArgs sA;
    __shared__ double sm[NQ * kBatchFaceTX * kBatchFaceTY];
    const int tid = threadIdx.x + kBatchFaceTX * threadIdx.y;
    int cur = -1;
    for (int t = blockIdx.x; t < B.ntiles; t += gridDim.x) {
        const int4 tile = __ldg(B.tiles + t);
        if (tile.x != cur) {           /* uniform over the block */
            __syncthreads();
            const unsigned long long *src = reinterpret_cast<const unsigned long long *>(B.args + tile.x);
            unsigned long long *dst = reinterpret_cast<unsigned long long *>(&sA);
            for (int w = tid; w < (int)(sizeof(StageArgs) / 8); w += kBatchFaceTX * kBatchFaceTY) dst[w] = src[w];
            __syncthreads();
            cur = tile.x;
        }
        /* an inactive member (nx = 0, and no state pointers in its
         * arguments): skip its tiles -- flux_faces_tile would otherwise take
         * the x face at index 2 for a valid face (uniform over the block) */
        if (sA.nx == 0) continue;
        flux_faces_tile<NQ, EOS, DIR, kBatchFaceTX, kBatchFaceTY>(sA, tile.y, tile.z, tile.w, sm);
    }
}

/* FP64: the flux along DIR over line pieces of every member, one block per
 * table entry (member, block index among its line blocks) -- the body of the
 * single-event kt_flux_lines_kernel, so a member's fluxes equal its
 * single-event ones.  Dynamic shared memory: 2 * NQ * FluxLines::plane(nd)
 * doubles for the member with the most. */
template <int NQ, int EOS, int DIR>
__global__ void __launch_bounds__(128, 5) kt_batch_lines_kernel(const __grid_constant__ BatchLaunch B)
{
    __shared__ __align__(16) StageArgs sA;
    extern __shared__ double smd[];
    int cur = -1;
    for (int t = blockIdx.x; t < B.ntiles; t += gridDim.x) {
        const int4 tile = __ldg(B.tiles + t);
        __syncthreads();               /* the previous entry's staged values are read to its end */
        if (tile.x != cur) {           /* uniform over the block */
            const unsigned long long *src = reinterpret_cast<const unsigned long long *>(B.args + tile.x);
            unsigned long long *dst = reinterpret_cast<unsigned long long *>(&sA);
            for (int w = threadIdx.x; w < (int)(sizeof(StageArgs) / 8); w += blockDim.x) dst[w] = src[w];
            __syncthreads();
            cur = tile.x;
        }
        if (sA.nx == 0) continue;      /* an inactive member (uniform over the block) */
        flux_lines_block<NQ, EOS, DIR, 3, false>(sA, smd, tile.y);
    }
}

/* Mixed precision along y and eta: the face-once flux over line pieces of
 * every member, one block per entry (member, block index among its face
 * blocks) -- flux_faces_lines, as the single-event
 * kt_flux_face_lines_kernel runs it. */
template <int NQ, int EOS, int DIR>
__global__ void __launch_bounds__(128, 5) kt_batch_face_lines_kernel(const __grid_constant__ BatchLaunch B)
{
    __shared__ __align__(16) StageArgs sA;
    __shared__ double sm[NQ * 128];
    int cur = -1;
    for (int t = blockIdx.x; t < B.ntiles; t += gridDim.x) {
        const int4 tile = __ldg(B.tiles + t);
        __syncthreads();               /* the previous entry's faces are read to its end */
        if (tile.x != cur) {           /* uniform over the block */
            const unsigned long long *src = reinterpret_cast<const unsigned long long *>(B.args + tile.x);
            unsigned long long *dst = reinterpret_cast<unsigned long long *>(&sA);
            for (int w = threadIdx.x; w < (int)(sizeof(StageArgs) / 8); w += blockDim.x) dst[w] = src[w];
            __syncthreads();
            cur = tile.x;
        }
        if (sA.nx == 0) continue;      /* an inactive member (uniform over the block) */
        flux_faces_lines<NQ, EOS, DIR, false>(sA, sm, tile.y);
    }
}

template <int NQ, int EOS, int PHASE, bool MIXED>
static BatchKernel batch_kernel_z(bool st2, int zm)
{
    if (zm == 0) return st2 ? kt_batch_kernel<NQ, EOS, PHASE, true, 0, MIXED> : kt_batch_kernel<NQ, EOS, PHASE, false, 0, MIXED>;
    if (zm == 1) return st2 ? kt_batch_kernel<NQ, EOS, PHASE, true, 1, MIXED> : kt_batch_kernel<NQ, EOS, PHASE, false, 1, MIXED>;
    return st2 ? kt_batch_kernel<NQ, EOS, PHASE, true, 2, MIXED> : kt_batch_kernel<NQ, EOS, PHASE, false, 2, MIXED>;
}

template <int NQ, int EOS, bool MIXED>
static BatchKernel batch_kernel_t(int phase, bool st2, int zm)
{
    switch (phase) {
    case 0: return kt_batch_kernel<NQ, EOS, 0, false, 0, MIXED>;
    case 1: return kt_batch_kernel<NQ, EOS, 1, false, 0, MIXED>;
    case 2: return kt_batch_kernel<NQ, EOS, 2, false, 0, MIXED>;
    case 3: return kt_batch_kernel<NQ, EOS, 3, false, 0, MIXED>;
    case 4: return batch_kernel_z<NQ, EOS, 4, MIXED>(st2, zm);
    default: return batch_kernel_z<NQ, EOS, 5, MIXED>(st2, zm);
    }
}

template <bool MIXED>
static BatchKernel batch_kernel_of(int nq, int eos_kind, int phase, bool st2, int zm)
{
    if (nq == 15) return eos_kind == 1 ? batch_kernel_t<15, 1, MIXED>(phase, st2, zm) : batch_kernel_t<15, 0, MIXED>(phase, st2, zm);
    return eos_kind == 1 ? batch_kernel_t<14, 1, MIXED>(phase, st2, zm) : batch_kernel_t<14, 0, MIXED>(phase, st2, zm);
}

} // namespace vh

#endif
