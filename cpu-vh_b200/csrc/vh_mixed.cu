/*
 * vh_mixed.cu -- the mixed-precision KT stage (vh_config.precision =
 * VH_PREC_MIXED), single-event and batched launch forms.
 *
 * FP32: the minmod limiter slopes, the flux arithmetic (F = v q / u^tau,
 * the spectral-radius term, H) and the source terms (velocity and pressure
 * gradients, sigma, omega, the pi/Pi relaxation right-hand side).
 * FP64: the conserved variables and their RK accumulation, the half-site
 * states the root solve receives, the root solve and the EoS (infer), the
 * d pi/dx direction sources, regulation and the stored e, p, u.
 *
 * Unlike the FP64 translation units this one is compiled with fused
 * multiply-adds and fast FP32 division and square root: the mixed result is
 * a numerical approximation of the FP64 one (its error against the FP64
 * path is measured by the tests), not a reproduction of its rounding.
 */
#include "vh_stage_kernels.cuh"
#include "vh_batch_kernels.cuh"

namespace vh {

void launch_stage_mixed(const StageArgs &a, int nq, int eos_kind, cudaStream_t s, StageMarks *m)
{
    if (nq == 15) {
        if (eos_kind == 1) launch_stage_t<15, 1, true>(a, s, m); else launch_stage_t<15, 0, true>(a, s, m);
    } else {
        if (eos_kind == 1) launch_stage_t<14, 1, true>(a, s, m); else launch_stage_t<14, 0, true>(a, s, m);
    }
}

BatchKernel batch_kernel_mixed(int nq, int eos_kind, int phase, bool st2, int zm)
{
    return batch_kernel_of<true>(nq, eos_kind, phase, st2, zm);
}

template <int NQ, int EOS>
static BatchKernel batch_face_t(int dir)
{
    return dir == 1 ? kt_batch_face_kernel<NQ, EOS, 1> : dir == 2 ? kt_batch_face_kernel<NQ, EOS, 2>
                                                                   : kt_batch_face_kernel<NQ, EOS, 3>;
}

BatchKernel batch_face_kernel_mixed(int nq, int eos_kind, int dir)
{
    if (nq == 15) return eos_kind == 1 ? batch_face_t<15, 1>(dir) : batch_face_t<15, 0>(dir);
    return eos_kind == 1 ? batch_face_t<14, 1>(dir) : batch_face_t<14, 0>(dir);
}

template <int NQ, int EOS>
static BatchKernel batch_face_lines_t(int dir)
{
    return dir == 3 ? kt_batch_face_lines_kernel<NQ, EOS, 3> : kt_batch_face_lines_kernel<NQ, EOS, 2>;
}

BatchKernel batch_face_lines_kernel_mixed(int nq, int eos_kind, int dir)
{
    if (nq == 15) return eos_kind == 1 ? batch_face_lines_t<15, 1>(dir) : batch_face_lines_t<15, 0>(dir);
    return eos_kind == 1 ? batch_face_lines_t<14, 1>(dir) : batch_face_lines_t<14, 0>(dir);
}

} // namespace vh
