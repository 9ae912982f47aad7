// Mixed-precision cell-model kernels: right-hand sides in FP32 with the
// hardware exp2/log2 approximations (this file is compiled with
// MB_FAST_FP32_MATH, -ftz=true, -prec-div=false), V and the ion
// concentrations accumulated in FP64.
#include "ode_common.cuh"

using namespace mb;

extern "C" int mbk_ode_step_mixed(const mb_ode_dev *o, mb_ctrl *ctrl, const double *vin, double *vout,
                                  cudaStream_t s) {
    if (o->n == 0) return 0;
    const unsigned blocks = (o->n + ODE_THREADS - 1) / ODE_THREADS;
    const mb_ode_dev &a = *o;
#define MB_STAGED(KERNEL, N64, N32)                                                       \
    do {                                                                                  \
        const size_t sm = staged_smem(N64, N32);                                          \
        auto *kfn = KERNEL;                                                               \
        const unsigned gb = staged_grid((const void *)kfn, sm, blocks);                   \
        if (!gb) return (int)cudaErrorInvalidConfiguration;                               \
        kfn<<<gb, ODE_THREADS, sm, s>>>(a, ctrl, vin, vout);                              \
    } while (0)
    if (o->model == MB_MODEL_TT2006) {
#define L(MB) k_tt2006_mixed<MB><<<blocks, ODE_THREADS, 0, s>>>(a, ctrl, vin, vout)
#define LS(MB) MB_STAGED(k_tt2006_mixed_s<MB>, 6, 13)
        MB_VARIANT_SWITCH(o->variant, L, LS)
#undef L
#undef LS
    } else if (o->rl_rule == MB_RL_TRUE) {
#define L(MB) k_torord_mixed<MB_RL_TRUE, MB><<<blocks, ODE_THREADS, 0, s>>>(a, ctrl, vin, vout)
#define LS(MB) MB_STAGED((k_torord_mixed_s<MB_RL_TRUE, MB>), TOR_N64, TOR_N32)
        MB_VARIANT_SWITCH(o->variant, L, LS)
#undef L
#undef LS
    } else {
#define L(MB) k_torord_mixed<MB_RL_REFERENCE_CPU, MB><<<blocks, ODE_THREADS, 0, s>>>(a, ctrl, vin, vout)
#define LS(MB) MB_STAGED((k_torord_mixed_s<MB_RL_REFERENCE_CPU, MB>), TOR_N64, TOR_N32)
        MB_VARIANT_SWITCH(o->variant, L, LS)
#undef L
#undef LS
    }
#undef MB_STAGED
    return (int)cudaGetLastError();
}
