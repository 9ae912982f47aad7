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
    if (o->model == MB_MODEL_TT2006) {
#define L(MB) k_tt2006_mixed<MB><<<blocks, ODE_THREADS, 0, s>>>(a, ctrl, vin, vout)
        MB_VARIANT_SWITCH(o->variant, L)
#undef L
    } else if (o->rl_rule == MB_RL_TRUE) {
#define L(MB) k_torord_mixed<MB_RL_TRUE, MB><<<blocks, ODE_THREADS, 0, s>>>(a, ctrl, vin, vout)
        MB_VARIANT_SWITCH(o->variant, L)
#undef L
    } else {
#define L(MB) k_torord_mixed<MB_RL_REFERENCE_CPU, MB><<<blocks, ODE_THREADS, 0, s>>>(a, ctrl, vin, vout)
        MB_VARIANT_SWITCH(o->variant, L)
#undef L
    }
    return (int)cudaGetLastError();
}
