// ten Tusscher & Panfilov 2006 human ventricular myocyte, epicardial variant
// with the constants of the reference model library
// (src/models_library/ten_tusscher/ten_tusscher_2006_RS_CPU.c:137-351).
//
// One Rush-Larsen sub-step: gates 1..12 advance with
//     y <- y_inf + (y - y_inf) * exp(-dt / tau)
// (the reference's RL update, _RS_CPU.c:337-348); V and the six
// concentration-like states advance with explicit Euler (_RS_CPU.c:112,128-133).
//
// The arithmetic type T is double for the plain method and float for the
// mixed-precision form.  Every literal keeps the reference's spelling: a
// constant written with an `f` suffix there is the float value promoted to
// double here too, which the FP64 parity bar depends on.
#pragma once
#include "mb_math.cuh"

MB_NS_BEGIN

constexpr int TT_NEQ = 19;

// Indices of the state rows (the reference sv[] order, _RS_CPU.c:140-158).
enum TTIdx {
    TT_V = 0, TT_XR1, TT_XR2, TT_XS, TT_M, TT_H, TT_J, TT_D, TT_F, TT_F2, TT_FCASS,
    TT_S, TT_R, TT_CAI, TT_CASR, TT_CASS, TT_RPRIME, TT_NAI, TT_KI
};

// Default initial state (_RS_CPU.c:27-45); the literals are floats there.
__host__ __device__ inline double tt2006_default_state(int i) {
    switch (i) {
    case 0: return -85.23f;   case 1: return 0.00621f;  case 2: return 0.4712f;
    case 3: return 0.0095f;   case 4: return 0.00172f;  case 5: return 0.7444f;
    case 6: return 0.7045f;   case 7: return 3.373e-5f; case 8: return 0.7888f;
    case 9: return 0.9755f;   case 10: return 0.9953f;  case 11: return 0.999998f;
    case 12: return 2.42e-8f; case 13: return 0.000126f; case 14: return 3.64f;
    case 15: return 0.00036f; case 16: return 0.9073f;  case 17: return 8.604f;
    default: return 136.89f;
    }
}

// Conductance scalings applied to gNa, gKr, gKs, gCaL, gK1 (1 = reference).
template <typename T>
struct TTScale { T gNa, gKr, gKs, gCaL, gK1; };

// Outputs of one evaluation: dV/dt, the six Euler derivatives and the twelve
// already-advanced gate values.
template <typename T>
struct TTUpdate {
    T dV;
    T gate[12];          // new values of states 1..12
    T dCai, dCaSR, dCaSS, dRprime, dNai, dKi;
};

// y: the 19 state values (in T), stim: merged stimulus current.
template <typename T>
__device__ __forceinline__ void tt2006_rhs(const T *y, T stim, T dt, const TTScale<T> &sc,
                                           TTUpdate<T> &u) {
    const T V = y[TT_V];
    const T Xr1 = y[TT_XR1], Xr2 = y[TT_XR2], Xs = y[TT_XS];
    const T m = y[TT_M], h = y[TT_H], j = y[TT_J];
    const T d = y[TT_D], f = y[TT_F], f2 = y[TT_F2], fCass = y[TT_FCASS];
    const T s = y[TT_S], r = y[TT_R];
    const T Ca_i = y[TT_CAI], Ca_SR = y[TT_CASR], Ca_ss = y[TT_CASS];
    const T R_prime = y[TT_RPRIME], Na_i = y[TT_NAI], K_i = y[TT_KI];

    // physical constants and cell geometry
    const T R = T(8314.472), Tk = T(310.0), F = T(96485.3415f);
    const T Cm = T(0.185), V_c = T(0.016404);
    const T Ko = T(5.4), Nao = T(140.0), Cao = T(2.0);
    const T P_kna = T(0.03), K_mk = T(1.0), P_NaK = T(2.724), K_mNa = T(40.0), K_pCa = T(0.0005);
    // calcium handling
    const T V_rel = T(0.102), k1_prime = T(0.15), max_sr = T(2.5), min_sr = T(1.0);
    const T EC = T(1.5), Vmax_up = T(0.006375);
    // Na/Ca exchanger
    const T n_alpha = T(2.5), n_gamma = T(0.35), K_sat = T(0.1), Km_Ca = T(1.38);
    const T Km_Nai = T(87.5), K_NaCa = T(1000.0);
    // maximal conductances
    const T g_to = T(0.294), g_Kr = T(0.153) * sc.gKr, g_Ks = T(0.098) * sc.gKs;
    const T g_CaL = T(3.98e-05) * sc.gCaL, g_Na = T(14.838) * sc.gNa, g_pK = T(0.0146);
    const T g_bca = T(0.000592), g_pCa = T(0.1238), g_K1 = T(5.405) * sc.gK1, g_bna = T(0.00029);

    const T RTF = (R * Tk) / F;
    const T EK = RTF * mlog(Ko / K_i);
    const T EKs = RTF * mlog((Ko + (P_kna * Nao)) / (K_i + (P_kna * Na_i)));
    const T ENa = RTF * mlog(Nao / Na_i);
    const T ECa = ((T(0.5f) * R * Tk) / F) * mlog(Cao / Ca_i);

    // inward rectifier
    const T vek = V - EK;
    const T beta_K1 = ((T(3.0f) * mexp(T(0.0002f) * (vek + T(100.0f)))) + mexp(T(0.1f) * (vek - T(10.0f)))) /
                      (T(1.0f) + mexp(T(-0.5f) * vek));
    const T alpha_K1 = T(0.1f) / (T(1.0f) + mexp(T(0.06f) * (vek - T(200.0f))));
    const T xK1_inf = alpha_K1 / (alpha_K1 + beta_K1);

    const T IK1 = g_K1 * xK1_inf * vek;
    const T Ito = g_to * r * s * vek;
    const T IKr = g_Kr * Xr1 * Xr2 * vek * msqrt(Ko / T(5.4f));
    const T IKs = g_Ks * (Xs * Xs) * (V - EKs);
    const T IpK = (g_pK * vek) / (T(1.0f) + mexp((T(25.0f) - V) / T(5.98f)));

    // L-type calcium current; the removable singularity at V = 15 mV uses
    // the limit value inside a +-1e-5 mV band (_RS_CPU.c:221)
    const T FRT = F / (R * Tk);
    T ICaL;
    const T v15 = V - T(15.0f);
    if (V < T(15.0f - 1.0e-5f) || V > T(15.0f + 1.0e-5f)) {
        const T ea = (T(2.0f) * v15 * F) / (R * Tk);
        ICaL = (((g_CaL * d * f * f2 * fCass * T(4.0f) * v15 * (F * F)) / (R * Tk)) *
                ((T(0.25f) * Ca_ss * mexp(ea)) - Cao)) / mexpm1(ea);
    } else {
        ICaL = g_CaL * d * f * f2 * fCass * T(2.0f) * F * (T(0.25f) * Ca_ss - Cao);
    }
    const T IbCa = g_bca * (V - ECa);
    const T IpCa = (g_pCa * Ca_i) / (Ca_i + K_pCa);

    const T INaK = ((((P_NaK * Ko) / (Ko + K_mk)) * Na_i) / (Na_i + K_mNa)) /
                   (T(1.0f) + (T(0.1245f) * mexp(((T(-0.1f)) * V * F) / (R * Tk))) +
                    (T(0.0353f) * mexp(((-V) * F) / (R * Tk))));
    const T INa = g_Na * (m * m * m) * h * j * (V - ENa);
    const T IbNa = g_bna * (V - ENa);
    const T e_gm1 = mexp(((n_gamma - T(1.0f)) * V * F) / (R * Tk));
    const T INaCa = (K_NaCa * ((mexp((n_gamma * V * F) / (R * Tk)) * (Na_i * Na_i * Na_i) * Cao) -
                               (e_gm1 * (Nao * Nao * Nao) * Ca_i * n_alpha))) /
                    (((Km_Nai * Km_Nai * Km_Nai) + (Nao * Nao * Nao)) * (Km_Ca + Cao) *
                     (T(1.0f) + (K_sat * e_gm1)));
    (void)FRT;

    // gating variables: steady states and time constants
    const T xr1_inf = T(1.0f) / (T(1.0f) + mexp((T(-26.0f) - V) / T(7.0f)));
    const T tau_xr1 = (T(450.0f) / (T(1.0f) + mexp((T(-45.0f) - V) / T(10.0f)))) *
                      (T(6.0f) / (T(1.0f) + mexp((V + T(30.0f)) / T(11.5f))));
    const T xr2_inf = T(1.0f) / (T(1.0f) + mexp((V + T(88.0f)) / T(24.0f)));
    const T tau_xr2 = (T(3.0f) / (T(1.0f) + mexp((T(-60.0f) - V) / T(20.0f)))) *
                      (T(1.12f) / (T(1.0f) + mexp((V - T(60.0f)) / T(20.0f))));
    const T xs_inf = T(1.0f) / (T(1.0f) + mexp((T(-5.0f) - V) / T(14.0f)));
    const T tau_xs = ((T(1400.0f) / msqrt(T(1.0f) + mexp((T(5.0f) - V) / T(6.0f)))) *
                      (T(1.0f) / (T(1.0f) + mexp((V - T(35.0f)) / T(15.0f))))) + T(80.0f);

    const T em = T(1.0f) + mexp((T(-56.86f) - V) / T(9.03f));
    const T m_inf = T(1.0f) / (em * em);
    const T tau_m = (T(1.0f) / (T(1.0f) + mexp((T(-60.0f) - V) / T(5.0f)))) *
                    ((T(0.1f) / (T(1.0f) + mexp((V + T(35.0f)) / T(5.0f)))) +
                     (T(0.1f) / (T(1.0f) + mexp((V - T(50.0f)) / T(200.0f)))));

    const T eh = T(1.0f) + mexp((V + T(71.55f)) / T(7.43f));
    const T h_inf = T(1.0f) / (eh * eh);
    const T j_inf = h_inf;
    T alpha_h, beta_h, alpha_j, beta_j;
    if (V < T(-40.0f)) {
        alpha_h = T(0.057f) * mexp((-(V + T(80.0f))) / T(6.8f));
        beta_h = (T(2.7f) * mexp(T(0.079f) * V)) + (T(310000.0f) * mexp(T(0.3485f) * V));
        alpha_j = ((((T(-25428.0f)) * mexp(T(0.2444f) * V)) - (T(6.948e-06f) * mexp(T(-0.04391f) * V))) *
                   (V + T(37.78f))) / (T(1.0f) + mexp(T(0.311f) * (V + T(79.23f))));
        beta_j = (T(0.02424f) * mexp(T(-0.01052f) * V)) / (T(1.0f) + mexp(T(-0.1378f) * (V + T(40.14f))));
    } else {
        alpha_h = T(0.0f);
        beta_h = T(0.77f) / (T(0.13f) * (T(1.0f) + mexp((V + T(10.66f)) / T(-11.1f))));
        alpha_j = T(0.0f);
        beta_j = (T(0.6f) * mexp(T(0.057f) * V)) / (T(1.0f) + mexp(T(-0.1f) * (V + T(32.0f))));
    }
    const T tau_h = T(1.0f) / (alpha_h + beta_h);
    const T tau_j = T(1.0f) / (alpha_j + beta_j);

    const T d_inf = T(1.0f) / (T(1.0f) + mexp((T(-8.0f) - V) / T(7.5f)));
    const T tau_d = ((T(1.4f) / (T(1.0f) + mexp((T(-35.0f) - V) / T(13.0f)))) + T(0.25f)) *
                        (T(1.4f) / (T(1.0f) + mexp((V + T(5.0f)) / T(5.0f)))) +
                    (T(1.0f) / (T(1.0f) + mexp((T(50.0f) - V) / T(20.0f))));

    const T e30 = mexp((V + T(30.0f)) / T(10.0f));
    const T v27 = V + T(27.0f);
    const T f_inf = T(1.0f) / (T(1.0f) + mexp((V + T(20.0f)) / T(7.0f)));
    const T tau_f = (T(1102.5f) * mexp((-(v27 * v27)) / T(225.0f))) +
                    (T(200.0f) / (T(1.0f) + mexp((T(13.0f) - V) / T(10.0f)))) +
                    (T(180.0f) / (T(1.0f) + e30)) + T(20.0f);
    const T f2_inf = (T(0.67f) / (T(1.0f) + mexp((V + T(35.0f)) / T(7.0f)))) + T(0.33f);
    const T tau_f2 = (T(562.0f) * mexp((-(v27 * v27)) / T(240.0f))) +
                     (T(31.0f) / (T(1.0f) + mexp((T(25.0f) - V) / T(10.0f)))) +
                     (T(80.0f) / (T(1.0f) + e30));

    const T cr = Ca_ss / T(0.05f);
    const T fCass_inf = (T(0.6f) / (T(1.0f) + cr * cr)) + T(0.4f);
    const T tau_fCass = (T(80.0f) / (T(1.0f) + cr * cr)) + T(2.0f);

    const T s_inf = T(1.0f) / (T(1.0f) + mexp((V + T(20.0f)) / T(5.0f)));
    const T v45 = V + T(45.0f);
    const T tau_s = (T(85.0f) * mexp((-(v45 * v45)) / T(320.0f))) +
                    (T(5.0f) / (T(1.0f) + mexp((V - T(20.0f)) / T(5.0f)))) + T(3.0f);
    const T r_inf = T(1.0f) / (T(1.0f) + mexp((T(20.0f) - V) / T(6.0f)));
    const T v40 = V + T(40.0f);
    const T tau_r = (T(9.5f) * mexp((-(v40 * v40)) / T(1800.0f))) + T(0.8f);

    // calcium dynamics
    const T ecs = EC / Ca_SR;
    const T kcasr = max_sr - ((max_sr - min_sr) / (T(1.0f) + ecs * ecs));
    const T k1 = k1_prime / kcasr;
    const T k3 = T(0.06);
    const T css2 = Ca_ss * Ca_ss;
    const T O = (k1 * css2 * R_prime) / (k3 + (k1 * css2));
    const T Irel = V_rel * O * (Ca_SR - Ca_ss);
    const T K_up = T(0.00025);
    const T i_up = Vmax_up / (T(1.0f) + ((K_up * K_up) / (Ca_i * Ca_i)));
    const T i_leak = T(0.00036f) * (Ca_SR - Ca_i);
    const T i_xfer = T(0.0038f) * (Ca_ss - Ca_i);
    const T k2 = T(0.045f) * kcasr;
    const T k4 = T(0.005f);
    const T Buf_c = T(0.2f), K_buf_c = T(0.001f);
    const T cbc = Ca_i + K_buf_c;
    const T Ca_i_bufc = T(1.0f) / (T(1.0f) + ((Buf_c * K_buf_c) / (cbc * cbc)));
    const T K_buf_sr = T(0.3f), Buf_sr = T(10.0f);
    const T cbs = Ca_SR + K_buf_sr;
    const T Ca_sr_bufsr = T(1.0f) / (T(1.0f) + ((Buf_sr * K_buf_sr) / (cbs * cbs)));
    const T Buf_ss = T(0.4f), K_buf_ss = T(0.00025f);
    const T cbss = Ca_ss + K_buf_ss;
    const T Ca_ss_bufss = T(1.0f) / (T(1.0f) + ((Buf_ss * K_buf_ss) / (cbss * cbss)));
    const T V_sr = T(0.001094f), V_ss = T(5.468e-05f);

    u.dV = -(IK1 + Ito + IKr + IKs + ICaL + INaK + INa + IbNa + INaCa + IbCa + IpK + IpCa + stim);
    u.dRprime = ((-k2) * Ca_ss * R_prime) + (k4 * (T(1.0f) - R_prime));
    u.dCai = Ca_i_bufc * (((((i_leak - i_up) * V_sr) / V_c) + i_xfer) -
                          ((((IbCa + IpCa) - (T(2.0f) * INaCa)) * Cm) / (T(2.0f) * V_c * F)));
    u.dCaSR = Ca_sr_bufsr * (i_up - (Irel + i_leak));
    u.dCaSS = Ca_ss_bufss * (((((-ICaL) * Cm) / (T(2.0f) * V_ss * F)) + ((Irel * V_sr) / V_ss)) -
                             ((i_xfer * V_c) / V_ss));
    u.dNai = ((-(INa + IbNa + (T(3.0f) * INaK) + (T(3.0f) * INaCa))) / (V_c * F)) * Cm;
    u.dKi = ((-((IK1 + Ito + IKr + IKs + IpK + stim) - (T(2.0f) * INaK))) / (V_c * F)) * Cm;

    // Rush-Larsen gate updates
    u.gate[0] = xr1_inf + (Xr1 - xr1_inf) * mexp(-dt / tau_xr1);
    u.gate[1] = xr2_inf + (Xr2 - xr2_inf) * mexp(-dt / tau_xr2);
    u.gate[2] = xs_inf + (Xs - xs_inf) * mexp(-dt / tau_xs);
    u.gate[3] = m_inf + (m - m_inf) * mexp(-dt / tau_m);
    u.gate[4] = h_inf + (h - h_inf) * mexp(-dt / tau_h);
    u.gate[5] = j_inf + (j - j_inf) * mexp(-dt / tau_j);
    u.gate[6] = d_inf + (d - d_inf) * mexp(-dt / tau_d);
    u.gate[7] = f_inf + (f - f_inf) * mexp(-dt / tau_f);
    u.gate[8] = f2_inf + (f2 - f2_inf) * mexp(-dt / tau_f2);
    u.gate[9] = fCass_inf + (fCass - fCass_inf) * mexp(-dt / tau_fCass);
    u.gate[10] = s_inf + (s - s_inf) * mexp(-dt / tau_s);
    u.gate[11] = r_inf + (r - r_inf) * mexp(-dt / tau_r);
}

MB_NS_END
