/* ten Tusscher & Panfilov 2006 epicardial myocyte, Rush-Larsen, FP64 --
 * TEST INFRASTRUCTURE (oracle).  Restates
 * src/models_library/ten_tusscher/ten_tusscher_2006_RS_CPU.c: the default
 * state (:27-45), the per-cell sub-step (:100-134) and RHS_cpu (:137-351).
 * As in the reference, rDY[1..12] returns the already advanced gate values
 * (y_inf + (y - y_inf) exp(-dt/tau), :337-348) and every other entry a time
 * derivative for explicit Euler.  Literals keep the reference's spelling,
 * `f` suffixes included, because the float-rounded constants are part of
 * the model the reference integrates.
 */
#include <math.h>
#include <stddef.h>

#include "oracle.h"

void orc_tt2006_initial_state(double *sv) {
    static const float s0[ORC_TT_NEQ] = {-85.23f,  0.00621f, 0.4712f,   0.0095f, 0.00172f, 0.7444f, 0.7045f,
                                         3.373e-5f, 0.7888f, 0.9755f,   0.9953f, 0.999998f, 2.42e-8f, 0.000126f,
                                         3.64f,    0.00036f, 0.9073f,   8.604f,  136.89f};
    for (int i = 0; i < ORC_TT_NEQ; ++i) sv[i] = (double)s0[i];
}

/* RHS_cpu (ten_tusscher_2006_RS_CPU.c:137-351). */
static void tt2006_rhs(const double *y, double *rDY, double stim, double dt, const double *sc) {
    const double V = y[0];
    const double Xr1 = y[1], Xr2 = y[2], Xs = y[3];
    const double m = y[4], h = y[5], j = y[6];
    const double d = y[7], f = y[8], f2 = y[9], fCass = y[10];
    const double s = y[11], r = y[12];
    const double Ca_i = y[13], Ca_SR = y[14], Ca_ss = y[15];
    const double R_prime = y[16], Na_i = y[17], K_i = y[18];

    // physical constants and cell geometry
    const double R = 8314.472, Tk = 310.0, F = (double)(96485.3415f);
    const double Cm = 0.185, V_c = 0.016404;
    const double Ko = 5.4, Nao = 140.0, Cao = 2.0;
    const double P_kna = 0.03, K_mk = 1.0, P_NaK = 2.724, K_mNa = 40.0, K_pCa = 0.0005;
    // calcium handling
    const double V_rel = 0.102, k1_prime = 0.15, max_sr = 2.5, min_sr = 1.0;
    const double EC = 1.5, Vmax_up = 0.006375;
    // Na/Ca exchanger
    const double n_alpha = 2.5, n_gamma = 0.35, K_sat = 0.1, Km_Ca = 1.38;
    const double Km_Nai = 87.5, K_NaCa = 1000.0;
    // maximal conductances
    const double g_to = 0.294, g_Kr = 0.153 * sc[1], g_Ks = 0.098 * sc[2];
    const double g_CaL = 3.98e-05 * sc[3], g_Na = 14.838 * sc[0], g_pK = 0.0146;
    const double g_bca = 0.000592, g_pCa = 0.1238, g_K1 = 5.405 * sc[4], g_bna = 0.00029;

    const double RTF = (R * Tk) / F;
    const double EK = RTF * log(Ko / K_i);
    const double EKs = RTF * log((Ko + (P_kna * Nao)) / (K_i + (P_kna * Na_i)));
    const double ENa = RTF * log(Nao / Na_i);
    const double ECa = (((double)(0.5f) * R * Tk) / F) * log(Cao / Ca_i);

    // inward rectifier
    const double vek = V - EK;
    const double beta_K1 = (((double)(3.0f) * exp((double)(0.0002f) * (vek + (double)(100.0f)))) + exp((double)(0.1f) * (vek - (double)(10.0f)))) /
                      ((double)(1.0f) + exp((double)(-0.5f) * vek));
    const double alpha_K1 = (double)(0.1f) / ((double)(1.0f) + exp((double)(0.06f) * (vek - (double)(200.0f))));
    const double xK1_inf = alpha_K1 / (alpha_K1 + beta_K1);

    const double IK1 = g_K1 * xK1_inf * vek;
    const double Ito = g_to * r * s * vek;
    const double IKr = g_Kr * Xr1 * Xr2 * vek * sqrt(Ko / (double)(5.4f));
    const double IKs = g_Ks * (Xs * Xs) * (V - EKs);
    const double IpK = (g_pK * vek) / ((double)(1.0f) + exp(((double)(25.0f) - V) / (double)(5.98f)));

    // L-type calcium current; the removable singularity at V = 15 mV uses
    // the limit value inside a +-1e-5 mV band (_RS_CPU.c:221)
        double ICaL;
    const double v15 = V - (double)(15.0f);
    if (V < (double)(15.0f - 1.0e-5f) || V > (double)(15.0f + 1.0e-5f)) {
        const double ea = ((double)(2.0f) * v15 * F) / (R * Tk);
        ICaL = (((g_CaL * d * f * f2 * fCass * (double)(4.0f) * v15 * (F * F)) / (R * Tk)) *
                (((double)(0.25f) * Ca_ss * exp(ea)) - Cao)) / expm1(ea);
    } else {
        ICaL = g_CaL * d * f * f2 * fCass * (double)(2.0f) * F * ((double)(0.25f) * Ca_ss - Cao);
    }
    const double IbCa = g_bca * (V - ECa);
    const double IpCa = (g_pCa * Ca_i) / (Ca_i + K_pCa);

    const double INaK = ((((P_NaK * Ko) / (Ko + K_mk)) * Na_i) / (Na_i + K_mNa)) /
                   ((double)(1.0f) + ((double)(0.1245f) * exp((((double)(-0.1f)) * V * F) / (R * Tk))) +
                    ((double)(0.0353f) * exp(((-V) * F) / (R * Tk))));
    const double INa = g_Na * (m * m * m) * h * j * (V - ENa);
    const double IbNa = g_bna * (V - ENa);
    const double e_gm1 = exp(((n_gamma - (double)(1.0f)) * V * F) / (R * Tk));
    const double INaCa = (K_NaCa * ((exp((n_gamma * V * F) / (R * Tk)) * (Na_i * Na_i * Na_i) * Cao) -
                               (e_gm1 * (Nao * Nao * Nao) * Ca_i * n_alpha))) /
                    (((Km_Nai * Km_Nai * Km_Nai) + (Nao * Nao * Nao)) * (Km_Ca + Cao) *
                     ((double)(1.0f) + (K_sat * e_gm1)));

    // gating variables: steady states and time constants
    const double xr1_inf = (double)(1.0f) / ((double)(1.0f) + exp(((double)(-26.0f) - V) / (double)(7.0f)));
    const double tau_xr1 = ((double)(450.0f) / ((double)(1.0f) + exp(((double)(-45.0f) - V) / (double)(10.0f)))) *
                      ((double)(6.0f) / ((double)(1.0f) + exp((V + (double)(30.0f)) / (double)(11.5f))));
    const double xr2_inf = (double)(1.0f) / ((double)(1.0f) + exp((V + (double)(88.0f)) / (double)(24.0f)));
    const double tau_xr2 = ((double)(3.0f) / ((double)(1.0f) + exp(((double)(-60.0f) - V) / (double)(20.0f)))) *
                      ((double)(1.12f) / ((double)(1.0f) + exp((V - (double)(60.0f)) / (double)(20.0f))));
    const double xs_inf = (double)(1.0f) / ((double)(1.0f) + exp(((double)(-5.0f) - V) / (double)(14.0f)));
    const double tau_xs = (((double)(1400.0f) / sqrt((double)(1.0f) + exp(((double)(5.0f) - V) / (double)(6.0f)))) *
                      ((double)(1.0f) / ((double)(1.0f) + exp((V - (double)(35.0f)) / (double)(15.0f))))) + (double)(80.0f);

    const double em = (double)(1.0f) + exp(((double)(-56.86f) - V) / (double)(9.03f));
    const double m_inf = (double)(1.0f) / (em * em);
    const double tau_m = ((double)(1.0f) / ((double)(1.0f) + exp(((double)(-60.0f) - V) / (double)(5.0f)))) *
                    (((double)(0.1f) / ((double)(1.0f) + exp((V + (double)(35.0f)) / (double)(5.0f)))) +
                     ((double)(0.1f) / ((double)(1.0f) + exp((V - (double)(50.0f)) / (double)(200.0f)))));

    const double eh = (double)(1.0f) + exp((V + (double)(71.55f)) / (double)(7.43f));
    const double h_inf = (double)(1.0f) / (eh * eh);
    const double j_inf = h_inf;
    double alpha_h, beta_h, alpha_j, beta_j;
    if (V < (double)(-40.0f)) {
        alpha_h = (double)(0.057f) * exp((-(V + (double)(80.0f))) / (double)(6.8f));
        beta_h = ((double)(2.7f) * exp((double)(0.079f) * V)) + ((double)(310000.0f) * exp((double)(0.3485f) * V));
        alpha_j = (((((double)(-25428.0f)) * exp((double)(0.2444f) * V)) - ((double)(6.948e-06f) * exp((double)(-0.04391f) * V))) *
                   (V + (double)(37.78f))) / ((double)(1.0f) + exp((double)(0.311f) * (V + (double)(79.23f))));
        beta_j = ((double)(0.02424f) * exp((double)(-0.01052f) * V)) / ((double)(1.0f) + exp((double)(-0.1378f) * (V + (double)(40.14f))));
    } else {
        alpha_h = (double)(0.0f);
        beta_h = (double)(0.77f) / ((double)(0.13f) * ((double)(1.0f) + exp((V + (double)(10.66f)) / (double)(-11.1f))));
        alpha_j = (double)(0.0f);
        beta_j = ((double)(0.6f) * exp((double)(0.057f) * V)) / ((double)(1.0f) + exp((double)(-0.1f) * (V + (double)(32.0f))));
    }
    const double tau_h = (double)(1.0f) / (alpha_h + beta_h);
    const double tau_j = (double)(1.0f) / (alpha_j + beta_j);

    const double d_inf = (double)(1.0f) / ((double)(1.0f) + exp(((double)(-8.0f) - V) / (double)(7.5f)));
    const double tau_d = (((double)(1.4f) / ((double)(1.0f) + exp(((double)(-35.0f) - V) / (double)(13.0f)))) + (double)(0.25f)) *
                        ((double)(1.4f) / ((double)(1.0f) + exp((V + (double)(5.0f)) / (double)(5.0f)))) +
                    ((double)(1.0f) / ((double)(1.0f) + exp(((double)(50.0f) - V) / (double)(20.0f))));

    const double e30 = exp((V + (double)(30.0f)) / (double)(10.0f));
    const double v27 = V + (double)(27.0f);
    const double f_inf = (double)(1.0f) / ((double)(1.0f) + exp((V + (double)(20.0f)) / (double)(7.0f)));
    const double tau_f = ((double)(1102.5f) * exp((-(v27 * v27)) / (double)(225.0f))) +
                    ((double)(200.0f) / ((double)(1.0f) + exp(((double)(13.0f) - V) / (double)(10.0f)))) +
                    ((double)(180.0f) / ((double)(1.0f) + e30)) + (double)(20.0f);
    const double f2_inf = ((double)(0.67f) / ((double)(1.0f) + exp((V + (double)(35.0f)) / (double)(7.0f)))) + (double)(0.33f);
    const double tau_f2 = ((double)(562.0f) * exp((-(v27 * v27)) / (double)(240.0f))) +
                     ((double)(31.0f) / ((double)(1.0f) + exp(((double)(25.0f) - V) / (double)(10.0f)))) +
                     ((double)(80.0f) / ((double)(1.0f) + e30));

    const double cr = Ca_ss / (double)(0.05f);
    const double fCass_inf = ((double)(0.6f) / ((double)(1.0f) + cr * cr)) + (double)(0.4f);
    const double tau_fCass = ((double)(80.0f) / ((double)(1.0f) + cr * cr)) + (double)(2.0f);

    const double s_inf = (double)(1.0f) / ((double)(1.0f) + exp((V + (double)(20.0f)) / (double)(5.0f)));
    const double v45 = V + (double)(45.0f);
    const double tau_s = ((double)(85.0f) * exp((-(v45 * v45)) / (double)(320.0f))) +
                    ((double)(5.0f) / ((double)(1.0f) + exp((V - (double)(20.0f)) / (double)(5.0f)))) + (double)(3.0f);
    const double r_inf = (double)(1.0f) / ((double)(1.0f) + exp(((double)(20.0f) - V) / (double)(6.0f)));
    const double v40 = V + (double)(40.0f);
    const double tau_r = ((double)(9.5f) * exp((-(v40 * v40)) / (double)(1800.0f))) + (double)(0.8f);

    // calcium dynamics
    const double ecs = EC / Ca_SR;
    const double kcasr = max_sr - ((max_sr - min_sr) / ((double)(1.0f) + ecs * ecs));
    const double k1 = k1_prime / kcasr;
    const double k3 = 0.06;
    const double css2 = Ca_ss * Ca_ss;
    const double O = (k1 * css2 * R_prime) / (k3 + (k1 * css2));
    const double Irel = V_rel * O * (Ca_SR - Ca_ss);
    const double K_up = 0.00025;
    const double i_up = Vmax_up / ((double)(1.0f) + ((K_up * K_up) / (Ca_i * Ca_i)));
    const double i_leak = (double)(0.00036f) * (Ca_SR - Ca_i);
    const double i_xfer = (double)(0.0038f) * (Ca_ss - Ca_i);
    const double k2 = (double)(0.045f) * kcasr;
    const double k4 = (double)(0.005f);
    const double Buf_c = (double)(0.2f), K_buf_c = (double)(0.001f);
    const double cbc = Ca_i + K_buf_c;
    const double Ca_i_bufc = (double)(1.0f) / ((double)(1.0f) + ((Buf_c * K_buf_c) / (cbc * cbc)));
    const double K_buf_sr = (double)(0.3f), Buf_sr = (double)(10.0f);
    const double cbs = Ca_SR + K_buf_sr;
    const double Ca_sr_bufsr = (double)(1.0f) / ((double)(1.0f) + ((Buf_sr * K_buf_sr) / (cbs * cbs)));
    const double Buf_ss = (double)(0.4f), K_buf_ss = (double)(0.00025f);
    const double cbss = Ca_ss + K_buf_ss;
    const double Ca_ss_bufss = (double)(1.0f) / ((double)(1.0f) + ((Buf_ss * K_buf_ss) / (cbss * cbss)));
    const double V_sr = (double)(0.001094f), V_ss = (double)(5.468e-05f);

    rDY[0] = -(IK1 + Ito + IKr + IKs + ICaL + INaK + INa + IbNa + INaCa + IbCa + IpK + IpCa + stim);
    rDY[16] = ((-k2) * Ca_ss * R_prime) + (k4 * ((double)(1.0f) - R_prime));
    rDY[13] = Ca_i_bufc * (((((i_leak - i_up) * V_sr) / V_c) + i_xfer) -
                          ((((IbCa + IpCa) - ((double)(2.0f) * INaCa)) * Cm) / ((double)(2.0f) * V_c * F)));
    rDY[14] = Ca_sr_bufsr * (i_up - (Irel + i_leak));
    rDY[15] = Ca_ss_bufss * (((((-ICaL) * Cm) / ((double)(2.0f) * V_ss * F)) + ((Irel * V_sr) / V_ss)) -
                             ((i_xfer * V_c) / V_ss));
    rDY[17] = ((-(INa + IbNa + ((double)(3.0f) * INaK) + ((double)(3.0f) * INaCa))) / (V_c * F)) * Cm;
    rDY[18] = ((-((IK1 + Ito + IKr + IKs + IpK + stim) - ((double)(2.0f) * INaK))) / (V_c * F)) * Cm;

    // Rush-Larsen gate updates
    rDY[1] = xr1_inf + (Xr1 - xr1_inf) * exp(-dt / tau_xr1);
    rDY[2] = xr2_inf + (Xr2 - xr2_inf) * exp(-dt / tau_xr2);
    rDY[3] = xs_inf + (Xs - xs_inf) * exp(-dt / tau_xs);
    rDY[4] = m_inf + (m - m_inf) * exp(-dt / tau_m);
    rDY[5] = h_inf + (h - h_inf) * exp(-dt / tau_h);
    rDY[6] = j_inf + (j - j_inf) * exp(-dt / tau_j);
    rDY[7] = d_inf + (d - d_inf) * exp(-dt / tau_d);
    rDY[8] = f_inf + (f - f_inf) * exp(-dt / tau_f);
    rDY[9] = f2_inf + (f2 - f2_inf) * exp(-dt / tau_f2);
    rDY[10] = fCass_inf + (fCass - fCass_inf) * exp(-dt / tau_fCass);
    rDY[11] = s_inf + (s - s_inf) * exp(-dt / tau_s);
    rDY[12] = r_inf + (r - r_inf) * exp(-dt / tau_r);
}

/* solve_model_ode_cpu (ten_tusscher_2006_RS_CPU.c:100-134). */
void orc_tt2006_step(double *sv, double stim, double dt, const double *scale) {
    static const double one[5] = {1.0, 1.0, 1.0, 1.0, 1.0};
    double rY[ORC_TT_NEQ], rDY[ORC_TT_NEQ];
    for (int i = 0; i < ORC_TT_NEQ; ++i) rY[i] = sv[i];
    tt2006_rhs(rY, rDY, stim, dt, scale ? scale : one);
    sv[0] = dt * rDY[0] + rY[0];
    for (int i = 1; i <= 12; ++i) sv[i] = rDY[i];
    for (int i = 13; i < ORC_TT_NEQ; ++i) sv[i] = dt * rDY[i] + rY[i];
}
