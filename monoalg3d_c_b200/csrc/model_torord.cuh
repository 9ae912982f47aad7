// ToRORd-fkatp human ventricular model (Tomek et al. 2019) with endo/mid/epi
// cell types, as the reference's Rush-Larsen library evaluates it
// (src/models_library/ToROrd/ToRORd_fkatp_mixed_endo_mid_epi_RL.common.c:1-754,
//  driver ToRORd_fkatp_mixed_endo_mid_epi.c:252-310).
//
// Each evaluation yields dy/dt for the 17 explicitly-integrated states
// (0-9, 32-38) and the linearisation dy/dt = a*y + b for the 26 gates
// (10-31, 39-42), a = -1/tau, b = y_inf/tau.  The gate update is
//     y <- exp(a dt) (y + b/a) - b/a           (Rush-Larsen)
//     y <- y + dt (a y + b)                    (when |a| is "small")
// where "small" follows the reference macro (ToRORd_fkatp_mixed_endo_mid_epi.h:20):
// MB_RL_REFERENCE_CPU reproduces the CPU build, in which abs() of a double
// truncates to int, so |a| < 1 takes the Euler form; MB_RL_TRUE uses the
// written threshold |a| < 1e-8.
//
// Model features reproduced as the reference has them: the IClb multiplier is
// 1 (the reference CPU driver leaves it uninitialised), INaK has no MID
// scaling (the reference tests celltype == 2 after testing EPI == 2), and
// I_katp is identically zero (fkatp = 0).
#pragma once
#include "mb_math.cuh"

MB_NS_BEGIN

constexpr int TOR_NEQ = 43;
constexpr int TOR_N64 = 9;    // mixed form: V and the 8 ion concentrations in FP64
constexpr int TOR_N32 = 34;   // mixed form: everything else in FP32

// Mixed-form row of state s: rows64 = {V, cass, nai, nass, ki, kss, cansr,
// cajsr, cai}; rows32 = {CaMKt, states 10..42}.
__host__ __device__ inline int tor_mixed_row(int s, bool &is64) {
    if (s == 0) { is64 = true; return 0; }
    if (s >= 2 && s <= 9) { is64 = true; return s - 1; }
    is64 = false;
    if (s == 1) return 0;
    return s - 9;
}

template <typename T>
struct TorScale { T INa, IKr, IKs, ICaL, IK1; };

template <typename T>
__device__ __forceinline__ void load_tor_scale(const float *scale, size_t ld, uint32_t t, TorScale<T> &sc) {
    if (scale) {
        sc.INa = T(scale[0 * ld + t]);
        sc.IKr = T(scale[1 * ld + t]);
        sc.IKs = T(scale[2 * ld + t]);
        sc.ICaL = T(scale[3 * ld + t]);
        sc.IK1 = T(scale[4 * ld + t]);
    } else {
        sc.INa = sc.IKr = sc.IKs = sc.ICaL = sc.IK1 = T(1);
    }
}

// 1.82e6 * (74 * 310)^-1.5, the Davies-equation constant of the driving-force
// activity coefficients, evaluated once in double precision.
#define MB_TOR_CONSTA 0x1.0c3201d875e3fp-1  /* 0.52381902472820474 */

template <typename T>
struct TorRhs {
    T d[TOR_NEQ];   // dy/dt of the Euler states (other entries unused)
    T a[TOR_NEQ];   // RL linearisation (gates)
    T b[TOR_NEQ];
};

template <typename T>
__device__ __forceinline__ T sq(T x) { return x * x; }

// x / (exp(x) - 1), with its limit 1 - x/2 near x = 0.  The GHK fluxes
// divide by exp(z V F/RT) - 1, which vanishes at V = 0; in single precision
// exp(x) rounds to 1 once |V| is below a few microvolts and the quotient
// becomes 0/0, which a travelling wave crossing 0 mV in a million cells meets
// about once per beat.  The single-precision form therefore evaluates the
// flux through this function (the plain FP64 form keeps the reference's
// expression, whose singularity double precision does not reach).
__device__ __forceinline__ float ghk_b(float x) {
    if (fabsf(x) < 1e-4f) return 1.0f - 0.5f * x;
    return x / mexpm1(x);
}

// Activity-coefficient factor exp(-A z^2 (sqrt(I)/(1+sqrt(I)) - 0.3 I)).
template <typename T>
__device__ __forceinline__ T davies(T z2, T I) {
    const T s = msqrt(I);
    return mexp(-T(MB_TOR_CONSTA) * z2 * (s / (T(1) + s) - T(0.3) * I));
}

// Na/Ca exchanger flux for one compartment (RL.common.c:364-451).
template <typename T>
__device__ __forceinline__ T torord_ncx(T na, T ca, T hna, T hca, T nao, T cao, T &allo_out) {
    const T kna1 = T(15.0), kna2 = T(5.0), kna3 = T(88.12), kasymm = T(12.5);
    const T wna = T(6.0e4), wca = T(6.0e4), wnaca = T(5.0e3);
    const T kcaon = T(1.5e6), kcaoff = T(5.0e3);
    const T zna = T(1.0), zca = T(2.0);
    const T h1 = T(1) + na / kna3 * (T(1) + hna);
    const T h2 = (na * hna) / (kna3 * h1);
    const T h3 = T(1.0) / h1;
    const T h4 = T(1.0) + na / kna1 * (T(1) + na / kna2);
    const T h5 = na * na / (h4 * kna1 * kna2);
    const T h6 = T(1.0) / h4;
    const T h7 = T(1.0) + nao / kna3 * (T(1.0) + T(1.0) / hna);
    const T h8 = nao / (kna3 * hna * h7);
    const T h9 = T(1.0) / h7;
    const T h10 = kasymm + T(1.0) + nao / kna1 * (T(1.0) + nao / kna2);
    const T h11 = nao * nao / (h10 * kna1 * kna2);
    const T h12 = T(1.0) / h10;
    const T k1 = h12 * cao * kcaon;
    const T k2 = kcaoff;
    const T k3p = h9 * wca;
    const T k3pp = h8 * wnaca;
    const T k3 = k3p + k3pp;
    const T k4p = h3 * wca / hca;
    const T k4pp = h2 * wnaca;
    const T k4 = k4p + k4pp;
    const T k5 = kcaoff;
    const T k6 = h6 * ca * kcaon;
    const T k7 = h5 * h2 * wna;
    const T k8 = h8 * h11 * wna;
    const T x1 = k2 * k4 * (k7 + k6) + k5 * k7 * (k2 + k3);
    const T x2 = k1 * k7 * (k4 + k5) + k4 * k6 * (k1 + k8);
    const T x3 = k1 * k3 * (k7 + k6) + k8 * k6 * (k2 + k3);
    const T x4 = k2 * k8 * (k4 + k5) + k3 * k5 * (k1 + k8);
    const T xs = x1 + x2 + x3 + x4;
    const T E1 = x1 / xs, E2 = x2 / xs, E3 = x3 / xs, E4 = x4 / xs;
    const T KmCaAct = T(150.0e-6);
    allo_out = T(1.0) / (T(1.0) + sq(KmCaAct / ca));
    const T JncxNa = T(3.0) * (E4 * k7 - E1 * k8) + E3 * k4pp - E2 * k3pp;
    const T JncxCa = E2 * k2 - E1 * k1;
    return zna * JncxNa + zca * JncxCa;
}

// y: all 43 states; celltype 0 endo, 1 mid, 2 epi.
template <typename T>
__device__ __forceinline__ void torord_rhs(const T *y, T stim, T celltype, const TorScale<T> &sc,
                                           TorRhs<T> &o) {
    const T v = y[0], CaMKt = y[1], cass = y[2], nai = y[3], nass = y[4], ki = y[5], kss = y[6];
    const T cansr = y[7], cajsr = y[8], cai = y[9];
    const T m = y[10], h = y[11], j = y[12], hp = y[13], jp = y[14], mL = y[15], hL = y[16];
    const T hLp = y[17], a = y[18], iF = y[19], iS = y[20], ap = y[21], iFp = y[22], iSp = y[23];
    const T d = y[24], ff = y[25], fs = y[26], fcaf = y[27], fcas = y[28], jca = y[29];
    const T ffp = y[30], fcafp = y[31], nca = y[32], nca_i = y[33];
    const T c0 = y[34], c1 = y[35], c2 = y[36], I = y[37], o_ = y[38];
    const T xs1 = y[39], xs2 = y[40], Jrel_np = y[41], Jrel_p = y[42];

    const bool EPI = celltype == T(2.0);
    const bool MID = celltype == T(1.0);

    const T nao = T(140.0), cao = T(1.8), ko = T(5.0);
    const T ICaL_fractionSS = T(0.8), INaCa_fractionSS = T(0.35);
    const T R = T(8314.0), Tk = T(310.0), F = T(96485.0);

    // cell geometry
    const T L = T(0.01), rad = T(0.0011);
    const T vcell = T(1000) * T(3.14) * rad * rad * L;
    const T Ageo = T(2) * T(3.14) * rad * rad + T(2) * T(3.14) * rad * L;
    const T Acap = T(2) * Ageo;
    const T vmyo = T(0.68) * vcell, vnsr = T(0.0552) * vcell, vjsr = T(0.0048) * vcell;
    const T vss = T(0.02) * vcell;
    const T cli = T(24), clo = T(150);

    // CaMK
    const T KmCaMK = T(0.15), aCaMK = T(0.05), bCaMK = T(0.00068), CaMKo = T(0.05), KmCaM = T(0.0015);
    const T CaMKb = CaMKo * (T(1.0) - CaMKt) / (T(1.0) + KmCaM / cass);
    const T CaMKa = CaMKb + CaMKt;
    o.d[1] = aCaMK * CaMKb * (CaMKb + CaMKt) - bCaMK * CaMKt;

    const T RTF = R * Tk / F;
    const T ENa = RTF * mlog(nao / nai);
    const T EK = RTF * mlog(ko / ki);
    const T PKNa = T(0.01833);
    const T EKs = RTF * mlog((ko + PKNa * nao) / (ki + PKNa * nai));

    const T vffrt = v * F * F / (R * Tk);
    const T vfrt = v * F / (R * Tk);
    const T fCaMKp = T(1.0) / (T(1.0) + KmCaMK / CaMKa);   // fINap = fINaLp = fItop = fICaLp = fJrelp = fJupp

    // INa (Grandi formulation with CaMK phosphorylation)
    const T mss = T(1) / sq(T(1) + mexp(-(T(56.86) + v) / T(9.03)));
    const T tm = T(0.1292) * mexp(-sq((v + T(45.79)) / T(15.54))) + T(0.06487) * mexp(-sq((v - T(4.823)) / T(51.12)));
    T ah, bh, aj, bj;
    if (v >= T(-40)) {
        ah = T(0);
        bh = T(0.77) / (T(0.13) * (T(1) + mexp(-(v + T(10.66)) / T(11.1))));
        aj = T(0);
        bj = (T(0.6) * mexp(T(0.057) * v)) / (T(1) + mexp(T(-0.1) * (v + T(32))));
    } else {
        ah = T(0.057) * mexp(-(v + T(80)) / T(6.8));
        bh = T(2.7) * mexp(T(0.079) * v) + T(3.1) * T(100000.0) * mexp(T(0.3485) * v);
        aj = ((T(-2.5428) * T(10000.0) * mexp(T(0.2444) * v) - T(6.948) * T(1.0e-6) * mexp(T(-0.04391) * v)) *
              (v + T(37.78))) / (T(1) + mexp(T(0.311) * (v + T(79.23))));
        bj = (T(0.02424) * mexp(T(-0.01052) * v)) / (T(1) + mexp(T(-0.1378) * (v + T(40.14))));
    }
    const T tauh = T(1) / (ah + bh);
    const T hss = T(1) / sq(T(1) + mexp((v + T(71.55)) / T(7.43)));
    const T tauj = T(1) / (aj + bj);
    const T jss = hss;
    const T hssp = T(1) / sq(T(1) + mexp((v + T(71.55) + T(6)) / T(7.43)));
    const T taujp = T(1.46) * tauj;
    const T GNa = T(11.7802);
    const T INa = sc.INa * GNa * (v - ENa) * (m * m * m) * ((T(1.0) - fCaMKp) * h * j + fCaMKp * hp * jp);

    // INaL
    const T mLss = T(1.0) / (T(1.0) + mexp((-(v + T(42.85))) / T(5.264)));
    const T tmL = tm;
    const T hLss = T(1.0) / (T(1.0) + mexp((v + T(87.61)) / T(7.488)));
    const T thL = T(200.0);
    const T hLssp = T(1.0) / (T(1.0) + mexp((v + T(93.81)) / T(7.488)));
    const T thLp = T(3.0) * thL;
    T GNaL = T(0.0279);
    if (EPI) GNaL = GNaL * T(0.6);
    const T INaL = GNaL * (v - ENa) * mL * ((T(1.0) - fCaMKp) * hL + fCaMKp * hLp);

    // Ito
    const T ass = T(1.0) / (T(1.0) + mexp((-(v - T(14.34))) / T(14.82)));
    const T ta = T(1.0515) / (T(1.0) / (T(1.2089) * (T(1.0) + mexp(-(v - T(18.4099)) / T(29.3814)))) +
                              T(3.5) / (T(1.0) + mexp((v + T(100.0)) / T(29.3814))));
    const T iss = T(1.0) / (T(1.0) + mexp((v + T(43.94)) / T(5.711)));
    const T delta_epi = EPI ? T(1.0) - (T(0.95) / (T(1.0) + mexp((v + T(70.0)) / T(5.0)))) : T(1.0);
    T tiF = T(4.562) + T(1) / (T(0.3933) * mexp((-(v + T(100.0))) / T(100.0)) + T(0.08004) * mexp((v + T(50.0)) / T(16.59)));
    T tiS = T(23.62) + T(1) / (T(0.001416) * mexp((-(v + T(96.52))) / T(59.05)) + T(1.780e-8) * mexp((v + T(114.1)) / T(8.079)));
    tiF = tiF * delta_epi;
    tiS = tiS * delta_epi;
    const T AiF = T(1.0) / (T(1.0) + mexp((v - T(213.6)) / T(151.2)));
    const T AiS = T(1.0) - AiF;
    const T ii = AiF * iF + AiS * iS;
    const T assp = T(1.0) / (T(1.0) + mexp((-(v - T(24.34))) / T(14.82)));
    const T dti_develop = T(1.354) + T(1.0e-4) / (mexp((v - T(167.4)) / T(15.89)) + mexp(-(v - T(12.23)) / T(0.2154)));
    const T dti_recover = T(1.0) - T(0.5) / (T(1.0) + mexp((v + T(70.0)) / T(20.0)));
    const T tiFp = dti_develop * dti_recover * tiF;
    const T tiSp = dti_develop * dti_recover * tiS;
    const T ip = AiF * iFp + AiS * iSp;
    T Gto = T(0.16);
    if (EPI || MID) Gto = Gto * T(2.0);
    const T Ito = Gto * (v - EK) * ((T(1.0) - fCaMKp) * a * ii + fCaMKp * ap * ip);

    // ICaL, ICaNa, ICaK
    T dss = T(1.0763) * mexp(T(-1.0070) * mexp(T(-0.0829) * (v)));
    if (v > T(31.4978)) dss = T(1);
    const T td = T(0.6) + T(1.0) / (mexp(T(-0.05) * (v + T(6.0))) + mexp(T(0.09) * (v + T(14.0))));
    const T fss = T(1.0) / (T(1.0) + mexp((v + T(19.58)) / T(3.696)));
    const T tff = T(7.0) + T(1.0) / (T(0.0045) * mexp(-(v + T(20.0)) / T(10.0)) + T(0.0045) * mexp((v + T(20.0)) / T(10.0)));
    const T tfs = T(1000.0) + T(1.0) / (T(0.000035) * mexp(-(v + T(5.0)) / T(4.0)) + T(0.000035) * mexp((v + T(5.0)) / T(6.0)));
    const T Aff = T(0.6);
    const T Afs = T(1.0) - Aff;
    const T f = Aff * ff + Afs * fs;
    const T fcass = fss;
    const T tfcaf = T(7.0) + T(1.0) / (T(0.04) * mexp(-(v - T(4.0)) / T(7.0)) + T(0.04) * mexp((v - T(4.0)) / T(7.0)));
    const T tfcas = T(100.0) + T(1.0) / (T(0.00012) * mexp(-v / T(3.0)) + T(0.00012) * mexp(v / T(7.0)));
    const T Afcaf = T(0.3) + T(0.6) / (T(1.0) + mexp((v - T(10.0)) / T(10.0)));
    const T Afcas = T(1.0) - Afcaf;
    const T fca = Afcaf * fcaf + Afcas * fcas;
    const T tjca = T(75);
    const T jcass = T(1.0) / (T(1.0) + mexp((v + T(18.08)) / (T(2.7916))));
    const T tffp = T(2.5) * tff;
    const T fp = Aff * ffp + Afs * fs;
    const T tfcafp = T(2.5) * tfcaf;
    const T fcap = Afcaf * fcafp + Afcas * fcas;

    const T Kmn = T(0.002), k2n = T(500.0);
    const T km2n = jca * T(1);
    const T anca = T(1.0) / (k2n / km2n + sq(sq(T(1.0) + Kmn / cass)));
    o.d[32] = anca * k2n - nca * km2n;
    const T anca_i = T(1.0) / (k2n / km2n + sq(sq(T(1.0) + Kmn / cai)));
    o.d[33] = anca_i * k2n - nca_i * km2n;

    // driving forces with Davies activity coefficients
    const T Io = T(0.5) * (nao + ko + clo + T(4) * cao) / T(1000);
    T Ii = T(0.5) * (nass + kss + cli + T(4) * cass) / T(1000);
    T gamma_cai = davies(T(4), Ii);
    const T gamma_cao = davies(T(4), Io);
    T gamma_nai = davies(T(1), Ii);
    const T gamma_nao = davies(T(1), Io);
    T gamma_ki = davies(T(1), Ii);
    const T gamma_kao = gamma_nao;
    const T e2 = mexp(T(2.0) * vfrt);
    const T e1 = mexp(T(1.0) * vfrt);
    // q1 = vffrt / (e1 - 1), q2 = vffrt / (e2 - 1); used by the FP32 form only
    T q1 = T(0), q2 = T(0);
    if constexpr (sizeof(T) == 4) {
        q1 = F * ghk_b(vfrt);
        q2 = T(0.5) * F * ghk_b(T(2.0) * vfrt);
    }
    // z2x * vffrt * num / (e - 1), the reference's form in FP64
#define MB_GHK(z2x, num, e, q) (sizeof(T) == 8 ? (z2x) * vffrt * (num) / ((e) - T(1.0)) : (z2x) * (q) * (num))
    const T PhiCaL_ss = MB_GHK(T(4.0), gamma_cai * cass * e2 - gamma_cao * cao, e2, q2);
    const T PhiCaNa_ss = MB_GHK(T(1.0), gamma_nai * nass * e1 - gamma_nao * nao, e1, q1);
    const T PhiCaK_ss = MB_GHK(T(1.0), gamma_ki * kss * e1 - gamma_kao * ko, e1, q1);
    Ii = T(0.5) * (nai + ki + cli + T(4) * cai) / T(1000);
    gamma_cai = davies(T(4), Ii);
    gamma_nai = davies(T(1), Ii);
    gamma_ki = davies(T(1), Ii);
    const T PhiCaL_i = MB_GHK(T(4.0), gamma_cai * cai * e2 - gamma_cao * cao, e2, q2);
    const T PhiCaNa_i = MB_GHK(T(1.0), gamma_nai * nai * e1 - gamma_nao * nao, e1, q1);
    const T PhiCaK_i = MB_GHK(T(1.0), gamma_ki * ki * e1 - gamma_kao * ko, e1, q1);

    T PCa = T(8.3757e-05) * sc.ICaL;
    if (EPI) PCa = PCa * T(1.2);
    else if (MID) PCa = PCa * T(2);
    const T PCap = T(1.1) * PCa;
    const T PCaNa = T(0.00125) * PCa, PCaK = T(3.574e-4) * PCa;
    const T PCaNap = T(0.00125) * PCap, PCaKp = T(3.574e-4) * PCap;
    const T one_m = T(1.0) - fCaMKp;
    const T gss = f * (T(1.0) - nca) + jca * fca * nca;
    const T gssp = fp * (T(1.0) - nca) + jca * fcap * nca;
    const T gi = f * (T(1.0) - nca_i) + jca * fca * nca_i;
    const T gip = fp * (T(1.0) - nca_i) + jca * fcap * nca_i;
    T ICaL_ss = one_m * PCa * PhiCaL_ss * d * gss + fCaMKp * PCap * PhiCaL_ss * d * gssp;
    T ICaNa_ss = one_m * PCaNa * PhiCaNa_ss * d * gss + fCaMKp * PCaNap * PhiCaNa_ss * d * gssp;
    T ICaK_ss = one_m * PCaK * PhiCaK_ss * d * gss + fCaMKp * PCaKp * PhiCaK_ss * d * gssp;
    T ICaL_i = one_m * PCa * PhiCaL_i * d * gi + fCaMKp * PCap * PhiCaL_i * d * gip;
    T ICaNa_i = one_m * PCaNa * PhiCaNa_i * d * gi + fCaMKp * PCaNap * PhiCaNa_i * d * gip;
    T ICaK_i = one_m * PCaK * PhiCaK_i * d * gi + fCaMKp * PCaKp * PhiCaK_i * d * gip;
    const T fi = T(1) - ICaL_fractionSS;
    ICaL_i = ICaL_i * fi;
    ICaNa_i = ICaNa_i * fi;
    ICaK_i = ICaK_i * fi;
    ICaL_ss = ICaL_ss * ICaL_fractionSS;
    ICaNa_ss = ICaNa_ss * ICaL_fractionSS;
    ICaK_ss = ICaK_ss * ICaL_fractionSS;
    const T ICaL = ICaL_ss + ICaL_i;
    const T ICaNa = ICaNa_ss + ICaNa_i;
    const T ICaK = ICaK_ss + ICaK_i;

    // IKr, Lu-Vandenberg Markov model
    const T alpha = T(0.1161) * mexp(T(0.2990) * vfrt);
    const T beta = T(0.2442) * mexp(T(-1.604) * vfrt);
    const T alpha1 = T(1.25) * T(0.1235);
    const T beta1 = T(0.1911);
    const T alpha2 = T(0.0578) * mexp(T(0.9710) * vfrt);
    const T beta2 = T(0.349e-3) * mexp(T(-1.062) * vfrt);
    const T alphai = T(0.2533) * mexp(T(0.5953) * vfrt);
    const T betai = T(1.25) * T(0.0522) * mexp(T(-0.8209) * vfrt);
    const T alphac2ToI = T(0.52e-4) * mexp(T(1.525) * vfrt);
    const T betaItoC2 = (beta2 * betai * alphac2ToI) / (alpha2 * alphai);
    o.d[34] = c1 * beta - c0 * alpha;
    o.d[35] = c0 * alpha + c2 * beta1 - c1 * (beta + alpha1);
    o.d[36] = c1 * alpha1 + o_ * beta2 + I * betaItoC2 - c2 * (beta1 + alpha2 + alphac2ToI);
    o.d[38] = c2 * alpha2 + I * betai - o_ * (beta2 + alphai);
    o.d[37] = c2 * alphac2ToI + o_ * alphai - I * (betaItoC2 + betai);
    T GKr = T(0.0321) * msqrt(ko / T(5)) * sc.IKr;
    if (EPI) GKr = GKr * T(1.3);
    else if (MID) GKr = GKr * T(0.8);
    const T IKr = GKr * o_ * (v - EK);

    // IKs
    const T xs1ss = T(1.0) / (T(1.0) + mexp((-(v + T(11.60))) / T(8.932)));
    const T txs1 = T(817.3) + T(1.0) / (T(2.326e-4) * mexp((v + T(48.28)) / T(17.80)) +
                                       T(0.001292) * mexp((-(v + T(210.0))) / T(230.0)));
    const T xs2ss = xs1ss;
    const T txs2 = T(1.0) / (T(0.01) * mexp((v - T(50.0)) / T(20.0)) + T(0.0193) * mexp((-(v + T(66.54))) / T(31.0)));
    const T KsCa = T(1.0) + T(0.6) / (T(1.0) + mpow((T(3.8e-5) / cai), T(1.4)));
    T GKs = T(0.0011) * sc.IKs;
    if (EPI) GKs = GKs * T(1.4);
    const T IKs = GKs * KsCa * xs1 * xs2 * (v - EKs);

    // IK1
    const T vek = v - EK;
    const T aK1 = T(4.094) / (T(1) + mexp(T(0.1217) * (vek - T(49.934))));
    const T bK1 = (T(15.72) * mexp(T(0.0674) * (vek - T(3.257))) + mexp(T(0.0618) * (vek - T(594.31)))) /
                  (T(1) + mexp(T(-0.1629) * (vek + T(14.207))));
    const T K1ss = aK1 / (aK1 + bK1);
    T GK1 = sc.IK1 * T(0.6992);
    if (EPI) GK1 = GK1 * T(1.2);
    else if (MID) GK1 = GK1 * T(1.3);
    const T IK1 = GK1 * msqrt(ko / T(5)) * K1ss * vek;

    // INaCa (myoplasm and junctional subspace)
    const T qna = T(0.5224), qca = T(0.1670);
    const T hca = mexp((qca * v * F) / (R * Tk));
    const T hna = mexp((qna * v * F) / (R * Tk));
    T Gncx = T(0.0034);
    if (EPI) Gncx = Gncx * T(1.1);
    else if (MID) Gncx = Gncx * T(1.4);
    T allo_i, allo_ss;
    const T jn_i = torord_ncx(nai, cai, hna, hca, nao, cao, allo_i);
    const T INaCa_i = (T(1) - INaCa_fractionSS) * Gncx * allo_i * jn_i;
    const T jn_ss = torord_ncx(nass, cass, hna, hca, nao, cao, allo_ss);
    const T INaCa_ss = INaCa_fractionSS * Gncx * allo_ss * jn_ss;

    // INaK
    const T k1p = T(949.5), k1m = T(182.4), k2p = T(687.2), k2m = T(39.4);
    const T k3p = T(1899.0), k3m = T(79300.0), k4p = T(639.0), k4m = T(40.0);
    const T Knai0 = T(9.073), Knao0 = T(27.78), delta = T(-0.1550);
    const T Knai = Knai0 * mexp((delta * v * F) / (T(3.0) * R * Tk));
    const T Knao = Knao0 * mexp(((T(1.0) - delta) * v * F) / (T(3.0) * R * Tk));
    const T Kki = T(0.5), Kko = T(0.3582), MgADP = T(0.05), MgATP = T(9.8), Kmgatp = T(1.698e-7);
    const T H = T(1.0e-7), eP = T(4.2), Khp = T(1.698e-7), Knap = T(224.0), Kxkur = T(292.0);
    const T P = eP / (T(1.0) + H / Khp + nai / Knap + ki / Kxkur);
    const T nk3 = (T(1.0) + nai / Knai) * (T(1.0) + nai / Knai) * (T(1.0) + nai / Knai);
    const T kk2 = sq(T(1.0) + ki / Kki);
    const T no3 = (T(1.0) + nao / Knao) * (T(1.0) + nao / Knao) * (T(1.0) + nao / Knao);
    const T ko2 = sq(T(1.0) + ko / Kko);
    const T rn = nai / Knai, rno = nao / Knao;
    const T a1 = (k1p * (rn * rn * rn)) / (nk3 + kk2 - T(1.0));
    const T b1 = k1m * MgADP;
    const T a2 = k2p;
    const T b2 = (k2m * (rno * rno * rno)) / (no3 + ko2 - T(1.0));
    const T a3 = (k3p * sq(ko / Kko)) / (no3 + ko2 - T(1.0));
    const T b3 = (k3m * P * H) / (T(1.0) + MgATP / Kmgatp);
    const T a4 = (k4p * MgATP / Kmgatp) / (T(1.0) + MgATP / Kmgatp);
    const T b4 = (k4m * sq(ki / Kki)) / (nk3 + kk2 - T(1.0));
    const T x1 = a4 * a1 * a2 + b2 * b4 * b3 + a2 * b4 * b3 + b3 * a1 * a2;
    const T x2 = b2 * b1 * b4 + a1 * a2 * a3 + a3 * b1 * b4 + a2 * a3 * b4;
    const T x3 = a2 * a3 * a4 + b3 * b2 * b1 + b2 * b1 * a4 + a3 * a4 * b1;
    const T x4 = b4 * b3 * b2 + a3 * a4 * a1 + b2 * a4 * a1 + b3 * b2 * a1;
    const T xs = x1 + x2 + x3 + x4;
    const T E1 = x1 / xs, E2 = x2 / xs, E3 = x3 / xs, E4 = x4 / xs;
    const T JnakNa = T(3.0) * (E1 * a3 - E2 * b3);
    const T JnakK = T(2.0) * (E4 * b1 - E3 * a1);
    T Pnak = T(15.4509);
    if (EPI) Pnak = Pnak * T(0.9);
    const T INaK = Pnak * (T(1.0) * JnakNa + T(1.0) * JnakK);

    // background currents
    const T xkb = T(1.0) / (T(1.0) + mexp(-(v - T(10.8968)) / (T(23.9871))));
    T GKb = T(0.0189);
    if (EPI) GKb = GKb * T(0.6);
    const T IKb = GKb * xkb * (v - EK);
    const T PNab = T(1.9239e-09);
    const T INab = sizeof(T) == 8 ? PNab * vffrt * (nai * e1 - nao) / (e1 - T(1.0)) : PNab * q1 * (nai * e1 - nao);
    const T PCab = T(5.9194e-08);
    const T ICab = sizeof(T) == 8 ? PCab * T(4.0) * vffrt * (gamma_cai * cai * e2 - gamma_cao * cao) / (e2 - T(1.0))
                                  : PCab * T(4.0) * q2 * (gamma_cai * cai * e2 - gamma_cao * cao);
#undef MB_GHK
    const T GpCa = T(5e-04);
    const T IpCa = GpCa * cai / (T(0.0005) + cai);

    // chloride
    const T ECl = RTF * mlog(cli / clo);
    const T GClCa = T(0.2843), GClB = T(1.98e-3), KdClCa = T(0.1);
    const T I_ClCa = T(1) * GClCa / (T(1) + KdClCa / cass) * (v - ECl);
    const T I_Clbk = GClB * (v - ECl);

    // SR release
    const T jsrMidpoint = T(1.7), bt = T(4.75);
    const T a_rel = T(0.5) * bt;
    const T jr = jsrMidpoint / cajsr;
    const T jr8 = sq(sq(sq(jr)));
    T Jrel_inf = a_rel * (-ICaL) / (T(1.0) + jr8);
    if (MID) Jrel_inf = Jrel_inf * T(1.7);
    T tau_rel = bt / (T(1.0) + T(0.0123) / cajsr);
    if (tau_rel < T(0.001)) tau_rel = T(0.001);
    const T btp = T(1.25) * bt;
    const T a_relp = T(0.5) * btp;
    T Jrel_infp = a_relp * (-ICaL) / (T(1.0) + jr8);
    if (MID) Jrel_infp = Jrel_infp * T(1.7);
    T tau_relp = btp / (T(1.0) + T(0.0123) / cajsr);
    if (tau_relp < T(0.001)) tau_relp = T(0.001);
    const T Jrel = T(1.5378) * ((T(1.0) - fCaMKp) * Jrel_np + fCaMKp * Jrel_p);

    // SERCA uptake, leak, translocation
    T Jupnp = T(0.005425) * cai / (cai + T(0.00092));
    T Jupp = T(2.75) * T(0.005425) * cai / (cai + T(0.00092) - T(0.00017));
    if (EPI) {
        Jupnp = Jupnp * T(1.3);
        Jupp = Jupp * T(1.3);
    }
    const T Jleak = T(0.0048825) * cansr / T(15.0);
    const T Jup = (T(1.0) - fCaMKp) * Jupnp + fCaMKp * Jupp - Jleak;
    const T Jtr = (cansr - cajsr) / T(60);

    o.d[0] = -(INa + INaL + Ito + ICaL + ICaNa + ICaK + IKr + IKs + IK1 + INaCa_i + INaCa_ss + INaK + INab +
               IKb + IpCa + ICab + I_ClCa + I_Clbk + stim);

    const T JdiffNa = (nass - nai) / T(2.0);
    const T JdiffK = (kss - ki) / T(2.0);
    const T Jdiff = (cass - cai) / T(0.2);
    T cmdnmax = T(0.05);
    if (EPI) cmdnmax = cmdnmax * T(1.3);
    const T kmcmdn = T(0.00238), trpnmax = T(0.07), kmtrpn = T(0.0005);
    const T BSRmax = T(0.047), KmBSR = T(0.00087), BSLmax = T(1.124), KmBSL = T(0.0087);
    const T csqnmax = T(10.0), kmcsqn = T(0.8);

    o.d[3] = -(ICaNa_i + INa + INaL + T(3.0) * INaCa_i + T(3.0) * INaK + INab) * Acap / (F * vmyo) + JdiffNa * vss / vmyo;
    o.d[4] = -(ICaNa_ss + T(3.0) * INaCa_ss) * Acap / (F * vss) - JdiffNa;
    o.d[5] = -(ICaK_i + Ito + IKr + IKs + IK1 + IKb + stim - T(2.0) * INaK) * Acap / (F * vmyo) + JdiffK * vss / vmyo;
    o.d[6] = -(ICaK_ss)*Acap / (F * vss) - JdiffK;
    const T Bcai = T(1.0) / (T(1.0) + cmdnmax * kmcmdn / sq(kmcmdn + cai) + trpnmax * kmtrpn / sq(kmtrpn + cai));
    o.d[9] = Bcai * (-(ICaL_i + IpCa + ICab - T(2.0) * INaCa_i) * Acap / (T(2.0) * F * vmyo) - Jup * vnsr / vmyo +
                     Jdiff * vss / vmyo);
    const T Bcass = T(1.0) / (T(1.0) + BSRmax * KmBSR / sq(KmBSR + cass) + BSLmax * KmBSL / sq(KmBSL + cass));
    o.d[2] = Bcass * (-(ICaL_ss - T(2.0) * INaCa_ss) * Acap / (T(2.0) * F * vss) + Jrel * vjsr / vss - Jdiff);
    o.d[7] = Jup - Jtr * vjsr / vnsr;
    const T Bcajsr = T(1.0) / (T(1.0) + csqnmax * kmcsqn / sq(kmcsqn + cajsr));
    o.d[8] = Bcajsr * (Jtr - Jrel);

    // linearised gates: a = -1/tau, b = y_inf/tau
#define MB_GATE(id, tau, ss) do { o.a[id] = T(-1.0) / (tau); o.b[id] = (ss) / (tau); } while (0)
    MB_GATE(10, tm, mss);
    MB_GATE(11, tauh, hss);
    MB_GATE(12, tauj, jss);
    MB_GATE(13, tauh, hssp);
    MB_GATE(14, taujp, jss);
    MB_GATE(15, tmL, mLss);
    MB_GATE(16, thL, hLss);
    MB_GATE(17, thLp, hLssp);
    MB_GATE(18, ta, ass);
    MB_GATE(19, tiF, iss);
    MB_GATE(20, tiS, iss);
    MB_GATE(21, ta, assp);
    MB_GATE(22, tiFp, iss);
    MB_GATE(23, tiSp, iss);
    MB_GATE(24, td, dss);
    MB_GATE(25, tff, fss);
    MB_GATE(26, tfs, fss);
    MB_GATE(27, tfcaf, fcass);
    MB_GATE(28, tfcas, fcass);
    MB_GATE(29, tjca, jcass);
    MB_GATE(30, tffp, fss);
    MB_GATE(31, tfcafp, fcass);
    MB_GATE(39, txs1, xs1ss);
    MB_GATE(40, txs2, xs2ss);
    MB_GATE(41, tau_rel, Jrel_inf);
    MB_GATE(42, tau_relp, Jrel_infp);
#undef MB_GATE
}

// Gate update for one linearised state.
template <typename T, int RULE>
__device__ __forceinline__ T rl_update(T y, T a, T b, T dt) {
    const bool euler = (RULE == MB_RL_REFERENCE_CPU) ? (a > T(-1) && a < T(1)) : (fabs(a) < T(1e-8));
    if (euler) return y + dt * (y * a + b);
    const T ba = b / a;
    return mexp(a * dt) * (y + ba) - ba;
}

__host__ __device__ constexpr bool tor_is_euler(int s) { return s <= 9 || (s >= 32 && s <= 38); }

// One sub-step in a single precision T (FP64 plain method).
template <typename T, typename S, int RULE>
__device__ __forceinline__ void torord_rl_step(T *y, double stim, double dt, T celltype, const TorScale<T> &sc) {
    TorRhs<T> r;
    torord_rhs<T>(y, T(stim), celltype, sc, r);
    const T dtt = T(dt);
#pragma unroll
    for (int s = 0; s < TOR_NEQ; ++s) {
        if (tor_is_euler(s)) y[s] = dtt * r.d[s] + y[s];
        else y[s] = rl_update<T, RULE>(y[s], r.a[s], r.b[s], dtt);
    }
}

struct TorMixedState {
    double d[TOR_N64];
    float f[TOR_N32];
};

// One sub-step of the mixed form: right-hand side in FP32, V and the ion
// concentrations accumulated in FP64.
template <int RULE>
__device__ __forceinline__ void torord_mixed_step(TorMixedState &st, double stim, double dt, float celltype,
                                                  const TorScale<float> &sc) {
    float y[TOR_NEQ];
#pragma unroll
    for (int s = 0; s < TOR_NEQ; ++s) {
        bool is64 = false;
        const int row = tor_mixed_row(s, is64);
        y[s] = is64 ? (float)st.d[row] : st.f[row];
    }
    TorRhs<float> r;
    torord_rhs<float>(y, (float)stim, celltype, sc, r);
    const float dtf = (float)dt;
#pragma unroll
    for (int s = 0; s < TOR_NEQ; ++s) {
        bool is64 = false;
        const int row = tor_mixed_row(s, is64);
        if (is64) {
            st.d[row] = dt * (double)r.d[s] + st.d[row];
        } else if (tor_is_euler(s)) {
            st.f[row] = dtf * r.d[s] + st.f[row];
        } else {
            st.f[row] = rl_update<float, RULE>(st.f[row], r.a[s], r.b[s], dtf);
        }
    }
}

// Default initial states (steady state after 200 beats) for endo, mid, epi,
// as the reference tabulates them (ToRORd_fkatp_mixed_endo_mid_epi.c:110-154,
// extra_data_library/helper_functions.c:166-300).
__host__ __device__ inline double torord_default_state(int celltype, int s) {
    const double endo[TOR_NEQ] = {
        -8.890585e+01, 1.107642e-02, 6.504164e-05, 1.210818e+01, 1.210851e+01, 1.426206e+02,
        1.426205e+02, 1.530373e+00, 1.528032e+00, 7.455488e-05, 7.814592e-04, 8.313839e-01,
        8.311938e-01, 6.752873e-01, 8.308255e-01, 1.585610e-04, 5.294475e-01, 2.896996e-01,
        9.419166e-04, 9.996194e-01, 5.938602e-01, 4.799180e-04, 9.996194e-01, 6.543754e-01,
        -2.898677e-33, 1.000000e+00, 9.389659e-01, 1.000000e+00, 9.999003e-01, 9.999773e-01,
        1.000000e+00, 1.000000e+00, 4.920606e-04, 8.337021e-04, 6.962775e-04, 8.425453e-04,
        9.980807e-01, 1.289824e-05, 3.675442e-04, 2.471690e-01, 1.742987e-04, 5.421027e-24,
        6.407933e-23};
    const double mid[TOR_NEQ] = {
        -8.924177e+01, 1.922391e-02, 6.585066e-05, 1.503347e+01, 1.503401e+01, 1.434407e+02,
        1.434406e+02, 1.959747e+00, 1.963459e+00, 8.177438e-05, 7.269124e-04, 8.379059e-01,
        8.377164e-01, 6.860578e-01, 8.372100e-01, 1.487602e-04, 5.350003e-01, 2.851164e-01,
        9.208259e-04, 9.996411e-01, 5.673539e-01, 4.691672e-04, 9.996412e-01, 6.265825e-01,
        -4.922960e-40, 1.000000e+00, 9.200354e-01, 1.000000e+00, 9.997888e-01, 9.999665e-01,
        1.000000e+00, 1.000000e+00, 5.161178e-04, 1.189422e-03, 6.917041e-04, 8.225453e-04,
        9.979358e-01, 1.835276e-05, 5.316232e-04, 2.650323e-01, 1.678628e-04, 2.091039e-25,
        2.438403e-23};
    const double epi[TOR_NEQ] = {
        -8.917755e+01, 1.288116e-02, 5.767956e-05, 1.284260e+01, 1.284291e+01, 1.429114e+02,
        1.429113e+02, 1.812268e+00, 1.810520e+00, 6.631866e-05, 7.370422e-04, 8.366816e-01,
        8.366012e-01, 6.840260e-01, 8.363958e-01, 1.505860e-04, 5.412669e-01, 3.043382e-01,
        9.248184e-04, 9.996371e-01, 9.996342e-01, 4.712023e-04, 9.996371e-01, 9.996366e-01,
        4.333129e-43, 1.000000e+00, 9.485160e-01, 1.000000e+00, 9.999339e-01, 9.999822e-01,
        1.000000e+00, 1.000000e+00, 3.086885e-04, 5.303737e-04, 6.775197e-04, 8.264829e-04,
        9.982135e-01, 9.433146e-06, 2.730221e-04, 2.308784e-01, 1.690386e-04, -1.103286e-23,
        -6.177055e-22};
    if (celltype == 1) return mid[s];
    if (celltype == 2) return epi[s];
    return endo[s];
}

MB_NS_END
