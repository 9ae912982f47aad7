/* ToRORd-fkatp (Tomek et al. 2019) with endo/mid/epi cell types, Rush-Larsen,
 * FP64 -- TEST INFRASTRUCTURE (oracle).  Restates
 * src/models_library/ToROrd/ToRORd_fkatp_mixed_endo_mid_epi.c (initial
 * states :38-154, sub-step :252-310, RHS_RL_cpu :718-791) and the model body
 * ToRORd_fkatp_mixed_endo_mid_epi_RL.common.c:1-754.
 *
 * As the reference CPU build runs it: the 17 current multipliers are 1 (the
 * IClb one, which the reference driver leaves unset, is taken as 1), INaK
 * has no MID scaling (the reference tests celltype == 2 a second time where
 * MID is meant), I_katp is zero (fkatp = 0), and the Rush-Larsen test
 * `abs(a) < 1e-8` (ToRORd_fkatp_mixed_endo_mid_epi.h:20) is applied to
 * abs() of a double, which C truncates to int: any -1 < a < 1 takes the
 * Euler form (MB_RL_REFERENCE_CPU).  MB_RL_TRUE applies |a| < 1e-8.
 */
#include <math.h>
#include <stddef.h>

#include "oracle.h"

static double sq(double x) { return x * x; }

/* 1.82e6 * (74 * 310)^-1.5, the Davies-equation constant of the activity
 * coefficients (RL.common.c:262-296), evaluated once in double precision. */
#define ORC_TOR_CONSTA 0x1.0c3201d875e3fp-1

/* Activity-coefficient factor exp(-A z^2 (sqrt(I)/(1+sqrt(I)) - 0.3 I)). */
static double davies(double z2, double I) {
    const double s = sqrt(I);
    return exp(-ORC_TOR_CONSTA * z2 * (s / (1.0 + s) - 0.3 * I));
}

/* Na/Ca exchanger flux of one compartment (RL.common.c:364-451). */
static double torord_ncx(double na, double ca, double hna, double hca, double nao, double cao, double *allo_out) {
    const double kna1 = 15.0, kna2 = 5.0, kna3 = 88.12, kasymm = 12.5;
    const double wna = 6.0e4, wca = 6.0e4, wnaca = 5.0e3;
    const double kcaon = 1.5e6, kcaoff = 5.0e3;
    const double zna = 1.0, zca = 2.0;
    const double h1 = 1.0 + na / kna3 * (1.0 + hna);
    const double h2 = (na * hna) / (kna3 * h1);
    const double h3 = 1.0 / h1;
    const double h4 = 1.0 + na / kna1 * (1.0 + na / kna2);
    const double h5 = na * na / (h4 * kna1 * kna2);
    const double h6 = 1.0 / h4;
    const double h7 = 1.0 + nao / kna3 * (1.0 + 1.0 / hna);
    const double h8 = nao / (kna3 * hna * h7);
    const double h9 = 1.0 / h7;
    const double h10 = kasymm + 1.0 + nao / kna1 * (1.0 + nao / kna2);
    const double h11 = nao * nao / (h10 * kna1 * kna2);
    const double h12 = 1.0 / h10;
    const double k1 = h12 * cao * kcaon;
    const double k2 = kcaoff;
    const double k3p = h9 * wca;
    const double k3pp = h8 * wnaca;
    const double k3 = k3p + k3pp;
    const double k4p = h3 * wca / hca;
    const double k4pp = h2 * wnaca;
    const double k4 = k4p + k4pp;
    const double k5 = kcaoff;
    const double k6 = h6 * ca * kcaon;
    const double k7 = h5 * h2 * wna;
    const double k8 = h8 * h11 * wna;
    const double x1 = k2 * k4 * (k7 + k6) + k5 * k7 * (k2 + k3);
    const double x2 = k1 * k7 * (k4 + k5) + k4 * k6 * (k1 + k8);
    const double x3 = k1 * k3 * (k7 + k6) + k8 * k6 * (k2 + k3);
    const double x4 = k2 * k8 * (k4 + k5) + k3 * k5 * (k1 + k8);
    const double xs = x1 + x2 + x3 + x4;
    const double E1 = x1 / xs, E2 = x2 / xs, E3 = x3 / xs, E4 = x4 / xs;
    const double KmCaAct = 150.0e-6;
    *allo_out = 1.0 / (1.0 + sq(KmCaAct / ca));
    const double JncxNa = 3.0 * (E4 * k7 - E1 * k8) + E3 * k4pp - E2 * k3pp;
    const double JncxCa = E2 * k2 - E1 * k1;
    return zna * JncxNa + zca * JncxCa;
}

/* RHS_RL_cpu (ToRORd_fkatp_mixed_endo_mid_epi.c:718-791) with the model body of
 * ToRORd_fkatp_mixed_endo_mid_epi_RL.common.c:1-754: rd = dy/dt of the Euler
 * states, (ra, rb) = the linearisation dy/dt = a y + b of the gates
 * (RL.common.c:657-710).  celltype 0 endo, 1 mid, 2 epi; sc = multipliers of
 * INa, IKr, IKs, ICaL, IK1. */
static void torord_rhs(const double *y, double stim, int celltype, const double *sc, double *rd, double *ra,
                       double *rb) {
    const double v = y[0], CaMKt = y[1], cass = y[2], nai = y[3], nass = y[4], ki = y[5], kss = y[6];
    const double cansr = y[7], cajsr = y[8], cai = y[9];
    const double m = y[10], h = y[11], j = y[12], hp = y[13], jp = y[14], mL = y[15], hL = y[16];
    const double hLp = y[17], a = y[18], iF = y[19], iS = y[20], ap = y[21], iFp = y[22], iSp = y[23];
    const double d = y[24], ff = y[25], fs = y[26], fcaf = y[27], fcas = y[28], jca = y[29];
    const double ffp = y[30], fcafp = y[31], nca = y[32], nca_i = y[33];
    const double c0 = y[34], c1 = y[35], c2 = y[36], I = y[37], o_ = y[38];
    const double xs1 = y[39], xs2 = y[40], Jrel_np = y[41], Jrel_p = y[42];

    const int EPI = celltype == 2;
    const int MID = celltype == 1;

    const double nao = 140.0, cao = 1.8, ko = 5.0;
    const double ICaL_fractionSS = 0.8, INaCa_fractionSS = 0.35;
    const double R = 8314.0, Tk = 310.0, F = 96485.0;

    // cell geometry
    const double L = 0.01, rad = 0.0011;
    const double vcell = 1000.0 * 3.14 * rad * rad * L;
    const double Ageo = 2.0 * 3.14 * rad * rad + 2.0 * 3.14 * rad * L;
    const double Acap = 2.0 * Ageo;
    const double vmyo = 0.68 * vcell, vnsr = 0.0552 * vcell, vjsr = 0.0048 * vcell;
    const double vss = 0.02 * vcell;
    const double cli = 24.0, clo = 150.0;

    // CaMK
    const double KmCaMK = 0.15, aCaMK = 0.05, bCaMK = 0.00068, CaMKo = 0.05, KmCaM = 0.0015;
    const double CaMKb = CaMKo * (1.0 - CaMKt) / (1.0 + KmCaM / cass);
    const double CaMKa = CaMKb + CaMKt;
    rd[1] = aCaMK * CaMKb * (CaMKb + CaMKt) - bCaMK * CaMKt;

    const double RTF = R * Tk / F;
    const double ENa = RTF * log(nao / nai);
    const double EK = RTF * log(ko / ki);
    const double PKNa = 0.01833;
    const double EKs = RTF * log((ko + PKNa * nao) / (ki + PKNa * nai));

    const double vffrt = v * F * F / (R * Tk);
    const double vfrt = v * F / (R * Tk);
    const double fCaMKp = 1.0 / (1.0 + KmCaMK / CaMKa);   // fINap = fINaLp = fItop = fICaLp = fJrelp = fJupp

    // INa (Grandi formulation with CaMK phosphorylation)
    const double mss = 1.0 / sq(1.0 + exp(-(56.86 + v) / 9.03));
    const double tm = 0.1292 * exp(-sq((v + 45.79) / 15.54)) + 0.06487 * exp(-sq((v - 4.823) / 51.12));
    double ah, bh, aj, bj;
    if (v >= (-40.0)) {
        ah = 0.0;
        bh = 0.77 / (0.13 * (1.0 + exp(-(v + 10.66) / 11.1)));
        aj = 0.0;
        bj = (0.6 * exp(0.057 * v)) / (1.0 + exp((-0.1) * (v + 32.0)));
    } else {
        ah = 0.057 * exp(-(v + 80.0) / 6.8);
        bh = 2.7 * exp(0.079 * v) + 3.1 * 100000.0 * exp(0.3485 * v);
        aj = (((-2.5428) * 10000.0 * exp(0.2444 * v) - 6.948 * 1.0e-6 * exp((-0.04391) * v)) *
              (v + 37.78)) / (1.0 + exp(0.311 * (v + 79.23)));
        bj = (0.02424 * exp((-0.01052) * v)) / (1.0 + exp((-0.1378) * (v + 40.14)));
    }
    const double tauh = 1.0 / (ah + bh);
    const double hss = 1.0 / sq(1.0 + exp((v + 71.55) / 7.43));
    const double tauj = 1.0 / (aj + bj);
    const double jss = hss;
    const double hssp = 1.0 / sq(1.0 + exp((v + 71.55 + 6.0) / 7.43));
    const double taujp = 1.46 * tauj;
    const double GNa = 11.7802;
    const double INa = sc[0] * GNa * (v - ENa) * (m * m * m) * ((1.0 - fCaMKp) * h * j + fCaMKp * hp * jp);

    // INaL
    const double mLss = 1.0 / (1.0 + exp((-(v + 42.85)) / 5.264));
    const double tmL = tm;
    const double hLss = 1.0 / (1.0 + exp((v + 87.61) / 7.488));
    const double thL = 200.0;
    const double hLssp = 1.0 / (1.0 + exp((v + 93.81) / 7.488));
    const double thLp = 3.0 * thL;
    double GNaL = 0.0279;
    if (EPI) GNaL = GNaL * 0.6;
    const double INaL = GNaL * (v - ENa) * mL * ((1.0 - fCaMKp) * hL + fCaMKp * hLp);

    // Ito
    const double ass = 1.0 / (1.0 + exp((-(v - 14.34)) / 14.82));
    const double ta = 1.0515 / (1.0 / (1.2089 * (1.0 + exp(-(v - 18.4099) / 29.3814))) +
                              3.5 / (1.0 + exp((v + 100.0) / 29.3814)));
    const double iss = 1.0 / (1.0 + exp((v + 43.94) / 5.711));
    const double delta_epi = EPI ? 1.0 - (0.95 / (1.0 + exp((v + 70.0) / 5.0))) : 1.0;
    double tiF = 4.562 + 1.0 / (0.3933 * exp((-(v + 100.0)) / 100.0) + 0.08004 * exp((v + 50.0) / 16.59));
    double tiS = 23.62 + 1.0 / (0.001416 * exp((-(v + 96.52)) / 59.05) + 1.780e-8 * exp((v + 114.1) / 8.079));
    tiF = tiF * delta_epi;
    tiS = tiS * delta_epi;
    const double AiF = 1.0 / (1.0 + exp((v - 213.6) / 151.2));
    const double AiS = 1.0 - AiF;
    const double ii = AiF * iF + AiS * iS;
    const double assp = 1.0 / (1.0 + exp((-(v - 24.34)) / 14.82));
    const double dti_develop = 1.354 + 1.0e-4 / (exp((v - 167.4) / 15.89) + exp(-(v - 12.23) / 0.2154));
    const double dti_recover = 1.0 - 0.5 / (1.0 + exp((v + 70.0) / 20.0));
    const double tiFp = dti_develop * dti_recover * tiF;
    const double tiSp = dti_develop * dti_recover * tiS;
    const double ip = AiF * iFp + AiS * iSp;
    double Gto = 0.16;
    if (EPI || MID) Gto = Gto * 2.0;
    const double Ito = Gto * (v - EK) * ((1.0 - fCaMKp) * a * ii + fCaMKp * ap * ip);

    // ICaL, ICaNa, ICaK
    double dss = 1.0763 * exp((-1.0070) * exp((-0.0829) * (v)));
    if (v > 31.4978) dss = 1.0;
    const double td = 0.6 + 1.0 / (exp((-0.05) * (v + 6.0)) + exp(0.09 * (v + 14.0)));
    const double fss = 1.0 / (1.0 + exp((v + 19.58) / 3.696));
    const double tff = 7.0 + 1.0 / (0.0045 * exp(-(v + 20.0) / 10.0) + 0.0045 * exp((v + 20.0) / 10.0));
    const double tfs = 1000.0 + 1.0 / (0.000035 * exp(-(v + 5.0) / 4.0) + 0.000035 * exp((v + 5.0) / 6.0));
    const double Aff = 0.6;
    const double Afs = 1.0 - Aff;
    const double f = Aff * ff + Afs * fs;
    const double fcass = fss;
    const double tfcaf = 7.0 + 1.0 / (0.04 * exp(-(v - 4.0) / 7.0) + 0.04 * exp((v - 4.0) / 7.0));
    const double tfcas = 100.0 + 1.0 / (0.00012 * exp(-v / 3.0) + 0.00012 * exp(v / 7.0));
    const double Afcaf = 0.3 + 0.6 / (1.0 + exp((v - 10.0) / 10.0));
    const double Afcas = 1.0 - Afcaf;
    const double fca = Afcaf * fcaf + Afcas * fcas;
    const double tjca = 75.0;
    const double jcass = 1.0 / (1.0 + exp((v + 18.08) / (2.7916)));
    const double tffp = 2.5 * tff;
    const double fp = Aff * ffp + Afs * fs;
    const double tfcafp = 2.5 * tfcaf;
    const double fcap = Afcaf * fcafp + Afcas * fcas;

    const double Kmn = 0.002, k2n = 500.0;
    const double km2n = jca * 1.0;
    const double anca = 1.0 / (k2n / km2n + sq(sq(1.0 + Kmn / cass)));
    rd[32] = anca * k2n - nca * km2n;
    const double anca_i = 1.0 / (k2n / km2n + sq(sq(1.0 + Kmn / cai)));
    rd[33] = anca_i * k2n - nca_i * km2n;

    // driving forces with Davies activity coefficients
    const double Io = 0.5 * (nao + ko + clo + 4.0 * cao) / 1000.0;
    double Ii = 0.5 * (nass + kss + cli + 4.0 * cass) / 1000.0;
    double gamma_cai = davies(4.0, Ii);
    const double gamma_cao = davies(4.0, Io);
    double gamma_nai = davies(1.0, Ii);
    const double gamma_nao = davies(1.0, Io);
    double gamma_ki = davies(1.0, Ii);
    const double gamma_kao = gamma_nao;
    const double e2 = exp(2.0 * vfrt);
    const double e1 = exp(1.0 * vfrt);
    const double PhiCaL_ss = 4.0 * vffrt * (gamma_cai * cass * e2 - gamma_cao * cao) / (e2 - 1.0);
    const double PhiCaNa_ss = 1.0 * vffrt * (gamma_nai * nass * e1 - gamma_nao * nao) / (e1 - 1.0);
    const double PhiCaK_ss = 1.0 * vffrt * (gamma_ki * kss * e1 - gamma_kao * ko) / (e1 - 1.0);
    Ii = 0.5 * (nai + ki + cli + 4.0 * cai) / 1000.0;
    gamma_cai = davies(4.0, Ii);
    gamma_nai = davies(1.0, Ii);
    gamma_ki = davies(1.0, Ii);
    const double PhiCaL_i = 4.0 * vffrt * (gamma_cai * cai * e2 - gamma_cao * cao) / (e2 - 1.0);
    const double PhiCaNa_i = 1.0 * vffrt * (gamma_nai * nai * e1 - gamma_nao * nao) / (e1 - 1.0);
    const double PhiCaK_i = 1.0 * vffrt * (gamma_ki * ki * e1 - gamma_kao * ko) / (e1 - 1.0);

    double PCa = 8.3757e-05 * sc[3];
    if (EPI) PCa = PCa * 1.2;
    else if (MID) PCa = PCa * 2.0;
    const double PCap = 1.1 * PCa;
    const double PCaNa = 0.00125 * PCa, PCaK = 3.574e-4 * PCa;
    const double PCaNap = 0.00125 * PCap, PCaKp = 3.574e-4 * PCap;
    const double one_m = 1.0 - fCaMKp;
    const double gss = f * (1.0 - nca) + jca * fca * nca;
    const double gssp = fp * (1.0 - nca) + jca * fcap * nca;
    const double gi = f * (1.0 - nca_i) + jca * fca * nca_i;
    const double gip = fp * (1.0 - nca_i) + jca * fcap * nca_i;
    double ICaL_ss = one_m * PCa * PhiCaL_ss * d * gss + fCaMKp * PCap * PhiCaL_ss * d * gssp;
    double ICaNa_ss = one_m * PCaNa * PhiCaNa_ss * d * gss + fCaMKp * PCaNap * PhiCaNa_ss * d * gssp;
    double ICaK_ss = one_m * PCaK * PhiCaK_ss * d * gss + fCaMKp * PCaKp * PhiCaK_ss * d * gssp;
    double ICaL_i = one_m * PCa * PhiCaL_i * d * gi + fCaMKp * PCap * PhiCaL_i * d * gip;
    double ICaNa_i = one_m * PCaNa * PhiCaNa_i * d * gi + fCaMKp * PCaNap * PhiCaNa_i * d * gip;
    double ICaK_i = one_m * PCaK * PhiCaK_i * d * gi + fCaMKp * PCaKp * PhiCaK_i * d * gip;
    const double fi = 1.0 - ICaL_fractionSS;
    ICaL_i = ICaL_i * fi;
    ICaNa_i = ICaNa_i * fi;
    ICaK_i = ICaK_i * fi;
    ICaL_ss = ICaL_ss * ICaL_fractionSS;
    ICaNa_ss = ICaNa_ss * ICaL_fractionSS;
    ICaK_ss = ICaK_ss * ICaL_fractionSS;
    const double ICaL = ICaL_ss + ICaL_i;
    const double ICaNa = ICaNa_ss + ICaNa_i;
    const double ICaK = ICaK_ss + ICaK_i;

    // IKr, Lu-Vandenberg Markov model
    const double alpha = 0.1161 * exp(0.2990 * vfrt);
    const double beta = 0.2442 * exp((-1.604) * vfrt);
    const double alpha1 = 1.25 * 0.1235;
    const double beta1 = 0.1911;
    const double alpha2 = 0.0578 * exp(0.9710 * vfrt);
    const double beta2 = 0.349e-3 * exp((-1.062) * vfrt);
    const double alphai = 0.2533 * exp(0.5953 * vfrt);
    const double betai = 1.25 * 0.0522 * exp((-0.8209) * vfrt);
    const double alphac2ToI = 0.52e-4 * exp(1.525 * vfrt);
    const double betaItoC2 = (beta2 * betai * alphac2ToI) / (alpha2 * alphai);
    rd[34] = c1 * beta - c0 * alpha;
    rd[35] = c0 * alpha + c2 * beta1 - c1 * (beta + alpha1);
    rd[36] = c1 * alpha1 + o_ * beta2 + I * betaItoC2 - c2 * (beta1 + alpha2 + alphac2ToI);
    rd[38] = c2 * alpha2 + I * betai - o_ * (beta2 + alphai);
    rd[37] = c2 * alphac2ToI + o_ * alphai - I * (betaItoC2 + betai);
    double GKr = 0.0321 * sqrt(ko / 5.0) * sc[1];
    if (EPI) GKr = GKr * 1.3;
    else if (MID) GKr = GKr * 0.8;
    const double IKr = GKr * o_ * (v - EK);

    // IKs
    const double xs1ss = 1.0 / (1.0 + exp((-(v + 11.60)) / 8.932));
    const double txs1 = 817.3 + 1.0 / (2.326e-4 * exp((v + 48.28) / 17.80) +
                                       0.001292 * exp((-(v + 210.0)) / 230.0));
    const double xs2ss = xs1ss;
    const double txs2 = 1.0 / (0.01 * exp((v - 50.0) / 20.0) + 0.0193 * exp((-(v + 66.54)) / 31.0));
    const double KsCa = 1.0 + 0.6 / (1.0 + pow((3.8e-5 / cai), 1.4));
    double GKs = 0.0011 * sc[2];
    if (EPI) GKs = GKs * 1.4;
    const double IKs = GKs * KsCa * xs1 * xs2 * (v - EKs);

    // IK1
    const double vek = v - EK;
    const double aK1 = 4.094 / (1.0 + exp(0.1217 * (vek - 49.934)));
    const double bK1 = (15.72 * exp(0.0674 * (vek - 3.257)) + exp(0.0618 * (vek - 594.31))) /
                  (1.0 + exp((-0.1629) * (vek + 14.207)));
    const double K1ss = aK1 / (aK1 + bK1);
    double GK1 = sc[4] * 0.6992;
    if (EPI) GK1 = GK1 * 1.2;
    else if (MID) GK1 = GK1 * 1.3;
    const double IK1 = GK1 * sqrt(ko / 5.0) * K1ss * vek;

    // INaCa (myoplasm and junctional subspace)
    const double qna = 0.5224, qca = 0.1670;
    const double hca = exp((qca * v * F) / (R * Tk));
    const double hna = exp((qna * v * F) / (R * Tk));
    double Gncx = 0.0034;
    if (EPI) Gncx = Gncx * 1.1;
    else if (MID) Gncx = Gncx * 1.4;
    double allo_i, allo_ss;
    const double jn_i = torord_ncx(nai, cai, hna, hca, nao, cao, &allo_i);
    const double INaCa_i = (1.0 - INaCa_fractionSS) * Gncx * allo_i * jn_i;
    const double jn_ss = torord_ncx(nass, cass, hna, hca, nao, cao, &allo_ss);
    const double INaCa_ss = INaCa_fractionSS * Gncx * allo_ss * jn_ss;

    // INaK
    const double k1p = 949.5, k1m = 182.4, k2p = 687.2, k2m = 39.4;
    const double k3p = 1899.0, k3m = 79300.0, k4p = 639.0, k4m = 40.0;
    const double Knai0 = 9.073, Knao0 = 27.78, delta = (-0.1550);
    const double Knai = Knai0 * exp((delta * v * F) / (3.0 * R * Tk));
    const double Knao = Knao0 * exp(((1.0 - delta) * v * F) / (3.0 * R * Tk));
    const double Kki = 0.5, Kko = 0.3582, MgADP = 0.05, MgATP = 9.8, Kmgatp = 1.698e-7;
    const double H = 1.0e-7, eP = 4.2, Khp = 1.698e-7, Knap = 224.0, Kxkur = 292.0;
    const double P = eP / (1.0 + H / Khp + nai / Knap + ki / Kxkur);
    const double nk3 = (1.0 + nai / Knai) * (1.0 + nai / Knai) * (1.0 + nai / Knai);
    const double kk2 = sq(1.0 + ki / Kki);
    const double no3 = (1.0 + nao / Knao) * (1.0 + nao / Knao) * (1.0 + nao / Knao);
    const double ko2 = sq(1.0 + ko / Kko);
    const double rn = nai / Knai, rno = nao / Knao;
    const double a1 = (k1p * (rn * rn * rn)) / (nk3 + kk2 - 1.0);
    const double b1 = k1m * MgADP;
    const double a2 = k2p;
    const double b2 = (k2m * (rno * rno * rno)) / (no3 + ko2 - 1.0);
    const double a3 = (k3p * sq(ko / Kko)) / (no3 + ko2 - 1.0);
    const double b3 = (k3m * P * H) / (1.0 + MgATP / Kmgatp);
    const double a4 = (k4p * MgATP / Kmgatp) / (1.0 + MgATP / Kmgatp);
    const double b4 = (k4m * sq(ki / Kki)) / (nk3 + kk2 - 1.0);
    const double x1 = a4 * a1 * a2 + b2 * b4 * b3 + a2 * b4 * b3 + b3 * a1 * a2;
    const double x2 = b2 * b1 * b4 + a1 * a2 * a3 + a3 * b1 * b4 + a2 * a3 * b4;
    const double x3 = a2 * a3 * a4 + b3 * b2 * b1 + b2 * b1 * a4 + a3 * a4 * b1;
    const double x4 = b4 * b3 * b2 + a3 * a4 * a1 + b2 * a4 * a1 + b3 * b2 * a1;
    const double xs = x1 + x2 + x3 + x4;
    const double E1 = x1 / xs, E2 = x2 / xs, E3 = x3 / xs, E4 = x4 / xs;
    const double JnakNa = 3.0 * (E1 * a3 - E2 * b3);
    const double JnakK = 2.0 * (E4 * b1 - E3 * a1);
    double Pnak = 15.4509;
    if (EPI) Pnak = Pnak * 0.9;
    const double INaK = Pnak * (1.0 * JnakNa + 1.0 * JnakK);

    // background currents
    const double xkb = 1.0 / (1.0 + exp(-(v - 10.8968) / (23.9871)));
    double GKb = 0.0189;
    if (EPI) GKb = GKb * 0.6;
    const double IKb = GKb * xkb * (v - EK);
    const double PNab = 1.9239e-09;
    const double INab = PNab * vffrt * (nai * e1 - nao) / (e1 - 1.0);
    const double PCab = 5.9194e-08;
    const double ICab = PCab * 4.0 * vffrt * (gamma_cai * cai * e2 - gamma_cao * cao) / (e2 - 1.0);
    const double GpCa = 5e-04;
    const double IpCa = GpCa * cai / (0.0005 + cai);

    // chloride
    const double ECl = RTF * log(cli / clo);
    const double GClCa = 0.2843, GClB = 1.98e-3, KdClCa = 0.1;
    const double I_ClCa = 1.0 * GClCa / (1.0 + KdClCa / cass) * (v - ECl);
    const double I_Clbk = GClB * (v - ECl);

    // SR release
    const double jsrMidpoint = 1.7, bt = 4.75;
    const double a_rel = 0.5 * bt;
    const double jr = jsrMidpoint / cajsr;
    const double jr8 = sq(sq(sq(jr)));
    double Jrel_inf = a_rel * (-ICaL) / (1.0 + jr8);
    if (MID) Jrel_inf = Jrel_inf * 1.7;
    double tau_rel = bt / (1.0 + 0.0123 / cajsr);
    if (tau_rel < 0.001) tau_rel = 0.001;
    const double btp = 1.25 * bt;
    const double a_relp = 0.5 * btp;
    double Jrel_infp = a_relp * (-ICaL) / (1.0 + jr8);
    if (MID) Jrel_infp = Jrel_infp * 1.7;
    double tau_relp = btp / (1.0 + 0.0123 / cajsr);
    if (tau_relp < 0.001) tau_relp = 0.001;
    const double Jrel = 1.5378 * ((1.0 - fCaMKp) * Jrel_np + fCaMKp * Jrel_p);

    // SERCA uptake, leak, translocation
    double Jupnp = 0.005425 * cai / (cai + 0.00092);
    double Jupp = 2.75 * 0.005425 * cai / (cai + 0.00092 - 0.00017);
    if (EPI) {
        Jupnp = Jupnp * 1.3;
        Jupp = Jupp * 1.3;
    }
    const double Jleak = 0.0048825 * cansr / 15.0;
    const double Jup = (1.0 - fCaMKp) * Jupnp + fCaMKp * Jupp - Jleak;
    const double Jtr = (cansr - cajsr) / 60.0;

    rd[0] = -(INa + INaL + Ito + ICaL + ICaNa + ICaK + IKr + IKs + IK1 + INaCa_i + INaCa_ss + INaK + INab +
               IKb + IpCa + ICab + I_ClCa + I_Clbk + stim);

    const double JdiffNa = (nass - nai) / 2.0;
    const double JdiffK = (kss - ki) / 2.0;
    const double Jdiff = (cass - cai) / 0.2;
    double cmdnmax = 0.05;
    if (EPI) cmdnmax = cmdnmax * 1.3;
    const double kmcmdn = 0.00238, trpnmax = 0.07, kmtrpn = 0.0005;
    const double BSRmax = 0.047, KmBSR = 0.00087, BSLmax = 1.124, KmBSL = 0.0087;
    const double csqnmax = 10.0, kmcsqn = 0.8;

    rd[3] = -(ICaNa_i + INa + INaL + 3.0 * INaCa_i + 3.0 * INaK + INab) * Acap / (F * vmyo) + JdiffNa * vss / vmyo;
    rd[4] = -(ICaNa_ss + 3.0 * INaCa_ss) * Acap / (F * vss) - JdiffNa;
    rd[5] = -(ICaK_i + Ito + IKr + IKs + IK1 + IKb + stim - 2.0 * INaK) * Acap / (F * vmyo) + JdiffK * vss / vmyo;
    rd[6] = -(ICaK_ss)*Acap / (F * vss) - JdiffK;
    const double Bcai = 1.0 / (1.0 + cmdnmax * kmcmdn / sq(kmcmdn + cai) + trpnmax * kmtrpn / sq(kmtrpn + cai));
    rd[9] = Bcai * (-(ICaL_i + IpCa + ICab - 2.0 * INaCa_i) * Acap / (2.0 * F * vmyo) - Jup * vnsr / vmyo +
                     Jdiff * vss / vmyo);
    const double Bcass = 1.0 / (1.0 + BSRmax * KmBSR / sq(KmBSR + cass) + BSLmax * KmBSL / sq(KmBSL + cass));
    rd[2] = Bcass * (-(ICaL_ss - 2.0 * INaCa_ss) * Acap / (2.0 * F * vss) + Jrel * vjsr / vss - Jdiff);
    rd[7] = Jup - Jtr * vjsr / vnsr;
    const double Bcajsr = 1.0 / (1.0 + csqnmax * kmcsqn / sq(kmcsqn + cajsr));
    rd[8] = Bcajsr * (Jtr - Jrel);

    // linearised gates: a = -1/tau, b = y_inf/tau
#define ORC_GATE(id, tau, ss) do { ra[id] = (-1.0) / (tau); rb[id] = (ss) / (tau); } while (0)
    ORC_GATE(10, tm, mss);
    ORC_GATE(11, tauh, hss);
    ORC_GATE(12, tauj, jss);
    ORC_GATE(13, tauh, hssp);
    ORC_GATE(14, taujp, jss);
    ORC_GATE(15, tmL, mLss);
    ORC_GATE(16, thL, hLss);
    ORC_GATE(17, thLp, hLssp);
    ORC_GATE(18, ta, ass);
    ORC_GATE(19, tiF, iss);
    ORC_GATE(20, tiS, iss);
    ORC_GATE(21, ta, assp);
    ORC_GATE(22, tiFp, iss);
    ORC_GATE(23, tiSp, iss);
    ORC_GATE(24, td, dss);
    ORC_GATE(25, tff, fss);
    ORC_GATE(26, tfs, fss);
    ORC_GATE(27, tfcaf, fcass);
    ORC_GATE(28, tfcas, fcass);
    ORC_GATE(29, tjca, jcass);
    ORC_GATE(30, tffp, fss);
    ORC_GATE(31, tfcafp, fcass);
    ORC_GATE(39, txs1, xs1ss);
    ORC_GATE(40, txs2, xs2ss);
    ORC_GATE(41, tau_rel, Jrel_inf);
    ORC_GATE(42, tau_relp, Jrel_infp);
#undef ORC_GATE
}

void orc_torord_initial_state(int celltype, double *sv) {
    const double endo[ORC_TOR_NEQ] = {
        -8.890585e+01, 1.107642e-02, 6.504164e-05, 1.210818e+01, 1.210851e+01, 1.426206e+02,
        1.426205e+02, 1.530373e+00, 1.528032e+00, 7.455488e-05, 7.814592e-04, 8.313839e-01,
        8.311938e-01, 6.752873e-01, 8.308255e-01, 1.585610e-04, 5.294475e-01, 2.896996e-01,
        9.419166e-04, 9.996194e-01, 5.938602e-01, 4.799180e-04, 9.996194e-01, 6.543754e-01,
        -2.898677e-33, 1.000000e+00, 9.389659e-01, 1.000000e+00, 9.999003e-01, 9.999773e-01,
        1.000000e+00, 1.000000e+00, 4.920606e-04, 8.337021e-04, 6.962775e-04, 8.425453e-04,
        9.980807e-01, 1.289824e-05, 3.675442e-04, 2.471690e-01, 1.742987e-04, 5.421027e-24,
        6.407933e-23};
    const double mid[ORC_TOR_NEQ] = {
        -8.924177e+01, 1.922391e-02, 6.585066e-05, 1.503347e+01, 1.503401e+01, 1.434407e+02,
        1.434406e+02, 1.959747e+00, 1.963459e+00, 8.177438e-05, 7.269124e-04, 8.379059e-01,
        8.377164e-01, 6.860578e-01, 8.372100e-01, 1.487602e-04, 5.350003e-01, 2.851164e-01,
        9.208259e-04, 9.996411e-01, 5.673539e-01, 4.691672e-04, 9.996412e-01, 6.265825e-01,
        -4.922960e-40, 1.000000e+00, 9.200354e-01, 1.000000e+00, 9.997888e-01, 9.999665e-01,
        1.000000e+00, 1.000000e+00, 5.161178e-04, 1.189422e-03, 6.917041e-04, 8.225453e-04,
        9.979358e-01, 1.835276e-05, 5.316232e-04, 2.650323e-01, 1.678628e-04, 2.091039e-25,
        2.438403e-23};
    const double epi[ORC_TOR_NEQ] = {
        -8.917755e+01, 1.288116e-02, 5.767956e-05, 1.284260e+01, 1.284291e+01, 1.429114e+02,
        1.429113e+02, 1.812268e+00, 1.810520e+00, 6.631866e-05, 7.370422e-04, 8.366816e-01,
        8.366012e-01, 6.840260e-01, 8.363958e-01, 1.505860e-04, 5.412669e-01, 3.043382e-01,
        9.248184e-04, 9.996371e-01, 9.996342e-01, 4.712023e-04, 9.996371e-01, 9.996366e-01,
        4.333129e-43, 1.000000e+00, 9.485160e-01, 1.000000e+00, 9.999339e-01, 9.999822e-01,
        1.000000e+00, 1.000000e+00, 3.086885e-04, 5.303737e-04, 6.775197e-04, 8.264829e-04,
        9.982135e-01, 9.433146e-06, 2.730221e-04, 2.308784e-01, 1.690386e-04, -1.103286e-23,
        -6.177055e-22};
    const double *src = celltype == 1 ? mid : (celltype == 2 ? epi : endo);
    for (int i = 0; i < ORC_TOR_NEQ; ++i) sv[i] = src[i];
}

static int is_euler_state(int s) { return s <= 9 || (s >= 32 && s <= 38); }

/* solve_model_ode_cpu (ToRORd_fkatp_mixed_endo_mid_epi.c:252-310) with the
 * SOLVE_EQUATION_* macros of ToRORd_fkatp_mixed_endo_mid_epi.h:18-22. */
void orc_torord_step(double *sv, double stim, double dt, int celltype, int rl_rule, const double *scale) {
    static const double one[5] = {1.0, 1.0, 1.0, 1.0, 1.0};
    double rY[ORC_TOR_NEQ], rd[ORC_TOR_NEQ], ra[ORC_TOR_NEQ], rb[ORC_TOR_NEQ];
    for (int i = 0; i < ORC_TOR_NEQ; ++i) {
        rY[i] = sv[i];
        rd[i] = ra[i] = rb[i] = 0.0;
    }
    torord_rhs(rY, stim, celltype, scale ? scale : one, rd, ra, rb);
    for (int i = 0; i < ORC_TOR_NEQ; ++i) {
        if (is_euler_state(i)) {
            sv[i] = dt * rd[i] + rY[i];
            continue;
        }
        const double a = ra[i], b = rb[i];
        const int small = rl_rule == MB_RL_TRUE ? fabs(a) < 1e-8 : (a > -1.0 && a < 1.0);
        sv[i] = small ? rY[i] + dt * (rY[i] * a + b) : exp(a * dt) * (rY[i] + b / a) - b / a;
    }
}
