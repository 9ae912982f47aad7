// ToRORd-fkatp endocardial cell with the forward-Euler integrators: the model
// of the reference's libToRORd_fkatp_endo (src/models_library/ToROrd/
// ToRORd_fkatp_endo.c:1-130, right-hand side ToROrd_common.inc.c:1-720),
// stepped by the default solvers (default_solvers.c:9-175,
// default_solvers.cu:1-235):
//
//   fixed step     y <- y + dt f(y) for all 43 states, num_steps times per
//                  loop step (default_solvers.c:37-53);
//   adaptive step  the Euler / Heun error-controlled scheme with a per-cell
//                  step size carried across loop steps (default_solvers.c:
//                  55-175, default_solvers.cu:84-203).
//
// The library is generated from CellML.  Every parameter is written as a
// single-precision literal while the arithmetic is double (real = double), so
// each parameter is the double value of a float; the two products of two
// literals (the 1000 * 3.14 of the cell volume and the 2 * 3.14 of the cell
// area) are float products; a few rate constants are double literals.  Those
// precisions move the solution at the 1e-8 level and are kept here: the
// parameters are float constants, the two products are formed in float, and
// the double literals stay double.  The cell type is fixed to ENDO (celltype
// = 0: no cell-type scaling applies) and I_katp is zero (fkatp = 0).
//
// State order (the library's):
//   0 v, 1 CaMKt, 2 nai, 3 nass, 4 ki, 5 kss, 6 cai, 7 cass, 8 cansr,
//   9 cajsr, 10 m, 11 h, 12 j, 13 hp, 14 jp, 15 mL, 16 hL, 17 hLp, 18 a,
//   19 iF, 20 iS, 21 ap, 22 iFp, 23 iSp, 24 d, 25 ff, 26 fs, 27 fcaf,
//   28 fcas, 29 jca, 30 ffp, 31 fcafp, 32 nca_ss, 33 nca_i, 34 C3, 35 C2,
//   36 C1, 37 O, 38 I, 39 xs1, 40 xs2, 41 Jrel_np, 42 Jrel_p.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace mb_tore {

constexpr int NEQ = 43;

// ---- parameters (single-precision literals of the generated library) -------
// physical constants and cell geometry
constexpr float F = 96485.0f, R = 8314.0f, T = 310.0f;
constexpr float rad = 0.0011f, L = 0.01f;
constexpr float nao = 140.0f, ko = 5.0f, cao = 1.8f, clo = 150.0f, cli = 24.0f;
// CaMK
constexpr float CaMKo = 0.05f, KmCaM = 0.0015f, aCaMK = 0.05f, bCaMK = 0.00068f, KmCaMK = 0.15f;
// buffers
constexpr float cmdnmax = 0.05f, kmcmdn = 0.00238f, trpnmax = 0.07f, kmtrpn = 0.0005f;
constexpr float BSRmax = 0.047f, KmBSR = 0.00087f, BSLmax = 1.124f, KmBSL = 0.0087f;
constexpr float csqnmax = 10.0f, kmcsqn = 0.8f;
// reversal potentials, K_ATP (inactive)
constexpr float PKNa = 0.01833f;
// channel conductances and permeabilities (endo values)
constexpr float GNa = 11.7802f, thL = 200.0f, GNaL = 0.0279f, Gto = 0.16f;
constexpr float Aff = 0.6f, tjca = 75.0f, k2n = 500.0f, Kmn = 0.002f;
constexpr float dielConstant = 74.0f, PCa = 8.3757e-05f, ICaL_fractionSS = 0.8f;
constexpr float beta_1 = 0.1911f, alpha_1 = 0.154375f, GKr = 0.0321f, GKs = 0.0011f, GK1 = 0.6992f;
// NCX
constexpr float qca = 0.167f, qna = 0.5224f, kna1 = 15.0f, kna2 = 5.0f, kna3 = 88.12f, kasymm = 12.5f;
constexpr float kcaon = 1.5e6f, kcaoff = 5000.0f, wca = 60000.0f, wnaca = 5000.0f, wna = 60000.0f;
constexpr float KmCaAct = 0.00015f, Gncx = 0.0034f, INaCa_fractionSS = 0.35f;
// NaK pump
constexpr float Knai0 = 9.073f, Knao0 = 27.78f, delta = -0.155f, eP = 4.2f, H = 1.0e-7f, Khp = 1.698e-7f;
constexpr float Knap = 224.0f, Kxkur = 292.0f, k1p = 949.5f, Kki = 0.5f, k1m = 182.4f, MgADP = 0.05f;
constexpr float k2p = 687.2f, k2m = 39.4f, Kko = 0.3582f, k3p = 1899.0f, k3m = 79300.0f, MgATP = 9.8f;
constexpr float Kmgatp = 1.698e-7f, k4p = 639.0f, k4m = 40.0f, Pnak = 15.4509f;
// background currents, Cl
constexpr float GKb = 0.0189f, PNab = 1.9239e-09f, PCab = 5.9194e-08f, GpCa = 0.0005f, KmCap = 0.0005f;
constexpr float GClCa = 0.2843f, KdClCa = 0.1f, GClb = 0.00198f;
// diffusion and SR fluxes
constexpr float tauNa = 2.0f, tauK = 2.0f, tauCa = 0.2f, bt = 4.75f, cajsr_half = 1.7f;
constexpr float Jrel_b = 1.5378f, Jup_b = 1.0f;

__host__ __device__ inline double sq(double x) { return x * x; }

// Driving-force activity coefficient exp(-A z^2 (sqrt(I)/(1+sqrt(I)) - 0.3 I)).
__host__ __device__ inline double activity(double constA, double z2, double I) {
    const double s = pow(I, 0.5);
    return exp(-constA * z2 * (s / (1.0 + s) - (double)0.3f * I));
}

// GHK flux of an ion of valence z (z2 = z^2) between concentration c (with
// its activity coefficient g) and the bath co (gamma go).
__host__ __device__ inline double ghk(double z2, double vffrt, double vfrt_z, double g, double c, double go,
                                      double co) {
    const double e = exp(vfrt_z);
    return z2 * vffrt * (g * c * e - go * co) / (e - 1.0);
}

// NCX of one compartment (sodium na, calcium ca): the allosteric factor and
// the transported charge zNa JNa + zCa JCa.
struct Ncx {
    double allo, J;
};

__host__ __device__ inline Ncx ncx(double na, double ca, double hna, double hca) {
    const double h1 = 1.0 + (na / kna3) * (1.0 + hna);
    const double h2 = (na * hna) / (kna3 * h1);
    const double h3 = 1.0 / h1;
    const double h4 = 1.0 + (na / kna1) * (1.0 + na / kna2);
    const double h5 = (na * na) / (h4 * kna1 * kna2);
    const double h6 = 1.0 / h4;
    const double h7 = 1.0 + ((double)nao / kna3) * (1.0 + 1.0 / hna);
    const double h8 = (double)nao / (kna3 * hna * h7);
    const double h9 = 1.0 / h7;
    const double h10 = (double)kasymm + 1.0 + ((double)nao / kna1) * (1.0 + (double)nao / kna2);
    const double h11 = ((double)nao * nao) / (h10 * kna1 * kna2);
    const double h12 = 1.0 / h10;
    const double k1 = h12 * cao * kcaon, k2 = kcaoff;
    const double k3p_ = h9 * wca, k3pp = h8 * wnaca, k3 = k3p_ + k3pp;
    const double k4p_ = (h3 * wca) / hca, k4pp = h2 * wnaca, k4 = k4p_ + k4pp;
    const double k5 = kcaoff, k6 = h6 * ca * kcaon, k7 = h5 * h2 * wna, k8 = h8 * h11 * wna;
    const double x1 = k2 * k4 * (k7 + k6) + k5 * k7 * (k2 + k3);
    const double x2 = k1 * k7 * (k4 + k5) + k4 * k6 * (k1 + k8);
    const double x3 = k1 * k3 * (k7 + k6) + k8 * k6 * (k2 + k3);
    const double x4 = k2 * k8 * (k4 + k5) + k3 * k5 * (k1 + k8);
    const double sum = x1 + x2 + x3 + x4;
    const double E1 = x1 / sum, E2 = x2 / sum, E3 = x3 / sum, E4 = x4 / sum;
    const double allo = 1.0 / (1.0 + sq((double)KmCaAct / ca));
    const double JNa = (3.0 * (E4 * k7 - E1 * k8) + E3 * k4pp) - E2 * k3pp;
    const double JCa = E2 * k2 - E1 * k1;
    return {allo, JNa + 2.0 * JCa};    // zna = 1, zca = 2
}

// dy/dt of the 43 states for the total stimulus current stim.
__host__ __device__ inline void rhs(const double *y, double stim, double *dy) {
    const double v = y[0], CaMKt = y[1], nai = y[2], nass = y[3], ki = y[4], kss = y[5];
    const double cai = y[6], cass = y[7], cansr = y[8], cajsr = y[9];
    const double m = y[10], h = y[11], j = y[12], hp = y[13], jp = y[14], mL = y[15], hL = y[16];
    const double hLp = y[17], a = y[18], iF = y[19], iS = y[20], ap = y[21], iFp = y[22], iSp = y[23];
    const double d = y[24], ff = y[25], fs = y[26], fcaf = y[27], fcas = y[28], jca = y[29];
    const double ffp = y[30], fcafp = y[31], nca_ss = y[32], nca_i = y[33];
    const double C3 = y[34], C2 = y[35], C1 = y[36], O = y[37], I = y[38];
    const double xs1 = y[39], xs2 = y[40], Jrel_np = y[41], Jrel_p = y[42];

    // geometry: the literal products are float products
    const double vcell = (double)(1000.0f * 3.14f) * rad * rad * L;
    const double Ageo = (double)(2.0f * 3.14f) * rad * rad + (double)(2.0f * 3.14f) * rad * L;
    const double Acap = 2.0 * Ageo;
    const double vmyo = (double)0.68f * vcell, vnsr = (double)0.0552f * vcell;
    const double vjsr = (double)0.0048f * vcell, vss = (double)0.02f * vcell;

    const double RT = (double)R * T;
    const double vffrt = (v * F * F) / RT, vfrt = (v * F) / RT;
    const double RTF = RT / F;                 // zna = zk = 1
    const double ENa = RTF * log((double)nao / nai);
    const double EK = RTF * log((double)ko / ki);
    const double EKs = RTF * log(((double)ko + (double)PKNa * nao) / (ki + (double)PKNa * nai));
    const double ECl = (RT / (-1.0 * F)) * log((double)clo / cli);   // zcl = -1

    // CaMK and the phosphorylated fractions of INa, INaL, Ito, ICaL, Jrel, Jup
    const double CaMKb = (CaMKo * (1.0 - CaMKt)) / (1.0 + KmCaM / cass);
    const double CaMKa = CaMKb + CaMKt;
    const double fp_ = 1.0 / (1.0 + KmCaMK / CaMKa);

    // buffering factors
    const double Bcai = 1.0 / (1.0 + (cmdnmax * (double)kmcmdn) / sq(kmcmdn + cai) +
                               ((double)trpnmax * kmtrpn) / sq(kmtrpn + cai));
    const double Bcass = 1.0 / (1.0 + ((double)BSRmax * KmBSR) / sq(KmBSR + cass) +
                                ((double)BSLmax * KmBSL) / sq(KmBSL + cass));
    const double Bcajsr = 1.0 / (1.0 + ((double)csqnmax * kmcsqn) / sq(kmcsqn + cajsr));

    // INa
    const double mss = 1.0 / sq(1.0 + exp(-(v + 56.86f) / 9.03f));
    const double tm = 0.1292f * exp(-sq((v + 45.79f) / 15.54f)) + 0.06487f * exp(-sq((v - 4.823f) / 51.12f));
    const double hss = 1.0 / sq(1.0 + exp((v + 71.55f) / 7.43f));
    const double hssp = 1.0 / sq(1.0 + exp((v + 77.55f) / 7.43f));
    double ah, bh, aj, bj;
    if (v >= -40.0f) {
        ah = 0.0;
        bh = 0.77f / (0.13f * (1.0 + exp(-(v + 10.66f) / 11.1f)));
        aj = 0.0;
        bj = (0.6f * exp(0.057f * v)) / (1.0 + exp(-0.1f * (v + 32.0f)));
    } else {
        ah = 0.057f * exp(-(v + 80.0f) / 6.8f);
        bh = 2.7f * exp(0.079f * v) + 3.1e5 * exp(0.3485f * v);
        aj = ((-2.5428e4 * exp(0.2444f * v) - 6.948e-6 * exp(-0.04391f * v)) * (v + 37.78f)) /
             (1.0 + exp(0.311f * (v + 79.23f)));
        bj = (0.02424f * exp(-0.01052f * v)) / (1.0 + exp(-0.1378f * (v + 40.14f)));
    }
    const double th = 1.0 / (ah + bh), tj = 1.0 / (aj + bj), tjp = 1.46f * tj;
    const double INa = GNa * (v - ENa) * (m * m * m) * ((1.0 - fp_) * h * j + fp_ * hp * jp);

    // INaL
    const double mLss = 1.0 / (1.0 + exp(-(v + 42.85f) / 5.264f));
    const double hLss = 1.0 / (1.0 + exp((v + 87.61f) / 7.488f));
    const double hLssp = 1.0 / (1.0 + exp((v + 93.81f) / 7.488f));
    const double thLp = 3.0f * thL;
    const double INaL = GNaL * (v - ENa) * mL * ((1.0 - fp_) * hL + fp_ * hLp);

    // Ito (EKshift = 0, endo: delta_epi = 1)
    const double ass = 1.0 / (1.0 + exp(-(v - 14.34f) / 14.82f));
    const double assp = 1.0 / (1.0 + exp(-(v - 24.34f) / 14.82f));
    const double ta = 1.0515f / (1.0 / (1.2089f * (1.0 + exp(-(v - 18.4099f) / 29.3814f))) +
                                 3.5f / (1.0 + exp((v + 100.0f) / 29.3814f)));
    const double iss = 1.0 / (1.0 + exp((v + 43.94f) / 5.711f));
    const double tiF = 4.562f + 1.0 / (0.3933f * exp(-(v + 100.0f) / 100.0f) + 0.08004f * exp((v + 50.0f) / 16.59f));
    const double tiS = 23.62f + 1.0 / (0.001416f * exp(-(v + 96.52f) / 59.05f) + 1.78e-8 * exp((v + 114.1f) / 8.079f));
    const double AiF = 1.0 / (1.0 + exp((v - 213.6f) / 151.2f)), AiS = 1.0 - AiF;
    const double dti_develop = 1.354f + 1.0e-4 / (exp((v - 167.4f) / 15.89f) + exp(-(v - 12.23f) / 0.2154f));
    const double dti_recover = 1.0 - 0.5f / (1.0 + exp((v + 70.0f) / 20.0f));
    const double tiFp = dti_develop * dti_recover * tiF, tiSp = dti_develop * dti_recover * tiS;
    const double ii = AiF * iF + AiS * iS, ip = AiF * iFp + AiS * iSp;
    const double Ito = Gto * (v - EK) * ((1.0 - fp_) * a * ii + fp_ * ap * ip);

    // ICaL, ICaNa, ICaK (offset = vShift = 0)
    const double dss = (v >= 31.4978f) ? 1.0 : 1.0763f * exp(-1.007f * exp(-0.0829f * v));
    const double td = 0.6f + 1.0 / (exp(-0.05f * (v + 6.0f)) + exp(0.09f * (v + 14.0f)));
    const double fss = 1.0 / (1.0 + exp((v + 19.58f) / 3.696f));
    const double tff = 7.0f + 1.0 / (0.0045f * exp(-(v + 20.0f) / 10.0f) + 0.0045f * exp((v + 20.0f) / 10.0f));
    const double tfs = 1000.0f + 1.0 / (3.5e-5f * exp(-(v + 5.0f) / 4.0f) + 3.5e-5f * exp((v + 5.0f) / 6.0f));
    const double Afs = 1.0 - (double)Aff;
    const double f = Aff * ff + Afs * fs, fp = Aff * ffp + Afs * fs;
    const double tfcaf = 7.0f + 1.0 / (0.04f * exp(-(v - 4.0f) / 7.0f) + 0.04f * exp((v - 4.0f) / 7.0f));
    const double tfcas = 100.0f + 1.0 / (0.00012f * exp(-v / 3.0f) + 0.00012f * exp(v / 7.0f));
    const double Afcaf = 0.3f + 0.6f / (1.0 + exp((v - 10.0f) / 10.0f)), Afcas = 1.0 - Afcaf;
    const double fca = Afcaf * fcaf + Afcas * fcas, fcap = Afcaf * fcafp + Afcas * fcas;
    const double jcass = 1.0 / (1.0 + exp((v + 18.08f) / 2.7916f));
    const double tffp = 2.5f * tff, tfcafp = 2.5f * tfcaf;
    const double km2n = jca;
    const double anca_ss = 1.0 / (k2n / km2n + pow(1.0 + Kmn / cass, 4.0));
    const double anca_i = 1.0 / (k2n / km2n + pow(1.0 + Kmn / cai, 4.0));
    const double constA = 1.82e6 * pow((double)dielConstant * T, -1.5);
    const double Io = (0.5f * ((double)nao + ko + clo + 4.0f * cao)) / 1000.0f;
    const double Iss = (0.5f * (nass + kss + cli + 4.0f * cass)) / 1000.0f;
    const double Ii = (0.5f * (nai + ki + cli + 4.0f * cai)) / 1000.0f;
    const double g_cass = activity(constA, 4.0, Iss), g_cao = activity(constA, 4.0, Io);
    const double g_nass = activity(constA, 1.0, Iss), g_nao = activity(constA, 1.0, Io);
    const double g_kss = activity(constA, 1.0, Iss), g_ko = activity(constA, 1.0, Io);
    const double g_cai = activity(constA, 4.0, Ii), g_nai = activity(constA, 1.0, Ii);
    const double g_ki = activity(constA, 1.0, Ii);
    const double PhiCaL_ss = ghk(4.0, vffrt, 2.0 * vfrt, g_cass, cass, g_cao, cao);
    const double PhiCaNa_ss = ghk(1.0, vffrt, vfrt, g_nass, nass, g_nao, nao);
    const double PhiCaK_ss = ghk(1.0, vffrt, vfrt, g_kss, kss, g_ko, ko);
    const double PhiCaL_i = ghk(4.0, vffrt, 2.0 * vfrt, g_cai, cai, g_cao, cao);
    const double PhiCaNa_i = ghk(1.0, vffrt, vfrt, g_nai, nai, g_nao, nao);
    const double PhiCaK_i = ghk(1.0, vffrt, vfrt, g_ki, ki, g_ko, ko);
    const double PCap = 1.1f * (double)PCa;
    const double PCaNa = 0.00125f * (double)PCa, PCaNap = 0.00125f * PCap;
    const double PCaK = 3.574e-4 * (double)PCa, PCaKp = 3.574e-4 * PCap;
    // the L-type channel carrying one ion (permeabilities P, Pp when
    // phosphorylated; flux Phi) in the subspace (nca = nca_ss) or in the bulk
    // myoplasm (nca = nca_i)
    auto chan = [&](double frac, double P_, double Pp_, double Phi, double nca) {
        return frac * ((1.0 - fp_) * P_ * Phi * d * (f * (1.0 - nca) + jca * fca * nca) +
                       fp_ * Pp_ * Phi * d * (fp * (1.0 - nca) + jca * fcap * nca));
    };
    const double fSS = ICaL_fractionSS, fI = 1.0 - (double)ICaL_fractionSS;
    const double ICaL_ss = chan(fSS, PCa, PCap, PhiCaL_ss, nca_ss);
    const double ICaNa_ss = chan(fSS, PCaNa, PCaNap, PhiCaNa_ss, nca_ss);
    const double ICaK_ss = chan(fSS, PCaK, PCaKp, PhiCaK_ss, nca_ss);
    const double ICaL_i = chan(fI, PCa, PCap, PhiCaL_i, nca_i);
    const double ICaNa_i = chan(fI, PCaNa, PCaNap, PhiCaNa_i, nca_i);
    const double ICaK_i = chan(fI, PCaK, PCaKp, PhiCaK_i, nca_i);
    const double ICaL = ICaL_ss + ICaL_i, ICaNa = ICaNa_ss + ICaNa_i, ICaK = ICaK_ss + ICaK_i;

    // IKr: five-state Markov chain
    const double al = 0.1161f * exp(0.299f * vfrt), be = 0.2442f * exp(-1.604f * vfrt);
    const double al2 = 0.0578f * exp(0.971f * vfrt), be2 = 0.349e-3 * exp(-1.062f * vfrt);
    const double ali = 0.2533f * exp(0.5953f * vfrt), bei = 0.06525f * exp(-0.8209f * vfrt);
    const double alC2I = 0.52e-4 * exp(1.525f * vfrt);
    const double beIC2 = (be2 * bei * alC2I) / (al2 * ali);
    const double sqrt_ko5 = pow((double)ko / 5.0f, 0.5);
    const double IKr = GKr * sqrt_ko5 * O * (v - EK);

    // IKs
    const double xs1ss = 1.0 / (1.0 + exp(-(v + 11.6f) / 8.932f));
    const double txs1 = 817.3f + 1.0 / (2.326e-4 * exp((v + 48.28f) / 17.8f) + 0.001292f * exp(-(v + 210.0f) / 230.0f));
    const double txs2 = 1.0 / (0.01f * exp((v - 50.0f) / 20.0f) + 0.0193f * exp(-(v + 66.54f) / 31.0f));
    const double KsCa = 1.0 + 0.6f / (1.0 + pow(3.8e-5 / cai, (double)1.4f));
    const double IKs = GKs * KsCa * xs1 * xs2 * (v - EKs);

    // IK1
    const double dvk = v - EK;
    const double aK1 = 4.094f / (1.0 + exp(0.1217f * (dvk - 49.934f)));
    const double bK1 = (15.72f * exp(0.0674f * (dvk - 3.257f)) + exp(0.0618f * (dvk - 594.31f))) /
                       (1.0 + exp(-0.1629f * (dvk + 14.207f)));
    const double IK1 = GK1 * sqrt_ko5 * (aK1 / (aK1 + bK1)) * dvk;

    // INaCa
    const double hca = exp(qca * vfrt), hna = exp(qna * vfrt);
    const Ncx nx_i = ncx(nai, cai, hna, hca), nx_ss = ncx(nass, cass, hna, hca);
    const double INaCa_i = (1.0 - (double)INaCa_fractionSS) * Gncx * nx_i.allo * nx_i.J;
    const double INaCa_ss = INaCa_fractionSS * (double)Gncx * nx_ss.allo * nx_ss.J;

    // INaK
    const double Knai = Knai0 * exp((delta * vfrt) / 3.0f);
    const double Knao = Knao0 * exp(((1.0 - (double)delta) * vfrt) / 3.0f);
    const double P = eP / (1.0 + (double)H / Khp + nai / Knap + ki / Kxkur);
    const double den_i = (pow(1.0 + nai / Knai, 3.0) + sq(1.0 + ki / Kki)) - 1.0;
    const double den_o = (pow(1.0 + nao / Knao, 3.0) + sq(1.0 + (double)ko / Kko)) - 1.0;
    const double a1 = (k1p * pow(nai / Knai, 3.0)) / den_i;
    const double b1 = (double)k1m * MgADP, a2 = k2p;
    const double b2 = (k2m * pow(nao / Knao, 3.0)) / den_o;
    const double a3 = (k3p * sq((double)ko / Kko)) / den_o;
    const double b3 = (k3m * P * H) / (1.0 + (double)MgATP / Kmgatp);
    const double a4 = (((double)k4p * MgATP) / Kmgatp) / (1.0 + (double)MgATP / Kmgatp);
    const double b4 = (k4m * sq(ki / Kki)) / den_i;
    const double x1 = a4 * a1 * a2 + b2 * b4 * b3 + a2 * b4 * b3 + b3 * a1 * a2;
    const double x2 = b2 * b1 * b4 + a1 * a2 * a3 + a3 * b1 * b4 + a2 * a3 * b4;
    const double x3 = a2 * a3 * a4 + b3 * b2 * b1 + b2 * b1 * a4 + a3 * a4 * b1;
    const double x4 = b4 * b3 * b2 + a3 * a4 * a1 + b2 * a4 * a1 + b3 * b2 * a1;
    const double xs = x1 + x2 + x3 + x4;
    const double JnakNa = 3.0 * ((x1 / xs) * a3 - (x2 / xs) * b3);
    const double JnakK = 2.0 * ((x4 / xs) * b1 - (x3 / xs) * a1);
    const double INaK = Pnak * (JnakNa + JnakK);

    // background and chloride currents
    const double xkb = 1.0 / (1.0 + exp(-(v - 10.8968f) / 23.9871f));
    const double IKb = GKb * xkb * (v - EK);
    const double INab = (PNab * vffrt * (nai * exp(vfrt) - nao)) / (exp(vfrt) - 1.0);
    const double ICab = (PCab * 4.0f * vffrt * (g_cai * cai * exp(2.0 * vfrt) - g_cao * cao)) / (exp(2.0 * vfrt) - 1.0);
    const double IpCa = (GpCa * cai) / (KmCap + cai);
    const double IClCa = (GClCa / (1.0 + KdClCa / cass)) * (v - ECl);   // Fjunc = 1: junctional part only
    const double IClb = GClb * (v - ECl);

    // SR release, uptake, transfer, diffusion
    const double JdiffNa = (nass - nai) / tauNa, JdiffK = (kss - ki) / tauK, Jdiff = (cass - cai) / tauCa;
    const double relK = 1.0 + pow((double)cajsr_half / cajsr, 8.0);
    const double Jrel_inf = ((-(0.5f * (double)bt)) * ICaL_ss) / relK;
    const double btp = 1.25f * (double)bt;
    const double Jrel_infp = ((-(0.5f * btp)) * ICaL_ss) / relK;
    double tau_rel = bt / (1.0 + 0.0123f / cajsr);
    if (tau_rel < 0.001f) tau_rel = 0.001f;
    double tau_relp = btp / (1.0 + 0.0123f / cajsr);
    if (tau_relp < 0.001f) tau_relp = 0.001f;
    const double Jrel = Jrel_b * ((1.0 - fp_) * Jrel_np + fp_ * Jrel_p);
    const double Jupnp = (0.005425f * cai) / (cai + 0.00092f);
    const double Jupp = (2.75f * (double)0.005425f * cai) / ((cai + 0.00092f) - 0.00017f);
    const double Jleak = (0.0048825f * cansr) / 15.0f;
    const double Jup = Jup_b * (((1.0 - fp_) * Jupnp + fp_ * Jupp) - Jleak);
    const double Jtr = (cansr - cajsr) / 60.0f;

    // derivatives
    dy[0] = -(INa + INaL + Ito + ICaL + ICaNa + ICaK + IKr + IKs + IK1 + INaCa_i + INaCa_ss + INaK + INab + IKb +
              IpCa + ICab + IClCa + IClb + stim);
    dy[1] = aCaMK * CaMKb * (CaMKb + CaMKt) - bCaMK * CaMKt;
    dy[2] = (-(INa + INaL + 3.0 * INaCa_i + ICaNa_i + 3.0 * INaK + INab) * Acap) / (F * vmyo) + (JdiffNa * vss) / vmyo;
    dy[3] = (-(ICaNa_ss + 3.0 * INaCa_ss) * Acap) / (F * vss) - JdiffNa;
    dy[4] = (-(ICaK_i + Ito + IKr + IKs + IK1 + IKb + stim - 2.0 * INaK) * Acap) / (F * vmyo) + (JdiffK * vss) / vmyo;
    dy[5] = (-ICaK_ss * Acap) / (F * vss) - JdiffK;
    dy[6] = Bcai * (((-(ICaL_i + IpCa + ICab - 2.0 * INaCa_i)) * Acap) / (2.0 * F * vmyo) - (Jup * vnsr) / vmyo +
                    (Jdiff * vss) / vmyo);
    dy[7] = Bcass * ((-(ICaL_ss - 2.0 * INaCa_ss) * Acap) / (2.0 * F * vss) + (Jrel * vjsr) / vss - Jdiff);
    dy[8] = Jup - (Jtr * vjsr) / vnsr;
    dy[9] = Bcajsr * (Jtr - Jrel);
    dy[10] = (mss - m) / tm;
    dy[11] = (hss - h) / th;
    dy[12] = (hss - j) / tj;            // jss = hss
    dy[13] = (hssp - hp) / th;
    dy[14] = (hss - jp) / tjp;
    dy[15] = (mLss - mL) / tm;          // tmL = tm
    dy[16] = (hLss - hL) / thL;
    dy[17] = (hLssp - hLp) / thLp;
    dy[18] = (ass - a) / ta;
    dy[19] = (iss - iF) / tiF;
    dy[20] = (iss - iS) / tiS;
    dy[21] = (assp - ap) / ta;
    dy[22] = (iss - iFp) / tiFp;
    dy[23] = (iss - iSp) / tiSp;
    dy[24] = (dss - d) / td;
    dy[25] = (fss - ff) / tff;
    dy[26] = (fss - fs) / tfs;
    dy[27] = (fss - fcaf) / tfcaf;      // fcass = fss
    dy[28] = (fss - fcas) / tfcas;
    dy[29] = (jcass - jca) / tjca;
    dy[30] = (fss - ffp) / tffp;
    dy[31] = (fss - fcafp) / tfcafp;
    dy[32] = anca_ss * k2n - nca_ss * km2n;
    dy[33] = anca_i * k2n - nca_i * km2n;
    dy[34] = be * C2 - al * C3;
    dy[35] = (al * C3 + beta_1 * C1) - (be + alpha_1) * C2;
    dy[36] = (alpha_1 * C2 + be2 * O + beIC2 * I) - (beta_1 + al2 + alC2I) * C1;
    dy[37] = (al2 * C1 + bei * I) - (be2 + ali) * O;
    dy[38] = (alC2I * C1 + ali * O) - (beIC2 + bei) * I;
    dy[39] = (xs1ss - xs1) / txs1;
    dy[40] = (xs1ss - xs2) / txs2;      // xs2ss = xs1ss
    dy[41] = (Jrel_inf - Jrel_np) / tau_rel;
    dy[42] = (Jrel_infp - Jrel_p) / tau_relp;
}

// Initial state of the library's CPU build (ToRORd_fkatp_endo.c:30-76): float
// literals.  INITIAL_V (ToRORd_fkatp_endo.h:5) is its V.
__host__ __device__ inline double initial_state_cpu(int s) {
    const float y0[NEQ] = {
        -88.7638f, 0.0111f, 12.1025f, 12.1029f, 142.3002f, 142.3002f, 8.1583e-05f, 7.0305e-05f, 1.5211f, 1.5214f,
        8.0572e-04f, 0.8286f, 0.8284f, 0.6707f, 0.8281f, 1.629e-04f, 0.5255f, 0.2872f, 9.5098e-04f, 0.9996f,
        0.5936f, 4.8454e-04f, 0.9996f, 0.6538f, 8.1084e-09f, 1.0f, 0.939f, 1.0f, 0.9999f, 1.0f,
        1.0f, 1.0f, 6.6462e-04f, 0.0012f, 0.9981f, 8.5109e-04f, 7.0344e-04f, 3.7585e-04f, 1.3289e-05f, 0.248f,
        1.7707e-04f, 1.6129e-22f, 1.2475e-20f};
    return (double)y0[s];
}

// Initial state of the library's GPU build (ToRORd_fkatp_endo.cu:8-50):
// double literals, a different steady state.
__host__ __device__ inline double initial_state_gpu(int s) {
    const double y0[NEQ] = {
        -88.8691566357934, 0.0110752904836162, 12.0996647655188, 12.1000028563765, 142.412524737626,
        142.412481425842, 7.45541572746214e-05, 6.50418928341426e-05, 1.53037019085812, 1.52803094224238,
        0.000787657400526199, 0.830658198588696, 0.830466744399495, 0.674096901201792, 0.830093612199637,
        0.000159670117055769, 0.528261721740178, 0.288775833197764, 0.000944249645410894, 0.999616956857814,
        0.593680589620082, 0.000481107253796778, 0.999616964658062, 0.654092074678260, 8.86091322819384e-29,
        0.999999992783113, 0.938965241412012, 0.999999992783179, 0.999900458262832, 0.999977476316330,
        0.999999992566681, 0.999999992766279, 0.000492094765239740, 0.000833711885764158, 0.998073652444028,
        0.000844745297078649, 0.000698171876592920, 0.000370404872169913, 1.30239063420973e-05, 0.247156543918935,
        0.000175017075236424, 3.90843796133124e-24, -1.88428892080206e-22};
    return y0[s];
}

// Adaptive Euler / Heun step of one cell to final_time (default_solvers.c:
// 55-175): an Euler step of size dt is accepted when half the difference of
// the slopes at its two ends, over max(abs_tol, rel_tol |y_new|), stays below
// 1 for every state (or dt is already min_dt); the next dt is
// 0.8 dt / sqrt(error), clamped to [min_dt, max_dt] and to the time left.
// The cell's dt, time_new and previous_dt persist between calls.  Returns
// false if max_iterations passes did not reach final_time (the state is left
// as it stands).
struct Adaptive {
    double min_dt, max_dt, abs_tol, rel_tol;
    int max_iterations;
};

__host__ __device__ inline bool adaptive_step(double *y, double stim, double final_time, const Adaptive &p,
                                              double &dt, double &time_new, double &previous_dt) {
    double k1[NEQ], k2[NEQ], old[NEQ], eul[NEQ];
    const double tiny = pow(p.abs_tol, 2.0);
    previous_dt = dt;
    if (time_new + dt > final_time) dt = final_time - time_new;
    rhs(y, stim, k1);
    time_new += dt;
    for (int it = 0; it < p.max_iterations; ++it) {
        for (int s = 0; s < NEQ; ++s) {
            old[s] = y[s];
            eul[s] = k1[s] * dt + old[s];
            y[s] = eul[s];
        }
        rhs(y, stim, k2);
        double err = 0.0;
        for (int s = 0; s < NEQ; ++s) {
            const double rt = fabs(eul[s]) * p.rel_tol;
            const double tol = p.abs_tol > rt ? p.abs_tol : rt;
            const double e = fabs(((dt / 2.0) * (k1[s] - k2[s])) / tol);
            err = e > err ? e : err;
        }
        err += tiny;
        previous_dt = dt;
        dt = 0.8 * dt * sqrt(1.0f / err);
        if (dt < p.min_dt) dt = p.min_dt;
        else if (dt > p.max_dt) dt = p.max_dt;
        if (time_new + dt > final_time) dt = final_time - time_new;
        if (err >= 1.0f && dt > p.min_dt) {
            for (int s = 0; s < NEQ; ++s) y[s] = old[s];     // rejected: again from the old state
            continue;
        }
        for (int s = 0; s < NEQ; ++s) {
            k1[s] = k2[s];
            y[s] = eul[s];
        }
        if (time_new + previous_dt >= final_time) {
            if (final_time == time_new) return true;
            if (time_new < final_time) {
                dt = previous_dt = final_time - time_new;
                time_new += previous_dt;
                return true;
            }
        } else {
            time_new += previous_dt;
        }
    }
    return false;
}

}  // namespace mb_tore
