/*
 * CPU oracle for the NeuroGPU simulation step -- TEST INFRASTRUCTURE ONLY
 * (the checker; see oracle.h).  Compiled twice: ONG_REAL=double -> *_f64,
 * ONG_REAL=float -> *_f32.  The f32 build keeps the reference's storage
 * split (U/Util.h:7-9): voltages, gating states, parameters and channel
 * arithmetic in float (MYFTYPE), the tree matrix and its solve in double
 * (MYSECONDFTYPE).  It does not reproduce the double promotions inside the
 * reference's generated channel expressions; it is a precision probe, the
 * f64 build is the parity reference.
 *
 * Every function below restates the reference's arithmetic; each cites the
 * file:line it follows.  Paths are relative to the reference project:
 *   U/  = GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/
 *   MN/ = Figures/FigureS4_mainen/CParsed/
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef ONG_REAL
#define ONG_REAL double
#endif
typedef ONG_REAL real;

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#ifdef ONG_SUFFIX_F32
#define SFX(name) CAT(name, _f32)
#else
#define SFX(name) CAT(name, _f64)
#endif

/* ---- universal constants, U/AllModels.cu:10-36 and MN/AllModels.cu:9-67 ---- */
#define FARADAY 96485.309
#define DEF_CAI 5.e-5
#define DEF_CAO 2.
static real ktf_of(real celsius) { return (real)(1000. * 8.3134 * (celsius + 273.15) / FARADAY); }

/* cnexp update x += (1 - exp(-dt/tau)) (xinf - x)   (U/AllModels.cu:303-304) */
static inline real cnexp(real x, real xinf, real tau, real dt) {
    return x + ((real)1. - exp(-dt / tau)) * (xinf - x);
}

/* ======================= TTPC set: U/AllModels.cu ======================= */
#define T_NSTATES 19
#define T_NPARAMS 19
#define T_NMECH 13
#define T_CELSIUS 34.0
#define T_ENA 50.0
#define T_EK (-85.0)
static real t_qt(void) { return (real)pow(2.3, (34.0 - 21.0) / 10.0); } /* U/AllModels.cu:81 */

/* U/AllModels.cu:66-78 */
static void t_rates_Ca_HVA(real v, real *mInf, real *mTau, real *hInf, real *hTau) {
    if (v == -27.0) v = v + 0.0001;
    real mA = (0.055 * (-27.0 - v)) / (exp((-27.0 - v) / 3.8) - 1.0);
    real mB = (0.94 * exp((-75.0 - v) / 17.0));
    *mInf = mA / (mA + mB);
    *mTau = 1.0 / (mA + mB);
    real hA = (0.000457 * exp((-13.0 - v) / 50.0));
    real hB = (0.0065 / (exp((-v - 15.0) / 28.0) + 1.0));
    *hInf = hA / (hA + hB);
    *hTau = 1.0 / (hA + hB);
}
/* U/AllModels.cu:79-88 */
static void t_rates_Ca_LVAst(real v, real *mInf, real *mTau, real *hInf, real *hTau) {
    real qt = t_qt();
    v = v + 10.0;
    *mInf = 1.0 / (1.0 + exp((v + 30.0) / -6.0));
    *mTau = (5.0 + 20.0 / (1.0 + exp((v + 25.0) / 5.0))) / qt;
    *hInf = 1.0 / (1.0 + exp((v + 80.0) / 6.4));
    *hTau = (20.0 + 50.0 / (1.0 + exp((v + 40.0) / 7.0))) / qt;
}
/* U/AllModels.cu:89-97 */
static void t_rates_Ih(real v, real *mInf, real *mTau) {
    if (v == -154.9) v = v + 0.0001;
    real mA = 0.001 * 6.43 * (v + 154.9) / (exp((v + 154.9) / 11.9) - 1.0);
    real mB = 0.001 * 193.0 * exp(v / 33.1);
    *mInf = mA / (mA + mB);
    *mTau = 1.0 / (mA + mB);
}
/* U/AllModels.cu:98-105 */
static void t_rates_Im(real v, real *mInf, real *mTau) {
    real qt = t_qt();
    real mA = 3.3e-3 * exp(2.5 * 0.04 * (v + 35.0));
    real mB = 3.3e-3 * exp(-2.5 * 0.04 * (v + 35.0));
    *mInf = mA / (mA + mB);
    *mTau = (1.0 / (mA + mB)) / qt;
}
/* U/AllModels.cu:106-120 */
static void t_rates_K_Pst(real v, real *mInf, real *mTau, real *hInf, real *hTau) {
    real qt = t_qt();
    v = v + 10.0;
    *mInf = (1.0 / (1.0 + exp(-(v + 1.0) / 12.0)));
    if (v < -50.0) *mTau = (1.25 + 175.03 * exp(-v * -0.026)) / qt;
    else *mTau = ((1.25 + 13.0 * exp(-v * 0.026))) / qt;
    *hInf = 1.0 / (1.0 + exp(-(v + 54.0) / -11.0));
    real z = (v + 75.0) / 48.0;
    *hTau = (360.0 + (1010.0 + 24.0 * (v + 55.0)) * exp(-(z * z))) / qt;
}
/* U/AllModels.cu:121-130 */
static void t_rates_K_Tst(real v, real *mInf, real *mTau, real *hInf, real *hTau) {
    real qt = t_qt();
    v = v + 10.0;
    *mInf = 1.0 / (1.0 + exp(-(v + 0.0) / 19.0));
    real zm = (v + 71.0) / 59.0;
    *mTau = (0.34 + 0.92 * exp(-(zm * zm))) / qt;
    *hInf = 1.0 / (1.0 + exp(-(v + 66.0) / -10.0));
    real zh = (v + 73.0) / 23.0;
    *hTau = (8.0 + 49.0 * exp(-(zh * zh))) / qt;
}
/* U/AllModels.cu:131-151 */
static void t_rates_Nap_Et2(real v, real *mInf, real *mTau, real *hInf, real *hTau) {
    real qt = t_qt();
    *mInf = 1.0 / (1.0 + exp((v + 52.6) / -4.6));
    if (v == -38.0) v = v + 0.0001;
    real mA = (0.182 * (v + 38.0)) / (1.0 - (exp(-(v + 38.0) / 6.0)));
    real mB = (0.124 * (-v - 38.0)) / (1.0 - (exp(-(-v - 38.0) / 6.0)));
    *mTau = 6.0 * (1.0 / (mA + mB)) / qt;
    if (v == -17.0) v = v + 0.0001;
    if (v == -64.4) v = v + 0.0001;
    *hInf = 1.0 / (1.0 + exp((v + 48.8) / 10.0));
    real hA = -2.88e-6 * (v + 17.0) / (1.0 - exp((v + 17.0) / 4.63));
    real hB = 6.94e-6 * (v + 64.4) / (1.0 - exp(-(v + 64.4) / 2.63));
    *hTau = (1.0 / (hA + hB)) / qt;
}
/* U/AllModels.cu:152-169 (NaTa_t, vm=-38/-66) and :170-187 (NaTs2_t, -32/-60) */
static void t_rates_NaT(real v, real thm, real thh, real *mInf, real *mTau, real *hInf,
                        real *hTau) {
    real qt = t_qt();
    if (v == thm) v = v + 0.0001;
    real mA = (0.182 * (v - thm)) / (1.0 - (exp(-(v - thm) / 6.0)));
    real mB = (0.124 * (-v + thm)) / (1.0 - (exp(-(-v + thm) / 6.0)));
    *mTau = (1.0 / (mA + mB)) / qt;
    *mInf = mA / (mA + mB);
    if (v == thh) v = v + 0.0001;
    real hA = (-0.015 * (v - thh)) / (1.0 - (exp((v - thh) / 6.0)));
    real hB = (-0.015 * (-v + thh)) / (1.0 - (exp((-v + thh) / 6.0)));
    *hTau = (1.0 / (hA + hB)) / qt;
    *hInf = hA / (hA + hB);
}
/* U/AllModels.cu:188-193 */
static real t_zinf_SK_E2(real ca) {
    if (ca < 1e-7) ca = ca + 1e-07;
    return 1.0 / (1.0 + pow((0.00043 / ca), 4.8));
}
/* U/AllModels.cu:194-197 */
static void t_rates_SKv3_1(real v, real *mInf, real *mTau) {
    *mInf = 1.0 / (1.0 + exp(((v - (18.700)) / (-9.700))));
    *mTau = 0.2 * 20.000 / (1.0 + exp(((v - (-46.560)) / (-44.140))));
}

#define TS_CAI (T_NSTATES)
#define TS_ECA (T_NSTATES + 1)
#define TS_ICA (T_NSTATES + 2)

/* Channel init in mechanism order, U/CudaStuff.cu:219-221 and U/AllModels.cu:202-296.
 * Note the reference's order quirk: Ca_HVA/Ca_LVAst compute eca from cai
 * before CaDynamics_E2 sets cai (cai starts at 0, U/CudaStuff.cu:196-198). */
static void t_init(const unsigned char *mk, real v, const real *p, real *s) {
    real ktf = ktf_of(T_CELSIUS);
    real mi, mt, hi, ht;
    (void)p;
    if (mk[0]) { s[TS_ECA] = ktf / 2 * log(DEF_CAO / s[TS_CAI]);
                 t_rates_Ca_HVA(v, &mi, &mt, &hi, &ht); s[0] = mi; s[1] = hi; }
    if (mk[1]) { s[TS_ECA] = ktf / 2 * log(DEF_CAO / s[TS_CAI]);
                 t_rates_Ca_LVAst(v, &mi, &mt, &hi, &ht); s[2] = mi; s[3] = hi; }
    if (mk[2]) { s[TS_CAI] = DEF_CAI; s[TS_ECA] = ktf / 2 * log(DEF_CAO / s[TS_CAI]); }
    if (mk[3]) { t_rates_Ih(v, &mi, &mt); s[5] = mi; }
    if (mk[4]) { t_rates_Im(v, &mi, &mt); s[6] = mi; }
    if (mk[5]) { t_rates_K_Pst(v, &mi, &mt, &hi, &ht); s[7] = mi; s[8] = hi; }
    if (mk[6]) { t_rates_K_Tst(v, &mi, &mt, &hi, &ht); s[9] = mi; s[10] = hi; }
    if (mk[7]) { t_rates_Nap_Et2(v, &mi, &mt, &hi, &ht); s[11] = mi; s[12] = hi; }
    if (mk[8]) { t_rates_NaT(v, -38.0, -66.0, &mi, &mt, &hi, &ht); s[13] = mi; s[14] = hi; }
    if (mk[9]) { t_rates_NaT(v, -32.0, -60.0, &mi, &mt, &hi, &ht); s[15] = mi; s[16] = hi; }
    if (mk[11]) { s[TS_ECA] = ktf / 2 * log(DEF_CAO / s[TS_CAI]); s[17] = t_zinf_SK_E2(s[TS_CAI]); }
    if (mk[12]) { t_rates_SKv3_1(v, &mi, &mt); s[18] = mi; }
}

/* nrn_state in mechanism order, U/CudaStuff.cu:324-326, U/AllModels.cu:299-377. */
static void t_deriv(const unsigned char *mk, real dt, real v, const real *p, real *s) {
    real ktf = ktf_of(T_CELSIUS);
    real mi, mt, hi, ht;
    if (mk[0]) { t_rates_Ca_HVA(v, &mi, &mt, &hi, &ht);
                 s[0] = cnexp(s[0], mi, mt, dt); s[1] = cnexp(s[1], hi, ht, dt); }
    if (mk[1]) { t_rates_Ca_LVAst(v, &mi, &mt, &hi, &ht);
                 s[2] = cnexp(s[2], mi, mt, dt); s[3] = cnexp(s[3], hi, ht, dt); }
    if (mk[2]) { /* U/AllModels.cu:313-317 */
        real gamma = p[2], decay = p[3], depth = p[4], minCai = p[5];
        real cinf = (-(10000.0) * (s[TS_ICA] * gamma / (2.0 * FARADAY * depth)) + minCai / decay) * decay;
        s[TS_CAI] = cnexp(s[TS_CAI], cinf, decay, dt);
        s[TS_ECA] = ktf / 2 * log(DEF_CAO / s[TS_CAI]);
    }
    if (mk[3]) { t_rates_Ih(v, &mi, &mt); s[5] = cnexp(s[5], mi, mt, dt); }
    if (mk[4]) { t_rates_Im(v, &mi, &mt); s[6] = cnexp(s[6], mi, mt, dt); }
    if (mk[5]) { t_rates_K_Pst(v, &mi, &mt, &hi, &ht);
                 s[7] = cnexp(s[7], mi, mt, dt); s[8] = cnexp(s[8], hi, ht, dt); }
    if (mk[6]) { t_rates_K_Tst(v, &mi, &mt, &hi, &ht);
                 s[9] = cnexp(s[9], mi, mt, dt); s[10] = cnexp(s[10], hi, ht, dt); }
    if (mk[7]) { t_rates_Nap_Et2(v, &mi, &mt, &hi, &ht);
                 s[11] = cnexp(s[11], mi, mt, dt); s[12] = cnexp(s[12], hi, ht, dt); }
    if (mk[8]) { t_rates_NaT(v, -38.0, -66.0, &mi, &mt, &hi, &ht);
                 s[13] = cnexp(s[13], mi, mt, dt); s[14] = cnexp(s[14], hi, ht, dt); }
    if (mk[9]) { t_rates_NaT(v, -32.0, -60.0, &mi, &mt, &hi, &ht);
                 s[15] = cnexp(s[15], mi, mt, dt); s[16] = cnexp(s[16], hi, ht, dt); }
    if (mk[11]) { /* U/AllModels.cu:362-368 */
        real zi = t_zinf_SK_E2(s[TS_CAI]);
        s[17] = cnexp(s[17], zi, p[17], dt);
        s[TS_ECA] = ktf / 2 * log(DEF_CAO / s[TS_CAI]);
    }
    if (mk[12]) { t_rates_SKv3_1(v, &mi, &mt); s[18] = cnexp(s[18], mi, mt, dt); }
}

/* nrn_current in mechanism order, U/AllModels.cu:382-516.  Returns the summed
 * current (mA/cm2); *g the analytic dI/dv; s[ICA] accumulates when acc_ica. */
static real t_current(const unsigned char *mk, real v, const real *p, real *s, real *g,
                      int acc_ica) {
    real I = 0, G = 0, gx;
    if (mk[0]) { gx = p[0] * s[0] * s[0] * s[1]; real i = gx * (v - s[TS_ECA]);
                 I += i; G += gx; if (acc_ica) s[TS_ICA] += i; }
    if (mk[1]) { gx = p[1] * s[2] * s[2] * s[3]; real i = gx * (v - s[TS_ECA]);
                 I += i; G += gx; if (acc_ica) s[TS_ICA] += i; }
    if (mk[3]) { gx = p[6] * s[5]; I += gx * (v - p[7]); G += gx; }
    if (mk[4]) { gx = p[8] * s[6]; I += gx * (v - T_EK); G += gx; }
    if (mk[5]) { gx = p[9] * s[7] * s[7] * s[8]; I += gx * (v - T_EK); G += gx; }
    if (mk[6]) { real m2 = s[9] * s[9]; gx = p[10] * m2 * m2 * s[10]; I += gx * (v - T_EK); G += gx; }
    if (mk[7]) { gx = p[11] * s[11] * s[11] * s[11] * s[12]; I += gx * (v - T_ENA); G += gx; }
    if (mk[8]) { gx = p[12] * s[13] * s[13] * s[13] * s[14]; I += gx * (v - T_ENA); G += gx; }
    if (mk[9]) { gx = p[13] * s[15] * s[15] * s[15] * s[16]; I += gx * (v - T_ENA); G += gx; }
    if (mk[10]) { gx = p[14]; I += gx * (v - p[15]); G += gx; }
    if (mk[11]) { gx = p[16] * s[17]; I += gx * (v - T_EK); G += gx; }
    if (mk[12]) { gx = p[18] * s[18]; I += gx * (v - T_EK); G += gx; }
    *g = G;
    return I;
}

/* ====================== Mainen set: MN/AllModels.cu ====================== */
#define M_NSTATES 8
#define M_NPARAMS 34
#define M_NMECH 9
#define M_CELSIUS 37.0
#define M_ENA 60.0
#define M_EK (-90.0)
#define M_TADJ 3.2093639532679714   /* 2.3^((37-23)/10), MN/AllModels.cu:33 */
#define M_DEPTH_CAD 0.09334562733124982
#define M_CAINF_CAD 0.0001
#define M_TAUR_CAD 200.0
#define M_VSHIFT_NA (-5.0)

/* MN/AllModels.cu:92-112 (efun, trap0) */
static real m_efun(real z) {
    if (fabs(z) < 1e-4) return 1 - z / 2;
    return z / (exp(z) - 1);
}
static real m_trap0(real v, real th, real a, real q) {
    if (fabs((v - th) / q) > 1e-6) return a * (v - th) / (1 - exp(-(v - th) / q));
    return a * q;
}
/* MN/AllModels.cu:117-129 */
static void m_rates_ca(real vm, real *mi, real *mt, real *hi, real *ht) {
    real a = 0.209 * m_efun(-(27.0 + vm) / 3.8);
    real b = 0.94 * exp((-75.0 - vm) / 17.0);
    *mt = 1.0 / M_TADJ / (a + b);
    *mi = a / (a + b);
    a = 0.000457 * exp((-13.0 - vm) / 50.0);
    b = 0.0065 / (exp((-vm - 15.0) / 28.0) + 1.0);
    *ht = 1.0 / M_TADJ / (a + b);
    *hi = a / (a + b);
}
/* MN/AllModels.cu:130-136 */
static void m_rates_kca(real cai, real Ra, real Rb, real caix, real *ni, real *nt) {
    real a = Ra * pow(cai, caix);
    real b = Rb;
    *nt = 1.0 / M_TADJ / (a + b);
    *ni = a / (a + b);
}
/* MN/AllModels.cu:140-146 (km) and :150-156 (kv): same form */
static void m_rates_k(real v, real tha, real qa, real Ra, real Rb, real *ni, real *nt) {
    real a = Ra * qa * m_efun(-(v - tha) / qa);
    real b = Rb * qa * m_efun((v - tha) / qa);
    *nt = 1.0 / M_TADJ / (a + b);
    *ni = a / (a + b);
}
/* MN/AllModels.cu:160-172 */
static void m_rates_na(real vm, const real *q, real *mi, real *mt, real *hi, real *ht) {
    /* q = gbar, tha, qa, Ra, Rb, thi1, thi2, qi, thinf, qinf, Rg, Rd */
    real a = m_trap0(vm, q[1], q[3], q[2]);
    real b = m_trap0(-vm, -q[1], q[4], q[2]);
    *mt = 1.0 / M_TADJ / (a + b);
    *mi = a / (a + b);
    a = m_trap0(vm, q[5], q[11], q[7]);
    b = m_trap0(-vm, -q[6], q[10], q[7]);
    *ht = 1.0 / M_TADJ / (a + b);
    *hi = 1.0 / (1.0 + exp((vm - q[8]) / q[9]));
}
#define MS_CAI (M_NSTATES)
#define MS_ECA (M_NSTATES + 1)
#define MS_ICA (M_NSTATES + 2)

/* MN/AllModels.cu:175-222 in the order of CALL_TO_INIT_STATES_CU (MN/AllModels.cuh:63) */
static void m_init(const unsigned char *mk, real v, const real *p, real *s) {
    real ktf = ktf_of(M_CELSIUS);
    real mi, mt, hi, ht;
    if (mk[0]) { s[MS_ECA] = ktf / 2 * log(DEF_CAO / s[MS_CAI]);
                 m_rates_ca(v, &mi, &mt, &hi, &ht); s[0] = mi; s[1] = hi; }
    if (mk[1]) { s[MS_CAI] = DEF_CAI; s[MS_ECA] = ktf / 2 * log(DEF_CAO / s[MS_CAI]);
                 s[2] = M_CAINF_CAD; s[MS_CAI] = s[2]; }
    if (mk[2]) { s[MS_ECA] = ktf / 2 * log(DEF_CAO / s[MS_CAI]);
                 m_rates_kca(s[MS_CAI], p[4], p[5], p[3], &mi, &mt); s[3] = mi; }
    if (mk[3]) { m_rates_k(v, p[7], p[8], p[9], p[10], &mi, &mt); s[4] = mi; }
    if (mk[4]) { m_rates_k(v, p[12], p[13], p[14], p[15], &mi, &mt); s[5] = mi; }
    if (mk[5]) { m_rates_na(v + M_VSHIFT_NA, p + 16, &mi, &mt, &hi, &ht); s[6] = mi; s[7] = hi; }
}
/* MN/AllModels.cu:228-273 in the order of CALL_TO_DERIV_CU (MN/AllModels.cuh:65) */
static void m_deriv(const unsigned char *mk, real dt, real v, const real *p, real *s) {
    real ktf = ktf_of(M_CELSIUS);
    real mi, mt, hi, ht;
    if (mk[0]) { m_rates_ca(v, &mi, &mt, &hi, &ht);
                 s[0] = cnexp(s[0], mi, mt, dt); s[1] = cnexp(s[1], hi, ht, dt);
                 s[MS_ECA] = ktf / 2 * log(DEF_CAO / s[MS_CAI]); }
    if (mk[1]) {
        real drive = -(10000.0) * s[MS_ICA] / (2.0 * FARADAY * M_DEPTH_CAD);
        if (drive <= 0.) drive = 0.;
        s[2] = cnexp(s[2], (drive + M_CAINF_CAD / M_TAUR_CAD) * M_TAUR_CAD, M_TAUR_CAD, dt);
        s[MS_CAI] = s[2];
        s[MS_ECA] = ktf / 2 * log(DEF_CAO / s[MS_CAI]);
    }
    if (mk[2]) { m_rates_kca(s[MS_CAI], p[4], p[5], p[3], &mi, &mt);
                 s[3] = cnexp(s[3], mi, mt, dt);
                 s[MS_ECA] = ktf / 2 * log(DEF_CAO / s[MS_CAI]); }
    if (mk[3]) { m_rates_k(v, p[7], p[8], p[9], p[10], &mi, &mt); s[4] = cnexp(s[4], mi, mt, dt); }
    if (mk[4]) { m_rates_k(v, p[12], p[13], p[14], p[15], &mi, &mt); s[5] = cnexp(s[5], mi, mt, dt); }
    if (mk[5]) { m_rates_na(v + M_VSHIFT_NA, p + 16, &mi, &mt, &hi, &ht);
                 s[6] = cnexp(s[6], mi, mt, dt); s[7] = cnexp(s[7], hi, ht, dt); }
}
/* MN/AllModels.cu:276-340 in the order of CALL_TO_BREAK_CU (MN/AllModels.cuh:67) */
static real m_current(const unsigned char *mk, real v, const real *p, real *s, real *g,
                      int acc_ica) {
    real I = 0, G = 0, gx;
    if (mk[0]) { gx = 1e-4 * M_TADJ * p[0] * s[0] * s[0] * s[1]; real i = gx * (v - s[MS_ECA]);
                 I += i; G += gx; if (acc_ica) s[MS_ICA] += i; }
    if (mk[2]) { gx = 1e-4 * M_TADJ * p[2] * s[3]; I += gx * (v - M_EK); G += gx; }
    if (mk[3]) { gx = 1e-4 * M_TADJ * p[6] * s[4]; I += gx * (v - M_EK); G += gx; }
    if (mk[4]) { gx = 1e-4 * M_TADJ * p[11] * s[5]; I += gx * (v - M_EK); G += gx; }
    if (mk[5]) { gx = 1e-4 * M_TADJ * p[16] * s[6] * s[6] * s[6] * s[7]; I += gx * (v - M_ENA); G += gx; }
    if (mk[6]) { gx = p[28]; I += gx * (v - p[29]); G += gx; }
    if (mk[7]) { gx = p[30]; I += gx * (v - p[31]); G += gx; }
    if (mk[8]) { gx = p[32]; I += gx * (v - p[33]); G += gx; }
    *g = G;
    return I;
}

/* ============================ set dispatch ============================ */
static int n_states_of(int ms) { return ms == ONG_MECHSET_TTPC ? T_NSTATES : M_NSTATES; }
static int n_params_of(int ms) { return ms == ONG_MECHSET_TTPC ? T_NPARAMS : M_NPARAMS; }
static int n_mechs_of(int ms) { return ms == ONG_MECHSET_TTPC ? T_NMECH : M_NMECH; }

static void node_init(int ms, const unsigned char *mk, real v, const real *p, real *s) {
    if (ms == ONG_MECHSET_TTPC) t_init(mk, v, p, s); else m_init(mk, v, p, s);
}
static void node_deriv(int ms, const unsigned char *mk, real dt, real v, const real *p, real *s) {
    if (ms == ONG_MECHSET_TTPC) t_deriv(mk, dt, v, p, s); else m_deriv(mk, dt, v, p, s);
}
static real node_current(int ms, const unsigned char *mk, real v, const real *p, real *s, real *g,
                         int acc) {
    return ms == ONG_MECHSET_TTPC ? t_current(mk, v, p, s, g, acc) : m_current(mk, v, p, s, g, acc);
}

#ifndef ONG_SUFFIX_F32
int ong_n_params(int ms) { return n_params_of(ms); }
int ong_n_states(int ms) { return n_states_of(ms); }
int ong_n_mechs(int ms) { return n_mechs_of(ms); }

void ong_node_init_f64(int ms, const unsigned char *mask, double v, const double *p, double *s) {
    node_init(ms, mask, v, p, s);
}
void ong_node_deriv_f64(int ms, const unsigned char *mask, double dt, double v, const double *p,
                        double *s) {
    node_deriv(ms, mask, dt, v, p, s);
}
double ong_node_current_f64(int ms, const unsigned char *mask, double v, const double *p,
                            double *s, double *g) {
    return node_current(ms, mask, v, p, s, g, 1);
}
#endif

/*
 * One (parameter set, stimulus) instance for nt steps.
 * Step order follows U/CudaStuff.cu:227-330:
 *   record V (before update)               :243-248
 *   ica = 0; stimulus 100*amp/area at loc  :249-261
 *   currents at v+0.001 and v              :262-267
 *   g=(I(v+eps)-I(v))/eps; rhs=Istim-I;
 *   D=g+cm/(1000 dt)-f; axial terms        :268-291
 *   Hines forward elimination              :31-69 (in excess form, below)
 *   back-substitution                      :72-104
 *   v += dV                                :298-301
 *   cnexp gate / Ca updates at the new v   :324-326
 * The reference tracks dv = V_parent - V_node incrementally from the
 * previous solution; here it is taken directly (identical in exact
 * arithmetic, both start from a uniform v_init).
 */
static void run_instance(const ong_model *m, const float *pset, const float *amp, const float *dts,
                         int nt, int stim_node, double stim_area, int n_rec, const int *rec_nodes,
                         double v_init, int flags, double *out /* [n_rec][nt] */) {
    const int N = m->n_nodes, ms = m->mechset;
    const int NS = n_states_of(ms), NP = n_params_of(ms), NM = n_mechs_of(ms);
    const int SW = NS + 3; /* states + cai, eca, ica */
    real *V = (real *)calloc((size_t)N, sizeof(real));
    real *S = (real *)calloc((size_t)N * SW, sizeof(real));
    real *P = (real *)calloc((size_t)N * NP, sizeof(real));
    double *d = (double *)calloc((size_t)N, sizeof(double));    /* U/CudaStuff.cu:179-180: */
    double *rhs = (double *)calloc((size_t)N, sizeof(double));  /* D, rhs are MYSECONDFTYPE */
    real *tmp = (real *)calloc((size_t)SW, sizeof(real));
    unsigned char *mk = (unsigned char *)calloc((size_t)N * NM, 1);
    for (int i = 0; i < N; ++i) {
        V[i] = (real)v_init;
        for (int j = 0; j < NP; ++j)
            P[(size_t)i * NP + j] = (real)pset[(size_t)j * m->n_sections + m->section[i]];
        for (int k = 0; k < NM; ++k) mk[(size_t)i * NM + k] = m->mech_mask[(size_t)k * N + i];
        node_init(ms, mk + (size_t)i * NM, V[i], P + (size_t)i * NP, S + (size_t)i * SW);
    }
    const real eps = (real)0.001; /* EPS_V, U/Util.h:22 */
    for (int t = 0; t < nt; ++t) {
        const real dt = (real)dts[t];
        for (int r = 0; r < n_rec; ++r) out[(size_t)r * nt + t] = (double)V[rec_nodes[r]];
        for (int i = 0; i < N; ++i) {
            real *s = S + (size_t)i * SW;
            const real *p = P + (size_t)i * NP;
            const unsigned char *k = mk + (size_t)i * NM;
            s[NS + 2] = 0; /* ica reset, U/CudaStuff.cu:257 */
            real I, g;
            if (flags & ONG_FLAG_FD_CONDUCTANCE) {
                memcpy(tmp, s, sizeof(real) * SW);
                real gdum;
                real Idv = node_current(ms, k, V[i] + eps, p, tmp, &gdum, 1);
                I = node_current(ms, k, V[i], p, s, &gdum, 1);
                g = (Idv - I) / eps;
            } else {
                I = node_current(ms, k, V[i], p, s, &g, 1);
            }
            real istim = (i == stim_node) ? (real)(100.0 * (double)amp[t] / stim_area) : (real)0;
            rhs[i] = (double)istim - (double)I;
            /* the row's excess: its grounded conductance g + cm/(1000 dt) */
            d[i] = (double)g + (double)(real)((real)m->cm[i] / (dt * (real)1000));
        }
        for (int i = 1; i < N; ++i) {
            int p = m->parent[i];
            real dv = V[p] - V[i];
            rhs[i] -= m->a[i] * (double)dv;
            rhs[p] += m->b[i] * (double)dv;
        }
        /* leaf -> root elimination in excess form: row i's diagonal is its
         * excess minus its coupling a_i (children already folded in); the
         * child hands -b_i x_i / d_i to the parent's excess and -b_i rhs_i / d_i
         * to its right-hand side.  Algebraically the reference's update
         * u_p -= f e / u_i (U/CudaStuff.cu:31-69), without its cancellation of
         * nearly equal diagonal terms, which costs ~1e-5 relative in FP64 on
         * trees that join near zero-area compartments (couplings ~1e21) to
         * ordinary ones. */
        for (int i = N - 1; i >= 1; --i) {
            int p = m->parent[i];
            double di = d[i] - m->a[i];
            d[p] += -m->b[i] * (d[i] / di);
            rhs[p] += -m->b[i] * (rhs[i] / di);
            d[i] = di;
        }
        rhs[0] /= d[0];
        for (int i = 1; i < N; ++i) /* root -> leaf back-substitution */
            rhs[i] = (rhs[i] - m->a[i] * rhs[m->parent[i]]) / d[i];
        for (int i = 0; i < N; ++i) {
            V[i] += (real)rhs[i];
            node_deriv(ms, mk + (size_t)i * NM, dt, V[i], P + (size_t)i * NP, S + (size_t)i * SW);
        }
    }
    free(V); free(S); free(P); free(d); free(rhs); free(tmp); free(mk);
}

int SFX(ong_run)(const ong_model *m, int n_sets, const float *params, int n_stim, int nt,
                 const float *amps, const float *dts, int stim_node, double stim_area, int n_rec,
                 const int *rec_nodes, double v_init, int flags, double *out, int n_threads) {
    if (!m || m->n_nodes < 1 || n_sets < 0 || n_stim < 1 || nt < 0) return -1;
    if (m->mechset != ONG_MECHSET_TTPC && m->mechset != ONG_MECHSET_MAINEN) return -2;
    if (m->parent[0] != -1) return -3;
    for (int i = 1; i < m->n_nodes; ++i)
        if (m->parent[i] < 0 || m->parent[i] >= i) return -3;
    if (stim_node < 0 || stim_node >= m->n_nodes || !(stim_area > 0)) return -4;
    for (int r = 0; r < n_rec; ++r)
        if (rec_nodes[r] < 0 || rec_nodes[r] >= m->n_nodes) return -5;
    const int NP = n_params_of(m->mechset);
    const long total = (long)n_sets * n_stim;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 1)
#else
    (void)n_threads;
#endif
    for (long inst = 0; inst < total; ++inst) {
        int k = (int)(inst / n_stim), s = (int)(inst % n_stim);
        run_instance(m, params + (size_t)k * NP * m->n_sections, amps + (size_t)s * nt, dts, nt,
                     stim_node, stim_area, n_rec, rec_nodes, v_init, flags,
                     out + ((size_t)k * n_stim + s) * n_rec * nt);
    }
    return 0;
}
