// Mainen channel set (9 mechanisms) for the fused simulation kernel.
//
// Equations follow the reference's generated channel library for the
// Mainen & Sejnowski model, Figures/FigureS4_mainen/CParsed/AllModels.cu
// (efun/trap0 :92-112, rates :117-172, init :175-222, cnexp derivs
// :228-273, breakpoints :276-340), with the mechanism, parameter and state
// order of its CALL_TO_* expansion (CParsed/AllModels.cuh:63-67).
// trap0(v, th, a, q) is written as a*q*efun(-(v-th)/q), the same function.
// As in the TTPC set, the membrane conductance is the analytic dI/dv.
//
// State rows, in order, for the mechanisms present:
//   ca m,h | cad ca,ica | kca n | km n | kv n | na m,h | (pas, pas2, pasx: none)
#pragma once
#include "channels_ttpc.cuh"  // efun, sigm, ab_gate, cnexp_rate

namespace ngpu {

struct Mainen {
    static constexpr int kNMech = 9;
    static constexpr int kNParams = 34;
    enum : uint32_t {
        kCa = 1u << 0, kCad = 1u << 1, kKca = 1u << 2, kKm = 1u << 3, kKv = 1u << 4,
        kNa = 1u << 5, kPas = 1u << 6, kPas2 = 1u << 7, kPasx = 1u << 8
    };
    static constexpr double kCelsius = 37.0;
    static constexpr double kEna = 60.0, kEk = -90.0;
    static constexpr double kTadj = 3.2093639532679714;  // 2.3^((37-23)/10)
    static constexpr double kDepthCad = 0.09334562733124982;
    static constexpr double kCainfCad = 0.0001;
    static constexpr double kTaurCad = 200.0;
    static constexpr double kVshiftNa = -5.0;
};

template <typename R, bool INIT>
NGPU_HD void mainen_node(uint32_t mk, R v, R dt, R* __restrict__ st,
                                            const float* __restrict__ pr, R& I, R& G) {
    using M = Math<R>;
    constexpr int S = 32;
    const R tadj = (R)Mainen::kTadj;
    int s = 0, q = 0;
    R Itot = 0, Gtot = 0;
    R mi, mr, hi, hr;
    R ca_m = 0, ca_h = 0, ca_g = 0;
    if (mk & Mainen::kCa) {  // AllModels.cu:117-129, 228-233
        ca_g = (R)pr[q * S]; q += 1;
        R a = (R)0.209 * efun(-((R)27 + v) * (R)(1.0 / 3.8));
        R b = (R)0.94 * M::ex((-(R)75 - v) * (R)(1.0 / 17.0));
        mi = ab_gate(a, b, tadj, &mr);
        a = (R)0.000457 * M::ex((-(R)13 - v) * (R)(1.0 / 50.0));
        b = (R)0.0065 * sigm((-v - (R)15) * (R)(1.0 / 28.0));
        hi = ab_gate(a, b, tadj, &hr);
        ca_m = INIT ? mi : cnexp_rate(st[s * S], mi, mr, dt);
        ca_h = INIT ? hi : cnexp_rate(st[(s + 1) * S], hi, hr, dt);
        st[s * S] = ca_m; st[(s + 1) * S] = ca_h; s += 2;
    }
    R cai = 0;
    int ica_row = -1;
    if (mk & Mainen::kCad) {  // AllModels.cu:198-203, 234-242
        if (INIT) cai = (R)Mainen::kCainfCad;
        else {
            R ica = st[(s + 1) * S];
            R drive = (R)(-10000.0 / (2.0 * kFaraday * Mainen::kDepthCad)) * ica;
            if (drive <= (R)0) drive = (R)0;
            R cinf = (drive + (R)(Mainen::kCainfCad / Mainen::kTaurCad)) * (R)Mainen::kTaurCad;
            cai = cnexp_rate(st[s * S], cinf, (R)(1.0 / Mainen::kTaurCad), dt);
        }
        st[s * S] = cai;
        ica_row = s + 1;
        s += 2;
    }
    if (mk & Mainen::kKca) {  // AllModels.cu:130-136, 243-249
        R g = (R)pr[q * S], caix = (R)pr[(q + 1) * S];
        R Ra = (R)pr[(q + 2) * S], Rb = (R)pr[(q + 3) * S];
        q += 4;
        R a = Ra * M::pw(cai, caix);
        mi = ab_gate(a, Rb, tadj, &mr);
        R n = INIT ? mi : cnexp_rate(st[s * S], mi, mr, dt);
        st[s * S] = n; s += 1;
        R gx = (R)1e-4 * tadj * g * n; Itot += gx * (v - (R)Mainen::kEk); Gtot += gx;
    }
#define NGPU_MAINEN_K(BIT)                                                                \
    if (mk & (BIT)) { /* km AllModels.cu:140-146, kv :150-156 */                          \
        R g = (R)pr[q * S], tha = (R)pr[(q + 1) * S], qa = (R)pr[(q + 2) * S];            \
        R Ra = (R)pr[(q + 3) * S], Rb = (R)pr[(q + 4) * S];                               \
        q += 5;                                                                           \
        R z = M::dv(v - tha, qa);                                                         \
        R a = Ra * qa * efun(-z);                                                         \
        R b = Rb * qa * efun(z);                                                          \
        mi = ab_gate(a, b, tadj, &mr);                                                    \
        R n = INIT ? mi : cnexp_rate(st[s * S], mi, mr, dt);                              \
        st[s * S] = n; s += 1;                                                            \
        R gx = (R)1e-4 * tadj * g * n; Itot += gx * (v - (R)Mainen::kEk); Gtot += gx;    \
    }
    NGPU_MAINEN_K(Mainen::kKm)
    NGPU_MAINEN_K(Mainen::kKv)
#undef NGPU_MAINEN_K
    if (mk & Mainen::kNa) {  // AllModels.cu:160-172, 266-273 (rates at v + vshift)
        R g = (R)pr[q * S], tha = (R)pr[(q + 1) * S], qa = (R)pr[(q + 2) * S];
        R Ra = (R)pr[(q + 3) * S], Rb = (R)pr[(q + 4) * S], thi1 = (R)pr[(q + 5) * S];
        R thi2 = (R)pr[(q + 6) * S], qi = (R)pr[(q + 7) * S], thinf = (R)pr[(q + 8) * S];
        R qinf = (R)pr[(q + 9) * S], Rg = (R)pr[(q + 10) * S], Rd = (R)pr[(q + 11) * S];
        q += 12;
        R vm = v + (R)Mainen::kVshiftNa;
        R a = Ra * qa * efun(-M::dv(vm - tha, qa));
        R b = Rb * qa * efun(M::dv(vm - tha, qa));
        mi = ab_gate(a, b, tadj, &mr);
        a = Rd * qi * efun(-M::dv(vm - thi1, qi));
        b = Rg * qi * efun(M::dv(vm - thi2, qi));
        hr = tadj * (a + b);
        hi = sigm(M::dv(vm - thinf, qinf));
        R m = INIT ? mi : cnexp_rate(st[s * S], mi, mr, dt);
        R h = INIT ? hi : cnexp_rate(st[(s + 1) * S], hi, hr, dt);
        st[s * S] = m; st[(s + 1) * S] = h; s += 2;
        R gx = (R)1e-4 * tadj * g * m * m * m * h; Itot += gx * (v - (R)Mainen::kEna); Gtot += gx;
    }
#define NGPU_MAINEN_PAS(BIT)                                                              \
    if (mk & (BIT)) {                                                                     \
        R g = (R)pr[q * S], e = (R)pr[(q + 1) * S]; q += 2;                               \
        Itot += g * (v - e); Gtot += g;                                                   \
    }
    NGPU_MAINEN_PAS(Mainen::kPas)
    NGPU_MAINEN_PAS(Mainen::kPas2)
    NGPU_MAINEN_PAS(Mainen::kPasx)
#undef NGPU_MAINEN_PAS
    if (mk & Mainen::kCa) {  // AllModels.cu:276-285, eca from the updated cai
        R eca = (R)(ktf_of(Mainen::kCelsius) / 2) * M::lg(M::dv((R)kDefCao, cai));
        R gx = (R)1e-4 * tadj * ca_g * ca_m * ca_m * ca_h;
        R ica = gx * (v - eca);
        Itot += ica; Gtot += gx;
        if (ica_row >= 0) st[ica_row * S] = ica;
    } else if (ica_row >= 0) {
        st[ica_row * S] = (R)0;
    }
    I = Itot;
    G = Gtot;
}

}  // namespace ngpu
