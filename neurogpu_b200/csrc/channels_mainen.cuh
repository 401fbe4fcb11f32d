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

// One node, three phases (load every row / compute / store), as ttpc_node.
template <typename R, bool INIT, typename MK>
NGPU_HD void mainen_node(MK mk, R v, R dt, R* __restrict__ st, const float* __restrict__ pr, R& I,
                         R& G) {
    using M = Math<R>;
    constexpr int S = 32;
    const R tadj = (R)Mainen::kTadj;
    // ---------------------------------------------------------------- load
    R ca_m = 0, ca_h = 0, cai = 0, ica = 0, kca_n = 0, km_n = 0, kv_n = 0, na_m = 0, na_h = 0;
    R g_ca = 0, g_kca = 0, caix = 1, ra_kca = 0, rb_kca = 0;
    R km[5] = {0, 0, 1, 0, 0}, kv[5] = {0, 0, 1, 0, 0};  // gbar, tha, qa, Ra, Rb
    R na[12] = {0, 0, 1, 0, 0, 0, 0, 1, 0, 1, 0, 0};    // gbar tha qa Ra Rb thi1 thi2 qi thinf qinf Rg Rd
    R pas[6] = {0, 0, 0, 0, 0, 0};
    {
        int s = 0, q = 0;
        // parameter rows hold the set's parameters 0, 2-33 (ca's cao, 1, is not read)
        if (mk & Mainen::kCa) { if (!INIT) { ca_m = st[s * S]; ca_h = st[(s + 1) * S]; } s += 2; g_ca = pload<R, 0>(pr, q); q += 1; }
        if (mk & Mainen::kCad) { if (!INIT) { cai = st[s * S]; ica = st[(s + 1) * S]; } s += 2; }
        if (mk & Mainen::kKca) {
            if (!INIT) kca_n = st[s * S];
            s += 1;
            g_kca = pload<R, 2>(pr, q); caix = pload<R, 3>(pr, q + 1); ra_kca = pload<R, 4>(pr, q + 2);
            rb_kca = pload<R, 5>(pr, q + 3);
            q += 4;
        }
        if (mk & Mainen::kKm) {
            if (!INIT) km_n = st[s * S];
            s += 1;
            pload_n<R, 6, 5>(pr, q, km);
            q += 5;
        }
        if (mk & Mainen::kKv) {
            if (!INIT) kv_n = st[s * S];
            s += 1;
            pload_n<R, 11, 5>(pr, q, kv);
            q += 5;
        }
        if (mk & Mainen::kNa) {
            if (!INIT) { na_m = st[s * S]; na_h = st[(s + 1) * S]; }
            s += 2;
            pload_n<R, 16, 12>(pr, q, na);
            q += 12;
        }
        if (mk & Mainen::kPas) { pas[0] = pload<R, 28>(pr, q); pas[1] = pload<R, 29>(pr, q + 1); q += 2; }
        if (mk & Mainen::kPas2) { pas[2] = pload<R, 30>(pr, q); pas[3] = pload<R, 31>(pr, q + 1); q += 2; }
        if (mk & Mainen::kPasx) { pas[4] = pload<R, 32>(pr, q); pas[5] = pload<R, 33>(pr, q + 1); q += 2; }
    }
    // ------------------------------------------------------------- compute
    R Itot = 0, Gtot = 0;
    R mi, mr, hi, hr;
    if (mk & Mainen::kCa) {  // AllModels.cu:117-129, 228-233
        R a = (R)0.209 * efun(-((R)27 + v) * (R)(1.0 / 3.8));
        R b = (R)0.94 * M::ex((-(R)75 - v) * (R)(1.0 / 17.0));
        mi = ab_gate(a, b, tadj, &mr);
        a = (R)0.000457 * M::ex((-(R)13 - v) * (R)(1.0 / 50.0));
        b = (R)0.0065 * sigm((-v - (R)15) * (R)(1.0 / 28.0));
        hi = ab_gate(a, b, tadj, &hr);
        ca_m = INIT ? mi : cnexp_rate(ca_m, mi, mr, dt);
        ca_h = INIT ? hi : cnexp_rate(ca_h, hi, hr, dt);
    }
    if (mk & Mainen::kCad) {  // AllModels.cu:198-203, 234-242
        if (INIT) cai = (R)Mainen::kCainfCad;
        else {
            R drive = (R)(-10000.0 / (2.0 * kFaraday * Mainen::kDepthCad)) * ica;
            if (drive <= (R)0) drive = (R)0;
            R cinf = (drive + (R)(Mainen::kCainfCad / Mainen::kTaurCad)) * (R)Mainen::kTaurCad;
            cai = cnexp_rate(cai, cinf, (R)(1.0 / Mainen::kTaurCad), dt);
        }
    }
    if (mk & Mainen::kKca) {  // AllModels.cu:130-136, 243-249
        R a = ra_kca * M::pw(cai, caix);
        mi = ab_gate(a, rb_kca, tadj, &mr);
        kca_n = INIT ? mi : cnexp_rate(kca_n, mi, mr, dt);
        R gx = (R)1e-4 * tadj * g_kca * kca_n; Itot += gx * (v - (R)Mainen::kEk); Gtot += gx;
    }
    // km AllModels.cu:140-146, kv :150-156 (same rate form)
    auto kgate = [&](const R* p, R& n) {
        R z = M::dv(v - p[1], p[2]);
        R a = p[3] * p[2] * efun(-z);
        R b = p[4] * p[2] * efun(z);
        mi = ab_gate(a, b, tadj, &mr);
        n = INIT ? mi : cnexp_rate(n, mi, mr, dt);
        R gx = (R)1e-4 * tadj * p[0] * n; Itot += gx * (v - (R)Mainen::kEk); Gtot += gx;
    };
    if (mk & Mainen::kKm) kgate(km, km_n);
    if (mk & Mainen::kKv) kgate(kv, kv_n);
    if (mk & Mainen::kNa) {  // AllModels.cu:160-172, 266-273 (rates at v + vshift)
        R vm = v + (R)Mainen::kVshiftNa;
        R a = na[3] * na[2] * efun(-M::dv(vm - na[1], na[2]));
        R b = na[4] * na[2] * efun(M::dv(vm - na[1], na[2]));
        mi = ab_gate(a, b, tadj, &mr);
        a = na[11] * na[7] * efun(-M::dv(vm - na[5], na[7]));
        b = na[10] * na[7] * efun(M::dv(vm - na[6], na[7]));
        hr = tadj * (a + b);
        hi = sigm(M::dv(vm - na[8], na[9]));
        na_m = INIT ? mi : cnexp_rate(na_m, mi, mr, dt);
        na_h = INIT ? hi : cnexp_rate(na_h, hi, hr, dt);
        R gx = (R)1e-4 * tadj * na[0] * na_m * na_m * na_m * na_h; Itot += gx * (v - (R)Mainen::kEna); Gtot += gx;
    }
    if (mk & Mainen::kPas) { Itot += pas[0] * (v - pas[1]); Gtot += pas[0]; }
    if (mk & Mainen::kPas2) { Itot += pas[2] * (v - pas[3]); Gtot += pas[2]; }
    if (mk & Mainen::kPasx) { Itot += pas[4] * (v - pas[5]); Gtot += pas[4]; }
    ica = 0;
    if (mk & Mainen::kCa) {  // AllModels.cu:276-285, eca from the updated cai
        R eca = (R)(ktf_of(Mainen::kCelsius) / 2) * M::lg(M::dv((R)kDefCao, cai));
        R gx = (R)1e-4 * tadj * g_ca * ca_m * ca_m * ca_h;
        ica = gx * (v - eca);
        Itot += ica; Gtot += gx;
    }
    I = Itot;
    G = Gtot;
    // --------------------------------------------------------------- store
    {
        int s = 0;
        if (mk & Mainen::kCa) { st[s * S] = ca_m; st[(s + 1) * S] = ca_h; s += 2; }
        if (mk & Mainen::kCad) { st[s * S] = cai; st[(s + 1) * S] = ica; s += 2; }
        if (mk & Mainen::kKca) { st[s * S] = kca_n; s += 1; }
        if (mk & Mainen::kKm) { st[s * S] = km_n; s += 1; }
        if (mk & Mainen::kKv) { st[s * S] = kv_n; s += 1; }
        if (mk & Mainen::kNa) { st[s * S] = na_m; st[(s + 1) * S] = na_h; s += 2; }
    }
}

}  // namespace ngpu
