// TTPC channel set (13 mechanisms) for the fused simulation kernel.
//
// Equations follow the reference's generated channel library for the
// thick-tufted pyramidal cell, GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/
// AllModels.cu (rates :66-197, init :202-296, cnexp derivs :299-377,
// breakpoints :382-516), with the mechanism order, parameter order and
// per-mechanism state lists of its CALL_TO_* expansion (CudaStuff.cu:220,
// 264, 325).  Rewritten for the GPU:
//   * alpha/beta rates use efun(z) = z/(e^z - 1) with a series near z = 0
//     (the reference's exact-equality nudges v += 1e-4 at the singular
//     voltages are kept, so results agree at those points too);
//   * dt/tau is formed as dt*(alpha+beta)*qt, so one reciprocal per gate;
//   * the membrane conductance is the analytic dI/dv = sum of channel
//     conductances (every channel here is ohmic), which equals the
//     reference's finite difference (I(v+0.001)-I(v))/0.001 exactly in real
//     arithmetic and avoids its FP32 cancellation;
//   * eca is derived from cai when needed (the reference recomputes it
//     from cai after every cai change, AllModels.cu:316,367).
//
// State rows of a node, in order, for the mechanisms present:
//   Ca_HVA m,h | Ca_LVAst m,h | CaDynamics_E2 cai,ica | Ih m | Im m |
//   K_Pst m,h | K_Tst m,h | Nap_Et2 m,h | NaTa_t m,h | NaTs2_t m,h |
//   (pas: none) | SK_E2 z | SKv3_1 m
// Parameter rows: the reference parameter indices each mechanism reads.
#pragma once
#include "ngpu_math.cuh"

namespace ngpu {

struct TTPC {
    static constexpr int kNMech = 13;
    static constexpr int kNParams = 19;
    enum : uint32_t {
        kCaHVA = 1u << 0, kCaLVA = 1u << 1, kCaDyn = 1u << 2, kIh = 1u << 3, kIm = 1u << 4,
        kKP = 1u << 5, kKT = 1u << 6, kNap = 1u << 7, kNaTa = 1u << 8, kNaTs2 = 1u << 9,
        kPas = 1u << 10, kSK = 1u << 11, kSKv3 = 1u << 12
    };
    static constexpr double kCelsius = 34.0;
    static constexpr double kEna = 50.0, kEk = -85.0;
    static constexpr double kQt = 2.952882641412121;  // 2.3^((34-21)/10)
};

// z/(e^z - 1), with the series 1 - z/2 + z^2/12 near 0.
template <typename R>
NGPU_HD R efun(R z) {
    if (fabs(z) < (R)1e-2) return (R)1 - z * ((R)0.5 - z * (R)(1.0 / 12.0));
    return Math<R>::dv(z, Math<R>::ex(z) - (R)1);
}
// 1/(1 + e^z)
template <typename R>
NGPU_HD R sigm(R z) {
    return Math<R>::rc((R)1 + Math<R>::ex(z));
}
// Gate with alpha/beta rates: returns xinf, sets *rate = qt*(alpha+beta) = 1/tau.
template <typename R>
NGPU_HD R ab_gate(R a, R b, R qt, R* rate) {
    R s = a + b;
    *rate = qt * s;
    return Math<R>::dv(a, s);
}
// cnexp given 1/tau.
template <typename R>
NGPU_HD R cnexp_rate(R x, R xinf, R rate, R dt) {
    return x + Math<R>::one_minus_exp_neg(dt * rate) * (xinf - x);
}

template <typename R>
struct TTPCRates {
    using M = Math<R>;
    static constexpr R qt = (R)TTPC::kQt;
    // AllModels.cu:66-78
    static NGPU_HD void ca_hva(R v, R& mi, R& mr, R& hi, R& hr) {
        if (v == (R)-27.0) v = v + (R)0.0001;
        R ma = (R)(0.055 * 3.8) * efun((-(R)27 - v) * (R)(1.0 / 3.8));
        R mb = (R)0.94 * M::ex((-(R)75 - v) * (R)(1.0 / 17.0));
        mi = ab_gate(ma, mb, (R)1, &mr);
        R ha = (R)0.000457 * M::ex((-(R)13 - v) * (R)(1.0 / 50.0));
        R hb = (R)0.0065 * sigm((-v - (R)15) * (R)(1.0 / 28.0));
        hi = ab_gate(ha, hb, (R)1, &hr);
    }
    // AllModels.cu:79-88
    static NGPU_HD void ca_lva(R v, R& mi, R& mr, R& hi, R& hr) {
        v = v + (R)10;
        mi = sigm((v + (R)30) * (R)(-1.0 / 6.0));
        mr = qt * M::rc((R)5 + (R)20 * sigm((v + (R)25) * (R)(1.0 / 5.0)));
        hi = sigm((v + (R)80) * (R)(1.0 / 6.4));
        hr = qt * M::rc((R)20 + (R)50 * sigm((v + (R)40) * (R)(1.0 / 7.0)));
    }
    // AllModels.cu:89-97
    static NGPU_HD void ih(R v, R& mi, R& mr) {
        if (v == (R)-154.9) v = v + (R)0.0001;
        R ma = (R)(0.001 * 6.43 * 11.9) * efun((v + (R)154.9) * (R)(1.0 / 11.9));
        R mb = (R)(0.001 * 193.0) * M::ex(v * (R)(1.0 / 33.1));
        mi = ab_gate(ma, mb, (R)1, &mr);
    }
    // AllModels.cu:98-105
    static NGPU_HD void im(R v, R& mi, R& mr) {
        R ma = (R)3.3e-3 * M::ex((R)(2.5 * 0.04) * (v + (R)35));
        R mb = (R)3.3e-3 * M::ex((R)(-2.5 * 0.04) * (v + (R)35));
        mi = ab_gate(ma, mb, qt, &mr);
    }
    // AllModels.cu:106-120
    static NGPU_HD void k_pst(R v, R& mi, R& mr, R& hi, R& hr) {
        v = v + (R)10;
        mi = sigm(-(v + (R)1) * (R)(1.0 / 12.0));
        R mt = (v < (R)-50) ? (R)1.25 + (R)175.03 * M::ex(v * (R)0.026)
                            : (R)1.25 + (R)13 * M::ex(v * (R)-0.026);
        mr = qt * M::rc(mt);
        hi = sigm((v + (R)54) * (R)(1.0 / 11.0));
        R z = (v + (R)75) * (R)(1.0 / 48.0);
        hr = qt * M::rc((R)360 + ((R)1010 + (R)24 * (v + (R)55)) * M::ex(-(z * z)));
    }
    // AllModels.cu:121-130
    static NGPU_HD void k_tst(R v, R& mi, R& mr, R& hi, R& hr) {
        v = v + (R)10;
        mi = sigm(-v * (R)(1.0 / 19.0));
        R zm = (v + (R)71) * (R)(1.0 / 59.0);
        mr = qt * M::rc((R)0.34 + (R)0.92 * M::ex(-(zm * zm)));
        hi = sigm((v + (R)66) * (R)(1.0 / 10.0));
        R zh = (v + (R)73) * (R)(1.0 / 23.0);
        hr = qt * M::rc((R)8 + (R)49 * M::ex(-(zh * zh)));
    }
    // AllModels.cu:131-151
    static NGPU_HD void nap(R v, R& mi, R& mr, R& hi, R& hr) {
        mi = sigm((v + (R)52.6) * (R)(-1.0 / 4.6));
        if (v == (R)-38.0) v = v + (R)0.0001;
        R ma = (R)(0.182 * 6.0) * efun(-(v + (R)38) * (R)(1.0 / 6.0));
        R mb = (R)(0.124 * 6.0) * efun((v + (R)38) * (R)(1.0 / 6.0));
        mr = qt * (R)(1.0 / 6.0) * (ma + mb);
        if (v == (R)-17.0) v = v + (R)0.0001;
        if (v == (R)-64.4) v = v + (R)0.0001;
        hi = sigm((v + (R)48.8) * (R)(1.0 / 10.0));
        R ha = (R)(2.88e-6 * 4.63) * efun((v + (R)17) * (R)(1.0 / 4.63));
        R hb = (R)(6.94e-6 * 2.63) * efun(-(v + (R)64.4) * (R)(1.0 / 2.63));
        hr = qt * (ha + hb);
    }
    // AllModels.cu:152-169 (NaTa_t: th_m=-38, th_h=-66), :170-187 (NaTs2_t: -32, -60)
    static NGPU_HD void nat(R v, R thm, R thh, R& mi, R& mr, R& hi, R& hr) {
        if (v == thm) v = v + (R)0.0001;
        R ma = (R)(0.182 * 6.0) * efun(-(v - thm) * (R)(1.0 / 6.0));
        R mb = (R)(0.124 * 6.0) * efun((v - thm) * (R)(1.0 / 6.0));
        mi = ab_gate(ma, mb, qt, &mr);
        if (v == thh) v = v + (R)0.0001;
        R ha = (R)(0.015 * 6.0) * efun((v - thh) * (R)(1.0 / 6.0));
        R hb = (R)(0.015 * 6.0) * efun(-(v - thh) * (R)(1.0 / 6.0));
        hi = ab_gate(ha, hb, qt, &hr);
    }
    // AllModels.cu:188-193
    static NGPU_HD R sk_zinf(R ca) {
        if (ca < (R)1e-7) ca = ca + (R)1e-7;
        return M::rc((R)1 + M::pw((R)0.00043 * M::rc(ca), (R)4.8));
    }
    // AllModels.cu:194-197
    static NGPU_HD void skv3(R v, R& mi, R& mr) {
        mi = sigm((v - (R)18.7) * (R)(-1.0 / 9.7));
        mr = ((R)1 + M::ex((v + (R)46.56) * (R)(-1.0 / 44.14))) * (R)(1.0 / 4.0);
    }
};

// Channel update of one node for one lane.
//   INIT:  states := steady state at v (AllModels.cu:202-296; cai := 5e-5),
//          then currents at v.
//   !INIT: cnexp state update over dt at the new v (nrn_state), then
//          currents at v with the new states (nrn_current of the next step).
// st: the node's first state row (row stride 32 elements); pr: its first
// parameter row.  Returns I (mA/cm2) and G = dI/dv; writes the states back.
template <typename R, bool INIT>
NGPU_HD void ttpc_node(uint32_t mk, R v, R dt, R* __restrict__ st,
                                          const float* __restrict__ pr, R& I, R& G) {
    using Q = TTPCRates<R>;
    using M = Math<R>;
    constexpr int S = 32;
    int s = 0, q = 0;
    R Itot = 0, Gtot = 0;
    R mi, mr, hi, hr;
    // ---- Ca gates (their currents need cai, which CaDynamics updates first) ----
    R hva_m = 0, hva_h = 0, hva_g = 0;
    if (mk & TTPC::kCaHVA) {
        hva_g = (R)pr[q * S]; q += 1;
        Q::ca_hva(v, mi, mr, hi, hr);
        if (INIT) { hva_m = mi; hva_h = hi; }
        else {
            hva_m = cnexp_rate(st[s * S], mi, mr, dt);
            hva_h = cnexp_rate(st[(s + 1) * S], hi, hr, dt);
        }
        st[s * S] = hva_m; st[(s + 1) * S] = hva_h; s += 2;
    }
    R lva_m = 0, lva_h = 0, lva_g = 0;
    if (mk & TTPC::kCaLVA) {
        lva_g = (R)pr[q * S]; q += 1;
        Q::ca_lva(v, mi, mr, hi, hr);
        if (INIT) { lva_m = mi; lva_h = hi; }
        else {
            lva_m = cnexp_rate(st[s * S], mi, mr, dt);
            lva_h = cnexp_rate(st[(s + 1) * S], hi, hr, dt);
        }
        st[s * S] = lva_m; st[(s + 1) * S] = lva_h; s += 2;
    }
    R cai = 0;
    int ica_row = -1;
    if (mk & TTPC::kCaDyn) {
        // AllModels.cu:222-225 (init), :313-317 (cnexp with the previous step's ica)
        R gamma = (R)pr[q * S], decay = (R)pr[(q + 1) * S];
        R depth = (R)pr[(q + 2) * S], mincai = (R)pr[(q + 3) * S];
        q += 4;
        if (INIT) cai = (R)kDefCai;
        else {
            R ica = st[(s + 1) * S];
            R cinf = ((R)(-10000.0 / (2.0 * kFaraday)) * M::dv(ica * gamma, depth) +
                      M::dv(mincai, decay)) * decay;
            cai = cnexp_rate(st[s * S], cinf, M::rc(decay), dt);
        }
        st[s * S] = cai;
        ica_row = s + 1;
        s += 2;
    }
    if (mk & TTPC::kIh) {
        R g = (R)pr[q * S], e = (R)pr[(q + 1) * S]; q += 2;
        Q::ih(v, mi, mr);
        R m = INIT ? mi : cnexp_rate(st[s * S], mi, mr, dt);
        st[s * S] = m; s += 1;
        R gx = g * m; Itot += gx * (v - e); Gtot += gx;
    }
    if (mk & TTPC::kIm) {
        R g = (R)pr[q * S]; q += 1;
        Q::im(v, mi, mr);
        R m = INIT ? mi : cnexp_rate(st[s * S], mi, mr, dt);
        st[s * S] = m; s += 1;
        R gx = g * m; Itot += gx * (v - (R)TTPC::kEk); Gtot += gx;
    }
    if (mk & TTPC::kKP) {
        R g = (R)pr[q * S]; q += 1;
        Q::k_pst(v, mi, mr, hi, hr);
        R m = INIT ? mi : cnexp_rate(st[s * S], mi, mr, dt);
        R h = INIT ? hi : cnexp_rate(st[(s + 1) * S], hi, hr, dt);
        st[s * S] = m; st[(s + 1) * S] = h; s += 2;
        R gx = g * m * m * h; Itot += gx * (v - (R)TTPC::kEk); Gtot += gx;
    }
    if (mk & TTPC::kKT) {
        R g = (R)pr[q * S]; q += 1;
        Q::k_tst(v, mi, mr, hi, hr);
        R m = INIT ? mi : cnexp_rate(st[s * S], mi, mr, dt);
        R h = INIT ? hi : cnexp_rate(st[(s + 1) * S], hi, hr, dt);
        st[s * S] = m; st[(s + 1) * S] = h; s += 2;
        R m2 = m * m;
        R gx = g * m2 * m2 * h; Itot += gx * (v - (R)TTPC::kEk); Gtot += gx;
    }
    if (mk & TTPC::kNap) {
        R g = (R)pr[q * S]; q += 1;
        Q::nap(v, mi, mr, hi, hr);
        R m = INIT ? mi : cnexp_rate(st[s * S], mi, mr, dt);
        R h = INIT ? hi : cnexp_rate(st[(s + 1) * S], hi, hr, dt);
        st[s * S] = m; st[(s + 1) * S] = h; s += 2;
        R gx = g * m * m * m * h; Itot += gx * (v - (R)TTPC::kEna); Gtot += gx;
    }
    if (mk & TTPC::kNaTa) {
        R g = (R)pr[q * S]; q += 1;
        Q::nat(v, (R)-38, (R)-66, mi, mr, hi, hr);
        R m = INIT ? mi : cnexp_rate(st[s * S], mi, mr, dt);
        R h = INIT ? hi : cnexp_rate(st[(s + 1) * S], hi, hr, dt);
        st[s * S] = m; st[(s + 1) * S] = h; s += 2;
        R gx = g * m * m * m * h; Itot += gx * (v - (R)TTPC::kEna); Gtot += gx;
    }
    if (mk & TTPC::kNaTs2) {
        R g = (R)pr[q * S]; q += 1;
        Q::nat(v, (R)-32, (R)-60, mi, mr, hi, hr);
        R m = INIT ? mi : cnexp_rate(st[s * S], mi, mr, dt);
        R h = INIT ? hi : cnexp_rate(st[(s + 1) * S], hi, hr, dt);
        st[s * S] = m; st[(s + 1) * S] = h; s += 2;
        R gx = g * m * m * m * h; Itot += gx * (v - (R)TTPC::kEna); Gtot += gx;
    }
    if (mk & TTPC::kPas) {
        R g = (R)pr[q * S], e = (R)pr[(q + 1) * S]; q += 2;
        Itot += g * (v - e); Gtot += g;
    }
    if (mk & TTPC::kSK) {
        R g = (R)pr[q * S], ztau = (R)pr[(q + 1) * S]; q += 2;
        R zi = Q::sk_zinf(cai);
        R z = INIT ? zi : cnexp(st[s * S], zi, ztau, dt);
        st[s * S] = z; s += 1;
        R gx = g * z; Itot += gx * (v - (R)TTPC::kEk); Gtot += gx;
    }
    if (mk & TTPC::kSKv3) {
        R g = (R)pr[q * S]; q += 1;
        Q::skv3(v, mi, mr);
        R m = INIT ? mi : cnexp_rate(st[s * S], mi, mr, dt);
        st[s * S] = m; s += 1;
        R gx = g * m; Itot += gx * (v - (R)TTPC::kEk); Gtot += gx;
    }
    // ---- Ca currents with eca from the updated cai (AllModels.cu:382-407) ----
    if (mk & (TTPC::kCaHVA | TTPC::kCaLVA)) {
        R eca = (R)(ktf_of(TTPC::kCelsius) / 2) * M::lg(M::dv((R)kDefCao, cai));
        R gca = hva_g * hva_m * hva_m * hva_h + lva_g * lva_m * lva_m * lva_h;
        R ica = gca * (v - eca);
        Itot += ica; Gtot += gca;
        if (ica_row >= 0) st[ica_row * S] = ica;
    } else if (ica_row >= 0) {
        st[ica_row * S] = (R)0;
    }
    I = Itot;
    G = Gtot;
}

}  // namespace ngpu
