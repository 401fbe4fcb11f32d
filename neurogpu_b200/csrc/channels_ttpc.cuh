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
#include "param_fold.cuh"

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
// efun(z) and efun(-z) from one exponential: efun(-z) = efun(z) e^z, with the
// series 1 -+ z/2 + z^2/12 near 0.  The alpha/beta pairs of NaTa_t, NaTs2_t
// and Nap_Et2's activation are efun of opposite arguments.  Above z = 80,
// efun(-z) = z / (1 - e^-z) is z to well below FP64 rounding; there e^z may
// overflow FP32, where efun(z) e^z would be 0 * inf.
template <typename R>
NGPU_HD void efun_pair(R z, R& pos, R& neg) {
    if (fabs(z) < (R)1e-2) {
        const R c = z * z * (R)(1.0 / 12.0);
        pos = (R)1 - z * (R)0.5 + c;
        neg = (R)1 + z * (R)0.5 + c;
        return;
    }
    const R e = Math<R>::ex(z);
    pos = Math<R>::dv(z, e - (R)1);
    neg = z > (R)80 ? z : pos * e;
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
        R ep, en;
        efun_pair((v + (R)38) * (R)(1.0 / 6.0), ep, en);
        R ma = (R)(0.182 * 6.0) * en;
        R mb = (R)(0.124 * 6.0) * ep;
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
        R ep, en;
        efun_pair((v - thm) * (R)(1.0 / 6.0), ep, en);
        R ma = (R)(0.182 * 6.0) * en;
        R mb = (R)(0.124 * 6.0) * ep;
        mi = ab_gate(ma, mb, qt, &mr);
        if (v == thh) v = v + (R)0.0001;
        efun_pair((v - thh) * (R)(1.0 / 6.0), ep, en);
        R ha = (R)(0.015 * 6.0) * ep;
        R hb = (R)(0.015 * 6.0) * en;
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

// Channel update of one node for one lane, in three phases so that all of
// the node's state and parameter rows are requested from memory at once
// (one round trip instead of one per mechanism):
//   load     every state / parameter row of the mechanisms present
//   compute  INIT:  states := steady state at v (AllModels.cu:202-296;
//                   cai := 5e-5), then currents at v;
//            !INIT: cnexp state update over dt at the new v (nrn_state), then
//                   currents at v with the new states (nrn_current of the next
//                   step)
//   store    the updated states (and the Ca current for the next step's
//            CaDynamics update)
// st: the node's first state row (row stride 32 elements); pr: its first
// parameter row.  Returns I (mA/cm2) and G = dI/dv.
template <typename R, bool INIT, typename MK>
NGPU_HD void ttpc_node(MK mk, R v, R dt, R* __restrict__ st, const float* __restrict__ pr, R& I,
                       R& G) {
    using Q = TTPCRates<R>;
    using M = Math<R>;
    constexpr int S = 32;
    // ---------------------------------------------------------------- load
    R hva_m = 0, hva_h = 0, lva_m = 0, lva_h = 0, cai = 0, ica = 0, ih_m = 0, im_m = 0;
    R kp_m = 0, kp_h = 0, kt_m = 0, kt_h = 0, nap_m = 0, nap_h = 0, nta_m = 0, nta_h = 0;
    R nts_m = 0, nts_h = 0, sk_z = 0, skv_m = 0;
    R g_hva = 0, g_lva = 0, gamma = 0, decay = 1, depth = 1, mincai = 0, g_ih = 0, e_ih = 0;
    R g_im = 0, g_kp = 0, g_kt = 0, g_nap = 0, g_nta = 0, g_nts = 0, g_pas = 0, e_pas = 0;
    R g_sk = 0, ztau = 1, g_skv = 0;
    {
        int s = 0, q = 0;
#define LD2(A, B) { if (!INIT) { A = st[s * S]; B = st[(s + 1) * S]; } s += 2; }
#define LD1(A) { if (!INIT) A = st[s * S]; s += 1; }
// P1(A, I): A = parameter I of the set (a compile-time constant where folded)
#define P1(A, I) { A = pload<R, I>(pr, q); q += 1; }
        if (mk & TTPC::kCaHVA) { LD2(hva_m, hva_h) P1(g_hva, 0) }
        if (mk & TTPC::kCaLVA) { LD2(lva_m, lva_h) P1(g_lva, 1) }
        if (mk & TTPC::kCaDyn) { LD2(cai, ica) P1(gamma, 2) P1(decay, 3) P1(depth, 4) P1(mincai, 5) }
        if (mk & TTPC::kIh) { LD1(ih_m) P1(g_ih, 6) P1(e_ih, 7) }
        if (mk & TTPC::kIm) { LD1(im_m) P1(g_im, 8) }
        if (mk & TTPC::kKP) { LD2(kp_m, kp_h) P1(g_kp, 9) }
        if (mk & TTPC::kKT) { LD2(kt_m, kt_h) P1(g_kt, 10) }
        if (mk & TTPC::kNap) { LD2(nap_m, nap_h) P1(g_nap, 11) }
        if (mk & TTPC::kNaTa) { LD2(nta_m, nta_h) P1(g_nta, 12) }
        if (mk & TTPC::kNaTs2) { LD2(nts_m, nts_h) P1(g_nts, 13) }
        if (mk & TTPC::kPas) { P1(g_pas, 14) P1(e_pas, 15) }
        if (mk & TTPC::kSK) { LD1(sk_z) P1(g_sk, 16) P1(ztau, 17) }
        if (mk & TTPC::kSKv3) { LD1(skv_m) P1(g_skv, 18) }
#undef LD2
#undef LD1
#undef P1
    }
    // ------------------------------------------------------------- compute
    R Itot = 0, Gtot = 0;
    R mi, mr, hi, hr;
#define GATE2(M_, H_, CALL)                                                               \
    {                                                                                     \
        CALL;                                                                             \
        if (INIT) { M_ = mi; H_ = hi; }                                                   \
        else { M_ = cnexp_rate(M_, mi, mr, dt); H_ = cnexp_rate(H_, hi, hr, dt); }        \
    }
#define GATE1(M_, CALL)                                                                   \
    {                                                                                     \
        CALL;                                                                             \
        M_ = INIT ? mi : cnexp_rate(M_, mi, mr, dt);                                      \
    }
    if (mk & TTPC::kCaHVA) GATE2(hva_m, hva_h, Q::ca_hva(v, mi, mr, hi, hr))
    if (mk & TTPC::kCaLVA) GATE2(lva_m, lva_h, Q::ca_lva(v, mi, mr, hi, hr))
    if (mk & TTPC::kCaDyn) {  // AllModels.cu:222-225 (init), :313-317 (cnexp, previous step's ica)
        if (INIT) cai = (R)kDefCai;
        else {
            R cinf = ((R)(-10000.0 / (2.0 * kFaraday)) * M::dv(ica * gamma, depth) + M::dv(mincai, decay)) * decay;
            cai = cnexp_rate(cai, cinf, M::rc(decay), dt);
        }
    }
    if (mk & TTPC::kIh) {
        GATE1(ih_m, Q::ih(v, mi, mr))
        R gx = g_ih * ih_m; Itot += gx * (v - e_ih); Gtot += gx;
    }
    if (mk & TTPC::kIm) {
        GATE1(im_m, Q::im(v, mi, mr))
        R gx = g_im * im_m; Itot += gx * (v - (R)TTPC::kEk); Gtot += gx;
    }
    if (mk & TTPC::kKP) {
        GATE2(kp_m, kp_h, Q::k_pst(v, mi, mr, hi, hr))
        R gx = g_kp * kp_m * kp_m * kp_h; Itot += gx * (v - (R)TTPC::kEk); Gtot += gx;
    }
    if (mk & TTPC::kKT) {
        GATE2(kt_m, kt_h, Q::k_tst(v, mi, mr, hi, hr))
        R m2 = kt_m * kt_m;
        R gx = g_kt * m2 * m2 * kt_h; Itot += gx * (v - (R)TTPC::kEk); Gtot += gx;
    }
    if (mk & TTPC::kNap) {
        GATE2(nap_m, nap_h, Q::nap(v, mi, mr, hi, hr))
        R gx = g_nap * nap_m * nap_m * nap_m * nap_h; Itot += gx * (v - (R)TTPC::kEna); Gtot += gx;
    }
    if (mk & TTPC::kNaTa) {
        GATE2(nta_m, nta_h, Q::nat(v, (R)-38, (R)-66, mi, mr, hi, hr))
        R gx = g_nta * nta_m * nta_m * nta_m * nta_h; Itot += gx * (v - (R)TTPC::kEna); Gtot += gx;
    }
    if (mk & TTPC::kNaTs2) {
        GATE2(nts_m, nts_h, Q::nat(v, (R)-32, (R)-60, mi, mr, hi, hr))
        R gx = g_nts * nts_m * nts_m * nts_m * nts_h; Itot += gx * (v - (R)TTPC::kEna); Gtot += gx;
    }
    if (mk & TTPC::kPas) { Itot += g_pas * (v - e_pas); Gtot += g_pas; }
    if (mk & TTPC::kSK) {
        R zi = Q::sk_zinf(cai);
        sk_z = INIT ? zi : cnexp(sk_z, zi, ztau, dt);
        R gx = g_sk * sk_z; Itot += gx * (v - (R)TTPC::kEk); Gtot += gx;
    }
    if (mk & TTPC::kSKv3) {
        GATE1(skv_m, Q::skv3(v, mi, mr))
        R gx = g_skv * skv_m; Itot += gx * (v - (R)TTPC::kEk); Gtot += gx;
    }
#undef GATE2
#undef GATE1
    // Ca currents with eca from the updated cai (AllModels.cu:382-407)
    ica = 0;
    if (mk & (TTPC::kCaHVA | TTPC::kCaLVA)) {
        R eca = (R)(ktf_of(TTPC::kCelsius) / 2) * M::lg(M::dv((R)kDefCao, cai));
        R gca = g_hva * hva_m * hva_m * hva_h + g_lva * lva_m * lva_m * lva_h;
        ica = gca * (v - eca);
        Itot += ica; Gtot += gca;
    }
    I = Itot;
    G = Gtot;
    // --------------------------------------------------------------- store
    {
        int s = 0;
#define ST2(A, B) { st[s * S] = A; st[(s + 1) * S] = B; s += 2; }
#define ST1(A) { st[s * S] = A; s += 1; }
        if (mk & TTPC::kCaHVA) ST2(hva_m, hva_h)
        if (mk & TTPC::kCaLVA) ST2(lva_m, lva_h)
        if (mk & TTPC::kCaDyn) ST2(cai, ica)
        if (mk & TTPC::kIh) ST1(ih_m)
        if (mk & TTPC::kIm) ST1(im_m)
        if (mk & TTPC::kKP) ST2(kp_m, kp_h)
        if (mk & TTPC::kKT) ST2(kt_m, kt_h)
        if (mk & TTPC::kNap) ST2(nap_m, nap_h)
        if (mk & TTPC::kNaTa) ST2(nta_m, nta_h)
        if (mk & TTPC::kNaTs2) ST2(nts_m, nts_h)
        if (mk & TTPC::kSK) ST1(sk_z)
        if (mk & TTPC::kSKv3) ST1(skv_m)
#undef ST2
#undef ST1
    }
}

}  // namespace ngpu
