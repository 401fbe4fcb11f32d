// Test-only C entry points around the reference's OWN generated channel
// functions, which build_ref.sh compiles for the host from the reference tree
// (GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/AllModels.cu and
// Figures/FigureS4_mainen/CParsed/AllModels.cu, with __device__ defined away).
// Used only to pin the oracle's channel equations mechanism by mechanism.
//
// The declarations below repeat the reference's generated signatures
// (GUI/BBP_TTPC_EXAMPLE/pyNeuroGPU_unix/src/AllModels.cuh:25-60 and
// Figures/FigureS4_mainen/CParsed/AllModels.cuh:24-60) so that this file links
// against the objects built from them; float = the reference's MYFTYPE,
// double = MYSECONDFTYPE.
typedef float F;
typedef double D;

#ifdef REF_TTPC
void CuInitModel_Ca_HVA(F v, F &m, F &h, F g, F &ica, F &eca, F &cai);
void CuInitModel_Ca_LVAst(F v, F &m, F &h, F g, F &ica, F &eca, F &cai);
void CuInitModel_CaDynamics_E2(F v, F &cai, F gamma, F decay, F depth, F minCai, F ica, F &eca);
void CuInitModel_Ih(F v, F &m, F g, F ehcn);
void CuInitModel_Im(F v, F &m, F g);
void CuInitModel_K_Pst(F v, F &m, F &h, F g);
void CuInitModel_K_Tst(F v, F &m, F &h, F g);
void CuInitModel_Nap_Et2(F v, F &m, F &h, F g);
void CuInitModel_NaTa_t(F v, F &m, F &h, F g);
void CuInitModel_NaTs2_t(F v, F &m, F &h, F g);
void CuInitModel_SK_E2(F v, F &z, F g, F zTau, F cai, F &eca);
void CuInitModel_SKv3_1(F v, F &m, F g);
void CuDerivModel_Ca_HVA(F dt, F v, F &m, F &h, F g, F &ica);
void CuDerivModel_Ca_LVAst(F dt, F v, F &m, F &h, F g, F &ica);
void CuDerivModel_CaDynamics_E2(F dt, F v, F &cai, F gamma, F decay, F depth, F minCai, F ica, F &eca);
void CuDerivModel_Ih(F dt, F v, F &m, F g, F ehcn);
void CuDerivModel_Im(F dt, F v, F &m, F g);
void CuDerivModel_K_Pst(F dt, F v, F &m, F &h, F g);
void CuDerivModel_K_Tst(F dt, F v, F &m, F &h, F g);
void CuDerivModel_Nap_Et2(F dt, F v, F &m, F &h, F g);
void CuDerivModel_NaTa_t(F dt, F v, F &m, F &h, F g);
void CuDerivModel_NaTs2_t(F dt, F v, F &m, F &h, F g);
void CuDerivModel_SK_E2(F dt, F v, F &z, F g, F zTau, F cai, F &eca);
void CuDerivModel_SKv3_1(F dt, F v, F &m, F g);
void CuBreakpointModel_Ca_HVA(D &I, F &G, F v, F &m, F &h, F g, F &ica, F &eca, F &cai);
void CuBreakpointModel_Ca_LVAst(D &I, F &G, F v, F &m, F &h, F g, F &ica, F &eca, F &cai);
void CuBreakpointModel_Ih(D &I, F &G, F v, F &m, F g, F ehcn);
void CuBreakpointModel_Im(D &I, F &G, F v, F &m, F g);
void CuBreakpointModel_K_Pst(D &I, F &G, F v, F &m, F &h, F g);
void CuBreakpointModel_K_Tst(D &I, F &G, F v, F &m, F &h, F g);
void CuBreakpointModel_Nap_Et2(D &I, F &G, F v, F &m, F &h, F g);
void CuBreakpointModel_NaTa_t(D &I, F &G, F v, F &m, F &h, F g);
void CuBreakpointModel_NaTs2_t(D &I, F &G, F v, F &m, F &h, F g);
void CuBreakpointModel_pas(D &I, F &G, F v, F g, F e);
void CuBreakpointModel_SK_E2(D &I, F &G, F v, F &z, F g, F zTau, F cai, F &eca);
void CuBreakpointModel_SKv3_1(D &I, F &G, F v, F &m, F g);

// One mechanism of the TTPC set on one node.  s: 19 states (reference
// state_macro index), then cai, eca, ica.  p: 19 params (reference order).
// what: 0 = init, 1 = deriv, 2 = current (returns I, *G gets summed g).
extern "C" double ref_ttpc_mech(int mech, int what, float dt, float v, float *s, const float *p,
                                float *G) {
    F &cai = s[19], &eca = s[20], &ica = s[21];
    D I = 0;
    F g = 0;
    switch (mech) {
    case 0:
        if (what == 0) CuInitModel_Ca_HVA(v, s[0], s[1], p[0], ica, eca, cai);
        else if (what == 1) CuDerivModel_Ca_HVA(dt, v, s[0], s[1], p[0], ica);
        else CuBreakpointModel_Ca_HVA(I, g, v, s[0], s[1], p[0], ica, eca, cai);
        break;
    case 1:
        if (what == 0) CuInitModel_Ca_LVAst(v, s[2], s[3], p[1], ica, eca, cai);
        else if (what == 1) CuDerivModel_Ca_LVAst(dt, v, s[2], s[3], p[1], ica);
        else CuBreakpointModel_Ca_LVAst(I, g, v, s[2], s[3], p[1], ica, eca, cai);
        break;
    case 2:
        if (what == 0) CuInitModel_CaDynamics_E2(v, cai, p[2], p[3], p[4], p[5], ica, eca);
        else if (what == 1) CuDerivModel_CaDynamics_E2(dt, v, cai, p[2], p[3], p[4], p[5], ica, eca);
        break;
    case 3:
        if (what == 0) CuInitModel_Ih(v, s[5], p[6], p[7]);
        else if (what == 1) CuDerivModel_Ih(dt, v, s[5], p[6], p[7]);
        else CuBreakpointModel_Ih(I, g, v, s[5], p[6], p[7]);
        break;
    case 4:
        if (what == 0) CuInitModel_Im(v, s[6], p[8]);
        else if (what == 1) CuDerivModel_Im(dt, v, s[6], p[8]);
        else CuBreakpointModel_Im(I, g, v, s[6], p[8]);
        break;
    case 5:
        if (what == 0) CuInitModel_K_Pst(v, s[7], s[8], p[9]);
        else if (what == 1) CuDerivModel_K_Pst(dt, v, s[7], s[8], p[9]);
        else CuBreakpointModel_K_Pst(I, g, v, s[7], s[8], p[9]);
        break;
    case 6:
        if (what == 0) CuInitModel_K_Tst(v, s[9], s[10], p[10]);
        else if (what == 1) CuDerivModel_K_Tst(dt, v, s[9], s[10], p[10]);
        else CuBreakpointModel_K_Tst(I, g, v, s[9], s[10], p[10]);
        break;
    case 7:
        if (what == 0) CuInitModel_Nap_Et2(v, s[11], s[12], p[11]);
        else if (what == 1) CuDerivModel_Nap_Et2(dt, v, s[11], s[12], p[11]);
        else CuBreakpointModel_Nap_Et2(I, g, v, s[11], s[12], p[11]);
        break;
    case 8:
        if (what == 0) CuInitModel_NaTa_t(v, s[13], s[14], p[12]);
        else if (what == 1) CuDerivModel_NaTa_t(dt, v, s[13], s[14], p[12]);
        else CuBreakpointModel_NaTa_t(I, g, v, s[13], s[14], p[12]);
        break;
    case 9:
        if (what == 0) CuInitModel_NaTs2_t(v, s[15], s[16], p[13]);
        else if (what == 1) CuDerivModel_NaTs2_t(dt, v, s[15], s[16], p[13]);
        else CuBreakpointModel_NaTs2_t(I, g, v, s[15], s[16], p[13]);
        break;
    case 10:
        if (what == 2) CuBreakpointModel_pas(I, g, v, p[14], p[15]);
        break;
    case 11:
        if (what == 0) CuInitModel_SK_E2(v, s[17], p[16], p[17], cai, eca);
        else if (what == 1) CuDerivModel_SK_E2(dt, v, s[17], p[16], p[17], cai, eca);
        else CuBreakpointModel_SK_E2(I, g, v, s[17], p[16], p[17], cai, eca);
        break;
    case 12:
        if (what == 0) CuInitModel_SKv3_1(v, s[18], p[18]);
        else if (what == 1) CuDerivModel_SKv3_1(dt, v, s[18], p[18]);
        else CuBreakpointModel_SKv3_1(I, g, v, s[18], p[18]);
        break;
    default:
        break;
    }
    if (G) *G = g;
    return I;
}
#endif

#ifdef REF_MAINEN
void CuInitModel_ca(F v, F &m, F &h, F gbar, F cao, F cai, F &ica, F &eca);
void CuInitModel_cad(F v, F &ca, F ica, F &cai, F &eca);
void CuInitModel_kca(F v, F &n, F gbar, F caix, F Ra, F Rb, F cai, F &eca);
void CuInitModel_km(F v, F &n, F gbar, F tha, F qa, F Ra, F Rb);
void CuInitModel_kv(F v, F &n, F gbar, F tha, F qa, F Ra, F Rb);
void CuInitModel_na(F v, F &m, F &h, F gbar, F tha, F qa, F Ra, F Rb, F thi1, F thi2, F qi,
                    F thinf, F qinf, F Rg, F Rd);
void CuDerivModel_ca(F dt, F v, F &m, F &h, F gbar, F cao, F cai, F &ica, F &eca);
void CuDerivModel_cad(F dt, F v, F &ca, F ica, F &cai, F &eca);
void CuDerivModel_kca(F dt, F v, F &n, F gbar, F caix, F Ra, F Rb, F cai, F &eca);
void CuDerivModel_km(F dt, F v, F &n, F gbar, F tha, F qa, F Ra, F Rb);
void CuDerivModel_kv(F dt, F v, F &n, F gbar, F tha, F qa, F Ra, F Rb);
void CuDerivModel_na(F dt, F v, F &m, F &h, F gbar, F tha, F qa, F Ra, F Rb, F thi1, F thi2,
                     F qi, F thinf, F qinf, F Rg, F Rd);
void CuBreakpointModel_ca(D &I, F &G, F v, F &m, F &h, F gbar, F cao, F cai, F &ica, F &eca);
void CuBreakpointModel_kca(D &I, F &G, F v, F &n, F gbar, F caix, F Ra, F Rb, F cai, F &eca);
void CuBreakpointModel_km(D &I, F &G, F v, F &n, F gbar, F tha, F qa, F Ra, F Rb);
void CuBreakpointModel_kv(D &I, F &G, F v, F &n, F gbar, F tha, F qa, F Ra, F Rb);
void CuBreakpointModel_na(D &I, F &G, F v, F &m, F &h, F gbar, F tha, F qa, F Ra, F Rb, F thi1,
                          F thi2, F qi, F thinf, F qinf, F Rg, F Rd);
void CuBreakpointModel_pas(D &I, F &G, F v, F g, F e);
void CuBreakpointModel_pas2(D &I, F &G, F v, F g, F e);
void CuBreakpointModel_pasx(D &I, F &G, F v, F g, F e);

// One mechanism of the Mainen set.  s: 8 states, then cai, eca, ica; p: 34 params.
extern "C" double ref_mainen_mech(int mech, int what, float dt, float v, float *s, const float *p,
                                  float *G) {
    F &cai = s[8], &eca = s[9], &ica = s[10];
    D I = 0;
    F g = 0;
    const F *q = p + 16;
    switch (mech) {
    case 0:
        if (what == 0) CuInitModel_ca(v, s[0], s[1], p[0], p[1], cai, ica, eca);
        else if (what == 1) CuDerivModel_ca(dt, v, s[0], s[1], p[0], p[1], cai, ica, eca);
        else CuBreakpointModel_ca(I, g, v, s[0], s[1], p[0], p[1], cai, ica, eca);
        break;
    case 1:
        if (what == 0) CuInitModel_cad(v, s[2], ica, cai, eca);
        else if (what == 1) CuDerivModel_cad(dt, v, s[2], ica, cai, eca);
        break;
    case 2:
        if (what == 0) CuInitModel_kca(v, s[3], p[2], p[3], p[4], p[5], cai, eca);
        else if (what == 1) CuDerivModel_kca(dt, v, s[3], p[2], p[3], p[4], p[5], cai, eca);
        else CuBreakpointModel_kca(I, g, v, s[3], p[2], p[3], p[4], p[5], cai, eca);
        break;
    case 3:
        if (what == 0) CuInitModel_km(v, s[4], p[6], p[7], p[8], p[9], p[10]);
        else if (what == 1) CuDerivModel_km(dt, v, s[4], p[6], p[7], p[8], p[9], p[10]);
        else CuBreakpointModel_km(I, g, v, s[4], p[6], p[7], p[8], p[9], p[10]);
        break;
    case 4:
        if (what == 0) CuInitModel_kv(v, s[5], p[11], p[12], p[13], p[14], p[15]);
        else if (what == 1) CuDerivModel_kv(dt, v, s[5], p[11], p[12], p[13], p[14], p[15]);
        else CuBreakpointModel_kv(I, g, v, s[5], p[11], p[12], p[13], p[14], p[15]);
        break;
    case 5:
        if (what == 0)
            CuInitModel_na(v, s[6], s[7], q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8], q[9],
                           q[10], q[11]);
        else if (what == 1)
            CuDerivModel_na(dt, v, s[6], s[7], q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8],
                            q[9], q[10], q[11]);
        else
            CuBreakpointModel_na(I, g, v, s[6], s[7], q[0], q[1], q[2], q[3], q[4], q[5], q[6],
                                 q[7], q[8], q[9], q[10], q[11]);
        break;
    case 6:
        if (what == 2) CuBreakpointModel_pas(I, g, v, p[28], p[29]);
        break;
    case 7:
        if (what == 2) CuBreakpointModel_pas2(I, g, v, p[30], p[31]);
        break;
    case 8:
        if (what == 2) CuBreakpointModel_pasx(I, g, v, p[32], p[33]);
        break;
    default:
        break;
    }
    if (G) *G = g;
    return I;
}
#endif
