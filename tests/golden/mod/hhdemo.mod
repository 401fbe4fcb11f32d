: Hodgkin-Huxley squid axon sodium and potassium currents (Hodgkin & Huxley
: 1952, J Physiol 117:500), rates in the modern sign convention with the
: resting potential at -65 mV.  Test mechanism of neurogpu_b200.nmodl.
NEURON {
    SUFFIX hhdemo
    USEION na READ ena WRITE ina
    USEION k READ ek WRITE ik
    RANGE gnabar, gkbar
}
UNITS { (mV) = (millivolt) (mA) = (milliamp) (S) = (siemens) }
PARAMETER {
    gnabar = 0.12 (S/cm2)
    gkbar = 0.036 (S/cm2)
}
ASSIGNED {
    v (mV) ena (mV) ek (mV) ina (mA/cm2) ik (mA/cm2)
    minf hinf ninf mtau (ms) htau (ms) ntau (ms)
}
STATE { m h n }
BREAKPOINT {
    SOLVE gates METHOD cnexp
    ina = gnabar*m*m*m*h*(v - ena)
    ik = gkbar*n^4*(v - ek)
}
INITIAL {
    settle(v)
    m = minf
    h = hinf
    n = ninf
}
DERIVATIVE gates {
    settle(v)
    m' = (minf - m)/mtau
    h' = (hinf - h)/htau
    n' = (ninf - n)/ntau
}
PROCEDURE settle(u (mV)) {
    LOCAL am, bm, ah, bh, an, bn, q
    q = 3^((celsius - 6.3)/10)
    am = 0.1*vtrap(-(u + 40), 10)
    bm = 4*exp(-(u + 65)/18)
    ah = 0.07*exp(-(u + 65)/20)
    bh = 1/(exp(-(u + 35)/10) + 1)
    an = 0.01*vtrap(-(u + 55), 10)
    bn = 0.125*exp(-(u + 65)/80)
    minf = am/(am + bm)
    mtau = 1/(q*(am + bm))
    hinf = ah/(ah + bh)
    htau = 1/(q*(ah + bh))
    ninf = an/(an + bn)
    ntau = 1/(q*(an + bn))
}
FUNCTION vtrap(x, y) {
    if (fabs(x/y) < 1e-6) {
        vtrap = y*(1 - x/y/2)
    } else {
        vtrap = x/(exp(x/y) - 1)
    }
}
