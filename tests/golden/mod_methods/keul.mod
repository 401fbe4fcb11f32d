: Two-state potassium channel integrated by explicit Euler; h relaxes towards
: m, so the step shows whether every derivative reads the states the step
: started from.  Written for the integration-method tests of the NMODL
: generator.
NEURON {
    SUFFIX keul
    USEION k READ ek WRITE ik
    RANGE gbar
}
UNITS { (mA) = (milliamp) (mV) = (millivolt) (S) = (siemens) }
PARAMETER { gbar = 0.01 (S/cm2) }
ASSIGNED {
    v (mV)
    ek (mV)
    ik (mA/cm2)
    minf
    mtau (ms)
}
STATE { m h }
BREAKPOINT {
    SOLVE states METHOD euler
    ik = gbar * m * h * (v - ek)
}
INITIAL {
    rates(v)
    m = minf
    h = minf
}
DERIVATIVE states {
    rates(v)
    m' = (minf - m) / mtau
    h' = (m - h) / 20
}
PROCEDURE rates(v (mV)) {
    minf = 1 / (1 + exp(-(v + 30) / 8))
    mtau = 2 + 3 * exp(-((v + 40) / 20)^2)
}
