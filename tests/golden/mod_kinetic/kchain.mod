: Three-state potassium channel c1 <-> c2 <-> o with exponential rates.
: Written for the kinetic-scheme tests of the NMODL generator.
NEURON {
    SUFFIX kchain
    USEION k READ ek WRITE ik
    RANGE gbar, a0, b0
}
UNITS {
    (mA) = (milliamp)
    (mV) = (millivolt)
    (S) = (siemens)
}
PARAMETER {
    gbar = 0.01 (S/cm2)
    a0 = 0.2 (/ms)
    b0 = 0.05 (/ms)
}
ASSIGNED {
    v (mV)
    ek (mV)
    ik (mA/cm2)
    a1 (/ms)
    a2 (/ms)
    b1 (/ms)
    b2 (/ms)
}
STATE { c1 c2 o }
BREAKPOINT {
    SOLVE kin METHOD sparse
    ik = gbar * o * (v - ek)
}
INITIAL {
    SOLVE kin STEADYSTATE sparse
}
KINETIC kin {
    rates(v)
    ~ c1 <-> c2 (a1, b1)
    ~ c2 <-> o (a2, b2)
    CONSERVE c1 + c2 + o = 1
}
PROCEDURE rates(v (mV)) {
    a1 = a0 * exp((v + 40) / 20)
    b1 = b0 * exp(-(v + 40) / 25)
    a2 = 2 * a0 * exp((v + 30) / 15)
    b2 = b0 * exp(-(v + 30) / 30)
}
