: Potassium channel whose time constant is a FUNCTION_TABLE of the voltage
: (values supplied to the generator, as NEURON fills them from hoc).
: Written for the FUNCTION_TABLE tests of the NMODL generator.
NEURON {
    SUFFIX ktab
    USEION k READ ek WRITE ik
    RANGE gbar
}
UNITS {
    (mA) = (milliamp)
    (mV) = (millivolt)
    (S) = (siemens)
}
PARAMETER {
    gbar = 0.01 (S/cm2)
}
ASSIGNED {
    v (mV)
    ek (mV)
    ik (mA/cm2)
    ninf
    ntau (ms)
}
STATE { n }
FUNCTION_TABLE tautab(v (mV)) (ms)
BREAKPOINT {
    SOLVE states METHOD cnexp
    ik = gbar * n * n * (v - ek)
}
INITIAL {
    rates(v)
    n = ninf
}
DERIVATIVE states {
    rates(v)
    n' = (ninf - n) / ntau
}
PROCEDURE rates(v (mV)) {
    ninf = 1 / (1 + exp(-(v + 40) / 10))
    ntau = tautab(v)
}
