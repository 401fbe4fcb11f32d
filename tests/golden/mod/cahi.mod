: High-voltage-activated calcium current with m^2 h gating and Boltzmann
: steady states.  Test mechanism of neurogpu_b200.nmodl.
NEURON {
    SUFFIX cahi
    USEION ca READ eca WRITE ica
    RANGE gbar
}
UNITS { (mV) = (millivolt) (mA) = (milliamp) (S) = (siemens) }
PARAMETER { gbar = 0.001 (S/cm2) }
ASSIGNED { v (mV) eca (mV) ica (mA/cm2) g (S/cm2) }
STATE { m h }
BREAKPOINT {
    SOLVE kin METHOD cnexp
    g = gbar*m*m*h
    ica = g*(v - eca)
}
INITIAL {
    m = 1/(1 + exp(-(v + 20)/6))
    h = 1/(1 + exp((v + 45)/7))
}
DERIVATIVE kin {
    m' = (1/(1 + exp(-(v + 20)/6)) - m)/(0.5 + 2*exp(-((v + 20)/25)^2))
    h' = (1/(1 + exp((v + 45)/7)) - h)/80
}
