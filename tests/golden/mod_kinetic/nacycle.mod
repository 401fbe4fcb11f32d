: Four-state sodium channel: closed, open, fast- and slow-inactivated,
: with a closed-state inactivation path closing a cycle (c <-> o <-> i1 <-> c)
: so that the elimination fills in.  Written for the kinetic-scheme tests of
: the NMODL generator.
NEURON {
    SUFFIX nacycle
    USEION na READ ena WRITE ina
    RANGE gbar
}
UNITS {
    (mA) = (milliamp)
    (mV) = (millivolt)
    (S) = (siemens)
}
PARAMETER {
    gbar = 0.05 (S/cm2)
    kslow = 0.002 (/ms)
}
ASSIGNED {
    v (mV)
    ena (mV)
    ina (mA/cm2)
}
STATE { c o i1 i2 }
BREAKPOINT {
    SOLVE scheme METHOD sparse
    ina = gbar * o * (v - ena)
}
INITIAL {
    SOLVE scheme STEADYSTATE sparse
}
KINETIC scheme {
    LOCAL ao, bo, ai, bi
    ao = 3 * exp((v + 35) / 9)
    bo = 0.5 * exp(-(v + 35) / 12)
    ai = 0.8 * exp((v + 50) / 30)
    bi = 0.02 * exp(-(v + 70) / 10)
    ~ c <-> o (ao, bo)
    ~ o <-> i1 (ai, 0.01 * bi)
    ~ i1 <-> c (bi, 0.05 * ai)
    ~ i1 <-> i2 (kslow, 0.1 * kslow)
    CONSERVE c + o + i1 + i2 = 1
}
