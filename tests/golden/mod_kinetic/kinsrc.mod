: Two-state scheme with a constant source and no conservation law; a
: nonspecific current through the second state.  Written for the
: kinetic-scheme tests of the NMODL generator.
NEURON {
    SUFFIX kinsrc
    NONSPECIFIC_CURRENT i
    RANGE g, e, k1, k2, s
}
PARAMETER {
    g = 0.001 (S/cm2)
    e = -20 (mV)
    k1 = 0.3 (/ms)
    k2 = 0.1 (/ms)
    s = 0.02 (/ms)
}
ASSIGNED {
    v (mV)
    i (mA/cm2)
}
STATE { a b }
BREAKPOINT {
    SOLVE sch METHOD sparse
    i = g * b * (v - e)
}
INITIAL {
    a = 0.2
    b = 0.1
}
KINETIC sch {
    ~ a <-> b (k1 * exp(v / 40), k2)
    ~ a << (s)
}
