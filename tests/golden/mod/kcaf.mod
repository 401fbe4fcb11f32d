: Calcium-activated potassium current, Hill-type activation by cai with a
: fixed time constant.  Test mechanism of neurogpu_b200.nmodl.
NEURON {
    SUFFIX kcaf
    USEION k READ ek WRITE ik
    USEION ca READ cai
    RANGE gbar, kd, tauz
}
UNITS { (mV) = (millivolt) (mA) = (milliamp) (S) = (siemens) (mM) = (milli/liter) }
PARAMETER {
    gbar = 0.002 (S/cm2)
    kd = 5e-4 (mM)
    tauz = 10 (ms)
}
ASSIGNED { v (mV) ek (mV) ik (mA/cm2) cai (mM) zinf }
STATE { z }
BREAKPOINT {
    SOLVE act METHOD cnexp
    ik = gbar*z*(v - ek)
}
INITIAL {
    occupancy(cai)
    z = zinf
}
DERIVATIVE act {
    occupancy(cai)
    z' = (zinf - z)/tauz
}
PROCEDURE occupancy(c (mM)) {
    if (c < 1e-9) { c = 1e-9 }
    zinf = c^2/(c^2 + kd^2)
}
