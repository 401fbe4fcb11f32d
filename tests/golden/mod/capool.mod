: First-order intracellular calcium pool: influx from the calcium current
: into a shell of the given depth, relaxation to a resting level.  Test
: mechanism of neurogpu_b200.nmodl.
NEURON {
    SUFFIX capool
    USEION ca READ ica WRITE cai
    RANGE tau, shell, cai_rest
}
UNITS { (mV) = (millivolt) (mA) = (milliamp) (mM) = (milli/liter) (um) = (micron)
        FARADAY = (faraday) (coulomb) }
PARAMETER {
    tau = 50 (ms)
    shell = 0.2 (um)
    cai_rest = 1e-4 (mM)
}
ASSIGNED { ica (mA/cm2) }
STATE { cai (mM) }
INITIAL { cai = cai_rest }
BREAKPOINT { SOLVE pool METHOD cnexp }
DERIVATIVE pool {
    cai' = -ica*(10000)/(2*FARADAY*shell) + (cai_rest - cai)/tau
}
