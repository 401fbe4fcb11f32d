: Intracellular calcium pool integrated by derivimplicit (implicit Euler):
: influx from the calcium current into a shell, relaxation to a resting
: level.  Written for the integration-method tests of the NMODL generator.
NEURON {
    SUFFIX cabe
    USEION ca READ ica WRITE cai
    RANGE taur, cainf, depth
}
UNITS { (mM) = (milli/liter) (um) = (micron) (mA) = (milliamp)
        FARADAY = (faraday) (coulomb) }
PARAMETER {
    taur = 80 (ms)
    cainf = 1e-4 (mM)
    depth = 0.5 (um)
}
ASSIGNED { ica (mA/cm2) }
STATE { cai (mM) }
INITIAL { cai = cainf }
BREAKPOINT { SOLVE pool METHOD derivimplicit }
DERIVATIVE pool {
    cai' = -ica*(10000)/(2*FARADAY*depth) - (cai - cainf)/taur
}
