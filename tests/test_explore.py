"""Parameter exploration (GUI/run_neuroGPU.py, GUI/plot_param_explor.py):
the grid, the opt_table reader, and the dV/dt peak-count score.

The score is scipy.signal.find_peaks(dvdt, 15, distance=5) per trace in the
reference.  oracle/find_peaks_ref.py restates scipy's algorithm; the CPU
tests pin it against scipy itself, and the GPU tests check the CUDA kernel
(ngpu_trace_dvdt_peaks, ngpu_sim_dvdt_peaks) against both: counts exactly
equal.  Inputs with equal-height peaks closer than `distance` are checked
against the restatement only (scipy leaves their order to numpy's unstable
argsort)."""
import ctypes as C
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLD = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT / "oracle"))
import find_peaks_ref as fpr  # noqa: E402

from neurogpu_b200 import explore  # noqa: E402

scipy_signal = pytest.importorskip("scipy.signal")
DT = 0.1


def _scipy_count(v, dt=DT, height=15.0, distance=5):
    dvdt = np.diff(np.asarray(v, dtype=np.float64)) / dt
    return len(scipy_signal.find_peaks(dvdt, height, distance=distance)[0])


def _close_tie(v, dt=DT, height=15.0, distance=5):
    """Two candidate peaks of equal height closer than `distance` (the case
    whose outcome scipy leaves to numpy's argsort)."""
    x = np.diff(np.asarray(v, dtype=np.float64)) / dt
    pk = [p for p in fpr.local_maxima(x) if x[p] >= height]
    return any(pk[j] - pk[i] < distance and x[pk[i]] == x[pk[j]]
               for i in range(len(pk)) for j in range(i + 1, len(pk)))


def _check_against_scipy(traces, counts, dt=DT, height=15.0, distance=5):
    """counts equal scipy's on every trace without a close tie and the
    restatement's on every trace; returns the number compared with scipy."""
    n = 0
    for v, c in zip(traces, counts):
        assert c == fpr.dvdt_peak_count(v, dt, height, distance)
        if not _close_tie(v, dt, height, distance):
            assert c == _scipy_count(v, dt, height, distance)
            n += 1
    return n


def _spiky_traces(rng, n, nt):
    """Seeded float32 traces: rest plus noise, AP-like upstrokes at random
    times (some closer together than the distance), plateaus in dV/dt."""
    out = np.empty((n, nt), dtype=np.float32)
    for k in range(n):
        v = -70.0 + rng.normal(0.0, 0.05 + 0.5 * (k % 3), nt)
        n_sp = rng.integers(0, 12)
        for t0 in rng.integers(5, nt - 12, n_sp):
            w = rng.integers(2, 6)
            v[t0:t0 + w] += np.linspace(0, rng.uniform(2.0, 60.0), w)
            v[t0 + w:t0 + w + 4] += rng.uniform(2.0, 60.0)
        if k % 5 == 0:  # a linear ramp: a plateau of equal dV/dt values
            t0 = nt // 3
            v[t0:t0 + 6] = -70.0 + 2.0 * np.arange(6, dtype=np.float32)
        out[k] = v
    return out


def _edge_traces(nt=64):
    """Hand-made cases: flat, one sample, peaks at the ends, a long
    alternating cluster, a NaN, equal-height twins closer than the
    distance, a plateau ending in a rise."""
    cases = []
    cases.append(np.full(nt, -65.0))
    z = np.full(nt, -65.0)
    z[1] = 0.0
    cases.append(z)                                   # dV/dt peak at index 0: never a peak
    z = np.full(nt, -65.0)
    z[-1] = 0.0
    cases.append(z)                                   # rise into the last sample
    z = np.full(nt, -65.0)
    z[10:50:2] += 3.0 + 0.1 * np.arange(20)            # alternating: a 20-peak cluster
    cases.append(z)
    z = np.full(nt, -65.0)
    z[20] = 0.0
    z[21] = np.nan
    z[40] = 0.0
    cases.append(z)
    z = np.full(nt, -65.0)
    z[10] = -60.0
    z[11] = -65.0
    z[13] = -60.0                                      # equal heights 3 samples apart
    cases.append(z)
    z = np.full(nt, -65.0)
    z[10:14] = -65.0 + 2.0 * np.arange(1, 5)           # plateau of 2.0/dt, then
    z[14:] = z[13] + 5.0                               # a larger step: no peak on the plateau
    cases.append(z)
    return np.stack(cases).astype(np.float32)


def test_restatement_matches_scipy():
    rng = np.random.default_rng(11)
    tr = _spiky_traces(rng, 300, 400)
    for d in (1, 2, 5, 9):
        n = 0
        for v in tr:
            if not _close_tie(v, DT, 15.0, d):
                assert fpr.dvdt_peak_count(v, DT, 15.0, d) == _scipy_count(v, DT, 15.0, d)
                n += 1
        assert n >= 290
    edge = _edge_traces()
    assert [_close_tie(v) for v in edge] == [False] * 5 + [True, False]
    for k, v in enumerate(edge):
        if k != 5:
            assert fpr.dvdt_peak_count(v, DT) == _scipy_count(v, DT), k


def test_restatement_tie_rule():
    """Equal heights closer than the distance: the later peak is kept."""
    x = np.zeros(20)
    x[5] = x[8] = 20.0
    assert fpr.find_peaks(x, 15.0, 5) == [8]
    x[11] = 20.0
    assert fpr.find_peaks(x, 15.0, 5) == [5, 11]  # 11 first, drops 8; then 5


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    """The kernel's per-trace code (csrc/explore.cuh) built for the host."""
    src = ROOT / "tests" / "native" / "peaks_probe.cu"
    lib = tmp_path_factory.mktemp("peaks") / "peaks_probe.so"
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared", "-x", "cu", str(src),
                    "-o", str(lib)], check=True, capture_output=True)
    L = C.CDLL(str(lib))
    L.probe_dvdt_peaks.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_void_p]
    return L


def _probe_counts(L, traces, dt=DT, height=15.0, distance=5):
    tr = np.ascontiguousarray(traces, dtype=np.float32)
    out = np.zeros(tr.shape[0], dtype=np.int32)
    L.probe_dvdt_peaks(tr.ctypes.data, tr.shape[0], tr.shape[1], dt, height, distance, out.ctypes.data)
    return out


def test_kernel_code_on_the_host_matches_the_restatement(probe):
    """The same per-trace function the CUDA kernel runs, compiled for the
    host: equal counts to the restatement on seeded traces (every height
    and distance tried) and on the hand-made cases, ties included."""
    rng = np.random.default_rng(14)
    tr = _spiky_traces(rng, 200, 300)
    for dt, h, d in ((DT, 15.0, 5), (DT, 15.0, 1), (0.025, 40.0, 2), (DT, -np.inf, 7)):
        got = _probe_counts(probe, tr, dt, h, d)
        assert np.array_equal(got, [fpr.dvdt_peak_count(v, dt, h, d) for v in tr])
    edge = _edge_traces()
    assert np.array_equal(_probe_counts(probe, edge), [fpr.dvdt_peak_count(v, DT) for v in edge])
    # short traces: the shortest with a peak has 4 samples (3 of dV/dt)
    assert np.array_equal(_probe_counts(probe, np.array([[0, 0, 5, 0], [0, 5, 0, 0]], dtype=np.float32)), [1, 0])
    for n in (1, 2, 3):
        assert _probe_counts(probe, np.zeros((1, n), dtype=np.float32) + np.arange(n) * 5)[0] == 0


def test_kernel_code_on_oracle_traces(probe):
    """Spiking traces of the reference's shipped TTPC cell (the FP64 oracle,
    a 3 x 4 grid over g_pas and the soma's gNaTs2_t, 3168 steps of 0.1 ms),
    rounded to float32 as the simulator records them: the kernel's per-trace
    code built for the host counts what scipy counts."""
    import oracle_py
    from neurogpu_b200 import evaluator, formats
    m = formats.read_data_dir(GOLD / "ttpc512", stim_index=0, params_file="AllParams_reference.csv")
    mapping, g_na = _ttpc512_mapping(m)
    base = np.zeros(14)
    base[0], base[2] = 3e-5, g_na
    grid = explore.gen_params(base, 0, base[0] * np.array([0.5, 1.0, 2.0]), 2,
                              base[2] * np.array([0.25, 0.5, 1.0, 2.0]))
    rows = evaluator.allparams_from_mapping(grid, *mapping)
    nc = m.cell.n_sections
    fp = rows.reshape(len(rows), rows.shape[1] // nc, nc).astype(np.float32)
    params = formats.map_params(fp, int(m.raw["basic_const"]["NModels"][0]), fp.shape[1])
    c = m.cell
    v = np.asarray(oracle_py.run(c.parent, c.a, c.b, c.cm, c.section, c.n_sections, c.mechset.id, c.mech_mask,
                                 params, m.amps[:1], m.dts, m.stim_node, m.stim_area, m.rec_nodes[:1], m.v_init))
    tr = v[:, 0, 0, :].astype(np.float32)
    got = _probe_counts(probe, tr)
    assert _check_against_scipy(tr, got) >= 10
    assert got.min() >= 1 and got.max() >= 10


def test_gen_params_is_the_reference_grid():
    """The reference's nested loop (GUI/run_neuroGPU.py:15-31), restated."""
    names, lb, ub, base = explore.read_opt_table(GOLD / "ttpc512" / "opt_table.csv")
    t = np.genfromtxt(GOLD / "ttpc512" / "opt_table.csv", dtype=float, delimiter=",", names=True)
    assert list(t.dtype.names) == names
    assert np.array_equal(np.array(t[0].tolist()), lb) and np.array_equal(np.array(t[2].tolist()), base)
    assert np.array_equal(np.array(t[1].tolist()), ub)
    ref = []
    for p1 in np.linspace(0, 10, 100):
        for p2 in np.linspace(0, 20, 100):
            row = np.copy(base)
            row[0] = p1
            row[2] = p2
            ref.append(row)
    got = explore.gen_params(base)
    assert got.shape == (10000, base.size)
    assert np.array_equal(got, np.array(ref))
    with pytest.raises(ValueError):
        explore.gen_params(base, 1, None, 1, None)


def test_calc_scores_layout(tmp_path, monkeypatch):
    """calc_scores on the host side: a VHotP file read as the reference
    reads it, the overhang dropped, trace k at cell (k // nbins, k % nbins)
    (the counts themselves come from the restatement here)."""
    import torch
    from neurogpu_b200 import formats
    monkeypatch.setattr(explore, "dvdt_peak_counts", lambda v, dt, height, distance: torch.tensor(
        [fpr.dvdt_peak_count(x, dt, height, distance) for x in v], dtype=torch.int32))
    rng = np.random.default_rng(15)
    nb = 5
    tr = _spiky_traces(rng, nb * nb, 200)
    p = tmp_path / "VHotP0.dat"
    formats.write_vhot(p, np.concatenate([tr.reshape(-1).astype(np.float64), np.zeros(11)]))
    s = explore.calc_scores(p, nbins=nb)
    assert s.shape == (nb, nb) and s.dtype == np.float64
    assert np.array_equal(s.reshape(-1), [fpr.dvdt_peak_count(v, DT) for v in tr])
    assert s.max() > 0
    with pytest.raises(ValueError):
        explore.calc_scores(np.zeros(nb * nb - 1), nbins=nb)


def test_entry_points_reject_bad_arguments(ngpu_built):
    """Argument checks of the C ABI (they return before any launch)."""
    from neurogpu_b200 import _ffi
    L = _ffi.lib()
    assert L.ngpu_dvdt_peaks_scratch_bytes(10000, 3168) == 10000 * (3168 // 2 + 1) * 4
    out = C.c_void_p(0)
    args = lambda dt, dist, sb: (None, 1, 1, 4, 100, dt, 15.0, dist, None, sb, out, None)  # noqa: E731
    assert L.ngpu_trace_dvdt_peaks(*args(0.0, 5, 1 << 20)) == -1
    assert b"dt" in L.ngpu_last_error()
    assert L.ngpu_trace_dvdt_peaks(*args(0.1, 0, 1 << 20)) == -1
    assert b"distance" in L.ngpu_last_error()
    assert L.ngpu_trace_dvdt_peaks(*args(0.1, 5, 16)) == -1
    assert b"scratch" in L.ngpu_last_error()
    assert L.ngpu_trace_dvdt_peaks(*args(0.1, 5, 1 << 20)) == -1
    assert b"null" in L.ngpu_last_error()
    assert L.ngpu_trace_dvdt_peaks(None, 1, 1, 0, 100, 0.1, 15.0, 5, None, 0, None, None) == 0  # no traces


@pytest.mark.gpu
def test_kernel_matches_scipy_and_restatement(ngpu_built):
    import torch
    rng = np.random.default_rng(12)
    tr = _spiky_traces(rng, 1000, 600)
    got = explore.dvdt_peak_counts(tr).cpu().numpy()
    assert _check_against_scipy(tr, got) >= 950
    assert got.max() >= 5 and (got == 0).any()
    edge = _edge_traces()
    got = explore.dvdt_peak_counts(edge).cpu().numpy()
    _check_against_scipy(edge, got)
    # other heights and distances, and a strided view of device memory
    t = torch.from_numpy(np.ascontiguousarray(tr.T)).cuda()   # [sample][trace]
    got = explore.dvdt_peak_counts(t.T, dt=0.025, height=40.0, distance=2).cpu().numpy()
    _check_against_scipy(tr, got, 0.025, 40.0, 2)
    # float64 VHotP values holding float32 samples are taken as they are
    got = explore.dvdt_peak_counts(tr[:10].astype(np.float64)).cpu().numpy()
    _check_against_scipy(tr[:10], got)
    with pytest.raises(ValueError):
        explore.dvdt_peak_counts(tr[:2].astype(np.float64) + 1e-9)


@pytest.mark.gpu
def test_calc_scores_of_a_vhot_file(ngpu_built, tmp_path):
    """calc_scores reads a VHotP file as the reference does (overhang
    dropped) and maps trace k to cell (k // nbins, k % nbins)."""
    from neurogpu_b200 import formats
    rng = np.random.default_rng(13)
    nb = 6
    tr = _spiky_traces(rng, nb * nb, 300)
    flat = np.concatenate([tr.reshape(-1).astype(np.float64), np.zeros(7)])
    p = tmp_path / "VHotP0.dat"
    formats.write_vhot(p, flat)
    s = explore.calc_scores(p, nbins=nb)
    assert s.shape == (nb, nb)
    _check_against_scipy(tr, s.reshape(-1).astype(np.int64))


def _ttpc512_mapping(m):
    """GA parameter 0 -> g_pas in every section, 2 -> the soma's gNaTs2_t.
    The shipped AllParams_for_params.csv marks its GA parameters at entries
    that do not match opt_table.csv's names (parameter 0 marks two
    zero-valued entries), so the test states its own mapping."""
    from neurogpu_b200 import evaluator
    from neurogpu_b200.mechsets import TTPC
    tmpl, _, _ = evaluator.load_mapping(GOLD / "ttpc512")
    nc = m.cell.n_sections
    nats = tmpl.reshape(-1, nc)[TTPC.param_index("gNaTs2_tbar_NaTs2_t")]
    soma = np.nonzero(nats == nats.max())[0]
    return explore.mapping_for(tmpl, nc, {0: (TTPC.param_index("g_pas"), None),
                                          2: (TTPC.param_index("gNaTs2_tbar_NaTs2_t"), soma)}), nats.max()


def test_float32_rows_equal_the_rounded_float64_rows():
    """allparams_from_mapping(..., dtype=float32), the rows the exploration
    uploads, equal the float64 rows rounded entry by entry, bit for bit."""
    from neurogpu_b200 import evaluator, formats
    m = formats.read_data_dir(GOLD / "ttpc512", stim_index=0, params_file="AllParams_reference.csv")
    (tmpl, ind, _), g_na = _ttpc512_mapping(m)
    _, _, _, base = explore.read_opt_table(GOLD / "ttpc512" / "opt_table.csv")
    grid = explore.gen_params(base)
    r64 = evaluator.allparams_from_mapping(grid, tmpl, ind, {5: 0.25})
    r32 = evaluator.allparams_from_mapping(grid, tmpl, ind, {5: 0.25}, dtype=np.float32)
    assert r32.dtype == np.float32 and r64.dtype == np.float64
    assert np.array_equal(r32.view(np.uint32), r64.astype(np.float32).view(np.uint32))


def test_mapping_for_marks_the_given_entries():
    from neurogpu_b200 import evaluator, formats
    m = formats.read_data_dir(GOLD / "ttpc512", stim_index=0, params_file="AllParams_reference.csv")
    (tmpl, ind, corr), g_na = _ttpc512_mapping(m)
    nc = m.cell.n_sections
    assert corr == {} and ind.size == tmpl.size == 19 * nc
    assert (ind == 12300).sum() == 239 and (ind == 12302).sum() == 1
    rows = evaluator.allparams_from_mapping([[1e-4, 0.0, 0.5]], tmpl, ind)
    t, r = tmpl.reshape(19, nc), rows[0].reshape(19, nc)
    assert np.all(r[14][t[14] != 0] == 1e-4) and np.all(r[14][t[14] == 0] == 0)
    assert r[13].max() == 0.5 and np.array_equal(np.sort(r[13])[:-1], np.sort(t[13])[:-1])
    assert g_na == t[13].max()


@pytest.mark.gpu
def test_explore_on_the_reference_model(ngpu_built):
    """A 3 x 4 grid over the shipped TTPC cell's g_pas (every section) and
    somatic gNaTs2_t, 3168 steps of 0.1 ms under its Stim_raw0: the score
    computed where the traces lie equals scipy's count on the same
    simulation's read-back traces, and explore() returns that map.  (The
    FP64 oracle gives counts 2 to 14 over this grid.)"""
    from neurogpu_b200 import formats
    d = GOLD / "ttpc512"
    m = formats.read_data_dir(d, stim_index=0, params_file="AllParams_reference.csv")
    mapping, g_na = _ttpc512_mapping(m)
    base = np.zeros(14)
    base[0], base[2] = 3e-5, g_na
    v1 = base[0] * np.array([0.5, 1.0, 2.0])
    v2 = base[2] * np.array([0.25, 0.5, 1.0, 2.0])
    grid = explore.gen_params(base, 0, v1, 2, v2)
    sim, score_dt = explore.grid_simulation(m, mapping, grid)
    assert score_dt == 0.1
    got = sim.dvdt_peaks(score_dt).cpu().numpy()[:, 0]
    v = sim.trace()[:, 0, 0, :]
    assert _check_against_scipy(v, got) >= 10
    assert got.min() >= 1 and got.max() >= 10          # the grid spans few to many spikes
    scores, g2 = explore.explore(m, mapping, base, 0, v1, 2, v2)
    assert np.array_equal(g2, grid)
    assert np.array_equal(scores, got.reshape(3, 4).astype(np.float64))
