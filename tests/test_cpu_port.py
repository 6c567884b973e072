"""The OpenMP CPU port (oracle/cpu_port.*), which bench.py times as the
reference arm and as cpu_baseline, computes the same term as the FP64
oracle: a port that dropped a term or a pair would make the device path
look faster than it is.  Runs on the CPU."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle.cpu_port import CpuPort
from mdir_b200 import systems

# the port's pair loop is f32 (MDIR's mixed precision); its PME is f64 with
# the grid in i64 fixed point at 2^40
FORCE_RMS_TOL = 1e-5
ENERGY_TOL = 1e-6


def rms_rel(f, ref):
    return np.sqrt(np.mean(np.sum((f - ref) ** 2, 1))) / np.sqrt(np.mean(np.sum(ref ** 2, 1)))


@pytest.mark.parametrize("reach", [1.0, 1.05, 1.2])
def test_port_matches_the_oracle_on_a_water_box(reach):
    s = dict(systems.tip3p(waters=900, seed=7))
    s["reach"] = reach
    ref = O.evaluate(s, s["positions"])
    cp = CpuPort(s, threads=4)
    cp.build(s["positions"])
    f, terms = cp.force(s["positions"])
    assert rms_rel(f, ref["forces"]) < FORCE_RMS_TOL
    scale = sum(abs(v) for v in ref["terms"].values())
    for name in ("lj", "coulomb", "excluded", "reciprocal"):
        assert abs(terms[name] - ref["terms"][name]) <= ENERGY_TOL * scale, name


def test_port_keeps_every_pair_after_the_atoms_move():
    # lists built at x0 serve positions within half the skin of it
    s = dict(systems.tip3p(waters=600, seed=8))
    s["reach"] = 1.05
    x0 = s["positions"]
    rng = np.random.default_rng(3)
    x1 = x0 + rng.uniform(-0.07, 0.07, size=x0.shape) / np.sqrt(3.0)
    cp = CpuPort(s, threads=4)
    cp.build(x0)
    f, terms = cp.force(x1)
    ref = O.evaluate(s, x1)
    assert rms_rel(f, ref["forces"]) < FORCE_RMS_TOL
    scale = sum(abs(v) for v in ref["terms"].values())
    assert abs(terms["lj"] - ref["terms"]["lj"]) <= ENERGY_TOL * scale
    assert abs(terms["coulomb"] - ref["terms"]["coulomb"]) <= ENERGY_TOL * scale


def test_port_on_argon():
    s = systems.argon()
    ref = O.evaluate(s, s["positions"])
    cp = CpuPort(s, threads=4)
    cp.build(s["positions"])
    f, terms = cp.force(s["positions"])
    assert rms_rel(f, ref["forces"]) < FORCE_RMS_TOL
    assert abs(terms["lj"] - ref["terms"]["lj"]) <= ENERGY_TOL * abs(ref["terms"]["lj"])


def test_reference_fft_and_numpy_fallback_agree(monkeypatch):
    # with MDIR's mdrt_fft.c (built from the reference's sources) and
    # without it the port computes the same reciprocal sum
    import oracle.cpu_port as P
    s = dict(systems.tip3p(waters=300, seed=9))
    got = []
    for use in (True, False):
        P.port()
        if use and not P.reference_fft():
            continue
        monkeypatch.setattr(P, "_fft", use)
        cp = CpuPort(s, threads=2)
        cp.build(s["positions"])
        got.append(cp.force(s["positions"]))
    if len(got) == 2:
        (fa, ta), (fb, tb) = got
        assert ta["reciprocal"] == pytest.approx(tb["reciprocal"], rel=1e-12)
        np.testing.assert_allclose(fa, fb, rtol=1e-9, atol=1e-9 * np.abs(fb).max())
