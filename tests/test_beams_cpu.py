"""Several particle beams, predefined beams and the Twiss forms on the host (no GPU).

The golden cases flux_two_beams, traj_predefined_beam, pd_predefined_and_twiss and
traj_named_beam_ideal pin the sampling against the reference build (through the oracle, and the
trajectories directly in test_capi_cpu.py).  Here: the particle sequence of a two-beam request
(a beam picked by weight, then its own draws) against the oracle's, and the errors of
add_particle_beam / set_new_particle with the reference's wording.
"""
import numpy as np
import pytest

from cases import CASES, run_case


def _host():
    from oscars_b200.sr import sr
    return sr(gpu=1, device=-1)


def test_two_beam_particle_sequence_matches_oracle():
    from oracle.oracle import OracleSR
    setup = [c for c in CASES["flux_two_beams"] if not c[0].startswith("calculate")]
    s = _host()
    run_case(s, setup)
    seq = s.beam_particles(40)
    o = OracleSR()
    run_case(o, setup)
    ref = []
    for _ in range(40):
        o.set_new_particle()
        x0, b0 = o.get_particle()[:2]
        ref.append(list(x0) + list(b0))
    assert np.array_equal(seq, np.array(ref))


def test_named_and_predefined_beam_errors():
    s = _host()
    s.add_particle_beam(type="electron", name="a", energy_GeV=3, current=0.5)
    with pytest.raises(ValueError, match="possibly 'name' already exists"):
        s.add_particle_beam(type="electron", name="a", energy_GeV=3)
    with pytest.raises(ValueError, match="Error in predefined beam name / definition"):
        s.add_particle_beam(beam="SPEAR3")
    with pytest.raises(ValueError, match="Error in predefined beam name / definition"):
        s.add_particle_beam(beam="NSLSII", name="a")
    with pytest.raises(ValueError, match="Particle weight cannot be negative"):
        s.add_particle_beam(type="electron", name="w", energy_GeV=3, weight=-1)
    with pytest.raises(ValueError, match="Gamma cannot be <= 0"):
        s.add_particle_beam(type="electron", name="g", energy_GeV=3, alpha=[0, 0], gamma=[0, 1])
    with pytest.raises(ValueError, match="beam name not in map"):
        s.set_new_particle(beam="nobody")
    s.add_particle_beam(beam="NSLS-II", name="n")  # the default name of the next one is _beam2
    s.add_particle_beam(type="positron", energy_GeV=2)
    s.set_new_particle(beam="_beam2", particle="ideal")
    s.clear_particle_beams()
    with pytest.raises(ValueError, match="no beam defined"):
        s.set_new_particle()
