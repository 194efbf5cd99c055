"""End-to-end physics against eduPIC: the reference case of
C/ReferenceCase_RawData (eduPIC in FP64, converged over ~7900 RF cycles:
argon, 25 mm, 250 V, 13.56 MHz, 10 Pa) against this library's fused driver
(cudapic_b200.refcase: two seeds started from the reference's density
profiles, RELAX cycles of relaxation, MEASURE cycles measured).  Compared:
cycle-averaged n_e, n_i (Figure 10), the period-averaged potential (Figure
11c), the EEPF below 15 eV (Figure 12), the <j E> electron power (Figure
11g) and the electron count (Figure 9).  The tolerances are the stated
end-to-end error of the f32 path against the FP64 oracle; the two seeds'
difference (printed) is the statistical noise floor.
"""
import os

import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RELAX, MEASURE = 300, 100
# Measured: n_e 0.054, EEPF 0.042, power 0.014, N_e 0.051, potential 0.002
# at a seed-to-seed spread of 0.002-0.011; the few per cent of n_e and N_e
# follow the GPU reference's model differences from eduPIC (for example,
# electrons spawned in a step do not collide in the same step).
TOL = {"ne": 0.08, "ni": 0.08, "pot": 0.02, "eepf": 0.08, "power_e": 0.05, "count_e": 0.08}


def test_reference_case_profiles_against_edupic(cudapic, cuda_device):
    from cudapic_b200 import refcase
    ref = refcase.load_reference(GOLDEN)
    r = refcase.study(ref, "mixed", RELAX, MEASURE)
    print("\nreference case, %d relaxation + %d measured cycles, 2 seeds" % (RELAX, MEASURE))
    for key in TOL:
        print("  %-8s error %.4f  seed-to-seed %.4f  tolerance %.2f"
              % (key, r["errors"][key], r["seed_spread"][key], TOL[key]))
    assert r["device_errors"] == [0, 0]
    for key in TOL:
        assert r["errors"][key] <= TOL[key], (key, r["errors"][key], r["seed_spread"][key])
