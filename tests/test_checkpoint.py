"""eduPIC's particle checkpoint (picdata.bin, C/eduPIC.cc:726-781) through the
C ABI on the host: round trip, byte layout, and a run of eduPIC itself
(built from the reference sources by oracle/Makefile) from a file written here."""
import os
import re
import subprocess

import numpy as np
import pytest

EDUPIC = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "eduPIC")


def _population(n, seed):
    rng = np.random.default_rng(seed)
    x = (rng.random(n) * 0.025).astype(np.float32)
    v = [rng.normal(0.0, 1e5, n).astype(np.float32) for _ in range(3)]
    return (x, *v)


def test_picdata_round_trip(cudapic, tmp_path):
    from cudapic_b200.checkpoint import read_picdata, write_picdata
    e, i = _population(1001, 1), _population(77, 2)
    path = tmp_path / "picdata.bin"
    write_picdata(path, e, i, time=1.25e-6, cycles_done=17)
    t, cyc, e2, i2 = read_picdata(path)
    assert (t, cyc) == (1.25e-6, 17)
    for a, b in zip(e + i, e2 + i2):
        assert np.array_equal(a, b)
    assert os.path.getsize(path) == 8 * (2 + 1 + 4 * 1001 + 1 + 4 * 77)


def test_picdata_bytes_are_edupics_layout(cudapic, tmp_path):
    """Same bytes as a plain restatement of save_particle_data (doubles in
    the order of C/eduPIC.cc:731-745)."""
    from cudapic_b200.checkpoint import write_picdata
    e, i = _population(300, 3), _population(200, 4)
    write_picdata(tmp_path / "a.bin", e, i, time=3.5e-7, cycles_done=4)
    ref = [np.array([3.5e-7, 4.0, 300.0])] + [a.astype(np.float64) for a in e] + [np.array([200.0])] + \
        [a.astype(np.float64) for a in i]
    assert (tmp_path / "a.bin").read_bytes() == np.concatenate(ref).tobytes()


def test_picdata_rejects_malformed_files(cudapic, tmp_path):
    from cudapic_b200.checkpoint import read_picdata
    p = tmp_path / "bad.bin"
    np.array([0.0, 1.0, 10.0, 0.5], np.float64).tofile(p)   # 10 electrons announced, data missing
    with pytest.raises(cudapic.CudapicError):
        read_picdata(p)
    np.array([0.0, 1.0, -3.0], np.float64).tofile(p)
    with pytest.raises(cudapic.CudapicError):
        read_picdata(p)


@pytest.mark.skipif(not os.path.exists(EDUPIC), reason="eduPIC not built (make -C oracle ref)")
def test_edupic_continues_from_a_file_written_here(cudapic, tmp_path):
    """eduPIC loads the file, runs one RF cycle and writes its own; both
    files are read back here with the counts eduPIC reports."""
    from cudapic_b200.checkpoint import read_picdata, write_picdata
    from cudapic_b200.workloads import edupic_initial
    e, i = edupic_initial(1000, seed=0), edupic_initial(1000, seed=1)
    write_picdata(tmp_path / "picdata.bin", e, i, time=0.0, cycles_done=1)
    out = subprocess.run([os.path.abspath(EDUPIC), "1"], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "data loaded : 1000 electrons 1000 ions, 1 cycles completed before" in out.stdout
    m = re.search(r"data saved : (\d+) electrons (\d+) ions, (\d+) cycles completed, time is (\S+)", out.stdout)
    t, cyc, e2, i2 = read_picdata(tmp_path / "picdata.bin")
    assert (len(e2[0]), len(i2[0]), cyc) == (int(m.group(1)), int(m.group(2)), int(m.group(3))) == \
        (len(e2[0]), len(i2[0]), 2)
    assert t == pytest.approx(4000 / (13.56e6 * 4000), rel=1e-9)   # one period of DT_E steps
    assert np.all((e2[0] >= 0) & (e2[0] <= 0.025)) and len(e2[0]) > 0


@pytest.mark.skipif(not os.path.exists(EDUPIC), reason="eduPIC not built (make -C oracle ref)")
def test_stability_precheck_matches_edupics_report(cudapic, tmp_path):
    """The parameter-only lines of eduPIC's info.txt (max collision frequency
    x time step for electrons and ions, the CFL energy) equal the precheck
    to the printed digits."""
    exe = os.path.abspath(EDUPIC)
    for args in (["0"], ["1", "m"]):
        out = subprocess.run([exe] + args, cwd=tmp_path, capture_output=True, text=True, timeout=120)
        assert out.returncode == 0, out.stdout + out.stderr
    info = (tmp_path / "info.txt").read_text()

    def value(label):
        return float(re.search(re.escape(label) + r"\s*=\s*(\S+)", info).group(1))

    pc = cudapic.stability_precheck()
    assert round(pc["max_e_coll_dt_e"], 3) == value("Max. electron coll. frequency * DT_E")
    assert round(pc["max_i_coll_dt_i"], 3) == value("Max. ion coll. frequency * DT_I")
    assert round(pc["cfl_max_energy"], 3) == value("Max e- energy for CFL condition")
    assert pc["conditions_ok"] == 1


def test_stability_precheck_scales_with_density_and_step(cudapic):
    base = cudapic.stability_precheck()
    hi = cudapic.stability_precheck(pressure=50.0, n_t=1000)   # 5x the gas density, 4x the time step
    assert hi["max_e_coll_dt_e"] == pytest.approx(20 * base["max_e_coll_dt_e"], rel=1e-6)
    assert hi["max_i_coll_dt_i"] == pytest.approx(20 * base["max_i_coll_dt_i"], rel=1e-6)
    assert hi["cfl_max_energy"] == pytest.approx(base["cfl_max_energy"] / 16, rel=1e-12)
    assert hi["conditions_ok"] == 0
