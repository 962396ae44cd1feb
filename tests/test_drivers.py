"""The headless drivers (lbm-arrayfire_b200/drivers): the reference's cavity examples written against
the C ABI, built with g++ and linked to liblbm_b200.so like any C++ caller would."""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "lbm-arrayfire_b200"
BIN = PKG / "drivers" / "bin"
sys.path.insert(0, str(Path(__file__).resolve().parent))


def build():
    out = subprocess.run(["make", "-s", "-C", str(PKG), "drivers"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]


def test_drivers_build_and_link():
    build()
    for name in ("d2q9_bgk_lid", "d3q27_mrt_lid"):
        assert (BIN / name).exists()


@pytest.mark.gpu
def test_d2q9_driver_matches_oracle(tmp_path):
    """128^2 lid cavity, Re 200, lid 0.05 (the reference driver's parameters, C++ viscosity rule),
    500 iterations through the driver: DENSITY/UX/UY equal the FP64 oracle within the FP32 tolerance,
    and the CSV has the reference's header."""
    from helpers import O, cavity2d, oracle_problem, rel_l2

    build()
    dump, csv = tmp_path / "fields.bin", tmp_path / "mlups.csv"
    out = subprocess.run([str(BIN / "d2q9_bgk_lid"), "128", "128", "500", "--dump", str(dump), "--csv", str(csv)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "Iterations: 500" in out.stdout and "MLUPS:" in out.stdout
    lines = csv.read_text().splitlines()
    assert lines[0] == "Iterations,MLUPS" and len(lines) == 6 and lines[-1].startswith("500,")
    f = np.fromfile(dump, dtype=np.float64)
    n = 128 * 128
    rho, u = f[:n], f[n:]
    d, m, F0 = cavity2d(n=128, u_lid=0.05, re=200.0)
    _, rho_o, u_o = O.run(oracle_problem(d, m), F0, 500, dtype=np.float64)
    fluid = m == 0
    assert rel_l2(rho[fluid], rho_o[fluid]) < 1e-5
    uf = np.tile(fluid, 2)
    assert rel_l2(u[uf], u_o[uf]) < 1e-5


@pytest.mark.gpu
def test_d3q27_mrt_driver_runs_and_reports(tmp_path):
    build()
    dump = tmp_path / "fields.bin"
    out = subprocess.run([str(BIN / "d3q27_mrt_lid"), "32", "200", "--dump", str(dump)], capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "Iterations: 200" in out.stdout
    f = np.fromfile(dump, dtype=np.float64)
    assert f.size == 4 * 32 ** 3 and np.isfinite(f).all()
    ux = f[32 ** 3:2 * 32 ** 3].reshape(32, 32, 32, order="F")
    assert ux[16, 16, 30] > 0.0  # the lid on the z top drags the fluid below it along +x
