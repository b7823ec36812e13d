"""YaHMC itself on the engine: the reference's unmodified sources built with the shim
(integration/yahmc_gpu_shim.cpp replaces dirac.cpp, linalg.cpp, cg.cpp, bicgstab.cpp,
minres.cpp, inverter.cpp, forces.cpp and clover.cpp), against the same sources built for
the CPU.

* The reference's own self-checks (checks/dirac.cpp:7-189, checks/inverters.cpp:7-191,
  checks/group.cpp) pass through the shim.
* One trajectory of the Nf = 2 HMC + Hasenbusch setup (gauge monomial on level 0 with one
  o2mn step, HMC and Hasenbusch monomials on level 1 with ten o2mn steps; hmc.cpp:68-94,
  hasenbusch.cpp:67-96, integrator.cpp:42-64, update.cpp:281-339) run by the reference's
  monomials and integrator over the engine reproduces the CPU build's Hamiltonians and final
  links: both builds start from the same links and draw the same momenta and pseudo-fermions
  (the same generator and seed; spinor_random draws on the host in the reference's order).
* Integrating back with the momenta negated returns to the start: |delta H| <= 1e-8.
* YaHMC's `hmc` program (programs/hmc.cpp, unchanged) built on the shim prints the same
  trajectories (dH, acceptance, plaquette) as the CPU program from the same cfg and seed.
"""
import os
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import ref as oref
from yahmc_b200 import fields, heatbath

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
DIMS = (8, 8, 8, 8)

# configuration 2's monomials and integrator (16^3x32 there; 8^4 here so that the CPU build
# finishes in seconds); prec 1e-28 (squared) so that solver round-off stays below the
# tolerances checked
CFG = """
[integrator]
level = 0
type = o2mn
steps = 1
[integrator]
level = 1
type = o2mn
steps = 10
[monomial]
level = 0
type = gauge
beta = 5.6
c0 = 1.0
[monomial]
level = 1
type = hmc
mass = -0.75
dm = 0.2
prec = 1e-28
mre_past = 0
[monomial]
level = 1
type = hasenbusch
mass = -0.75
dm = 0.2
prec = 1e-28
"""
LEVELS = [("o2mn", 10), ("o2mn", 1)]


def need_shim(name="su3_fund_ap"):
    if not oref.shim_available(name):
        pytest.skip("oracle/_ref/libyahmc_shim_* not built (python oracle/build_ref.py --shim)")


_field = {}


def start_links():
    """A beta = 5.6 heatbath field (20 sweeps on 8^4): smooth enough for unit-length
    trajectories, the same in both builds."""
    if "U" not in _field:
        U, _ = heatbath.thermalised_field(DIMS, 5.6, 20, 7)
        _field["U"] = fields.complex_to_raw(U)
    return _field["U"]


def test_reference_checks_pass_through_the_shim():
    """run_checks (checks/check.cpp:4-26) on the reference's random start, as
    `hmc --run-checks` does; the covariance check reads and writes spinors on the host
    between operations, so the shim keeps host arrays in step (YAHMC_GPU_HOST_MIRROR=1)."""
    need_shim()
    os.environ["YAHMC_GPU_HOST_MIRROR"] = "1"
    try:
        G = oref.RefLattice("su3_fund_ap", DIMS, seed=4711, kind="shim")
    finally:
        del os.environ["YAHMC_GPU_HOST_MIRROR"]
    G.set_random_links()
    assert G.lib.yref_check_group() == 0
    assert G.lib.yref_check_dirac() == 0
    assert G.lib.yref_check_inverters() == 0


def _trajectory(R):
    R.set_links(start_links())
    R.hmc_init(CFG)
    R.call("hmc_reset")
    h0 = R.lib.yref_hmc_hamiltonian()
    R.call("mvm_reset")
    R.hmc_integrate(1.0, LEVELS)
    h1 = R.lib.yref_hmc_hamiltonian()
    return h0, h1, R.lib.yref_mvm_get(), R.get_links()


def test_trajectory_matches_cpu_build_and_reverses():
    need_shim()
    cpu = oref.RefLattice("su3_fund_ap", DIMS, seed=2024, kind="ref")
    gpu = oref.RefLattice("su3_fund_ap", DIMS, seed=2024, kind="shim")
    h0c, h1c, mvm_c, uc = _trajectory(cpu)
    h0g, h1g, mvm_g, ug = _trajectory(gpu)
    dhc, dhg = h1c - h0c, h1g - h0g
    # the same start: momenta, pseudo-fermions, actions and logdet agree to rounding
    assert abs(h0g - h0c) <= 1e-12 * abs(h0c), (h0g, h0c)
    # the same trajectory: solves to prec 1e-28 leave differences far below these bounds
    assert abs(dhg - dhc) <= 1e-9 * abs(h0c), (dhg, dhc)
    assert np.abs(ug - uc).max() <= 1e-10
    # the same solver iterations up to rounding (the engine counts MVMs like dirac.cpp:11-18)
    assert abs(mvm_g - mvm_c) <= 0.02 * mvm_c, (mvm_g, mvm_c)
    # reversibility on the GPU build: negate the momenta, integrate again
    u0 = start_links()
    gpu.set_momenta(-gpu.momenta())
    gpu.hmc_integrate(1.0, LEVELS)
    h2g = gpu.lib.yref_hmc_hamiltonian()
    assert abs(h2g - h0g) <= 1e-8, h2g - h0g
    assert np.abs(gpu.get_links() - u0).max() <= 1e-10


HMC_CFG = """[lattice]
dim_t = 8
dim_x = 8
dim_y = 8
dim_z = 8
[parallel]
threads = 0
np_t = 1
np_x = 1
np_y = 1
np_z = 1
[log]
level = 30
[rand]
seed = 4711
[cnfg]
dir = .
prefix = probe
start = random
last = 2
freq = 0
[clover]
csw = 1.0
cf = 1.0
[traj]
length = 1.0
[observables]
plaq_freq = 1
poly_freq = 0
mes_freq = 0
[integrator]
level = 0
type = o2mn
steps = 1
[integrator]
level = 1
type = o2mn
steps = 10
[monomial]
level = 0
type = gauge
beta = 5.6
c0 = 1.0
[monomial]
level = 1
type = hmc
mass = -0.75
dm = 0.2
prec = 1e-24
mre_past = 5
[monomial]
level = 1
type = hasenbusch
mass = -0.75
dm = 0.2
prec = 1e-24
"""


def _run_program(exe, tmp, name, env=None):
    cfg = tmp / "hmc.cfg"
    cfg.write_text(HMC_CFG)
    log = tmp / f"{name}.log"
    r = subprocess.run([str(exe), "-i", str(cfg), "-o", str(log)], cwd=tmp, capture_output=True, text=True,
                       timeout=600, env={**os.environ, **(env or {})})
    assert r.returncode == 0, r.stderr[-2000:]
    text = log.read_text()
    dh = [float(x) for x in re.findall(r"dH = ([-+0-9.e]+)", text)]
    plaq = [float(x) for x in re.findall(r"Plaquette: ([-+0-9.e]+)", text)]
    acc = re.findall(r"Configuration (accepted|rejected)", text)
    return dh, plaq, acc, text


def test_hmc_program_on_the_engine_prints_the_cpu_trajectories(tmp_path):
    exe_gpu = ROOT / "integration" / "_build" / "hmc_su3_fund_ap"
    exe_cpu = ROOT / "oracle" / "_ref" / "hmc_su3_fund_ap"
    if not (exe_gpu.exists() and exe_cpu.exists()):
        pytest.skip("integration/_build/hmc_su3_fund_ap or oracle/_ref/hmc_su3_fund_ap not built")
    dh_c, pl_c, acc_c, _ = _run_program(exe_cpu, tmp_path, "cpu")
    dh_g, pl_g, acc_g, text = _run_program(exe_gpu, tmp_path, "gpu")
    assert "B200 engine" in text
    assert len(dh_g) == len(dh_c) == 2 and acc_g == acc_c
    # printed with 7 significant digits (update.cpp:314, hmc.cpp:152-158)
    assert np.allclose(dh_g, dh_c, rtol=2e-6, atol=1e-9), (dh_g, dh_c)
    assert np.allclose(pl_g, pl_c, rtol=2e-6), (pl_g, pl_c)


def test_hmc_program_with_the_mixed_precision_solver(tmp_path):
    """YAHMC_GPU_SOLVER=mixed: the Hasenbusch force's Hphi_sq solves run the mixed CG, which
    stops on the true residual; the trajectory is the same to the solver tolerance."""
    exe_gpu = ROOT / "integration" / "_build" / "hmc_su3_fund_ap"
    if not exe_gpu.exists():
        pytest.skip("integration/_build/hmc_su3_fund_ap not built")
    dh_f, pl_f, acc_f, _ = _run_program(exe_gpu, tmp_path, "fp64")
    dh_m, pl_m, acc_m, text = _run_program(exe_gpu, tmp_path, "mixed", env={"YAHMC_GPU_SOLVER": "mixed"})
    assert "mixed CG" in text
    assert acc_m == acc_f
    assert np.allclose(dh_m, dh_f, rtol=1e-4, atol=1e-6), (dh_m, dh_f)
    assert np.allclose(pl_m, pl_f, rtol=1e-5), (pl_m, pl_f)
