"""The bench's CPU arms (no GPU): the reference arm and the CPU baseline time
the NumPy oracle on the bench's own geometry, and load nothing of the
package or its library, so the reference arm's process holds none of this
repository's compiled code.  Also the oracle on the full plain 2D
configuration against the reference's golden run of it."""

import os
import subprocess
import sys

import numpy as np

from conftest import ROOT, load_golden

PROBE = r"""
import sys
sys.argv = ["bench.py"]
import bench
r = bench.cpu_sample((1, 1))
assert r["its"] == 1 and r["steps"] == 1
mods = sorted(m for m in sys.modules if m.split(".")[0] == "prtlb_gpu")
maps = open("/proc/self/maps").read()
print("MODS", len(mods), "LIB", "libprtlb" in maps)
"""


def test_cpu_arm_loads_no_repo_library():
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True,
                       env=env, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "MODS 0 LIB False" in r.stdout, r.stdout


def test_host_geometry_is_the_bench_pack():
    sys.path.insert(0, ROOT)
    import bench
    z = load_golden("cfg_plain3d64")
    assert np.array_equal(bench.host_geometry(), z["g"])


def test_oracle_on_the_plain2d_configuration():
    """The whole plain 2D configuration (128^2 disks, D2Q9 to tol 1e-7, 4000
    first-order steps) through the oracle, against the reference's run."""
    from oracle import prtlb_oracle as O
    z = load_golden("cfg_plain2d")
    info = {}
    v = O.stokes(z["g"], nit=int(z["nit"]), force=float(z["force"]), tau_lb=float(z["tau"]),
                 tol=float(z["tol"]), info=info)
    assert info["flow_iters"] == int(z["info_flow_iters"])
    assert np.abs(v - z["v"]).max() / np.abs(z["v"]).max() < 1e-6
    ainfo, prog = {}, []
    out, tn = O.solve_adr(z["g"], z["v"], pe=float(z["arg_pe"]), da=float(z["arg_da"]),
                          n_t=int(z["arg_n_t"]), n_species=int(z["arg_n_species"]),
                          steps=int(z["arg_steps"]), info=ainfo,
                          on_progress=lambda *a: prog.append(a))
    assert np.array_equal(tn, z["t_norm"])
    assert np.array_equal(out, z["out"])
    assert np.array_equal(np.asarray(prog, np.float64).reshape(-1, 4), z["progress"])
