"""Drop-in check: the C++ driver gpu_ppm_b200/_build/ppm_run reads the
reference's own input files (tables/lensing/std text tables, the 5-column NSX
file, tables/ism_inst/std) from a scratch directory laid out like the
reference's, runs the reference's scenarios through the C ABI and writes the
reference's output files; those files are compared with the golden vectors
produced by the reference's own CPU programs on the same inputs."""
import os
import subprocess

import numpy as np
import pytest

from gpu_ppm_b200 import build as build_mod
from gpu_ppm_b200 import synth
from tests import golden_cases as gc
from tests.errors import max_rel

pytestmark = pytest.mark.gpu


def write_scenarios(path, lines):
    with open(path, "w") as f:
        for ln in lines:
            f.write(" ".join(repr(x) if isinstance(x, float) else str(x) for x in ln) + "\n")


def test_reference_layout_round_trip(golden, tmp_path):
    meta, z = golden
    d = str(tmp_path)
    synth.lensing("std").write_dir(os.path.join(d, "tables", "lensing", "std"))
    synth.nsx("v200804", seed=0).write_file(os.path.join(d, "ext", "model_data", "nsx_H_v200804.out"))
    E, rsp = gc.ism_inst(meta)
    synth.write_ism_inst(os.path.join(d, "tables", "ism_inst", "std"), E, rsp)
    os.makedirs(os.path.join(d, "output"))
    run = build_mod.RUN
    write_scenarios(os.path.join(d, "dev.txt"), meta["devarshi"])
    os1 = [(n, float(nu), th * np.pi / 180, ot * np.pi / 180, float(ar), b) for n, nu, th, ot, ar, b in meta["os1"]]
    write_scenarios(os.path.join(d, "os1.txt"), os1)
    write_scenarios(os.path.join(d, "ti.txt"), meta["tinterp"][:2])
    for mode, f in (("devarshi", "dev.txt"), ("os1", "os1.txt"), ("tinterp", "ti.txt")):
        r = subprocess.run([run, mode, f], cwd=d, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
    for s in meta["devarshi"]:
        counts = np.loadtxt(os.path.join(d, "output", f"{s[0]}_{s[4]}_counts_gpu.txt"))
        assert max_rel(counts, z["devarshi/" + s[0]]) < 1e-4, s[0]
    for s in meta["os1"]:
        row = np.loadtxt(os.path.join(d, "output", f"{s[0]}_gpu.txt"))
        assert max_rel(row, z["os1/" + s[0]]) < 1e-6, s[0]
    r0, r1, rs = meta["tinterp_rows"]
    c0, c1, cs = meta["tinterp_cols"]
    for s in meta["tinterp"][:2]:
        flux = np.loadtxt(os.path.join(d, "output", f"{s[0]}_flux_gpu.txt"))
        assert max_rel(flux[r0:r1:rs, c0:c1:cs], z["tinterp/" + s[0]]) < 1e-4, s[0]


def test_loader_errors_are_status_codes(tmp_path):
    """A missing table directory is a PPM_E_IO status, not a process exit
    (gpu/read_file.cuh:11-15 exits)."""
    from gpu_ppm_b200 import _abi
    from gpu_ppm_b200.engine import Engine

    e = Engine()
    with pytest.raises(_abi.PpmError) as ei:
        e.load_lensing_dir(tmp_path / "nope")
    assert ei.value.code == _abi.PPM_E_IO
    e.close()
