"""A compiled C++ consumer of the boundary: tests/cxx holds the reference's element /
force-contribution interface restated with its names and signatures (aperi_mirror.h),
the element shim a maintainer adds to aperi-mech (b200_element.h, the class INTEGRATION.md
shows) and a host program that drives one part through them and the C ABI without
Python (consumer.cpp). The header must compile as C and as C++; the program must build;
on a GPU its force and trajectory must match the oracle."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
CXX = ROOT / "tests" / "cxx"


def _cuda_home() -> Path:
    nvcc = shutil.which("nvcc")
    return Path(nvcc).resolve().parent.parent if nvcc else Path("/usr/local/cuda")


def build_consumer(out_dir: Path) -> Path:
    from aperi_mech_b200 import build

    lib = build.build()
    cuda = _cuda_home()
    exe = out_dir / "consumer"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}", f"-I{CXX}",
           f"-I{cuda / 'include'}", str(CXX / "consumer.cpp"), "-o", str(exe), f"-L{lib.parent}", "-laperi_b200",
           f"-L{cuda / 'lib64'}", "-lcudart", f"-Wl,-rpath,{lib.parent}", f"-Wl,-rpath,{cuda / 'lib64'}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    return exe


def test_header_compiles_as_c_and_cxx(tmp_path):
    src = tmp_path / "inc.c"
    src.write_text('#include "aperi_b200.h"\nint main(void) { return AM_OK; }\n')
    for tool, std in (("gcc", "-std=c99"), ("g++", "-std=c++11")):
        res = subprocess.run([tool, std, "-Wall", "-Werror", "-pedantic", f"-I{ROOT / 'include'}", "-x",
                              "c" if tool == "gcc" else "c++", str(src), "-c", "-o", str(tmp_path / f"inc_{tool}.o")],
                             capture_output=True, text=True)
        assert res.returncode == 0, res.stderr


def test_consumer_builds(capi_lib, tmp_path):
    assert build_consumer(tmp_path).exists()


def _write_input(path: Path, p, u, cells: bool):
    part = p.parts[0]
    mat = {"linear_elastic": 0, "neo_hookean": 1, "elastic": 2}[part.material.kind]
    fixed = np.concatenate([b.nodes for b in p.bcs]).astype(np.int32) if p.bcs else np.zeros(0, np.int32)
    with open(path, "wb") as f:
        np.array([p.num_nodes, part.num_elems, p.nsteps, int(cells), mat, fixed.size], dtype="<i8").tofile(f)
        np.array([part.material.lam, part.material.mu, part.material.density, p.dt], dtype="<f8").tofile(f)
        np.ascontiguousarray(p.coords, dtype="<f8").tofile(f)
        np.ascontiguousarray(part.conn, dtype="<i4").tofile(f)
        np.ascontiguousarray(u, dtype="<f8").tofile(f)
        np.ascontiguousarray(p.v0, dtype="<f8").tofile(f)
        fixed.astype("<i4").tofile(f)


@pytest.mark.gpu
@pytest.mark.parametrize("cells", [False, True], ids=["gauss", "smoothed_cells"])
def test_consumer_matches_oracle(gpu, oracle_lib, tmp_path, cells):
    from aperi_mech_b200 import problems, smoothing
    from helpers import l2_rel, rel_err

    p = problems.tet4_nh_shear(n=6, seed=4, nsteps=25)
    rng = np.random.default_rng(9)
    u = 1e-4 * rng.standard_normal(p.coords.shape)
    exe = build_consumer(tmp_path)
    _write_input(tmp_path / "in.bin", p, u, cells)
    res = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True,
                         text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    out = np.fromfile(tmp_path / "out.bin", dtype="<f8").reshape(4, p.num_nodes, 3)
    parts, mass = p.parts, None
    if cells:
        part, mass = smoothing.element_smoothing_part(p.coords, p.parts[0].conn, p.parts[0].material)
        parts = [part]
    op = oracle_lib.OracleProblem(p.coords, parts, p.bcs, mass=mass)
    assert rel_err(out[0], op.internal_force(u)) < 1e-12
    z = np.zeros_like(p.coords)
    want = op.steps(z, p.v0, op.init_acceleration(z), np.full(p.nsteps, p.dt))
    for g, w in zip(out[1:], want):
        assert l2_rel(g, w) < 1e-12


def test_integration_snippet_is_the_compiled_shim():
    """INTEGRATION.md shows the shim class exactly as tests/cxx/b200_element.h holds it."""
    doc = (ROOT / "INTEGRATION.md").read_text()
    shim = (CXX / "b200_element.h").read_text()
    cls = shim[shim.index("class B200Element"):].strip()
    assert cls in doc
