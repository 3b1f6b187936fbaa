"""The C++ class shim (ICARAT's LinearAnalysis / Filter / FilterHelmholtz / OC /
MMASolver over the C ABI) and its TOML-subset reader.

CPU: the reader against Python's tomllib on the same files, and its errors.
GPU: the two app drivers built on the shim against the oracle's app loops.
"""
import json
import os
import subprocess
import sys
import tomllib

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SHIM = os.path.join(REPO, "icarat-contact_b200", "shim")
LIB = os.path.join(REPO, "icarat-contact_b200", "lib")
TOMLS = os.path.join(REPO, "tests", "golden", "toml")


@pytest.fixture(scope="module")
def toml_dump(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("shim") / "toml_dump")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I" + SHIM,
                    os.path.join(REPO, "tests", "toml_dump.cpp"), "-o", exe], check=True)
    return exe


def _same(a, b):
    if isinstance(a, dict):
        return isinstance(b, dict) and a.keys() == b.keys() and all(_same(a[k], b[k]) for k in a)
    if isinstance(a, list):
        return isinstance(b, list) and len(a) == len(b) and all(_same(x, y) for x, y in zip(a, b))
    if isinstance(a, bool) or isinstance(b, bool):
        return a is b
    if isinstance(a, (int, float)):
        return type(a) is type(b) and a == b
    return a == b


def test_reader_matches_tomllib_on_fixtures(toml_dump):
    files = sorted(os.path.join(TOMLS, f) for f in os.listdir(TOMLS) if f.endswith(".toml"))
    assert len(files) >= 3
    out = subprocess.run([toml_dump] + files, capture_output=True, text=True, check=True).stdout
    for f, line in zip(files, out.splitlines()):
        with open(f, "rb") as fh:
            assert _same(tomllib.load(fh), json.loads(line)), f


def test_reader_subset_details(toml_dump, tmp_path):
    text = """# comment line
[mesh]
dimension = 3   # trailing comment
division = [
  8,      # x
  4,
  1_000,  # underscores
]
length = [1.5e1, -2.0, +3.25]
type = "hexa8"
flag = true
off = false
esc = "a\\"b\\\\c"

[boundary_condition]
dirichlet = [[[1,0,0,0,0,0],[0.0,0.0,0.0,0.0,0.0,0.0],[[0.0,0.0],[0.0,4.0],[0.0,1.0]]],]
neumann = []
"""
    p = tmp_path / "t.toml"
    p.write_text(text)
    got = json.loads(subprocess.run([toml_dump, str(p)], capture_output=True, text=True,
                                    check=True).stdout)
    assert _same(tomllib.loads(text), got)


@pytest.mark.parametrize("body,what", [
    ("[a]\nx = {y = 1}\n", "inline tables"),
    ("[a]\nx.y = 1\n", "dotted keys"),
    ("[a]\nx = 1\nx = 2\n", "defined twice"),
    ("[a]\n[a]\n", "defined twice"),
    ("[[a]]\n", "arrays of tables"),
    ("[a]\nx = [1, 2\n", "expected"),
    ("[a]\nx = 1 2\n", "unexpected text"),
])
def test_reader_rejects_outside_subset(toml_dump, tmp_path, body, what):
    p = tmp_path / "bad.toml"
    p.write_text(body)
    r = subprocess.run([toml_dump, str(p)], capture_output=True, text=True)
    assert r.returncode == 2 and what in r.stdout, r.stdout
    assert "bad.toml:" in r.stdout  # names file and line


def test_drivers_are_built():
    for name in ("opt_macro_oc_gpu", "opt_mma_helmholtz_gpu", "opt_heat_gpu"):
        assert os.access(os.path.join(LIB, name), os.X_OK), name


# ---------------------------------------------------------------- GPU --
def _oracle_from_toml(cfg):
    """The oracle problem for a TOML config, read with tomllib (independent
    of the shim's reader)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle as po
    m, mat, bc = cfg["mesh"], cfg["material"], cfg["boundary_condition"]
    dim = m["dimension"]
    nx, ny, nz = m["division"]
    lx, ly, lz = m["length"]
    state = 2 if dim == 3 else {"plane_stress": 0, "plane_strain": 1}[mat["state"]]
    p = po.Problem(dim, nx, ny, nz if dim == 3 else 1, lx, ly, lz if dim == 3 else 1.0,
                   state=state, young=tuple(mat["young"]), nu=mat["poisson"], penal=mat["penalty"])
    for flag, val, rng in bc["dirichlet"]:
        p.dirichlet_box(flag, val, np.asarray(rng, float).reshape(6))
    for val, rng in bc.get("neumann", []):
        p.traction_box(val[:3], np.asarray(rng, float).reshape(6))
    hx, hy = lx / nx, ly / ny
    hz = lz / nz if dim == 3 else 1.0
    for f, x in bc.get("point", []):
        i, j = int(round(x[0] / hx)), int(round(x[1] / hy))
        k = int(round(x[2] / hz)) if dim == 3 else 0
        n = i + (nx + 1) * (j + (ny + 1) * k)
        p.fext_full[n * dim:(n + 1) * dim] += np.asarray(f[:dim])
    return p, mat["designs_0"]


def _run(exe, toml):
    r = subprocess.run([os.path.join(LIB, exe), os.path.join(TOMLS, toml)], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return np.array([[float(v) for v in ln.split(",")] for ln in r.stdout.split()])


@pytest.mark.gpu
@pytest.mark.parametrize("toml", ["c1_cantilever.toml", "traction2d.toml"])
def test_oc_app_on_shim_matches_oracle(toml):
    with open(os.path.join(TOMLS, toml), "rb") as fh:
        cfg = tomllib.load(fh)
    tp = cfg["this_problem"]
    out = _run("opt_macro_oc_gpu", toml)
    assert out.shape == (tp["steps"], 3)
    p, rho0 = _oracle_from_toml(cfg)
    hist, _, _ = p.oc_loop(np.full(p.nel, rho0), tp["steps"], tp["filter_radius"],
                           tp["move_limit"], use_beta=True, tol=1e-10)
    rel = np.abs(out[:, 1] - hist) / np.abs(hist)
    assert rel.max() <= 1e-4, rel


@pytest.mark.gpu
def test_mma_app_on_shim_matches_oracle():
    toml = "traction3d.toml"
    with open(os.path.join(TOMLS, toml), "rb") as fh:
        cfg = tomllib.load(fh)
    steps = cfg["this_problem"]["steps"]
    out = _run("opt_mma_helmholtz_gpu", toml)
    assert out.shape == (steps, 3)
    p, rho0 = _oracle_from_toml(cfg)
    h = cfg["mesh"]["length"][0] / cfg["mesh"]["division"][0]
    hist, _ = p.mma_loop(np.full(p.nel, rho0), steps, 2.0 * h, 0.0, tol=1e-10)
    rel = np.abs(out[:, 1] - hist) / np.abs(hist)
    assert rel.max() <= 1e-4, rel
    assert out[0, 2] == 0.0  # step-1 constraint: V0 is the step-1 volume


@pytest.mark.gpu
def test_heat_app_on_shim_matches_oracle(tmp_path):
    """opt_heat_gpu (the opt-heat app on the library) against the oracle's
    heat loop, and the app's outputs: function.csv and res<step>.vtk with the
    temperature, threshold_s and design_s arrays."""
    toml = os.path.join(TOMLS, "heat2d.toml")
    with open(toml, "rb") as fh:
        cfg = tomllib.load(fh)
    m, mat, bc, tp = cfg["mesh"], cfg["material"], cfg["boundary_condition"], cfg["this_problem"]
    r = subprocess.run([os.path.join(LIB, "opt_heat_gpu"), toml], capture_output=True, text=True,
                       timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    out = np.array([[float(v) for v in ln.split(",")] for ln in r.stdout.split()])
    steps = tp["steps"]
    assert out.shape == (steps, 2)
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle as po
    nx, ny, _ = m["division"]
    lx, ly, _ = m["length"]
    o = po.Problem(2, nx, ny, 1, lx, ly, 1.0, state=3)
    for flag, val, rng in bc["dirichlet"]:
        o.dirichlet_box([flag[0], 0, 0, 0, 0, 0], [val[0], 0, 0, 0, 0, 0],
                        np.asarray(rng, float).reshape(6))
    for val, rng in bc["neumann"]:
        o.traction_box([val[0], 0, 0], np.asarray(rng, float).reshape(6))
    c1, c2 = mat["conductivity"]
    ho, _ = o.heat_loop(c1, c2, np.full(nx * ny, mat["designs_0"]), steps, tp["filterR"],
                        tol=1e-12)
    assert np.abs(out[:, 1] - ho).max() / np.abs(ho).max() <= 1e-4
    fn = np.loadtxt(tmp_path / "function.csv")
    assert fn.shape == (steps, 2) and np.allclose(fn[:, 1], out[:, 1], rtol=1e-5)
    vtk = (tmp_path / "res1.vtk").read_text()
    for key in ("POINT_DATA", "SCALARS temperature", "SCALARS threshold_s", "CELL_DATA",
                "SCALARS design_s", f"CELLS {nx * ny}"):
        assert key in vtk, key
    assert os.path.exists(tmp_path / f"res{steps}.vtk")
