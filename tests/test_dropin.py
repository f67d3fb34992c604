"""The C++ drop-in: the reference's own example programs, unmodified, built
against biofvm_b200's headers (biofvm_b200/shim) run on the GPU and write the
same MATLAB files as the same programs built against the reference."""
import glob
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
SHIM_INCLUDE = os.path.join(ROOT, "biofvm_b200", "shim", "include")
DROPIN = os.path.join(ROOT, "biofvm_b200", "shim", "_build", "dropin", "examples")
REFBIN = os.path.join(ROOT, "oracle", "_ref", "examples")
# the reference source tree (read only), named by BIOFVM_REFERENCE
REFERENCE_EXAMPLES = os.path.join(os.environ.get("BIOFVM_REFERENCE", "/root/reference"),
                                  "examples")

# example -> command-line arguments (dt, t_max, dx where the example takes them)
EXAMPLES = {
    "convergence_test1": ["0.01", "0.5", "20"],
    "convergence_test2": ["0.01", "1", "20"],
    "tutorial2_BioFVM": [],
    "tutorial3_BioFVM": [],
}


def read_mat4(path):
    """MATLAB Level-4 full real double matrix -> array [rows, cols]."""
    with open(path, "rb") as f:
        typ, rows, cols, imag, nlen = np.frombuffer(f.read(20), dtype="<i4")
        assert typ == 0 and imag == 0
        f.read(int(nlen))
        data = np.frombuffer(f.read(), dtype="<f8")
    return data.reshape(int(cols), int(rows)).T


@pytest.mark.skipif(not os.path.isdir(REFERENCE_EXAMPLES), reason="reference sources absent")
def test_every_reference_driver_compiles_against_the_dropin_headers(tmp_path):
    work = tmp_path / "examples"
    work.mkdir()
    os.symlink(os.path.join(SHIM_INCLUDE, "BioFVM.h"), tmp_path / "BioFVM.h")
    sources = sorted(glob.glob(os.path.join(REFERENCE_EXAMPLES, "*.cpp")))
    assert len(sources) >= 14
    for src in sources:
        with open(src, "rb") as f:
            r = subprocess.run(["/usr/bin/g++", "-std=c++14", "-fopenmp", "-fsyntax-only",
                                "-I", SHIM_INCLUDE, "-I", os.path.join(ROOT, "include"),
                                "-x", "c++", "-"], stdin=f, cwd=work, capture_output=True,
                               text=True)
        assert r.returncode == 0, (src, r.stderr[-2000:])


def test_dropin_library_exports_the_reference_api():
    lib = os.path.join(ROOT, "biofvm_b200", "libbiofvm_b200.so")
    out = subprocess.run(["nm", "-DC", "--defined-only", lib], capture_output=True, text=True,
                         check=True).stdout
    for sym in ["BioFVM::Microenvironment::simulate_diffusion_decay(double)",
                "BioFVM::Microenvironment::simulate_bulk_sources_and_sinks(double)",
                "BioFVM::Microenvironment::simulate_cell_sources_and_sinks(double)",
                "BioFVM::Microenvironment::apply_dirichlet_conditions()",
                "BioFVM::Microenvironment::resize_space_uniform(double, double, double, double, "
                "double, double, double)",
                "BioFVM::Basic_Agent::set_internal_uptake_constants(double)",
                "BioFVM::create_basic_agent()",
                "BioFVM::diffusion_decay_solver__constant_coefficients_LOD_3D("
                "BioFVM::Microenvironment&, double)"]:
        assert sym in out, sym


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(EXAMPLES))
def test_reference_example_runs_unchanged_on_the_gpu(name, tmp_path):
    dropin = os.path.join(DROPIN, name)
    ref = os.path.join(REFBIN, name)
    if not (os.path.exists(dropin) and os.path.exists(ref)):
        pytest.skip("example binaries not built (they need the reference sources)")
    outs = {}
    for tag, exe in (("ref", ref), ("gpu", dropin)):
        d = tmp_path / tag
        d.mkdir()
        r = subprocess.run([exe, *EXAMPLES[name]], cwd=d, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, (tag, r.stdout[-2000:], r.stderr[-2000:])
        outs[tag] = {os.path.basename(p): read_mat4(p) for p in glob.glob(str(d / "*.mat"))}
    assert outs["ref"] and set(outs["ref"]) == set(outs["gpu"])
    for fname, a in outs["ref"].items():
        b = outs["gpu"][fname]
        assert a.shape == b.shape, fname
        assert np.array_equal(a[:4], b[:4]), fname  # voxel centres and volumes
        den = np.maximum(np.abs(a[4:]).max(axis=1), 1e-300)
        err = np.abs(a[4:] - b[4:]).max(axis=1) / den
        assert np.all(err <= 1e-12), (fname, err)


def _parse_driver(text):
    """{tag: {key tuple: value}} from the driver's 'tag ints... value' lines."""
    out = {}
    for line in text.splitlines():
        f = line.split()
        if len(f) < 4 or f[0] not in ("G", "P", "L", "Q"):
            continue
        out.setdefault(f[0], {})[tuple(int(x) for x in f[1:-1])] = float(f[-1])
    return out


@pytest.mark.gpu
def test_api_driver_matches_the_reference_build():
    """tests/dropin/api_driver.cpp (agents sharing voxels, Dirichlet nodes,
    direct writes, gradients of every voxel and the lazy per-voxel path),
    built against the reference and against the drop-in headers.  Fields:
    relative max-norm per substrate <= 1e-12.  Gradients: within the error the
    field bound allows, |dg| <= 2e-12 * max|p_s| / dx."""
    gpu = os.path.join(ROOT, "biofvm_b200", "shim", "_build", "dropin", "drivers", "api_driver")
    ref = os.path.join(ROOT, "oracle", "_ref", "drivers", "api_driver")
    if not (os.path.exists(gpu) and os.path.exists(ref)):
        pytest.skip("driver binaries not built (they need the reference sources)")
    runs = {}
    for tag, exe in (("ref", ref), ("gpu", gpu)):
        r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, (tag, r.stdout[-2000:], r.stderr[-2000:])
        runs[tag] = _parse_driver(r.stdout)
    a, b = runs["ref"], runs["gpu"]
    assert set(a) == {"G", "P", "L", "Q"} and set(a) == set(b)
    dx = 10.0
    for field, grads in (("P", "G"), ("Q", "L")):
        assert a[field].keys() == b[field].keys() and a[grads].keys() == b[grads].keys()
        S = 1 + max(k[1] for k in a[field])
        pmax = [max(abs(v) for k, v in a[field].items() if k[1] == s) for s in range(S)]
        for s in range(S):
            err = max(abs(a[field][k] - b[field][k]) for k in a[field] if k[1] == s)
            assert err <= 1e-12 * pmax[s], (field, s, err)
            gerr = max(abs(a[grads][k] - b[grads][k]) for k in a[grads] if k[1] == s)
            assert gerr <= 2e-12 * pmax[s] / dx, (grads, s, gerr)


@pytest.mark.gpu
@pytest.mark.parametrize("data_matlab,mesh_matlab", [(1, 0), (0, 1), (0, 0)],
                         ids=["data-mat", "mesh-mat", "all-xml"])
def test_multicellds_files_match_the_reference_build(tmp_path, data_matlab, mesh_matlab):
    """tests/dropin/multicellds_driver.cpp saves a microenvironment twice (the
    second save updates the document of the first) and reads the first file
    back.  The XML files must be the same text as the reference build's, the
    MATLAB files the same numbers, and what is read back the same."""
    gpu = os.path.join(ROOT, "biofvm_b200", "shim", "_build", "dropin", "drivers",
                       "multicellds_driver")
    ref = os.path.join(ROOT, "oracle", "_ref", "drivers", "multicellds_driver")
    if not (os.path.exists(gpu) and os.path.exists(ref)):
        pytest.skip("driver binaries not built (they need the reference sources)")
    outs = {}
    for tag, exe in (("ref", ref), ("gpu", gpu)):
        d = tmp_path / tag
        d.mkdir()
        r = subprocess.run([exe, str(data_matlab), str(mesh_matlab)], cwd=d, capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0, (tag, r.stdout[-2000:], r.stderr[-2000:])
        files = {os.path.basename(p): p for p in glob.glob(str(d / "*"))}
        outs[tag] = (files, [l for l in r.stdout.splitlines() if l.startswith("R ")])
    (fa, la), (fb, lb) = outs["ref"], outs["gpu"]
    assert set(fa) == set(fb)
    for name, pa in fa.items():
        if name.endswith(".xml"):
            assert open(pa).read() == open(fb[name]).read(), name
        elif name.endswith(".mat"):
            assert np.array_equal(read_mat4(pa), read_mat4(fb[name])), name
    assert la == lb


def test_mesh_connectivity_and_vector_helpers_match_the_reference_build():
    """tests/dropin/mesh_vector_driver.cpp (host only): every voxel's list of
    face neighbours after Cartesian_Mesh::resize (the default one-voxel mesh,
    a 7 x 5 x 4 mesh, a mesh with a one-node axis) and the CSV helpers must
    print the same text in both builds.  The fused elementwise helpers, which
    the reference declares without defining, are checked against their
    stated formulas."""
    gpu = os.path.join(ROOT, "biofvm_b200", "shim", "_build", "dropin", "drivers",
                       "mesh_vector_driver")
    ref = os.path.join(ROOT, "oracle", "_ref", "drivers", "mesh_vector_driver")
    if not (os.path.exists(gpu) and os.path.exists(ref)):
        pytest.skip("driver binaries not built (they need the reference sources)")
    out = {}
    for tag, exe in (("ref", ref), ("gpu", gpu)):
        r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, (tag, r.stderr[-2000:])
        out[tag] = r.stdout.splitlines()
    keep = ("C0", "C1", "C2", "S1", "S2", "S3", "B ")
    a = [l for l in out["ref"] if l.startswith(keep)]
    b = [l for l in out["gpu"] if l.startswith(keep)]
    assert a and a == b
    assert "C1 size 140" in a
    v = {}
    for line in out["gpu"]:
        if line.startswith("V "):
            _, name, x = line.split()
            v.setdefault(name, []).append(float(x))
    y, a1, a2 = np.array([1.0, 2, 3]), np.array([0.5, -1, 2]), np.array([3.0, 0.25, -0.5])
    x1, x2, d = np.array([4.0, 5, -6]), np.array([-1.0, 2, 0.125]), np.array([2.0, 4, -8])
    assert v["axpy_div"] == list((y + a1 * x1) / d)
    assert v["double_axpy2"] == list(y + a1 * x1 + a2 * x2)
    assert v["double_axpy1"] == list(y + a1 * (x1 + x2))
    assert v["double_axpy_div1"] == list((y + a1 * (x1 + x2)) / d)
    assert v["double_axpy_div2"] == list((y + a1 * x1 + a2 * x2) / d)
