"""The drop-in C++ headers include/nukexc/*.hpp: the example program
tests/cpp/shim_h1s.cpp calls the reference's function names the way the
reference's tests do.  CPU: it compiles and links against libnkx.so.  GPU:
it reproduces the reference's known answers (tests/golden/reference_kats.json)."""
import json
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "nukexc_b200", "libnkx.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
KAT = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_kats.json")))


def build_example(outdir):
    if not os.path.exists(LIB):
        from nukexc_b200 import build as B
        B.build()
    exe = os.path.join(str(outdir), "shim_h1s")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "shim_h1s.cpp"),
           "-L" + os.path.dirname(LIB), "-lnkx", "-L" + os.path.join(CUDA, "lib64"), "-lcudart",
           "-Wl,-rpath," + os.path.dirname(LIB), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_shim_headers_compile_and_link(tmp_path):
    assert os.path.exists(build_example(tmp_path))


@pytest.mark.gpu
def test_shim_headers_reproduce_reference_known_answers(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA GPU")
    exe = build_example(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["int_rho"] == pytest.approx(KAT["h1s_density"]["int_rho"], rel=KAT["h1s_density"]["rel"])
    assert out["E_lda_x"] == pytest.approx(KAT["h1s_lda_x"]["E"], rel=1e-10)
    assert out["E_pbe_x"] == pytest.approx(KAT["h1s_pbe_x"]["E"], rel=1e-10)
    assert out["V00_pbe_x"] == pytest.approx(KAT["h1s_pbe_x"]["V00"], rel=1e-10)
    # open shell with all density in alpha: exchange spin scaling gives
    # E_x[rho, 0] = E_x[2 rho] / 2 -- not the closed-shell value
    assert out["E_pbe_x_pol"] < out["E_pbe_x"]
    assert out["int_sigma"] == pytest.approx(KAT["h1s_density_sigma"]["int_sigma"], rel=1e-10)
    assert out["J00"] == pytest.approx(KAT["h1s_coulomb"]["J00"], rel=1e-10)
    assert out["K"] >= 1
    assert out["becke_single_atom"] == pytest.approx(1.0, abs=1e-15)
