"""The drop-in C++ headers include/nukexc/*.hpp: the example programs
tests/cpp/shim_h1s.cpp (dense path) and tests/cpp/shim_sparse.cpp (bounding
boxes, neighbour lists, sparse / tiled functions) call the reference's
function names the way the reference's tests do.  CPU: they compile and link
against libnkx.so.  GPU: they reproduce the reference's known answers
(tests/golden/reference_kats.json) and its sparse-vs-tiled and
sparse-vs-dense agreement."""
import json
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "nukexc_b200", "libnkx.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
KAT = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_kats.json")))


def build_example(outdir, name="shim_h1s"):
    if not os.path.exists(LIB):
        from nukexc_b200 import build as B
        B.build()
    exe = os.path.join(str(outdir), name)
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
           "-L" + os.path.dirname(LIB), "-lnkx", "-L" + os.path.join(CUDA, "lib64"), "-lcudart",
           "-Wl,-rpath," + os.path.dirname(LIB), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_shim_headers_compile_and_link(tmp_path):
    assert os.path.exists(build_example(tmp_path))
    assert os.path.exists(build_example(tmp_path, "shim_sparse"))


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


@pytest.mark.gpu
def test_sparse_shims_match_reference_and_dense(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA GPU")
    exe = build_example(tmp_path, "shim_sparse")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    # H 1s self-repulsion 5/8 through the sparse and tiled J (test_hydrogen.cxx:633-686, :914-952)
    assert out["J_sparse_h1s"] == pytest.approx(KAT["h1s_coulomb"]["J00"], rel=1e-10)
    assert out["J_tiled_h1s"] == pytest.approx(KAT["h1s_coulomb"]["J00"], rel=1e-10)
    # boxes, in-place Morton permutation and neighbour lists (octree.hpp:70-144, :317-390)
    assert out["boxes_ok"] == 1 and out["weights_permuted"] == 1 and out["neighbor_list_ok"] == 1
    assert out["nnz"] > 0
    # tiled vs sparse element-wise at 1e-9 (test_hydrogen.cxx:994-1073)
    assert out["metric_tiled_vs_sparse"] <= 1e-9
    assert out["J_tiled_vs_sparse"] <= 1e-9
    # sparse vs dense on the same grid: equal up to what the 1e-10 cutoff drops
    assert out["J_sparse_vs_dense"] <= 1e-9 * max(1.0, out["J_scale"])
    assert out["rho_sparse_vs_dense"] <= 1e-9
    assert out["grad_sparse_vs_dense"] <= 1e-9
    assert out["sigma_sparse_vs_dense"] <= 1e-9 * max(1.0, out["sigma_scale"])
    assert out["rho_accumulated"] <= 1e-9
    assert out["xc_dE"] <= 1e-9
    assert out["xc_dV"] <= 1e-9
    assert out["E_lda_x"] < 0 and out["E_pbe_x"] < out["E_lda_x"] and out["E_pbe_c"] < 0
    assert out["family_checked"] == 1
    # RI-K self-exchange 5/8, dense / sparse / tiled (test_hydrogen.cxx:688-758, :760-822, :954-992)
    for key in ("K_dense_h1s", "K_sparse_h1s", "K_tiled_h1s"):
        assert out[key] == pytest.approx(KAT["h1s_exchange"]["K00"], rel=KAT["h1s_exchange"]["rel"])
    assert out["K_tiled_vs_sparse"] <= 1e-9
    assert out["K_sparse_vs_dense"] <= 1e-12 * max(1.0, out["K_scale"])
    # core Hamiltonian of H 1s (S = 1, T = 1/2, V = -1 analytically), and the
    # screened variants equal to it (test_integration.cxx:83-311 asks 1e-6)
    assert out["S00"] == pytest.approx(1.0, abs=1e-8)
    assert out["T00"] == pytest.approx(0.5, abs=1e-6)
    assert out["V00"] == pytest.approx(-1.0, abs=1e-6)
    assert out["H00"] == pytest.approx(out["T00"] + out["V00"], abs=1e-14)
    assert out["coreH_screened_diff"] <= 1e-6
    # set_precision(NKX_PREC_MIXED) moves the sparse XC and J onto the
    # tensor-core build: within the mixed scheme's gate of the FP64 results
    assert out["mixed_dE"] <= 1e-6 and out["mixed_dV"] <= 1e-7
    assert out["J_mixed_vs_fp64"] <= 1e-7 * max(1.0, out["J_scale"])
