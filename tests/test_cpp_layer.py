"""The C++ layer <mtlgpu/mtl.hpp>: reference-style programs on device types.

tests/cpp/itl_gpu_test.cpp (standalone mode) follows the reference's own test
programs case by case; tests/cpp/mtl4_dropin.cpp (MTL4 mode, built only where
the MTL4 tree is present) runs the same code on the reference's CPU types and
on device types side by side.  The CPU tests here only build the programs; the
GPU tests run them and check what they print against the golden fixtures and
against the reference run inside the same program."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")
BUILD = os.path.join(CPP, "_build")
# the MTL4 tree, where the environment names it (REFERENCE_ROOT)
REF_ROOT = os.environ.get("REFERENCE_ROOT", "")
REF_HEADERS = os.path.join(REF_ROOT, "boost", "numeric", "mtl", "mtl.hpp") if REF_ROOT else ""


def _make():
    subprocess.run(["make", "-C", CPP], check=True, capture_output=True)


def _run(prog, case):
    exe = os.path.join(BUILD, prog)
    p = subprocess.run([exe, case], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, (case, p.returncode, p.stderr[-2000:])
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    return json.loads(lines[-1])


def test_builds_standalone():
    _make()
    assert os.path.exists(os.path.join(BUILD, "itl_gpu_test"))


@pytest.mark.skipif(not REF_HEADERS or not os.path.exists(REF_HEADERS),
                    reason="REFERENCE_ROOT does not name the MTL4 tree here")
def test_builds_with_mtl4_headers():
    subprocess.run(["make", "-C", CPP, f"REFERENCE_ROOT={REF_ROOT}"], check=True,
                   capture_output=True)
    assert os.path.exists(os.path.join(BUILD, "mtl4_dropin"))


@pytest.fixture(scope="module")
def built():
    if not os.path.exists(os.path.join(BUILD, "itl_gpu_test")):
        _make()


@pytest.mark.gpu
def test_spmv_stencil(built):
    r = _run("itl_gpu_test", "spmv")
    assert r["w12"] == 20 and r["w18"] == 2


@pytest.mark.gpu
def test_dot(built):
    r = _run("itl_gpu_test", "dot")
    assert r["dot"] == 285.0


@pytest.mark.gpu
def test_ic0_float_known_answer(built, golden):
    y = np.array(_run("itl_gpu_test", "ic0_float")["y"])
    # ic_0_test.cpp's expected values, tolerance 1e-3 as there
    yc = np.array([1.03194, 1.60198, 1.45357, 2.5258, 3.55386, 3.16, 2.91787, 4.09338, 3.81335])
    assert np.linalg.norm(y - yc) <= 1e-3
    assert np.max(np.abs(y - golden["kat_ic0_float_iota"])) <= 1e-12


@pytest.mark.gpu
def test_cg_iteration_object(built, golden):
    r = _run("itl_gpu_test", "cg")
    ref_it = int(golden["cfg1_iters"][0])
    assert r["error"] == 0 and r["converged"] == 1
    assert abs(r["iterations"] - ref_it) <= 2
    assert r["resid"] <= 1e-10 * r["norm_r0"]
    assert r["true_rel"] <= 3e-10
    # cyclic_iteration(cycle 50) printed at iterations 0, 50, 100, ...
    assert r["log_lines"] == r["iterations"] // 50 + 1


@pytest.mark.gpu
def test_bicgstab_iteration_object(built, golden):
    r = _run("itl_gpu_test", "bicgstab")
    assert r["error"] == 0
    assert abs(r["iterations"] - int(golden["cd8_iters"][0])) <= 2
    assert r["true_rel"] <= 3e-10


@pytest.mark.gpu
def test_mixed_refinement(built):
    r = _run("itl_gpu_test", "mixed")
    assert r["error"] == 0 and r["true_rel"] <= 1e-10


@pytest.mark.gpu
def test_exceptions(built):
    assert _run("itl_gpu_test", "errors")["caught"] == 3


@pytest.mark.gpu
def test_linear_solve_gradients_vs_finite_differences(built):
    r = _run("itl_gpu_test", "adjoint")
    assert r["forward_iterations"] > 0 and r["backward_iterations"] > 0
    # central differences with h = 1e-6: truncation and rounding leave ~1e-6 relative
    assert r["fd_rel_err_b"] <= 5e-5 and r["fd_rel_err_vals"] <= 5e-5, r


def _dropin():
    exe = os.path.join(BUILD, "mtl4_dropin")
    if not os.path.exists(exe):
        pytest.skip("mtl4_dropin is built only where the MTL4 headers are present")


@pytest.mark.gpu
def test_mtl4_dropin_cg():
    _dropin()
    r = _run("mtl4_dropin", "cg")
    cpu, gpu, cls = r["cpu"], r["gpu"], r["gpu_solver_class"]
    assert cpu["error"] == gpu["error"] == cls["error"] == 0
    assert abs(gpu["iterations"] - cpu["iterations"]) <= 2
    assert cls["iterations"] == gpu["iterations"]
    assert gpu["norm_r0"] == cpu["norm_r0"]
    assert r["gpu_log_lines"] == gpu["iterations"] // 50 + 1
    assert r["x_max_diff"] <= 1e-8 and r["copy_back_max_diff"] == 0


@pytest.mark.gpu
def test_mtl4_dropin_bicgstab():
    _dropin()
    r = _run("mtl4_dropin", "bicgstab")
    assert r["cpu"]["error"] == r["gpu"]["error"] == 0
    assert abs(r["gpu"]["iterations"] - r["cpu"]["iterations"]) <= 2
    assert r["x_max_diff"] <= 1e-8


@pytest.mark.gpu
def test_mtl4_dropin_preconditioners():
    _dropin()
    r = _run("mtl4_dropin", "pc")
    assert r["ic0_float_max_diff"] <= 1e-12
    assert r["ilu0_max_diff"] <= 1e-14 and r["ilu0_adjoint_max_diff"] <= 1e-14


@pytest.mark.gpu
def test_device_inserter(built):
    r = _run("itl_gpu_test", "assemble")
    assert r["laplacian_equal"] and r["updaters"] and r["range_error"]
    assert r["nnz"] == 5 * 600 - 2 * (20 + 30)


@pytest.mark.gpu
def test_mtl4_dropin_inserter():
    _dropin()
    r = _run("mtl4_dropin", "assemble")
    assert r["identical"] and r["laplacian_identical"] and r["nnz"] > 0


@pytest.mark.gpu
def test_mtl4_dropin_other_krylov_methods():
    # itl::bicg ... itl::gmres called as the reference's tests call them, on
    # the reference's CPU types and on device types in one program
    _dropin()
    r = _run("mtl4_dropin", "krylov")
    for meth in ("bicg", "cgs", "bicgstab_2", "bicgstab_ell", "tfqmr", "qmr", "idr_s", "gmres"):
        cpu, gpu = r[meth]["cpu"], r[meth]["gpu"]
        assert cpu[1] == gpu[1], (meth, cpu, gpu)
        tol = 8 if meth == "gmres" else 2
        assert abs(cpu[0] - gpu[0]) <= tol, (meth, cpu, gpu)
        assert r[meth]["x_max_diff"] <= 1e-5, (meth, r[meth])
