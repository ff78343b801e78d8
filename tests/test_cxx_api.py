"""The C++ interface (include/hptt/hptt.h, libhptt.so) as a reference user sees
it: the test program tests/cxx/test_cxx_api.cpp is compiled with g++ against
the public header only.

CPU: libhptt.so exports hptt::create_plan<T> for the four element types and
the four create_trans_plan_impl_* factories under the mangled names the
reference's loader resolves (src/hptt.cc:67-81); the argument guard returns
nullptr where the reference's does.
GPU: every element type, reset_data, the complex-scalar overload and the
factories, each result bit-exact against the oracle.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hptt_b200")
LIBHPTT = os.path.join(PKG, "libhptt.so")
ORACLE_DIR = os.path.join(ROOT, "oracle")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
SRC = os.path.join(ROOT, "tests", "cxx", "test_cxx_api.cpp")

# Mangled names the reference's loader looks up (src/hptt.cc:67-81).
FACTORIES = [
    "_Z24create_trans_plan_impl_sPKfPfjRKSt6vectorIjSaIjEES6_ffjdS6_S6_",
    "_Z24create_trans_plan_impl_dPKdPdjRKSt6vectorIjSaIjEES6_ddjdS6_S6_",
    "_Z24create_trans_plan_impl_cPKCfPS_jRKSt6vectorIjSaIjEES7_ffjdS7_S7_",
    "_Z24create_trans_plan_impl_zPKCdPS_jRKSt6vectorIjSaIjEES7_ddjdS7_S7_",
]


@pytest.fixture(scope="module")
def cxx_binary(tmp_path_factory):
    if not os.path.exists(LIBHPTT):
        from hptt_b200 import build as b
        b.build()
    import oracle
    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build(with_ref=False)
    if shutil.which(os.environ.get("CXX", "g++")) is None:
        pytest.skip("no C++ compiler")
    out = str(tmp_path_factory.mktemp("cxx") / "test_cxx_api")
    cmd = [os.environ.get("CXX", "g++"), "-std=c++14", "-O1", "-Wall",
           "-I", os.path.join(ROOT, "include"), "-I", ORACLE_DIR,
           "-I", os.path.join(CUDA, "include"), SRC, "-o", out,
           "-L", PKG, "-lhptt", "-lhptt_cuda", "-L", ORACLE_DIR, "-loracle",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-ldl",
           f"-Wl,-rpath,{PKG}:{ORACLE_DIR}:{os.path.join(CUDA, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return out


def _dynamic_symbols(path):
    r = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return {line.split()[-1] for line in r.stdout.splitlines() if line.strip()}


def test_exports_reference_symbols():
    if not os.path.exists(LIBHPTT):
        from hptt_b200 import build as b
        b.build()
    syms = _dynamic_symbols(LIBHPTT)
    for name in FACTORIES:
        assert name in syms, name
    # hptt::create_plan<T> for T = float, double, float _Complex, double _Complex
    for t in ("If", "Id", "ICf", "ICd"):
        assert any(s.startswith(f"_ZN4hptt11create_plan{t}E") for s in syms), t


def test_guard_returns_nullptr(cxx_binary):
    r = subprocess.run([cxx_binary, "guard"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failure(s)" in r.stdout


@pytest.mark.gpu
def test_gpu_parity_through_cxx_api(cxx_binary):
    r = subprocess.run([cxx_binary, "gpu", LIBHPTT], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert "gpu checks done, 0 failure(s)" in r.stdout
