"""A compiled C++ caller of the C ABI (tests/cpp/abi_caller.cc): it is built
with the host compiler against include/nrgb.h and linked with -lnrgb, the way
the reference's C++ would bind the library (the eigensolver seam in place of
dsyev_, src/diag.h:54-89, and nrgb_run in place of start_calculation,
src/nrg.cc:3429-3469).  On the CPU it must build, link and fail cleanly for
want of a device; on the GPU its decompositions pass its own checkdiag, its
run matches the oracle, and a library error takes the my_error exit path."""
import os
import subprocess

import pytest

import nrg_cases as cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "nrgljubljana-old_b200")


@pytest.fixture(scope="module")
def caller(tmp_path_factory):
    import nrgb
    nrgb.load()  # the library must exist
    exe = str(tmp_path_factory.mktemp("cpp") / "abi_caller")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "abi_caller.cc"), "-o", exe, "-L" + PKG, "-lnrgb",
           "-Wl,-rpath," + PKG]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_caller_builds_and_fails_cleanly_without_a_device(caller, tmp_path):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    r = subprocess.run([caller, str(tmp_path), str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 2, (r.returncode, r.stdout, r.stderr)
    assert r.stdout.startswith("nrgb")


@pytest.mark.gpu
def test_cpp_caller_on_the_device(caller, tmp_path):
    import nrg_oracle as O
    wd = cases.make_case("siam_ph", str(tmp_path / "in"))
    out_g, out_o = str(tmp_path / "gpu"), str(tmp_path / "oracle")
    os.makedirs(out_g)
    r = subprocess.run([caller, wd, out_g], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "diagonalised 7 blocks" in r.stdout
    O.Oracle(wd).run(out_o)
    cases.compare_outputs(cases.load_outputs(out_g), cases.load_outputs(out_o), "cpp caller")
    # an error inside the library reaches the caller as a status and a message
    empty = tmp_path / "empty"
    empty.mkdir()
    r = subprocess.run([caller, "--bad-run", str(empty)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "ERROR: nrgb_run:" in r.stderr, (r.returncode, r.stderr)
