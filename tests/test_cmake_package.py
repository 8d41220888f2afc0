"""The CMake package (reference-implementation_b200/cmake/tapp-config.cmake):
a consumer project written against the reference's package (find_package
tapp, component reference, target tapp::reference) configures, builds and
runs against the B200 library. CPU only; skipped when cmake is absent."""
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("cmake") is None, reason="cmake not installed")
def test_consumer_builds_and_runs(tmp_path, tapp):
    src = os.path.join(REPO, "tests", "consume")
    pkg = os.path.join(REPO, "reference-implementation_b200", "cmake")
    b = tmp_path / "build"
    r = subprocess.run(["cmake", "-S", src, "-B", str(b), f"-Dtapp_DIR={pkg}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    r = subprocess.run(["cmake", "--build", str(b)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    r = subprocess.run([str(b / "consume")], capture_output=True, text=True)
    assert r.returncode == 0 and "consume ok" in r.stdout, r.stdout + r.stderr


@pytest.mark.skipif(shutil.which("cmake") is None, reason="cmake not installed")
def test_unknown_component_fails(tmp_path):
    proj = tmp_path / "p"
    proj.mkdir()
    (proj / "CMakeLists.txt").write_text(
        "cmake_minimum_required(VERSION 3.15)\nproject(x LANGUAGES C)\n"
        "find_package(tapp REQUIRED COMPONENTS nosuch)\n")
    pkg = os.path.join(REPO, "reference-implementation_b200", "cmake")
    r = subprocess.run(["cmake", "-S", str(proj), "-B", str(tmp_path / "b"), f"-Dtapp_DIR={pkg}"],
                       capture_output=True, text=True)
    assert r.returncode != 0 and "unknown component" in (r.stdout + r.stderr)
