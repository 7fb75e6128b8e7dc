"""The reference-compatible C++ header compiles against the C ABI library,
and a program written against silk::World runs on the GPU."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "cpp" / "drop_in_world.cpp"
EXE = ROOT / "tests" / "cpp" / "drop_in_world"


def _build():
    cmd = ["/usr/bin/g++", "-std=c++20", "-O1", "-I", str(ROOT / "include"), str(SRC),
           "-L", str(ROOT / "silk_physics_b200"), "-lsilk_b200",
           f"-Wl,-rpath,{ROOT / 'silk_physics_b200'}", "-o", str(EXE)]
    subprocess.run(cmd, check=True)


def test_header_compiles_and_links():
    _build()
    assert EXE.exists()


@pytest.mark.gpu
def test_dropin_program_runs():
    _build()
    out = subprocess.run([str(EXE)], capture_output=True, text=True, timeout=120)
    print(out.stdout, out.stderr)
    assert out.returncode == 0
    assert "ok" in out.stdout
