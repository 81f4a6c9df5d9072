"""The C++ mirror of the API (cubokit_b200/include/CuboPtycho.hpp): it compiles and links against the engine here;
tests/test_gpu_cpp.py runs it on a GPU against CuboKit's main pin."""
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "test_reconstruct.cpp"
EXE = ROOT / "tests" / "cpp" / "test_reconstruct"


def build():
    from cubokit_b200 import build as b
    lib = b.build(quiet=True)
    gxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
    subprocess.run([gxx, "-std=c++17", "-O2", "-I", str(ROOT / "cubokit_b200" / "include"), str(SRC), "-o", str(EXE),
                    "-L", str(lib.parent), "-lcuboptycho", f"-Wl,-rpath,{lib.parent}"], check=True)
    return EXE


ENGINES_SRC = ROOT / "tests" / "cpp" / "run_engines.cpp"
ENGINES_EXE = ROOT / "tests" / "cpp" / "run_engines"


def build_engines():
    from cubokit_b200 import build as b
    lib = b.build(quiet=True)
    gxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
    subprocess.run([gxx, "-std=c++17", "-O2", "-I", str(ROOT / "cubokit_b200" / "include"), str(ENGINES_SRC), "-o",
                    str(ENGINES_EXE), "-L", str(lib.parent), "-lcuboptycho", f"-Wl,-rpath,{lib.parent}"], check=True)
    return ENGINES_EXE


def test_cpp_mirror_compiles_and_links():
    assert build().exists()


def test_cpp_engine_mirrors_compile_and_link():
    """MixedstatePtychography and MultislicePtychography of the C++ mirror (run on a GPU by tests/test_gpu_cpp.py)."""
    assert build_engines().exists()
