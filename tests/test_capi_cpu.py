"""The C-ABI shared library loads and exports every declared entry point.

No compute call is made here (this suite runs without a GPU).
"""
import ctypes as C
import os
import re

import pytest

from n2p2_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "n2p2_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(n2p2b_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "n2p2b_evaluate" in names and "n2p2b_create" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_capi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_the_header():
    assert set(declared_functions()) <= set(_capi.SIGNATURES)


def test_create_without_gpu_reports_cuda_error():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    L = _capi.load()
    h = C.c_void_p()
    assert L.n2p2b_create(0, C.byref(h)) == _capi.ERR_CUDA
    assert not h.value


def test_null_context_is_rejected():
    L = _capi.load()
    assert L.n2p2b_evaluate(None, 1) == _capi.ERR_ARGUMENT
    assert L.n2p2b_last_error(None) == b"null context"


def test_cpp_wrapper_mirrors_mode_api(tmp_path):
    """The C++ header (nnp::Mode / Prediction / InterfaceLammps names over
    the C ABI) compiles and links a caller that uses the reference's
    evaluation steps (libnnp/Mode.h) and Prediction flow; nothing runs."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "caller.cpp"
    src.write_text(r'''
#include "n2p2_b200.hpp"
int main(int argc, char** argv)
{
    if (argc < 2) return 0;
    n2p2b::Prediction p(0);
    p.initialize();
    p.setup();
    p.setupSymmetryFunctionGroups();
    std::map<std::string, std::string> formats{
        {"short", p.formatWeightsFilesShort},
        {"elec", p.formatWeightsFilesCharge}};
    p.setupNeuralNetworkWeights(formats);
    p.setupNeuralNetworkWeights("weights.%03zu.data");
    p.readStructureFromFile(argv[1]);
    n2p2b::Structure& s = p.structure;
    p.calculateSymmetryFunctionGroups(s, true);
    p.calculateAtomicNeuralNetworks(s, true);
    p.calculateEnergy(s);
    p.calculateForces(s);
    p.evaluateNNP(s);
    p.evaluateNNP(s, false, true);
    p.predict();
    n2p2b::InterfaceLammps lmp(0);
    lmp.initialize(".", "", true, false, 0, -1, 1.0, 1.0, 12.0, 2, 0);
    char* buf = new char[lmp.getEWBufferSize() + 1];
    lmp.fillEWBuffer(buf, (int)lmp.getEWBufferSize());
    lmp.extractEWBuffer(buf, (int)lmp.getEWBufferSize());
    lmp.writeExtrapolationWarnings();
    lmp.clearExtrapolationWarnings();
    delete[] buf;
    return p.getMaxCutoffRadius() > 0.0 ? 0 : 1;
}
''')
    lib = os.path.join(root, "n2p2_b200")
    if not os.path.exists(os.path.join(lib, "libn2p2b200.so")):
        pytest.skip("library not built")
    r = subprocess.run([gxx, "-std=c++17", "-I" + os.path.join(root, "include"),
                        str(src), "-o", str(tmp_path / "caller"),
                        "-L" + lib, "-ln2p2b200"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_exponential_table_is_correctly_rounded():
    """The FP64 exponential of the staged symmetry-function kernel reads
    2^(j / 64), j = 0 .. 63, from a table in sf_staged.cuh; every entry is
    the double nearest to the exact value (checked at 200 bits), and the
    reduction constants are ln2 / 64 split into a 32-bit head and its
    tail, and 64 / ln2 rounded."""
    mpmath = pytest.importorskip("mpmath")
    src = os.path.join(os.path.dirname(__file__), "..", "n2p2_b200", "csrc",
                       "sf_staged.cuh")
    text = open(src).read()
    body = text[text.index("kExp2Table[64] = {"):]
    body = body[:body.index("};")]
    vals = [float.fromhex(h) for h in re.findall(r"0x[0-9a-f.]+p[+-]\d+",
                                                 body)]
    assert len(vals) == 64
    mpmath.mp.prec = 200
    for j, v in enumerate(vals):
        exact = mpmath.power(2, mpmath.mpf(j) / 64)
        assert v == float(exact)
    consts = dict(re.findall(r"constexpr double (k\w+) = (0x[0-9a-f.]+p[+-]\d+)",
                             text))
    hi = float.fromhex(consts["kLHi"])
    lo = float.fromhex(consts["kLLo"])
    ln2_64 = mpmath.log(2) / 64
    assert float(64 / mpmath.log(2)) == float.fromhex(consts["kInvL"])
    assert int(mpmath.mpf(hi) * 2 ** 38) == mpmath.mpf(hi) * 2 ** 38
    assert lo == float(ln2_64 - mpmath.mpf(hi))
