"""The C-ABI library builds, loads and exports every symbol the header declares (CPU only)."""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def header_symbols():
    text = (ROOT / "include" / "vsjoin.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|long long|const char\*)\s+(vs_\w+)\s*\(", text, re.M)))


def test_library_builds_and_exports_header_symbols():
    from vibespatial_b200 import _build

    lib = _build.build()
    assert lib.exists()
    import ctypes

    L = ctypes.CDLL(str(lib))
    syms = header_symbols()
    assert len(syms) >= 10
    missing = [s for s in syms if not hasattr(L, s)]
    assert missing == []


def test_binding_covers_header():
    from vibespatial_b200 import _abi

    assert sorted(_abi.EXPORTED) == header_symbols()
    L = _abi.load()
    assert L.vs_version() == 2
    assert L.vs_last_error() is not None


def test_hilbert_host_restatement_is_a_bijection_with_locality():
    from vibespatial_b200._abi import hilbert_key_host

    # level-4 grid: all 256 cells map to distinct keys, consecutive keys are neighbours
    cells = {}
    for x in range(16):
        for y in range(16):
            k = hilbert_key_host(x << 28, y << 28, levels=4)
            cells[k] = (x, y)
    assert sorted(cells) == list(range(256))
    for k in range(255):
        (x0, y0), (x1, y1) = cells[k], cells[k + 1]
        assert abs(x0 - x1) + abs(y0 - y1) == 1
