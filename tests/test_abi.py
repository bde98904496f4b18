"""CPU checks of the C-ABI library: it loads without a GPU, exports every
function include/alpineem_b200.h declares, and rejects invalid decks with
the reference's own error text (main_fdtd/fdtd_solver.f90:726-1298)."""
import ctypes
import os
import re

import pytest

import decks

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol(gpu_lib):
    import alpineem_b200 as ab

    with open(os.path.join(ROOT, "include", "alpineem_b200.h")) as f:
        declared = sorted(set(re.findall(r"\b(aem_[a-z_]+)\s*\(", f.read())))
    assert len(declared) >= 20
    lib = ctypes.CDLL(ab.LIB_PATH)
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert ab.exported_symbols() == declared


def test_version(gpu_lib):
    assert gpu_lib.aem_version() >= 10000


@pytest.mark.parametrize("name", sorted(decks.DECKS))
def test_check_deck_accepts_every_test_deck(name, tmp_path):
    import alpineem_b200 as ab

    path, kmax = decks.write_deck(name, str(tmp_path))
    ext = open(path + ".b200").read() if os.path.exists(path + ".b200") else None
    X, Y, Z = ab.check_deck(open(path).read(), ext, kmax=kmax)
    d = decks.DECKS[name]
    bc = d.get("bc", (0,) * 6)
    assert (X, Y, Z) == tuple(d["n"][a] + 1 + (1 if bc[2 * a] and bc[2 * a + 1] else 0) for a in range(3))


def _mutate(text, line_no, new):
    lines = text.splitlines()
    lines[line_no] = new
    return "\n".join(lines) + "\n"


def test_check_deck_reference_errors(tmp_path):
    import alpineem_b200 as ab

    base = decks.deck_text(decks.DECKS["pbc_sheets"])
    # oblique incidence on a periodic y boundary (ref :781-789)
    bad = _mutate(base, 9, "1,0")
    bad = _mutate(bad, 10, "60,30,90")
    with pytest.raises(ab.AemError, match="ERROR: INCIDENT PLANE WAVE W/ OBLIQUE ANGLE"):
        ab.check_deck(bad)
    with pytest.raises(ab.AemError):
        ab.check_deck("90,30,30\n")
    with pytest.raises(ab.AemError, match="unknown extension"):
        ab.check_deck(base, "no_such_key 3\n")
    with pytest.raises(ab.AemError, match="pml_cells"):
        ab.check_deck(base, "pml_cells -2\n")
    for ext in ("dft_freqs 1e9\n", "dft_freqs 2e9 1e9 8\n", "dft_freqs 1e9 2e9 0\n", "dft_freqs -1 2e9 8\n",
                "dft_freqs 1e9 2e9 x\n", "dft_freqs 1e9 2e9 5000\n"):
        with pytest.raises(ab.AemError, match="dft_freqs"):
            ab.check_deck(base, ext)
    assert ab.check_deck(base, "dft_freqs 1e9 2e10 128\n") == ab.check_deck(base)
    for ext in ("watchdog -1\n", "watchdog x\n"):
        with pytest.raises(ab.AemError, match="watchdog"):
            ab.check_deck(base, ext)
    assert ab.check_deck(base, "watchdog 100\n") == ab.check_deck(base)
