"""The C-ABI library: loads without a GPU, exports every entry point the
header declares, and reports errors as statuses (never exits)."""
import ctypes as C
import re
import subprocess

import pytest

from tests.conftest import REPO


def header_symbols():
    text = (REPO / "include" / "omcgpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(omc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from ompmc_b200 import engine
    lib = engine.lib()
    syms = header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, f"declared but not exported: {missing}"


def test_exported_symbols_match_nm():
    from ompmc_b200.engine import LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB_PATH)], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l and l.split()[-1].startswith("omc_")}
    assert set(header_symbols()) <= exported


def test_status_strings_and_version():
    from ompmc_b200 import engine
    L = engine.lib()
    assert L.omc_status_string(0) == b"ok"
    assert L.omc_status_string(-4) == b"medium not found"
    assert L.omc_version() >= 10000


def test_tables_missing_file_is_a_status(assets_root):
    from ompmc_b200.engine import OmcError, Tables
    with pytest.raises(OmcError) as ei:
        Tables(assets_root / "pegs4" / "nope.pegs4dat", assets_root / "pegs4" / "pgs4form.dat",
               assets_root / "data", ["H2O521ICRU"])
    assert ei.value.status == -2
    assert "nope.pegs4dat" in str(ei.value)


def test_tables_unknown_medium_is_a_status(assets_root):
    from ompmc_b200.engine import OmcError, Tables
    with pytest.raises(OmcError) as ei:
        Tables.from_assets(["H2O521ICRU", "UNOBTAINIUM"], assets_root)
    assert ei.value.status == -4
    assert "UNOBTAINIUM" in str(ei.value)


def test_engine_without_gpu_fails_cleanly(assets_root):
    """On a host without a device the engine reports OMC_E_CUDA."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from ompmc_b200 import assets as A
    from ompmc_b200.engine import Engine, OmcError, Tables
    t = Tables.from_assets(["H2O521ICRU"], assets_root)
    with pytest.raises(OmcError) as ei:
        Engine(t, A.water_cube(4, 1.0))
    assert ei.value.status == -10


def test_cli_usage_error_exit_code():
    from ompmc_b200.engine import CLI_PATH
    p = subprocess.run([str(CLI_PATH)], capture_output=True, text=True)
    assert p.returncode == 1
    assert "usage" in p.stderr
