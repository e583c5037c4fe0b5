"""The C ABI without a GPU: the library loads, exports every function that
include/jimwlk.h declares, parses configuration files like the reference, and
reports errors as status codes (no compute calls here)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "jimwlk.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jw_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import jimwlk
    so = jimwlk.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (jw_[a-z0-9_]+)", out))
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing
    assert len(declared_functions()) >= 40


def test_config_read_matches_reference_parse(tmp_path):
    import jimwlk
    from jwref import Reference, config_text, reference_available
    text = config_text(mu=30.72, mass=0.0001, wilson_lines=50, step=0.0004, langevin_steps=100, measurements=100,
                       coupling="SQRT_COUPLING_CONSTANT", kernel="LINEAR_KERNEL")
    p = tmp_path / "config"
    p.write_text(text)
    c = jimwlk.config_read(str(p))
    assert c.mu == float(np.float32(30.72)) and c.mass == float(np.float32(0.0001))
    assert c.step == float(np.float32(0.0004))
    assert (c.CouplingChoice, c.KernelChoice, c.EvolutionChoice) == (0, 0, 1)
    assert c.elementaryWilsonLines == 50 and c.langevin_steps == 100 and c.measurements == 100
    if reference_available(8):
        r = Reference(8, text).config()
        assert (r["mu"], r["mass"], r["step"]) == (c.mu, c.mass, c.step)


def test_config_read_missing_file_is_an_error():
    import jimwlk
    with pytest.raises(jimwlk.JimwlkError):
        jimwlk.config_read("/nonexistent/config")


def test_status_strings():
    import jimwlk
    L = jimwlk.lib()
    for s in range(0, -10, -1):
        assert L.jw_status_string(s)
