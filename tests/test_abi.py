"""The C-ABI boundary without a GPU: exports, config parsing and error codes.

Everything here runs before the library touches CUDA (JSON and .bin loading
happen first), so the error paths are exercised on a CPU-only host; a valid
model either opens on a GPU or fails with MFDM_ERR_CUDA - never silently on the CPU.
"""
import json
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mfdm.h")

ERR = {"ARG": -1, "IO": -2, "CONFIG": -3, "CUDA": -4, "NONFINITE": -5, "NOMEM": -6}


@pytest.fixture(scope="module")
def lib(mfdm):
    mfdm.build()
    return mfdm.load_library()


def header_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(mfdm_\w+)\s*\(", text, re.M)))


def test_header_matches_binding(mfdm):
    assert sorted(mfdm.EXPORTS) == header_functions()


def test_library_exports_every_declared_symbol(lib, mfdm):
    out = subprocess.run(["nm", "-D", "--defined-only", mfdm.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (mfdm_\w+)", out))
    for name in header_functions():
        assert name in exported, name
        assert hasattr(lib, name)


def test_error_codes_match_header():
    text = open(HEADER).read()
    for name, code in ERR.items():
        assert re.search(rf"#define MFDM_ERR_{name} \({code}\)", text), name


def _open(mfdm, path):
    import ctypes
    h = ctypes.c_void_p()
    rc = mfdm.load_library().mfdm_open_json(os.fsencode(str(path)), 0, ctypes.byref(h))
    msg = mfdm.load_library().mfdm_last_error().decode()
    if rc == 0:
        mfdm.load_library().mfdm_close(h)
    return rc, msg


@pytest.fixture()
def small_model(modelgen, tmp_path):
    m = modelgen.make_model(40, 16, 20, npd=4, nt=10)
    j = modelgen.write_model(m, str(tmp_path / "m"))
    return m, j


def _edit(jpath, fn):
    cfg = json.load(open(jpath))
    fn(cfg)
    json.dump(cfg, open(jpath, "w"))


def test_missing_json(lib, mfdm, tmp_path):
    rc, msg = _open(mfdm, tmp_path / "nope.json")
    assert rc == ERR["CONFIG"] and "Cannot open JSON file" in msg


def test_malformed_json(lib, mfdm, tmp_path):
    p = tmp_path / "bad.json"
    p.write_text('{"base": {"fpeak": 30.0,, }')
    rc, msg = _open(mfdm, p)
    assert rc == ERR["CONFIG"] and "Failed to parse JSON" in msg


def test_empty_json(lib, mfdm, tmp_path):
    p = tmp_path / "empty.json"
    p.write_text("")
    rc, msg = _open(mfdm, p)
    assert rc == ERR["CONFIG"] and "empty" in msg


def test_missing_key(lib, mfdm, small_model):
    _, j = small_model
    _edit(j, lambda c: c["PML"].pop("beta0"))
    rc, msg = _open(mfdm, j)
    assert rc == ERR["CONFIG"] and "JSON path not found: PML.beta0" in msg


def test_type_mismatch(lib, mfdm, small_model):
    _, j = small_model
    _edit(j, lambda c: c["base"].__setitem__("nt", "many"))
    rc, msg = _open(mfdm, j)
    assert rc == ERR["CONFIG"] and "expected int" in msg


def test_unsupported_configuration(lib, mfdm, small_model):
    _, j = small_model
    # Dirichlet boundaries (boundary_type 0) are not built; 1 and 2 are
    _edit(j, lambda c: c["grid"].__setitem__("boundary_type", 0))
    rc, msg = _open(mfdm, j)
    assert rc == ERR["ARG"] and "unsupported" in msg


def test_nx_mismatch(lib, mfdm, small_model):
    _, j = small_model
    _edit(j, lambda c: c["grid"]["fluid"].__setitem__("nx", 41))
    rc, msg = _open(mfdm, j)
    assert rc == ERR["CONFIG"] and "nx_fluid doesn't match nx_solid" in msg


def test_missing_bin(lib, mfdm, small_model):
    _, j = small_model
    cfg = json.load(open(j))
    os.remove(cfg["grid"]["solid"]["C55"])
    rc, msg = _open(mfdm, j)
    assert rc == ERR["IO"] and "Failed to open file" in msg


def test_truncated_bin(lib, mfdm, small_model):
    _, j = small_model
    cfg = json.load(open(j))
    p = cfg["grid"]["jacob"]["ze_z"]
    data = open(p, "rb").read()
    open(p, "wb").write(data[:-4])
    rc, msg = _open(mfdm, j)
    assert rc == ERR["IO"] and "Failed to read data" in msg


def test_float_int_semantics(lib, mfdm, small_model):
    """nt given as 10.9 is read as 10 (int truncation like cJSON's valueint)."""
    _, j = small_model
    _edit(j, lambda c: c["base"].__setitem__("nt", 10.9))
    rc, msg = _open(mfdm, j)
    # Valid config: opens on a GPU host; without a GPU the first CUDA call fails.
    assert rc in (0, ERR["CUDA"]), msg


def test_valid_model_never_falls_back_to_cpu(lib, mfdm, small_model):
    _, j = small_model
    rc, msg = _open(mfdm, j)
    assert rc in (0, ERR["CUDA"]), msg
    if rc == ERR["CUDA"]:
        assert "cuda" in msg.lower()


def test_cli_usage_and_bad_output_dir(mfdm, small_model):
    mfdm.build()
    r = subprocess.run([mfdm.CLI_PATH], capture_output=True, text=True)
    assert r.returncode == 1 and "usage" in r.stderr
    _, j = small_model
    for bad in (".", "/", ".."):
        r = subprocess.run([mfdm.CLI_PATH, j, bad], capture_output=True, text=True)
        assert r.returncode == 1 and "Invalid output dir" in r.stderr


def test_field_ids_match_header(mfdm):
    text = open(HEADER).read()
    for name, fid in mfdm.FIELDS.items():
        assert re.search(rf"#define MFDM_{name.upper()} {fid}\b", text), name


def test_desc_layout_matches_header(mfdm):
    """The ctypes mirror of mfdm_desc has the header's field order."""
    text = open(HEADER).read()
    body = text[text.index("typedef struct mfdm_desc"):text.index("} mfdm_desc;")]
    names = re.findall(r"\b(\w+)\s*(?:,|;)", re.sub(r"/\*.*?\*/", "", body, flags=re.S))
    assert [f for f, _ in mfdm.Desc._fields_] == names
