"""The C ABI library on the CPU: it loads, exports every declared symbol, and
its host-side parts (configuration, PlaneImpactResponse build) agree with the
oracle.  No compute kernel runs here."""

import json
import os
import re

import numpy as np
import pytest

from conftest import ROOT, rel_l2

HEADER = os.path.join(ROOT, "include", "wctb200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(wct_[a-z0-9_]+)\s*\(", src)))


def test_header_parses_and_lists_entry_points():
    names = declared_functions()
    assert "wct_dt_forward" in names and "wct_pir_create" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(wct):
    L = wct.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_python_bindings_cover_the_header(wct):
    assert sorted(wct.SIGNATURES) == declared_functions()


def test_version_and_default_configuration(wct):
    assert b"sm_100a" in wct.lib().wct_version()
    cfg = wct.DepoTransform.default_configuration()
    # gen/src/DepoTransform.cxx:114-153
    for k in ("nsigma", "fluctuate", "start_time", "readout_time", "tick", "drift_speed", "first_frame_number",
              "anode", "rng", "pirs", "dft"):
        assert k in cfg
    assert cfg["nsigma"] == 3.0 and cfg["tick"] == 500.0 and cfg["readout_time"] == 5.0e6 and cfg["dft"] == "FftwDFT"


def test_configuration_errors_are_status_codes(wct):
    """DepoTransform::configure throws on empty pirs (gen/src/DepoTransform.cxx:101-106);
    the C ABI reports WCT_ERR_CONFIG instead and never throws."""
    with pytest.raises(wct.WctError) as e:
        wct.DepoTransform({"pirs": []})
    assert e.value.code == wct.WCT_ERR_CONFIG
    with pytest.raises(wct.WctError) as e:
        wct.DepoTransform({"drift_speed": -1.0})
    assert e.value.code == wct.WCT_ERR_CONFIG
    import ctypes as C
    h = C.c_void_p()
    assert wct.lib().wct_dt_create(b"{not json", C.byref(h)) == wct.WCT_ERR_CONFIG
    assert wct.lib().wct_last_error()
    # integer keys out of range, and a readout shorter than one tick, are refused before any device work
    for bad in ({"seed": -1}, {"seed": 2.0 ** 64}, {"first_frame_number": 1e12}, {"device": -1},
                {"readout_time": 100.0, "tick": 500.0}, {"readout_time": 1e30}, {"nsigma": 3.0, "tick": 0.0}):
        assert wct.lib().wct_dt_create(json.dumps(bad).encode(), C.byref(h)) == wct.WCT_ERR_CONFIG, bad


def test_null_arguments_are_rejected(wct):
    import ctypes as C
    L = wct.lib()
    assert L.wct_dt_create(b"{}", None) == wct.WCT_ERR_ARG
    assert L.wct_pir_create(None, 0, None, None, 1.0, 1.0, 10, None) == wct.WCT_ERR_ARG
    assert L.wct_dt_forward(None, None, 0, None, None, None) == wct.WCT_ERR_ARG
    k = C.c_int()
    assert L.wct_pir_closest(None, 0.0, C.byref(k)) == wct.WCT_ERR_ARG


def test_pir_create_argument_checks(wct, synth):
    """Inconsistent response arguments are status codes: short responses
    announced but not given, a negative length, a non-positive field-response
    pitch (PlaneImpactResponse's wire numbering divides by it), and a field
    response sampled before t = 0 (the reference's bin index would not exist)."""
    import ctypes as C
    L = wct.lib()
    fr = synth.plane1_config(nticks=1000, nwire_half=10)["fr"][0]
    pp = np.ascontiguousarray(fr["pitchpos"], dtype=np.float64)
    cur = np.ascontiguousarray(fr["current"], dtype=np.float64)
    h = C.c_void_p()

    def create(pitch=fr["pitch"], tstart=fr["tstart"], nshort=0, sl=None, sw=None):
        d = wct.FrPlane(pp.shape[0], cur.shape[1], pp.ctypes.data, cur.ctypes.data, pitch, tstart, fr["period"])
        return L.wct_pir_create(C.byref(d), nshort, sl, sw, 100e3, 500.0, 1000, C.byref(h))

    assert create(nshort=1) == wct.WCT_ERR_ARG
    neg = np.array([-5], dtype=np.int32)
    wave = np.zeros(4)
    assert create(nshort=1, sl=neg.ctypes.data, sw=wave.ctypes.data) == wct.WCT_ERR_ARG
    assert create(pitch=0.0) == wct.WCT_ERR_CONFIG
    assert create(tstart=-10e3) == wct.WCT_ERR_CONFIG
    assert create() == wct.WCT_OK
    L.wct_pir_destroy(h)
    assert L.wct_pir_set_long_responses(None, 0, None, None, 0.0) == wct.WCT_ERR_ARG


@pytest.mark.parametrize("nwire_half", [10, 21])
def test_pir_build_matches_oracle(wct, oracle, synth, nwire_half):
    """PlaneImpactResponse::build_responses (gen/src/PlaneImpactResponse.cxx:89-269):
    the product's host build against the oracle's FP64 restatement."""
    cfg = synth.plane1_config(nticks=1000, nwire_half=nwire_half)
    ref = oracle.pir_build(cfg, 0, fp64=True)
    pir = wct.PlaneImpactResponse(cfg["fr"][0], cfg["short_responses"], cfg["overall_short_padding"], cfg["tick"],
                                  cfg["pir_nticks"])
    info = pir.info()
    assert info["nwires"] == ref["bywire"].shape[0]
    assert info["nimp_per_wire"] == ref["bywire"].shape[1] == 11
    assert info["pitch"] == ref["pitch"] and info["impact"] == ref["impact"]
    assert info["half_extent"] == ref["half_extent"]
    assert info["waveform_pad"] == 200
    for p in range(0, info["npaths"], 7):
        assert rel_l2(pir.waveform(p), ref["waveforms"][p]) < 1e-6
    # closest(): the reference rule, path for path
    rng = np.random.default_rng(3)
    for rp in rng.uniform(-ref["half_extent"], ref["half_extent"], 500):
        wi = ref["bywire"].shape[0] // 2 + oracle.cround(rp / ref["pitch"])
        rem = rp - oracle.cround(rp / ref["pitch"]) * ref["pitch"]
        ii = oracle.cround(rem / ref["impact"]) + ref["bywire"].shape[1] // 2
        if 0 <= wi < ref["bywire"].shape[0] and 0 <= ii < ref["bywire"].shape[1]:
            assert pir.closest(float(rp)) == ref["bywire"][wi][ii]
    with pytest.raises(wct.WctError) as e:
        pir.closest(ref["half_extent"] * 1.01)
    assert e.value.code == wct.WCT_ERR_RESPONSE


def test_dt_create_reports_cuda_state(wct):
    """Without a GPU the component cannot be created; the failure is a status
    code, not a crash (on a GPU machine creation succeeds)."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        dt = wct.DepoTransform({})
        assert dt.frame_shape()[0] == 0
    else:
        with pytest.raises(wct.WctError) as e:
            wct.DepoTransform({})
        assert e.value.code == wct.WCT_ERR_CUDA


def _header_prototypes():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"#[^\n]*", "", src)
    out = {}
    for m in re.finditer(r"([A-Za-z_][\w \t\*]*?)\b(wct_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", src):
        ret, name, params = m.group(1), m.group(2), m.group(3).strip()
        ps = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
        # drop the parameter name: the last identifier of each parameter
        types = [re.sub(r"\b\w+$", "", p).strip() if re.search(r"[\w\*]\s*\w+$", p) else p for p in ps]
        out[name] = (ret.strip(), types)
    return out


# argument classes of the x86-64 LP64 calling convention, which is what a
# ctypes prototype must match (ctypes itself aliases long long to long and
# size_t to unsigned long there)
def _c_kind(t):
    t = " ".join(t.replace("*", " * ").split())
    if "*" in t:
        return "ptr"
    t = t.replace("const ", "")
    return {"int": "i32", "long": "i64", "long long": "i64", "double": "f64", "size_t": "u64",
            "unsigned long long": "u64"}[t]


def _ct_kind(c):
    import ctypes as C
    if c in (C.c_void_p, C.c_char_p) or (isinstance(c, type) and issubclass(c, C._Pointer)):
        return "ptr"
    if C.sizeof(C.c_long) != 8:
        pytest.skip("an LP64 platform is assumed")
    return {C.c_int: "i32", C.c_long: "i64", C.c_double: "f64", C.c_ulong: "u64"}[c]


def test_python_argtypes_match_header(wct):
    """Every ctypes prototype has the header's arity and argument classes
    (pointer, 32-bit int, signed and unsigned 64-bit int, double) and return
    class."""
    protos = _header_prototypes()
    assert sorted(protos) == sorted(wct.SIGNATURES)
    for name, (rt, at) in wct.SIGNATURES.items():
        hret, htypes = protos[name]
        assert len(at) == len(htypes), (name, len(at), htypes)
        assert [_ct_kind(a) for a in at] == [_c_kind(t) for t in htypes], name
        assert _ct_kind(rt) == _c_kind(hret), name
