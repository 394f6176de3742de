"""The C ABI from plain C: include/wctb200.h compiles as C99 and as C++, its
structs have the layout of the Python mirrors, and a C program
(tests/c_consumer.c) linked against libwctb200.so builds a
PlaneImpactResponse through it with the same results as the Python binding.
Host-side entry points only; CPU."""

import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

INCLUDE = os.path.join(ROOT, "include")
PKG = os.path.join(ROOT, "wire-cell-toolkit_b200")


def _need(tool):
    if shutil.which(tool) is None:
        pytest.skip(tool + " not available")


def test_header_compiles_as_c_and_cxx(tmp_path):
    _need("gcc")
    _need("g++")
    hdr = os.path.join(INCLUDE, "wctb200.h")
    for cmd in (["gcc", "-std=c99", "-pedantic", "-Wall", "-Werror", "-fsyntax-only", "-x", "c", hdr],
                ["g++", "-std=c++11", "-pedantic", "-Wall", "-Werror", "-fsyntax-only", "-x", "c++", hdr]):
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_c_program_builds_a_pir(tmp_path, wct, synth):
    _need("gcc")
    wct.lib()  # builds libwctb200.so if needed
    exe = str(tmp_path / "c_consumer")
    r = subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Werror", "-I", INCLUDE,
                        os.path.join(ROOT, "tests", "c_consumer.c"), "-L", PKG, "-lwctb200",
                        "-Wl,-rpath," + PKG, "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

    cfg = synth.plane1_config(nticks=1000, nwire_half=3)
    fr = cfg["fr"][0]
    short = np.asarray(cfg["short_responses"][0], dtype=np.float64)
    pp = np.asarray(fr["pitchpos"], dtype=np.float64)
    cur = np.asarray(fr["current"], dtype=np.float64)
    rng = np.random.default_rng(11)
    half = 3.5 * fr["pitch"]
    rel = np.concatenate([rng.uniform(-half, half, 64), [1.2 * half, -1.2 * half]])
    hdr = [len(pp), cur.shape[1], fr["pitch"], fr["tstart"], fr["period"], cfg["overall_short_padding"],
           cfg["tick"], cfg["pir_nticks"], len(short), len(rel)]
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    np.concatenate([np.asarray(hdr, dtype=np.float64), pp, cur.ravel(), short, rel]).tofile(fin)
    r = subprocess.run([exe, fin, fout], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stderr)
    out = np.fromfile(fout, dtype=np.float64)

    assert out[0] == wct.WCT_ERR_ARG and out[1] == 1.0
    assert out[2] == wct.fft_best_length(984, True) == 1024
    assert out[3] == wct.fft_best_length(3334) == 3584
    pir = wct.PlaneImpactResponse(fr, cfg["short_responses"], cfg["overall_short_padding"], cfg["tick"],
                                  cfg["pir_nticks"])
    info = pir.info()
    keys = ["pitch", "impact", "half_extent", "nwires", "nimp_per_wire", "npaths", "nticks", "waveform_pad"]
    assert list(out[4:12]) == [float(info[k]) for k in keys]
    got = out[12:12 + len(rel)]
    for g, rp in zip(got, rel):
        try:
            want = pir.closest(float(rp))
        except wct.WctError as e:
            want = -1 - e.code
        assert g == want, (rp, g, want)
    waves = out[12 + len(rel):].reshape(info["npaths"], info["nticks"])
    for p in range(info["npaths"]):
        assert np.array_equal(waves[p].astype(np.float32), pir.waveform(p))


STRUCTS = {  # C struct of the header -> ctypes mirror in the package
    "wct_plane_desc": "PlaneDesc",
    "wct_fr_plane": "FrPlane",
    "wct_plane_window": "PlaneWindow",
    "wct_splat_config": "SplatConfig",
}


def test_struct_layouts_match_ctypes(tmp_path, wct):
    """sizeof and every member's offset of the header's structs, as the C
    compiler lays them out, equal the Python mirrors' (same member names in
    the same order)."""
    _need("gcc")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "wctb200.h"', "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for f, _ in getattr(wct, pyname)._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, f, cname, f))
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = str(tmp_path / "layout")
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", INCLUDE, str(src), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = {}
    for ln in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.splitlines():
        c, f, v = ln.split()
        got[(c, f)] = int(v)
    for cname, pyname in STRUCTS.items():
        cls = getattr(wct, pyname)
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert got[(cname, f)] == getattr(cls, f).offset, (cname, f)
